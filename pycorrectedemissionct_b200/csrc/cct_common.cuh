// Shared helpers of the corrct B200 kernels (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/corrct_b200.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "corrct_b200 kernels are written for sm_100a (B200) only"
#endif

namespace cct {

// Maps are stored as FP32 or BF16; both are read as FP32.
__device__ __forceinline__ float load_map(const void* base, int dtype, int64_t idx) {
  if (dtype == CCT_DTYPE_BF16) {
    return __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(base)[idx]);
  }
  return __ldg(reinterpret_cast<const float*>(base) + idx);
}

// floor() of a coordinate in [-2^22, 2^22) without the conversion pipe:
// adding 1.5*2^23 with round-down leaves floor(x) in the low mantissa bits.
struct FloorSplit {
  int i;     // floor(x) as an integer
  float f;   // x - floor(x), exact
};
__device__ __forceinline__ FloorSplit floor_split(float x) {
  const float magic = 12582912.0f;  // 1.5 * 2^23
  float t = __fadd_rd(x, magic);
  float fl = t - magic;  // exact
  FloorSplit r;
  r.i = __float_as_int(t) - 0x4B400000;
  r.f = x - fl;  // exact (Sterbenz)
  return r;
}

__device__ __forceinline__ double warp_sum_double(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float warp_sum_float(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace cct

#define CCT_CUDA_TRY(expr)                       \
  do {                                           \
    cudaError_t _e = (expr);                     \
    if (_e != cudaSuccess) {                     \
      cct_set_last_error(cudaGetErrorString(_e)); \
      return CCT_ERR_CUDA;                       \
    }                                            \
  } while (0)

#define CCT_REQUIRE(cond, msg)  \
  do {                          \
    if (!(cond)) {              \
      cct_set_last_error(msg);  \
      return CCT_ERR_VALUE;     \
    }                           \
  } while (0)

void cct_set_last_error(const char* msg);
