// Shared helpers of the corrct B200 kernels (sm_100a only).
#pragma once

#include <atomic>

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

// The map of one (slice, angle, detector): an image of stored maps, or the two line-integral
// planes of a fields slice and the channel's scale (map = exp(-(L_in + scale * L_out))).
struct MapRef {
  const void* base;
  int64_t off;     // map image, or the L_out plane
  int64_t off_in;  // fields: the L_in plane
  float scale;     // fields: the channel's s_c
};

__device__ __forceinline__ MapRef make_map_ref(const void* maps, int dtype, int64_t slice_stride, int n_angles,
                                               int n_det, int n, int s, int a, int d, int n_channels,
                                               const float* channel_scale) {
  const int64_t plane = (int64_t)n * n;
  MapRef r;
  r.base = maps;
  if (dtype == CCT_DTYPE_FIELDS_F32) {
    const int fs = s / n_channels;
    const int c = s - fs * n_channels;
    r.off_in = (int64_t)fs * slice_stride + (int64_t)a * (1 + n_det) * plane;
    r.off = r.off_in + (int64_t)(1 + d) * plane;
    r.scale = __ldg(channel_scale + c);
  } else {
    r.off = (int64_t)s * slice_stride + ((int64_t)a * n_det + d) * plane;
    r.off_in = 0;
    r.scale = 0.f;
  }
  return r;
}

template <int DT>
__device__ __forceinline__ float map_at(const MapRef& m, int64_t pix) {
  if (DT == CCT_DTYPE_FIELDS_F32) {
    const float* f = reinterpret_cast<const float*>(m.base);
    return expf(-fmaf(m.scale, __ldg(f + m.off + pix), __ldg(f + m.off_in + pix)));
  }
  return load_map(m.base, DT, m.off + pix);
}

// Four consecutive map values (pix % 4 == 0, 16-byte aligned FP32 / 8-byte aligned BF16 data).
template <int DT>
__device__ __forceinline__ float4 map_at4(const MapRef& m, int64_t pix) {
  if (DT == CCT_DTYPE_BF16) {
    const uint2 raw = __ldg(reinterpret_cast<const uint2*>(reinterpret_cast<const __nv_bfloat16*>(m.base) + m.off + pix));
    const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&raw.x));
    const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&raw.y));
    return make_float4(lo.x, lo.y, hi.x, hi.y);
  }
  const float* f = reinterpret_cast<const float*>(m.base);
  if (DT == CCT_DTYPE_FIELDS_F32) {
    const float4 li = __ldg(reinterpret_cast<const float4*>(f + m.off_in + pix));
    const float4 lo = __ldg(reinterpret_cast<const float4*>(f + m.off + pix));
    return make_float4(expf(-fmaf(m.scale, lo.x, li.x)), expf(-fmaf(m.scale, lo.y, li.y)),
                       expf(-fmaf(m.scale, lo.z, li.z)), expf(-fmaf(m.scale, lo.w, li.w)));
  }
  return __ldg(reinterpret_cast<const float4*>(f + m.off + pix));
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

// Two bilinear samples of a staged box z (row stride STRIDE, zoff moving the origin) at the
// positions (x.x, y.x) and (x.y, y.y), added to acc in that order, in packed FP32x2 arithmetic.
// Every lane of every packed operation rounds like the scalar sequence
//   (fx, fy) = floor_split(x), floor_split(y)
//   top = fmaf(fx.f, t1 - t0, t0); bot = fmaf(fx.f, b1 - b0, b0); acc += fmaf(fy.f, bot - top, top)
// (a - b is formed as fma(b, -1, a), which rounds the exact difference once), so the result is
// bit-identical to it.
template <int STRIDE>
__device__ __forceinline__ float bilerp2(const float* z, int zoff, float2 x, float2 y, float acc) {
  const float2 magic = make_float2(12582912.0f, 12582912.0f);  // 1.5 * 2^23, see floor_split
  const float2 nmagic = make_float2(-12582912.0f, -12582912.0f);
  const float2 neg1 = make_float2(-1.f, -1.f);
  const float2 tx = __fadd2_rd(x, magic), ty = __fadd2_rd(y, magic);
  const float2 fx = __ffma2_rn(__fadd2_rn(tx, nmagic), neg1, x);  // x - floor(x), exact
  const float2 fy = __ffma2_rn(__fadd2_rn(ty, nmagic), neg1, y);
  const int q0 = (__float_as_int(ty.x) - 0x4B400000) * STRIDE + (__float_as_int(tx.x) - 0x4B400000) + zoff;
  const int q1 = (__float_as_int(ty.y) - 0x4B400000) * STRIDE + (__float_as_int(tx.y) - 0x4B400000) + zoff;
  const float2 t0 = make_float2(z[q0], z[q1]), t1 = make_float2(z[q0 + 1], z[q1 + 1]);
  const float2 b0 = make_float2(z[q0 + STRIDE], z[q1 + STRIDE]);
  const float2 b1 = make_float2(z[q0 + STRIDE + 1], z[q1 + STRIDE + 1]);
  const float2 top = __ffma2_rn(fx, __ffma2_rn(t0, neg1, t1), t0);
  const float2 bot = __ffma2_rn(fx, __ffma2_rn(b0, neg1, b1), b0);
  const float2 res = __ffma2_rn(fy, __ffma2_rn(top, neg1, bot), top);
  acc += res.x;
  acc += res.y;
  return acc;
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

// The dynamic shared-memory limit is a per-device attribute of a kernel: set it once per device
// (and kernel), thread-safe.  Devices beyond the first 64 set it before every launch.
template <auto KERNEL>
inline bool ensure_dynamic_smem(int bytes) {
  static std::atomic<uint64_t> done{0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  const uint64_t bit = (dev >= 0 && dev < 64) ? (1ull << dev) : 0ull;
  if (bit != 0 && (done.load(std::memory_order_acquire) & bit) != 0) return true;
  if (cudaFuncSetAttribute(KERNEL, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  done.fetch_or(bit, std::memory_order_acq_rel);
  return true;
}

// After a launch with a fallback: false (and the launch error cleared) if it was refused.
inline bool launched_ok() { return cudaGetLastError() == cudaSuccess; }

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
