// Warm-start network kernels (no reference counterpart): 3x3 convolutions as implicit GEMMs on
// the 5th-generation tensor cores (tcgen05.mma, BF16 x BF16 -> FP32 accumulators in TMEM), and
// the elementwise pieces of a small encoder-decoder (bias/ReLU, 2x2 average pooling, nearest
// upsampling, skip additions, MSE, Adam).
//
// Activations are NHWC bfloat16 with channel counts that are multiples of 16.  Weights are
// [Cout][3][3][Cin] bfloat16 ("K-major": k = tap * Cin + ci).
//
// GEMM tile: M = 128 rows (one TMEM lane each), N = BN columns (16..128, FP32 TMEM columns),
// K blocks of 64 elements staged in shared memory.  Forward (and data-gradient) convolutions use
// the 128-byte swizzled K-major UMMA layout: 8 lanes gather one tile row's 128 contiguous bytes
// (four rows per warp load) and write them as 8 chunks XOR-permuted by the row, conflict-free;
// the weight-gradient GEMM uses the canonical no-swizzle layout (the 16-byte chunk kc of row r
// at byte kc * ROWS * 16 + r * 16; descriptor start = base + 2s * ROWS * 16, leading-byte offset
// ROWS * 16, stride-byte offset 128).  Two operand buffers alternate: all 128 threads gather block
// kb + 1 while the tensor core works on block kb; one elected thread issues the four MMAs of a
// block and commits them to that buffer's mbarrier.  Every wait is bounded; on timeout the
// kernel raises g_net_timeout and leaves after waiting once more for its own MMAs.

#include <cstdint>
#include <cstring>

#include "cct_common.cuh"
#include "cct_internal.cuh"

namespace cct {

__device__ int g_net_timeout = 0;

constexpr int NET_THREADS = 128;
constexpr int NET_BM = 128;
constexpr int NET_BK = 64;
constexpr uint32_t NET_WAIT_LIMIT = 1u << 24;

enum NetMode : int { NET_FWD = 0, NET_WGRAD = 1 };

struct ConvArgs {
  int batch, h, w, cin, cout;
  int log2_cin;
  const __nv_bfloat16* x;   // NHWC input (FWD / WGRAD)
  const __nv_bfloat16* wt;  // [cout][9][cin] (FWD)
  const __nv_bfloat16* dy;  // NHWC output gradient (WGRAD)
  const float* bias;        // [cout] or nullptr (FWD)
  __nv_bfloat16* y;         // NHWC output (FWD)
  float* dw;                // [cout][9][cin] FP32, accumulated (WGRAD)
  int relu;                 // FWD epilogue ReLU
  int64_t m_total, n_total, k_total;  // GEMM sizes
  int64_t k_split;          // WGRAD: K range per grid.z slice
};

__device__ __forceinline__ uint32_t net_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  // base offset 0, legacy LBO mode, layout type 0 = SWIZZLE_NONE
  return d;
}

// K-major operand in the 128-byte swizzle layout: row r's 64 K elements (128 bytes) at r * 128 with
// its 16-byte chunk c stored at chunk c ^ (r % 8), 8-row atoms 1024 bytes apart (stride-byte
// offset), atom bases 1024-byte aligned; the leading-byte offset (between the two 16-byte chunks
// of one K = 16 step) is one chunk.  A K = 16 step inside the row advances the start address by
// 32 bytes; the tensor core applies the swizzle to the address bits.
__device__ __forceinline__ uint64_t umma_sw128_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;            // leading-byte offset: 16 bytes
  d |= (uint64_t)(1024 >> 4) << 32;  // stride-byte offset: 1024 bytes
  d |= (uint64_t)1 << 46;            // descriptor version for sm_100
  d |= (uint64_t)2 << 61;            // layout type SWIZZLE_128B
  return d;
}

// Byte offset of 16-byte chunk kc of row r in a 128-byte swizzled K-major operand.
__device__ __forceinline__ uint32_t sw128_offset(int r, int kc) { return (uint32_t)(r * 128 + ((kc ^ (r & 7)) << 4)); }

__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
  return (1u << 4)                    // D format FP32
         | (1u << 7)                  // A format BF16
         | (1u << 10)                 // B format BF16
         | ((uint32_t)(n >> 3) << 17) // N / 8
         | ((uint32_t)(m >> 4) << 24);  // M / 16   (A and B K-major: bits 15, 16 = 0)
}

__device__ __forceinline__ void net_mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(net_smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool net_mbar_wait(uint64_t* bar, uint32_t phase) {
  for (uint32_t it = 0; it < NET_WAIT_LIMIT; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(net_smem_u32(bar)), "r"(phase)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ uint4 zero4() { return make_uint4(0u, 0u, 0u, 0u); }

// 8 consecutive k of the im2col row of output pixel m (k = tap * cin + ci, cin % 8 == 0), with the
// pixel's coordinates hoisted out of the K loop: px points at input pixel (b, y, x) of output row
// m (valid = m < m_total).  tap / 3 for tap < 9 is (tap * 11) >> 5.
__device__ __forceinline__ uint4 load_im2col_row(const ConvArgs& a, const __nv_bfloat16* px, int y, int x, bool valid,
                                                 int64_t k) {
  if (!valid || k >= a.k_total) return zero4();
  const int tap = (int)(k >> a.log2_cin);
  const int ci = (int)(k & (int64_t)(a.cin - 1));
  const int ty = (tap * 11) >> 5;
  const int dy = ty - 1, dx = tap - 3 * ty - 1;
  const int ys = y + dy, xs = x + dx;
  if ((unsigned)ys >= (unsigned)a.h || (unsigned)xs >= (unsigned)a.w) return zero4();
  return __ldg(reinterpret_cast<const uint4*>(px + ((int64_t)dy * a.w + dx) * a.cin + ci));
}

__device__ __forceinline__ uint4 pack8(const __nv_bfloat16 v[8]) {
  uint4 r;
  r.x = (uint32_t)__bfloat16_as_ushort(v[0]) | ((uint32_t)__bfloat16_as_ushort(v[1]) << 16);
  r.y = (uint32_t)__bfloat16_as_ushort(v[2]) | ((uint32_t)__bfloat16_as_ushort(v[3]) << 16);
  r.z = (uint32_t)__bfloat16_as_ushort(v[4]) | ((uint32_t)__bfloat16_as_ushort(v[5]) << 16);
  r.w = (uint32_t)__bfloat16_as_ushort(v[6]) | ((uint32_t)__bfloat16_as_ushort(v[7]) << 16);
  return r;
}

// WGRAD GEMM: rows m = (tap, ci) (k_total of the forward), columns n = co, k = pixel.
// A(m, k..k+7) = x[pixel k.. shifted by tap][ci]; B(n, k..k+7) = dy[pixel k..][co].
__device__ __forceinline__ uint4 load_wgrad_a(const ConvArgs& a, int64_t m, int64_t k) {
  const int64_t rows = 9LL * a.cin;
  __nv_bfloat16 v[8];
  const int tap = (int)(m >> a.log2_cin);
  const int ci = (int)(m - ((int64_t)tap << a.log2_cin));
  const int dy_ = tap / 3 - 1, dx_ = tap % 3 - 1;
  const int hw = a.h * a.w;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    v[j] = __ushort_as_bfloat16((unsigned short)0);
    const int64_t p = k + j;
    if (m < rows && p < a.k_total) {
      const int b = (int)(p / hw);
      const int rem = (int)(p - (int64_t)b * hw);
      const int y = rem / a.w, x = rem - (rem / a.w) * a.w;
      const int ys = y + dy_, xs = x + dx_;
      if (ys >= 0 && ys < a.h && xs >= 0 && xs < a.w) v[j] = a.x[(((int64_t)b * a.h + ys) * a.w + xs) * a.cin + ci];
    }
  }
  return pack8(v);
}

__device__ __forceinline__ uint4 load_wgrad_b(const ConvArgs& a, int64_t n, int64_t k) {
  __nv_bfloat16 v[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    v[j] = __ushort_as_bfloat16((unsigned short)0);
    const int64_t p = k + j;
    if (n < a.cout && p < a.k_total) v[j] = a.dy[p * a.cout + n];
  }
  return pack8(v);
}

template <int MODE, int BN>
__global__ void __launch_bounds__(NET_THREADS) conv_umma_kernel(ConvArgs a) {
  constexpr int A_BYTES = NET_BM * NET_BK * 2;
  constexpr int B_BYTES = BN * NET_BK * 2;
  constexpr int TMEM_COLS = BN < 32 ? 32 : BN;
  extern __shared__ __align__(1024) unsigned char net_smem[];
  __shared__ __align__(8) uint64_t mma_bar[2];
  __shared__ uint32_t tmem_base_sh;
  __shared__ int4 rows_sh[NET_BM];  // FWD: (y, x, output pixel or -1) of every tile row

  unsigned char* abuf[2] = {net_smem, net_smem + A_BYTES};
  unsigned char* bbuf[2] = {net_smem + 2 * A_BYTES, net_smem + 2 * A_BYTES + B_BYTES};

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t m0 = (int64_t)blockIdx.x * NET_BM;
  const int64_t n0 = (int64_t)blockIdx.y * BN;
  // forward gather: this thread's output pixel, decomposed once
  const int64_t m_row = m0 + tid;
  const bool row_valid = MODE == NET_FWD && m_row < a.m_total;
  int py = 0, px_ = 0;
  const __nv_bfloat16* prow = a.x;
  if (row_valid) {
    const int hw = a.h * a.w;
    const int b = (int)(m_row / hw);
    const int rem = (int)(m_row - (int64_t)b * hw);
    py = rem / a.w;
    px_ = rem - py * a.w;
    prow = a.x + m_row * a.cin;
  }
  if (MODE == NET_FWD) rows_sh[tid] = make_int4(py, px_, row_valid ? (int)m_row : -1, 0);
  int64_t k_begin = 0, k_end = a.k_total;
  if (MODE == NET_WGRAD) {
    k_begin = (int64_t)blockIdx.z * a.k_split;
    k_end = k_begin + a.k_split < a.k_total ? k_begin + a.k_split : a.k_total;
  }
  const int kblocks = (int)((k_end - k_begin + NET_BK - 1) / NET_BK);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(net_smem_u32(&tmem_base_sh)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    net_mbar_init(&mma_bar[0]);
    net_mbar_init(&mma_bar[1]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem_d = tmem_base_sh;
  constexpr uint32_t IDESC = umma_idesc_bf16(NET_BM, BN);

  // A wait that runs out sets this thread's flag; the flags are combined at the block's barrier
  // (__syncthreads_or), so every thread leaves the loop after the same block.
  bool timed_out = false;
  int committed = 0;  // blocks whose MMAs were issued and committed (uniform across the CTA)
  for (int kb = 0; kb < kblocks; ++kb) {
    const int buf = kb & 1;
    if (kb >= 2) {
      // the MMAs that read this buffer (block kb - 2) must be done before it is overwritten
      if (!net_mbar_wait(&mma_bar[buf], (uint32_t)(((kb - 2) >> 1) & 1))) timed_out = true;
    }
    const int64_t k0 = k_begin + (int64_t)kb * NET_BK;
    if (MODE == NET_FWD) {
      // ---- gather A: 8 lanes per tile row, one 16-byte chunk each, so that a warp's load covers
      // four rows' contiguous K segments; 128-byte swizzled K-major layout
      uint4 v[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int idx = i * NET_THREADS + tid;
        const int r = idx >> 3, kc = idx & 7;
        const int4 ri = rows_sh[r];
        v[i] = load_im2col_row(a, a.x + (int64_t)max(ri.z, 0) * a.cin, ri.x, ri.y, ri.z >= 0, k0 + 8 * kc);
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int idx = i * NET_THREADS + tid;
        *reinterpret_cast<uint4*>(abuf[buf] + sw128_offset(idx >> 3, idx & 7)) = v[i];
      }
      // ---- gather B: BN weight rows x 8 chunks, same layout
      for (int it = tid; it < BN * 8; it += NET_THREADS) {
        const int r = it >> 3, kc = it & 7;
        const int64_t n = n0 + r;
        const int64_t k = k0 + 8 * kc;
        uint4 w = zero4();
        if (n < a.n_total && k < a.k_total) w = __ldg(reinterpret_cast<const uint4*>(a.wt + n * a.k_total + k));
        *reinterpret_cast<uint4*>(bbuf[buf] + sw128_offset(r, kc)) = w;
      }
    } else {
      // ---- gather A: 128 rows x 8 chunks (thread = row), canonical no-swizzle layout
      const int64_t m = m0 + tid;
#pragma unroll
      for (int kc = 0; kc < 8; ++kc) {
        const int64_t k = k0 + 8 * kc;
        const uint4 v = (k < k_end) ? load_wgrad_a(a, m, k) : zero4();
        *reinterpret_cast<uint4*>(abuf[buf] + kc * (NET_BM * 16) + tid * 16) = v;
      }
      // ---- gather B: BN rows x 8 chunks
      for (int it = tid; it < BN * 8; it += NET_THREADS) {
        const int r = it % BN;
        const int kc = it / BN;
        const int64_t n = n0 + r;
        const int64_t k = k0 + 8 * kc;
        const uint4 v = (k < k_end) ? load_wgrad_b(a, n, k) : zero4();
        *reinterpret_cast<uint4*>(bbuf[buf] + kc * (BN * 16) + r * 16) = v;
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (__syncthreads_or(timed_out ? 1 : 0)) {
      timed_out = true;
      break;
    }
    committed = kb + 1;
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a_base = net_smem_u32(abuf[buf]);
      const uint32_t b_base = net_smem_u32(bbuf[buf]);
#pragma unroll
      for (int s = 0; s < NET_BK / 16; ++s) {
        const uint64_t ad = MODE == NET_FWD ? umma_sw128_desc(a_base + 32 * s)
                                            : umma_smem_desc(a_base + 2 * s * NET_BM * 16, NET_BM * 16, 128);
        const uint64_t bd = MODE == NET_FWD ? umma_sw128_desc(b_base + 32 * s)
                                            : umma_smem_desc(b_base + 2 * s * BN * 16, BN * 16, 128);
        const uint32_t acc = (kb > 0 || s > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
            "l"(ad), "l"(bd), "r"(IDESC), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       net_smem_u32(&mma_bar[buf]))
                   : "memory");
    }
  }
  // wait for the last committed block (its commit covers all earlier MMAs of this thread)
  if (committed > 0 && !timed_out) {
    const int last = committed - 1;
    if (!net_mbar_wait(&mma_bar[last & 1], (uint32_t)((last >> 1) & 1))) timed_out = true;
  }
  timed_out = __syncthreads_or(timed_out ? 1 : 0) != 0;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  if (timed_out) {
    if (tid == 0) {
      atomicExch(&g_net_timeout, 1);
      if (committed > 0) {  // one more bounded wait for the MMAs in flight before TMEM is freed
        const int last = committed - 1;
        net_mbar_wait(&mma_bar[last & 1], (uint32_t)((last >> 1) & 1));
      }
    }
  } else if (kblocks > 0) {
    // ---- epilogue: warp w owns rows 32w..32w+31 (TMEM lanes), 8 columns per load
    const int64_t m = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 8) {
      uint32_t r[8];
      const uint32_t taddr = tmem_d + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (MODE == NET_FWD) {
        if (m < a.m_total) {
          __nv_bfloat16 out[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int64_t n = n0 + c0 + j;
            float v = __uint_as_float(r[j]);
            if (a.bias != nullptr && n < a.n_total) v += a.bias[n];
            if (a.relu) v = fmaxf(v, 0.f);
            out[j] = __float2bfloat16_rn(v);
          }
          if (n0 + c0 + 8 <= a.n_total) {
            *reinterpret_cast<uint4*>(a.y + m * a.n_total + n0 + c0) = pack8(out);
          } else {
            for (int j = 0; j < 8; ++j)
              if (n0 + c0 + j < a.n_total) a.y[m * a.n_total + n0 + c0 + j] = out[j];
          }
        }
      } else {
        // dW[co][tap][ci]: row m = (tap, ci), column n = co
        if (m < 9LL * a.cin) {
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int64_t n = n0 + c0 + j;
            if (n < a.cout) atomicAdd(a.dw + n * (9LL * a.cin) + m, __uint_as_float(r[j]));
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_d), "r"(TMEM_COLS) : "memory");
  }
}

template <int MODE, int BN>
static int launch_conv_bn(const ConvArgs& a, cudaStream_t st) {
  // the double-buffered operands; every MMA descriptor addresses inside them (K chunks at
  // LBO = rows * 16 bytes, core matrices at SBO = 128 bytes), so 3-6 CTAs fit per SM, whose TMEM
  // columns (BN, at least 32, each) stay within the SM's 512
  const size_t smem = 2 * (NET_BM * NET_BK * 2) + 2 * (BN * NET_BK * 2);
  if (!ensure_dynamic_smem<conv_umma_kernel<MODE, BN>>((int)smem)) {
    cct_set_last_error("cudaFuncSetAttribute(MaxDynamicSharedMemorySize) failed for the convolution kernel");
    return CCT_ERR_CUDA;
  }
  dim3 grid((unsigned)((a.m_total + NET_BM - 1) / NET_BM), (unsigned)((a.n_total + BN - 1) / BN), 1);
  if (MODE == NET_WGRAD) grid.z = (unsigned)((a.k_total + a.k_split - 1) / a.k_split);
  conv_umma_kernel<MODE, BN><<<grid, NET_THREADS, smem, st>>>(a);
  return CCT_OK;
}

template <int MODE>
static int launch_conv_mode(const ConvArgs& a, int bn, cudaStream_t st) {
  switch (bn) {
    case 16: return launch_conv_bn<MODE, 16>(a, st);
    case 32: return launch_conv_bn<MODE, 32>(a, st);
    case 64: return launch_conv_bn<MODE, 64>(a, st);
    default: return launch_conv_bn<MODE, 128>(a, st);
  }
}

// ----------------------------------------------------------------------------------------------
// Elementwise kernels (NHWC bf16 activations, FP32 parameters / gradients)
// ----------------------------------------------------------------------------------------------
__global__ void relu_bwd_kernel(const __nv_bfloat16* y, const __nv_bfloat16* dy, __nv_bfloat16* dx, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float g = __bfloat162float(y[i]) > 0.f ? __bfloat162float(dy[i]) : 0.f;
    dx[i] = __float2bfloat16_rn(g);
  }
}

// 2x2 average pooling (stride 2) and its adjoint
__global__ void avgpool2_kernel(const __nv_bfloat16* x, __nv_bfloat16* y, int b, int h, int w, int c, int bwd) {
  const int ho = h / 2, wo = w / 2;
  const int64_t n = (int64_t)b * ho * wo * c;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int ch = (int)(i % c);
    int64_t p = i / c;
    const int xo = (int)(p % wo); p /= wo;
    const int yo = (int)(p % ho);
    const int bb = (int)(p / ho);
    const int64_t base = (((int64_t)bb * h + 2 * yo) * w + 2 * xo) * c + ch;
    if (!bwd) {
      const float s = __bfloat162float(x[base]) + __bfloat162float(x[base + c]) +
                      __bfloat162float(x[base + (int64_t)w * c]) + __bfloat162float(x[base + (int64_t)w * c + c]);
      y[i] = __float2bfloat16_rn(0.25f * s);
    } else {
      // x: gradient at the pooled resolution (index i), y: gradient at full resolution
      const __nv_bfloat16 g = __float2bfloat16_rn(0.25f * __bfloat162float(x[i]));
      y[base] = g; y[base + c] = g; y[base + (int64_t)w * c] = g; y[base + (int64_t)w * c + c] = g;
    }
  }
}

// nearest 2x upsampling and its adjoint (sum of the 4 children)
__global__ void upsample2_kernel(const __nv_bfloat16* x, __nv_bfloat16* y, int b, int h, int w, int c, int bwd) {
  // h, w: the small resolution
  const int64_t n = (int64_t)b * h * w * c;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int ch = (int)(i % c);
    int64_t p = i / c;
    const int xs = (int)(p % w); p /= w;
    const int ys = (int)(p % h);
    const int bb = (int)(p / h);
    const int64_t base = (((int64_t)bb * 2 * h + 2 * ys) * 2 * w + 2 * xs) * c + ch;
    const int64_t row = (int64_t)2 * w * c;
    if (!bwd) {
      const __nv_bfloat16 v = x[i];
      y[base] = v; y[base + c] = v; y[base + row] = v; y[base + row + c] = v;
    } else {
      const float s = __bfloat162float(x[base]) + __bfloat162float(x[base + c]) + __bfloat162float(x[base + row]) +
                      __bfloat162float(x[base + row + c]);
      y[i] = __float2bfloat16_rn(s);
    }
  }
}

__global__ void add_kernel(const __nv_bfloat16* a, const __nv_bfloat16* b, __nv_bfloat16* out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16_rn(__bfloat162float(a[i]) + __bfloat162float(b[i]));
}

// db[c] += sum over pixels of dy[p][c]
__global__ void bias_grad_kernel(const __nv_bfloat16* dy, float* db, int64_t pixels, int c) {
  const int ch = blockIdx.y * blockDim.x + threadIdx.x;
  if (ch >= c) return;
  float s = 0.f;
  for (int64_t p = blockIdx.x; p < pixels; p += gridDim.x) s += __bfloat162float(dy[p * c + ch]);
  atomicAdd(db + ch, s);
}

// MSE loss on channel 0 of an NHWC prediction vs an FP32 target [b][h][w]:
// loss += sum (pred - t)^2 / count; grad = 2 (pred - t) / count written to channel 0 (others 0)
__global__ void mse_kernel(const __nv_bfloat16* pred, const float* target, __nv_bfloat16* grad, double* loss,
                           int64_t pixels, int c) {
  double acc = 0.0;
  const float inv = 1.f / (float)pixels;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < pixels; p += (int64_t)gridDim.x * blockDim.x) {
    const float d = __bfloat162float(pred[p * c]) - target[p];
    acc += (double)d * d;
    grad[p * c] = __float2bfloat16_rn(2.f * d * inv);
    for (int ch = 1; ch < c; ++ch) grad[p * c + ch] = __float2bfloat16_rn(0.f);
  }
  acc = warp_sum_double(acc);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc / (double)pixels);
}

// Adam with FP32 master weights; writes the BF16 copy used by the GEMMs
__global__ void adam_kernel(float* p, const float* g, float* m, float* v, __nv_bfloat16* p16, int64_t n, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    if (p16 != nullptr) p16[i] = __float2bfloat16_rn(pi);
  }
}

// weights [co][3][3][ci] -> data-gradient weights [ci][3][3][co] with the taps flipped
__global__ void flip_weights_kernel(const __nv_bfloat16* w, __nv_bfloat16* wf, int cin, int cout) {
  const int64_t n = 9LL * cin * cout;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int co = (int)(i % cout);
    int64_t r = i / cout;
    const int tap = (int)(r % 9);
    const int ci = (int)(r / 9);
    wf[i] = w[((int64_t)co * 9 + (8 - tap)) * cin + ci];
  }
}

// FP32 planar images (channel k of `nch` sources, each [pixels]) -> NHWC bf16 with c channels
// (zero padded), every value divided by the scale of its slice (slices of slice_pixels pixels)
__global__ void pack_nhwc_kernel(const float* const* src, int nch, __nv_bfloat16* dst, int64_t pixels, int c,
                                 const float* slice_scale, int64_t slice_pixels) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < pixels; p += (int64_t)gridDim.x * blockDim.x) {
    const float inv = slice_scale != nullptr ? 1.f / slice_scale[p / slice_pixels] : 1.f;
    for (int ch = 0; ch < c; ++ch) {
      const float v = ch < nch ? src[ch][p] * inv : 0.f;
      dst[p * c + ch] = __float2bfloat16_rn(v);
    }
  }
}

// channel 0 of NHWC bf16 -> FP32 planar.  mode 0: out = max(base + scale_s * v, floor);
// mode 1 (multiplicative): out = max((base + scale_s * floor) * exp(v) - scale_s * floor, floor)
__global__ void unpack_c0_kernel(const __nv_bfloat16* src, int c, const float* base, const float* slice_scale,
                                 int64_t slice_pixels, int mode, float floor_v, float* out, int64_t pixels) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < pixels; p += (int64_t)gridDim.x * blockDim.x) {
    const float sc = slice_scale != nullptr ? slice_scale[p / slice_pixels] : 1.f;
    const float v = __bfloat162float(src[p * c]);
    const float b = base != nullptr ? base[p] : 0.f;
    float r;
    if (mode == 1) {
      const float off = sc * floor_v;
      r = (b + off) * expf(v) - off;
    } else {
      r = b + sc * v;
    }
    out[p] = fmaxf(r, floor_v);
  }
}

// out[i] = a[i] / b[i % b_count] (b broadcast over slices)
__global__ void ratio_kernel(const float* a, const float* b, float* out, int64_t n, int64_t b_count) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = a[i] / b[i % b_count];
}

static inline unsigned ew_blocks(int64_t n) {
  int64_t b = (n + 255) / 256;
  if (b > 4096) b = 4096;
  return (unsigned)(b < 1 ? 1 : b);
}

int read_net_timeout(int clear, int* value) {
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_net_timeout, sizeof(int));
  if (e != cudaSuccess) return (int)e;
  if (clear) {
    const int zero = 0;
    e = cudaMemcpyToSymbol(g_net_timeout, &zero, sizeof(int));
    if (e != cudaSuccess) return (int)e;
  }
  *value = v;
  return 0;
}

}  // namespace cct

// ------------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------------
static int net_check_conv(const cct_conv_desc* d) {
  CCT_REQUIRE(d != nullptr, "conv descriptor is NULL");
  CCT_REQUIRE(d->batch >= 1 && d->height >= 1 && d->width >= 1, "batch, height and width must be >= 1");
  CCT_REQUIRE(d->cin >= 16 && d->cin <= 512 && (d->cin & (d->cin - 1)) == 0, "cin must be a power of two in [16, 512]");
  CCT_REQUIRE(d->cout >= 16 && d->cout <= 512 && d->cout % 16 == 0, "cout must be a multiple of 16 in [16, 512]");
  return CCT_OK;
}

static cct::ConvArgs net_args(const cct_conv_desc* d) {
  cct::ConvArgs a;
  std::memset(&a, 0, sizeof(a));
  a.batch = d->batch; a.h = d->height; a.w = d->width; a.cin = d->cin; a.cout = d->cout;
  int l = 0;
  while ((1 << l) < d->cin) ++l;
  a.log2_cin = l;
  return a;
}

// the implicit-GEMM loads move 8 bf16 (16 bytes) at a time
static bool net_aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

static int net_bn(int cout) { return cout >= 128 ? 128 : cout; }

static int net_launch_check() {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    cct_set_last_error(cudaGetErrorString(e));
    return CCT_ERR_CUDA;
  }
  return CCT_OK;
}

extern "C" {

int cct_conv3x3_fwd(const cct_conv_desc* desc, const void* x, const void* w, const float* bias, int32_t relu,
                    void* y, void* stream) {
  int rc = net_check_conv(desc);
  if (rc != CCT_OK) return rc;
  CCT_REQUIRE(x != nullptr && w != nullptr && y != nullptr, "x, w and y are required");
  CCT_REQUIRE(net_aligned16(x) && net_aligned16(w) && net_aligned16(y), "x, w and y must be 16-byte aligned");
  cct::ConvArgs a = net_args(desc);
  a.x = reinterpret_cast<const __nv_bfloat16*>(x);
  a.wt = reinterpret_cast<const __nv_bfloat16*>(w);
  a.bias = bias;
  a.y = reinterpret_cast<__nv_bfloat16*>(y);
  a.relu = relu;
  a.m_total = (int64_t)desc->batch * desc->height * desc->width;
  a.n_total = desc->cout;
  a.k_total = 9LL * desc->cin;
  rc = cct::launch_conv_mode<cct::NET_FWD>(a, net_bn(desc->cout), reinterpret_cast<cudaStream_t>(stream));
  if (rc != CCT_OK) return rc;
  return net_launch_check();
}

int cct_conv3x3_wgrad(const cct_conv_desc* desc, const void* x, const void* dy, float* dw, void* stream) {
  int rc = net_check_conv(desc);
  if (rc != CCT_OK) return rc;
  CCT_REQUIRE(x != nullptr && dy != nullptr && dw != nullptr, "x, dy and dw are required");
  CCT_REQUIRE(net_aligned16(x) && net_aligned16(dy), "x and dy must be 16-byte aligned");
  cct::ConvArgs a = net_args(desc);
  a.x = reinterpret_cast<const __nv_bfloat16*>(x);
  a.dy = reinterpret_cast<const __nv_bfloat16*>(dy);
  a.dw = dw;
  a.m_total = 9LL * desc->cin;
  a.n_total = desc->cout;
  a.k_total = (int64_t)desc->batch * desc->height * desc->width;
  // split K (pixels) so that the grid has a few hundred CTAs
  const int64_t tiles = ((a.m_total + 127) / 128) * ((a.n_total + 127) / 128);
  int64_t splits = (512 + tiles - 1) / tiles;
  int64_t ks = (a.k_total + splits - 1) / splits;
  ks = ((ks + 63) / 64) * 64;
  if (ks < 64) ks = 64;
  a.k_split = ks;
  rc = cct::launch_conv_mode<cct::NET_WGRAD>(a, net_bn(desc->cout), reinterpret_cast<cudaStream_t>(stream));
  if (rc != CCT_OK) return rc;
  return net_launch_check();
}

int cct_net_flip_weights(const void* w, void* w_flipped, int32_t cin, int32_t cout, void* stream) {
  CCT_REQUIRE(w != nullptr && w_flipped != nullptr && cin > 0 && cout > 0, "bad flip_weights arguments");
  const int64_t n = 9LL * cin * cout;
  cct::flip_weights_kernel<<<cct::ew_blocks(n), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const __nv_bfloat16*>(w), reinterpret_cast<__nv_bfloat16*>(w_flipped), cin, cout);
  return net_launch_check();
}

int cct_net_relu_bwd(const void* y, const void* dy, void* dx, int64_t count, void* stream) {
  CCT_REQUIRE(y && dy && dx && count > 0, "bad relu_bwd arguments");
  cct::relu_bwd_kernel<<<cct::ew_blocks(count), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const __nv_bfloat16*>(y), reinterpret_cast<const __nv_bfloat16*>(dy),
      reinterpret_cast<__nv_bfloat16*>(dx), count);
  return net_launch_check();
}

int cct_net_avgpool2(const void* x, void* y, int32_t batch, int32_t height, int32_t width, int32_t channels,
                     int32_t backward, void* stream) {
  CCT_REQUIRE(x && y && batch > 0 && height % 2 == 0 && width % 2 == 0 && channels > 0, "bad avgpool2 arguments");
  const int64_t n = (int64_t)batch * (height / 2) * (width / 2) * channels;
  cct::avgpool2_kernel<<<cct::ew_blocks(n), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const __nv_bfloat16*>(x), reinterpret_cast<__nv_bfloat16*>(y), batch, height, width, channels,
      backward);
  return net_launch_check();
}

int cct_net_upsample2(const void* x, void* y, int32_t batch, int32_t height, int32_t width, int32_t channels,
                      int32_t backward, void* stream) {
  CCT_REQUIRE(x && y && batch > 0 && height > 0 && width > 0 && channels > 0, "bad upsample2 arguments");
  const int64_t n = (int64_t)batch * height * width * channels;
  cct::upsample2_kernel<<<cct::ew_blocks(n), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const __nv_bfloat16*>(x), reinterpret_cast<__nv_bfloat16*>(y), batch, height, width, channels,
      backward);
  return net_launch_check();
}

int cct_net_add(const void* a, const void* b, void* out, int64_t count, void* stream) {
  CCT_REQUIRE(a && b && out && count > 0, "bad add arguments");
  cct::add_kernel<<<cct::ew_blocks(count), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const __nv_bfloat16*>(a), reinterpret_cast<const __nv_bfloat16*>(b),
      reinterpret_cast<__nv_bfloat16*>(out), count);
  return net_launch_check();
}

int cct_net_bias_grad(const void* dy, float* db, int64_t pixels, int32_t channels, void* stream) {
  CCT_REQUIRE(dy && db && pixels > 0 && channels > 0, "bad bias_grad arguments");
  dim3 grid((unsigned)(pixels < 1024 ? pixels : 1024), (unsigned)((channels + 127) / 128));
  cct::bias_grad_kernel<<<grid, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const __nv_bfloat16*>(dy), db, pixels, channels);
  return net_launch_check();
}

int cct_net_mse(const void* pred, const float* target, void* grad, double* loss, int64_t pixels, int32_t channels,
                void* stream) {
  CCT_REQUIRE(pred && target && grad && loss && pixels > 0 && channels > 0, "bad mse arguments");
  cct::mse_kernel<<<cct::ew_blocks(pixels), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const __nv_bfloat16*>(pred), target, reinterpret_cast<__nv_bfloat16*>(grad), loss, pixels,
      channels);
  return net_launch_check();
}

int cct_net_adam(float* p, const float* g, float* m, float* v, void* p_bf16, int64_t count, float lr, float beta1,
                 float beta2, float eps, int32_t step, void* stream) {
  CCT_REQUIRE(p && g && m && v && count > 0 && step >= 1, "bad adam arguments");
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  cct::adam_kernel<<<cct::ew_blocks(count), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      p, g, m, v, reinterpret_cast<__nv_bfloat16*>(p_bf16), count, lr, beta1, beta2, eps, c1, c2);
  return net_launch_check();
}

int cct_net_pack_nhwc(const float* const* src, int32_t n_src, void* dst, int64_t pixels, int32_t channels,
                      const float* slice_scale, int64_t slice_pixels, void* stream) {
  CCT_REQUIRE(src && dst && n_src >= 1 && n_src <= channels && pixels > 0, "bad pack_nhwc arguments");
  CCT_REQUIRE(slice_scale == nullptr || (slice_pixels > 0 && pixels % slice_pixels == 0), "bad slice_pixels");
  cct::pack_nhwc_kernel<<<cct::ew_blocks(pixels), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      src, n_src, reinterpret_cast<__nv_bfloat16*>(dst), pixels, channels, slice_scale, slice_pixels);
  return net_launch_check();
}

int cct_net_unpack_c0(const void* src, int32_t channels, const float* base, const float* slice_scale,
                      int64_t slice_pixels, int32_t mode, float floor_value, float* out, int64_t pixels, void* stream) {
  CCT_REQUIRE(src && out && pixels > 0 && channels > 0 && (mode == 0 || mode == 1), "bad unpack_c0 arguments");
  CCT_REQUIRE(slice_scale == nullptr || (slice_pixels > 0 && pixels % slice_pixels == 0), "bad slice_pixels");
  cct::unpack_c0_kernel<<<cct::ew_blocks(pixels), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const __nv_bfloat16*>(src), channels, base, slice_scale, slice_pixels, mode, floor_value, out,
      pixels);
  return net_launch_check();
}

int cct_net_ratio(const float* a, const float* b, float* out, int64_t count, int64_t b_count, void* stream) {
  CCT_REQUIRE(a && b && out && count > 0 && b_count > 0 && count % b_count == 0, "bad ratio arguments");
  cct::ratio_kernel<<<cct::ew_blocks(count), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(a, b, out, count, b_count);
  return net_launch_check();
}

int cct_net_timeout(int32_t clear, int32_t* value) {
  CCT_REQUIRE(value != nullptr, "value is required");
  int v = 0;
  const int e = cct::read_net_timeout(clear, &v);
  if (e != 0) {
    cct_set_last_error(cudaGetErrorString((cudaError_t)e));
    return CCT_ERR_CUDA;
  }
  *value = v;
  return CCT_OK;
}

}  // extern "C"
