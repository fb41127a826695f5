// Forward and back projection kernels of the XRF path (sm_100a).
//
// Forward projection (scikit-image radon discretisation, corrct:
// src/corrct/_projector_backends.py:312-333, attenuated form projectors.py:502-531):
//   sino[s][d][a][c] = w[a][d] * sum_r bilin(vol[s] * maps[s][a][d], M_a (c, r))
// One CTA owns (slice, angle, detector, band of 64 detector bins) and walks the
// column band in chunks of 64 rows.  For each chunk the bounding box of the
// rotated chunk is staged in shared memory as z = vol * map (coalesced float4
// loads of both, zero outside the image, odd row stride so lanes on different
// rows hit different banks), then each thread samples 16 rows of one column
// from shared memory.  Column sums stay in registers; the CTA writes final
// values, so the result is deterministic and needs no atomics or partial sums.
// The map of every angle is read from HBM once; the volume is L2-resident.
//
// Back projection (scikit-image iradon, filter None, corrct:
// src/corrct/_projector_backends.py:335-359): one CTA owns a 32x32 pixel tile and
// loops over all (detector, angle) lines in chunks of 32; each chunk stages, per
// line, the <= 48 detector bins the tile can reach as (value, slope) pairs, and
// every pixel does one shared-memory lookup and one FMA per line.  np.interp's
// left=0 / right=0 edges are discontinuous, so lines whose range comes within
// 0.01 bin of an edge take a checked path that decides edge cases in double
// precision exactly as numpy does.

#include <cstring>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "cct_common.cuh"
#include "cct_internal.cuh"

namespace cct {

// Raised (never trapped) if a staged box would exceed its shared-memory bound; valid
// rotation matrices cannot reach it.  Read through cct_device_error().
__device__ int g_box_overflow = 0;

// ------------------------------------------------------------------------------------------
// Forward projection
// ------------------------------------------------------------------------------------------
constexpr int FP_TC = 64;                          // detector bins per CTA
constexpr int FP_TR = 64;                          // rows per staged chunk
constexpr int FP_THREADS = 256;
// Lanes of a warp cover an 8 (columns) x 4 (rows) block of samples: 32 points of a rotated
// lattice patch spread over ~2 wavefronts per shared load at any angle, where a 32 x 1 line
// of lanes hits 32-way bank conflicts at some angles.  Warp w owns columns 8w..8w+7.
constexpr int FP_LC = 8;
constexpr int FP_LR = 4;
constexpr int FP_RPT = FP_TR / FP_LR;              // 16 samples per thread per chunk
// Rotated 64x64 chunk: extent <= 63*sqrt(2) = 89.1, +1/+2 tap margins, +3 for float4
// alignment of the left edge, rounded up to a multiple of 4.
constexpr int FP_BOX_W = 100;
constexpr int FP_BOX_H = 96;
constexpr int FP_STRIDE = FP_BOX_W;                // 16-byte rows: conflict-free float4 fills
constexpr int FP_MAX_CHUNKS = (8192 + FP_TR - 1) / FP_TR;  // row chunks of the largest n
constexpr float FP_SLAB_EPS = 0.01f;               // slab widening of a box row (y)
constexpr float FP_ROW_MARGIN = 0.5f;              // column range widening (x)
static_assert(FP_MAX_CHUNKS <= FP_THREADS, "one thread per chunk box");
constexpr int FP_FILL_BATCH = 3;                   // float4 items whose loads are issued together

template <bool HAS_MAPS, int MAPS_DTYPE>
__device__ __forceinline__ float4 fp_load_item(const float* vol, const MapRef& mref, int n, int gy, int gx, bool vec4) {
  float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
  if (gy < 0 || gy >= n || gx + 3 < 0 || gx >= n) return v;
  const int off = gy * n + gx;  // < 2^31 for n <= 8192... n*n <= 2^26
  if (vec4 && gx >= 0 && gx + 3 < n) {
    v = __ldg(reinterpret_cast<const float4*>(vol + off));
    if (HAS_MAPS) {
      const float4 mv = map_at4<MAPS_DTYPE>(mref, off);
      v.x *= mv.x; v.y *= mv.y; v.z *= mv.z; v.w *= mv.w;
    }
    return v;
  }
  float e[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int xx = gx + k;
    float val = 0.f;
    if (xx >= 0 && xx < n) {
      val = __ldg(vol + off + k);
      if (HAS_MAPS) val *= map_at<MAPS_DTYPE>(mref, off + k);
    }
    e[k] = val;
  }
  return make_float4(e[0], e[1], e[2], e[3]);
}

// Bounding box of the sample positions of columns [c0, c_last] x rows [r0, r_last] (the corners
// of a rotated rectangle), widened by the bilinear taps; x origin floored to a multiple of 4.
__device__ __forceinline__ void chunk_box(float m00, float m01, float m02, float m10, float m11, float m12, int c0,
                                          int c_last, int r0, int r_last, int& bx0, int& bx1, int& by0, int& by1) {
  const float fc0 = (float)c0, fc1 = (float)c_last, fr0 = (float)r0, fr1 = (float)r_last;
  const float xa = sample_x(m00, m01, m02, fc0, fr0), xb = sample_x(m00, m01, m02, fc1, fr0);
  const float xc = sample_x(m00, m01, m02, fc0, fr1), xd = sample_x(m00, m01, m02, fc1, fr1);
  const float ya = sample_x(m10, m11, m12, fc0, fr0), yb = sample_x(m10, m11, m12, fc1, fr0);
  const float yc = sample_x(m10, m11, m12, fc0, fr1), yd = sample_x(m10, m11, m12, fc1, fr1);
  const float xmin = fminf(fminf(xa, xb), fminf(xc, xd)), xmax = fmaxf(fmaxf(xa, xb), fmaxf(xc, xd));
  const float ymin = fminf(fminf(ya, yb), fminf(yc, yd)), ymax = fmaxf(fmaxf(ya, yb), fmaxf(yc, yd));
  bx0 = ((int)floorf(xmin) - 1) & ~3;  // floor to a multiple of 4 (two's complement)
  bx1 = (int)floorf(xmax) + 2;
  by0 = (int)floorf(ymin) - 1;
  by1 = (int)floorf(ymax) + 2;
}

// Quads (4-column groups counted from the box origin bx0) of box row y that the bilinear taps
// of a chunk can read.  Samples whose floor(py) is y - 1 or y lie in the slab y - 1 <= py < y + 1;
// their x over the chunk's parallelogram (corners (px[k], py[k]) in cyclic order, the positions
// of the corner samples) is the range of its edges clipped to the slab, widened by
// FP_ROW_MARGIN against rounding (the approximate division moves it by far less) and by the
// right tap.  Returns (first, last) clipped to [0, q4 - 1]; first > last when no tap reads it.
__device__ __forceinline__ short2 fp_row_quads(const float (&px)[4], const float (&py)[4], int y, int bx0, int q4) {
  const float ylo = (float)y - 1.f - FP_SLAB_EPS, yhi = (float)y + 1.f + FP_SLAB_EPS;
  float xmin = 3.0e38f, xmax = -3.0e38f;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const float xa = px[e], ya = py[e], xb = px[(e + 1) & 3], yb = py[(e + 1) & 3];
    float t0 = 0.f, t1 = 1.f;
    const float dy = yb - ya;
    if (fabsf(dy) < 1e-6f) {
      if (ya < ylo || ya > yhi) continue;
    } else {
      float ta = __fdividef(ylo - ya, dy), tb = __fdividef(yhi - ya, dy);
      if (ta > tb) { const float t = ta; ta = tb; tb = t; }
      t0 = fmaxf(ta, 0.f);
      t1 = fminf(tb, 1.f);
      if (t0 > t1) continue;
    }
    const float x0 = fmaf(t0, xb - xa, xa), x1 = fmaf(t1, xb - xa, xa);
    xmin = fminf(xmin, fminf(x0, x1));
    xmax = fmaxf(xmax, fmaxf(x0, x1));
  }
  if (xmin > xmax) return make_short2(1, 0);
  const int lo = (int)floorf(xmin - FP_ROW_MARGIN) - bx0;
  const int hi = (int)floorf(xmax + FP_ROW_MARGIN) + 1 - bx0;
  return make_short2((short)(max(lo, 0) >> 2), (short)min(hi >> 2, q4 - 1));
}

// Positions of the four corner samples of chunk columns [c0, c1] x rows [r0, r1], cyclic order.
__device__ __forceinline__ void chunk_corners(float m00, float m01, float m02, float m10, float m11, float m12, int c0,
                                              int c1, int r0, int r1, float (&px)[4], float (&py)[4]) {
  const float fc0 = (float)c0, fc1 = (float)c1, fr0 = (float)r0, fr1 = (float)r1;
  px[0] = sample_x(m00, m01, m02, fc0, fr0); py[0] = sample_x(m10, m11, m12, fc0, fr0);
  px[1] = sample_x(m00, m01, m02, fc1, fr0); py[1] = sample_x(m10, m11, m12, fc1, fr0);
  px[2] = sample_x(m00, m01, m02, fc1, fr1); py[2] = sample_x(m10, m11, m12, fc1, fr1);
  px[3] = sample_x(m00, m01, m02, fc0, fr1); py[3] = sample_x(m10, m11, m12, fc0, fr1);
}

// CTA sum of one residual partial per thread (FP64, fixed order) into partials[slot]; red
// holds one double per warp.  Every thread of the CTA calls it.
__device__ __forceinline__ void fp_write_partial(double v, double* partials, int64_t slot, double* red, int lane,
                                                 int warp, int tid) {
  v = warp_sum_double(v);
  __syncthreads();  // red may still be read by a previous call
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < FP_TC / FP_LC; ++w) t += red[w];
    partials[slot] = t;
  }
}

// One CTA of the forward projection: detector band `band` of (angle, detector) `ad` of slice
// `s`; `n_bands` and `n_ad` are the batch's band and (angle, detector) counts (the residual
// partials are indexed by them).
template <int EPI, bool HAS_MAPS, int MAPS_DTYPE>
__device__ __forceinline__ void fp_cta(const FpArgs& args, const int band, const int ad, const int s, const int n_bands,
                                       const int n_ad) {
  __shared__ __align__(16) float z[FP_BOX_H * FP_STRIDE];
  __shared__ double red_d[FP_TC / FP_LC];
  __shared__ int4 box_sh[FP_MAX_CHUNKS];  // every chunk's box, computed once per CTA

  const int n = args.n;
  if (args.active != nullptr && args.active[s] == 0) return;
  const int a = ad / args.n_det;
  const int d = ad - a * args.n_det;

  const float* M = args.fp_matrix + 6 * a;
  const float m00 = M[0], m01 = M[1], m02 = M[2], m10 = M[3], m11 = M[4], m12 = M[5];

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int lc = lane & (FP_LC - 1);
  const int lr = lane / FP_LC;
  const int c0 = band * FP_TC;
  const int c = c0 + warp * FP_LC + lc;
  const int c_last = min(c0 + FP_TC, n) - 1;

  const float* vol = args.vol + (int64_t)s * n * n;
  const MapRef mref = make_map_ref(args.maps, MAPS_DTYPE, args.maps_slice_stride, args.n_angles, args.n_det, n, s, a,
                                   d, args.n_channels, args.chan_scale);
  const bool vec4 = args.vec4 != 0;
  const float fc = (float)c;
  const float pxc = fmaf(m00, fc, m02);
  const float pyc = fmaf(m10, fc, m12);

  // thread t computes the box of row chunk t (n <= 8192: at most FP_MAX_CHUNKS chunks)
  if (tid * FP_TR < n) {
    int4 b;
    chunk_box(m00, m01, m02, m10, m11, m12, c0, c_last, tid * FP_TR, min((tid + 1) * FP_TR, n) - 1, b.x, b.y, b.z,
              b.w);
    box_sh[tid] = b;
  }
  __syncthreads();

  float acc = 0.f;
  for (int r0 = 0; r0 < n; r0 += FP_TR) {
    const int r_last = min(r0 + FP_TR, n) - 1;
    const int4 box = box_sh[r0 / FP_TR];
    const int bx0 = box.x, bx1 = box.y, by0 = box.z, by1 = box.w;
    const int q4 = (bx1 - bx0) / 4 + 1;  // float4 columns
    const int bh = by1 - by0 + 1;
    if (4 * q4 > FP_BOX_W || bh > FP_BOX_H) {  // cannot happen for valid matrices; never trap
      if (tid == 0) atomicExch(&g_box_overflow, 1);
      return;
    }

    // Stage z = vol * map over the box (zeros outside the image); every thread takes items
    // tid, tid + 256, ... of the q4 x bh grid, issuing FP_FILL_BATCH items' loads at once.
    const int items = q4 * bh;
    // it / q4 = (it * ceil(2^20 / q4)) >> 20, exact for it < 2^12 and q4 <= 25 (the error
    // it * (magic - 2^20 / q4) / 2^20 < 2^-8 stays below 1 / q4), and the product fits 32 bits
    const unsigned magic = (1048576u + (unsigned)q4 - 1u) / (unsigned)q4;
    for (int base = tid; base < items; base += FP_THREADS * FP_FILL_BATCH) {
      float4 v[FP_FILL_BATCH];
      int dst[FP_FILL_BATCH];
#pragma unroll
      for (int k = 0; k < FP_FILL_BATCH; ++k) {
        const int it = base + k * FP_THREADS;
        dst[k] = -1;
        v[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (it < items) {
          const int rr = (int)(((unsigned)it * magic) >> 20);
          const int qq = it - rr * q4;
          const int gy = by0 + rr, gx = bx0 + 4 * qq;
          dst[k] = rr * FP_STRIDE + 4 * qq;
          if (vec4) {
            // n % 4 == 0 and gx % 4 == 0: a float4 is either fully inside or fully outside
            if ((unsigned)gy < (unsigned)n && (unsigned)gx < (unsigned)n) {
              const int off = gy * n + gx;
              v[k] = __ldg(reinterpret_cast<const float4*>(vol + off));
              if (HAS_MAPS) {
                const float4 mv = map_at4<MAPS_DTYPE>(mref, off);
                v[k].x *= mv.x; v[k].y *= mv.y; v[k].z *= mv.z; v[k].w *= mv.w;
              }
            }
          } else {
            v[k] = fp_load_item<HAS_MAPS, MAPS_DTYPE>(vol, mref, n, gy, gx, false);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < FP_FILL_BATCH; ++k) {
        if (dst[k] >= 0) *reinterpret_cast<float4*>(z + dst[k]) = v[k];
      }
    }
    __syncthreads();

    if (c <= c_last) {
      // Sample positions use exactly sample_x()'s expression so that the adjoint kernel (and
      // the box corners) see bit-identical coordinates.  Taps index the __shared__ array with
      // 32-bit offsets (zoff moves the box origin to (by0, bx0)).
      const int zoff = -by0 * FP_STRIDE - bx0;
      float fr = (float)(r0 + lr);
      const int rem = r_last - r0 - lr;                      // rows of this thread left in the chunk
      const int kmax = rem >= 0 ? rem / FP_LR + 1 : 0;       // samples of this thread in the chunk
      if (kmax >= FP_RPT) {
        // two samples (rows r and r + FP_LR) per packed FP32x2 instruction, with the roundings
        // of the scalar loop below
        const float2 mx = make_float2(m01, m01), my = make_float2(m11, m11);
        const float2 cx = make_float2(pxc, pxc), cy = make_float2(pyc, pyc);
        const float2 step2 = make_float2(2.f * FP_LR, 2.f * FP_LR);
        float2 fr2 = make_float2(fr, fr + (float)FP_LR);
#pragma unroll 4
        for (int k = 0; k < FP_RPT; k += 2) {
          acc = bilerp2<FP_STRIDE>(z, zoff, __ffma2_rn(mx, fr2, cx), __ffma2_rn(my, fr2, cy), acc);
          fr2 = __fadd2_rn(fr2, step2);
        }
      } else {
        for (int k = 0; k < kmax; ++k) {
          const FloorSplit fx = floor_split(fmaf(m01, fr, pxc));
          const FloorSplit fy = floor_split(fmaf(m11, fr, pyc));
          const int q = fy.i * FP_STRIDE + fx.i + zoff;
          const float t0 = z[q], t1 = z[q + 1], b0 = z[q + FP_STRIDE], b1 = z[q + FP_STRIDE + 1];
          const float top = fmaf(fx.f, t1 - t0, t0);
          const float bot = fmaf(fx.f, b1 - b0, b0);
          acc += fmaf(fy.f, bot - top, top);
          fr += (float)FP_LR;
        }
      }
    }
    __syncthreads();
  }

  // column sum over the 4 row-lanes of the 8x4 lane block (lanes lc, lc+8, lc+16, lc+24)
  acc += __shfl_xor_sync(0xffffffffu, acc, 8);
  acc += __shfl_xor_sync(0xffffffffu, acc, 16);
  double part = 0.0, ptest = 0.0;
  if (lr == 0 && c <= c_last) {
    float total = acc;
    if (args.weights != nullptr) total *= args.weights[a * args.n_det + d];
    const int64_t idx = (((int64_t)s * args.n_det + d) * args.n_angles + a) * n + c;
    part = fp_epilogue<EPI>(args, idx, total, &ptest);
  }
  // only the MLEM and SIRT epilogues produce residual partials (PDHG passes none)
  if (EPI == FP_EPI_MLEM || EPI == FP_EPI_SIRT) {
    const int64_t slot = (int64_t)s * n_bands * n_ad + (int64_t)ad * n_bands + band;
    fp_write_partial(part, args.partials, slot, red_d, lane, warp, tid);
    if (args.partials_test != nullptr) fp_write_partial(ptest, args.partials_test, slot, red_d, lane, warp, tid);
  }
}

template <int EPI, bool HAS_MAPS, int MAPS_DTYPE>
__global__ void __launch_bounds__(FP_THREADS, 5) fp_kernel(FpArgs args) {
  fp_cta<EPI, HAS_MAPS, MAPS_DTYPE>(args, blockIdx.x, blockIdx.y, blockIdx.z, gridDim.x, gridDim.y);
}

// Line-integral fields: the channels of a field slice read the same two planes per angle, so
// they run as neighbouring CTAs (grid x = band * C + channel, z = field slice) and all but the
// first find the planes in L2.  Same per-CTA work as fp_kernel.
template <int EPI>
__global__ void __launch_bounds__(FP_THREADS, 5) fp_fields_kernel(FpArgs args) {
  const int C = args.n_channels;
  const int band = blockIdx.x / C;
  const int ch = blockIdx.x - band * C;
  fp_cta<EPI, true, CCT_DTYPE_FIELDS_F32>(args, band, blockIdx.y, blockIdx.z * C + ch, gridDim.x / C, gridDim.y);
}

// Group g of a ragged launch owns CTAs [start[g], start[g + 1]); binary search over the groups.
__device__ __forceinline__ int ragged_group(const int64_t* __restrict__ start, int n_groups, int64_t cta) {
  int lo = 0, hi = n_groups - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(start + mid) <= cta) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Forward projection over groups of slices with different sizes, angle counts and buffers, in
// one launch: group g's CTAs are (band, angle * detector, slice) in band-fastest order.
template <int EPI, bool HAS_MAPS, int MAPS_DTYPE>
__global__ void __launch_bounds__(FP_THREADS, 5) fp_ragged_kernel(const FpArgs* __restrict__ groups,
                                                                  const int64_t* __restrict__ start, int n_groups) {
  const int64_t cta = blockIdx.x;
  const int g = ragged_group(start, n_groups, cta);
  const FpArgs& a = groups[g];
  const int n_bands = (a.n + FP_TC - 1) / FP_TC;
  const int n_ad = a.n_angles * a.n_det;
  const int64_t local = cta - start[g];
  const int band = (int)(local % n_bands);
  const int64_t rest = local / n_bands;
  const int ad = (int)(rest % n_ad);
  const int sl = (int)(rest / n_ad);
  fp_cta<EPI, HAS_MAPS, MAPS_DTYPE>(a, band, ad, sl, n_bands, n_ad);
}

// ------------------------------------------------------------------------------------------
// Forward projection, TMA-staged variant (n % 8 == 0)
//
// The chunk's x box and map box (fixed 96 x 104 boxes, zero-filled outside the image) arrive
// through two cp.async.bulk.tensor loads on one mbarrier; one vectorised pass multiplies them
// in place (z = x * map), then the same 8x4-lane sampling as fp_kernel runs on row stride 104.
// No load instruction per element, and the copy overlaps the other resident CTA's sampling.
// The left box edge is a multiple of 8 elements (16 bytes for BF16 maps too), as TMA needs.
// ------------------------------------------------------------------------------------------
constexpr int FPT_BOX_W = 104;
constexpr int FPT_BOX_H = 96;
constexpr int FPT_Q4 = FPT_BOX_W / 4;              // float4 per box row
constexpr uint32_t FPT_WAIT_LIMIT = 1u << 22;      // bounded mbarrier polling (never spins forever)

__device__ int g_tma_timeout = 0;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase) {
  for (uint32_t it = 0; it < FPT_WAIT_LIMIT; ++it) {
    if (mbar_try_wait(bar, phase)) return true;
  }
  return false;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

template <int EPI, bool HAS_MAPS, int MAPS_DTYPE>
__global__ void __launch_bounds__(FP_THREADS, 2)
    fp_tma_kernel(FpArgs args, const __grid_constant__ CUtensorMap tm_vol, const __grid_constant__ CUtensorMap tm_maps) {
  extern __shared__ __align__(128) unsigned char fpt_smem[];
  float* zb = reinterpret_cast<float*>(fpt_smem);                                  // [96][104] x, then z
  unsigned char* mraw = fpt_smem + FPT_BOX_H * FPT_BOX_W * sizeof(float);         // [96][104] map
  __shared__ __align__(8) uint64_t bar;
  __shared__ double red_d[FP_TC / FP_LC];
  __shared__ int timed_out;

  const int n = args.n;
  const int band = blockIdx.x;
  const int ad = blockIdx.y;
  const int s = blockIdx.z;
  if (args.active != nullptr && args.active[s] == 0) return;
  const int a = ad / args.n_det;
  const int d = ad - a * args.n_det;

  const float* M = args.fp_matrix + 6 * a;
  const float m00 = M[0], m01 = M[1], m02 = M[2], m10 = M[3], m11 = M[4], m12 = M[5];

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int lc = lane & (FP_LC - 1);
  const int lr = lane / FP_LC;
  const int c0 = band * FP_TC;
  const int c = c0 + warp * FP_LC + lc;
  const int c_last = min(c0 + FP_TC, n) - 1;
  const int map_img = (s * args.n_angles + a) * args.n_det + d;
  const uint32_t box_bytes = FPT_BOX_H * FPT_BOX_W * sizeof(float) +
                             (HAS_MAPS ? FPT_BOX_H * FPT_BOX_W * (MAPS_DTYPE == CCT_DTYPE_BF16 ? 2 : 4) : 0);
  const float fc = (float)c;
  const float pxc = fmaf(m00, fc, m02);
  const float pyc = fmaf(m10, fc, m12);

  if (tid == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    timed_out = 0;
  }
  __syncthreads();

  uint32_t phase = 0;
  float acc = 0.f;
  for (int r0 = 0; r0 < n; r0 += FP_TR) {
    const int r_last = min(r0 + FP_TR, n) - 1;
    const float fc0 = (float)c0, fc1 = (float)c_last, fr0 = (float)r0, fr1 = (float)r_last;
    const float xa = sample_x(m00, m01, m02, fc0, fr0), xb = sample_x(m00, m01, m02, fc1, fr0);
    const float xc = sample_x(m00, m01, m02, fc0, fr1), xd = sample_x(m00, m01, m02, fc1, fr1);
    const float ya = sample_x(m10, m11, m12, fc0, fr0), yb = sample_x(m10, m11, m12, fc1, fr0);
    const float yc = sample_x(m10, m11, m12, fc0, fr1), yd = sample_x(m10, m11, m12, fc1, fr1);
    const float xmin = fminf(fminf(xa, xb), fminf(xc, xd)), xmax = fmaxf(fmaxf(xa, xb), fmaxf(xc, xd));
    const float ymin = fminf(fminf(ya, yb), fminf(yc, yd)), ymax = fmaxf(fmaxf(ya, yb), fmaxf(yc, yd));
    const int bx0 = ((int)floorf(xmin) - 1) & ~7;  // 16-byte aligned TMA x coordinate (BF16 too)
    const int bx1 = (int)floorf(xmax) + 2;
    const int by0 = (int)floorf(ymin) - 1;
    const int by1 = (int)floorf(ymax) + 2;
    const int wq = (bx1 - bx0) / 4 + 1;  // float4 columns used
    const int bh = by1 - by0 + 1;
    if (4 * wq > FPT_BOX_W || bh > FPT_BOX_H) {  // cannot happen for valid matrices; never trap
      if (tid == 0) atomicExch(&g_box_overflow, 1);
      return;
    }

    if (tid == 0) {
      mbar_expect_tx(&bar, box_bytes);
      tma_load_3d(zb, &tm_vol, bx0, by0, s, &bar);
      if (HAS_MAPS) tma_load_3d(mraw, &tm_maps, bx0, by0, map_img, &bar);
    }
    // every thread observes the phase flip itself (acquire of the bulk-copy writes)
    if (!mbar_wait_bounded(&bar, phase)) timed_out = 1;
    __syncthreads();
    if (timed_out) {
      // give the copies in flight one more bounded wait, then leave without touching smem
      if (tid == 0) {
        atomicExch(&g_tma_timeout, 1);
        mbar_wait_bounded(&bar, phase);
      }
      return;
    }
    phase ^= 1u;

    if (HAS_MAPS) {
      float4* z4 = reinterpret_cast<float4*>(zb);
      for (int it = tid; it < bh * FPT_Q4; it += FP_THREADS) {
        const int rr = it / FPT_Q4;
        const int qq = it - rr * FPT_Q4;
        if (qq < wq) {
          float4 v = z4[it];
          if (MAPS_DTYPE == CCT_DTYPE_BF16) {
            const uint2 raw = reinterpret_cast<const uint2*>(mraw)[it];
            const float2 flo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&raw.x));
            const float2 fhi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&raw.y));
            v.x *= flo.x; v.y *= flo.y; v.z *= fhi.x; v.w *= fhi.y;
          } else {
            const float4 mv = reinterpret_cast<const float4*>(mraw)[it];
            v.x *= mv.x; v.y *= mv.y; v.z *= mv.z; v.w *= mv.w;
          }
          z4[it] = v;
        }
      }
      __syncthreads();
    }

    if (c <= c_last) {
      const int zoff = -by0 * FPT_BOX_W - bx0;
      float fr = (float)(r0 + lr);
      const int rem = r_last - r0 - lr;
      const int kmax = rem >= 0 ? rem / FP_LR + 1 : 0;
      if (kmax >= FP_RPT) {
        const float2 mx = make_float2(m01, m01), my = make_float2(m11, m11);
        const float2 cx = make_float2(pxc, pxc), cy = make_float2(pyc, pyc);
        const float2 step2 = make_float2(2.f * FP_LR, 2.f * FP_LR);
        float2 fr2 = make_float2(fr, fr + (float)FP_LR);
#pragma unroll 4
        for (int k = 0; k < FP_RPT; k += 2) {
          acc = bilerp2<FPT_BOX_W>(zb, zoff, __ffma2_rn(mx, fr2, cx), __ffma2_rn(my, fr2, cy), acc);
          fr2 = __fadd2_rn(fr2, step2);
        }
      } else {
        for (int k = 0; k < kmax; ++k) {
          const FloorSplit fx = floor_split(fmaf(m01, fr, pxc));
          const FloorSplit fy = floor_split(fmaf(m11, fr, pyc));
          const int q = fy.i * FPT_BOX_W + fx.i + zoff;
          const float t0 = zb[q], t1 = zb[q + 1], b0 = zb[q + FPT_BOX_W], b1 = zb[q + FPT_BOX_W + 1];
          const float top = fmaf(fx.f, t1 - t0, t0);
          const float bot = fmaf(fx.f, b1 - b0, b0);
          acc += fmaf(fy.f, bot - top, top);
          fr += (float)FP_LR;
        }
      }
    }
    __syncthreads();
    // generic-proxy writes/reads of the boxes are done; order them before the next bulk copy
    if (tid == 0) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }

  acc += __shfl_xor_sync(0xffffffffu, acc, 8);
  acc += __shfl_xor_sync(0xffffffffu, acc, 16);
  double part = 0.0, ptest = 0.0;
  if (lr == 0 && c <= c_last) {
    float total = acc;
    if (args.weights != nullptr) total *= args.weights[a * args.n_det + d];
    const int64_t idx = (((int64_t)s * args.n_det + d) * args.n_angles + a) * n + c;
    part = fp_epilogue<EPI>(args, idx, total, &ptest);
  }
  if (EPI == FP_EPI_MLEM || EPI == FP_EPI_SIRT) {
    const int64_t slot = (int64_t)s * gridDim.x * gridDim.y + (int64_t)blockIdx.y * gridDim.x + blockIdx.x;
    fp_write_partial(part, args.partials, slot, red_d, lane, warp, tid);
    if (args.partials_test != nullptr) fp_write_partial(ptest, args.partials_test, slot, red_d, lane, warp, tid);
  }
}

// ------------------------------------------------------------------------------------------
// Forward projection, two slices per CTA
//
// All slices of a batch share the angle's sample positions, so one CTA owns (band, angle *
// detector, pair of slices): it computes each sample's coordinates and tap offsets once, stages
// z = x * map of both slices interleaved (one float2 element per pixel) and reads every
// bilinear tap of both with one 8-byte shared load.  The arithmetic per sample and slice is
// fp_cta's (bit-identical results).  Chunks are 64 columns x 32 rows so that three CTAs fit per
// SM; like fp_cta, only the quads of each box row that the taps read are staged, and the row
// stride (80 + 2v elements, v in 0..4, even so that 16-byte stores stay aligned) is chosen per angle on
// the host (column 1 of cct_xrf_desc::fp_box_strides).  The fill loads float4 quads of both
// slices, and writes a quad as two 16-byte element pairs; lanes 4-7 of every 8-lane store phase
// write their second pair first, which keeps the 16-byte stores of a phase on distinct banks.
// Four CTAs fit per SM (64 registers, < 56 KB of shared memory each).
// ------------------------------------------------------------------------------------------
constexpr int FP2_TR = 32;                          // rows per staged chunk
constexpr int FP2_RPT = FP2_TR / FP_LR;             // 8 samples per thread per chunk
// 64 x 32 chunk rotated: x extent <= sqrt(63^2 + 31^2) = 70.2 (+ 11 for taps, margins and the
// float4-aligned origin) -> 80; y extent 70.2 + 5 -> 75 rows.
constexpr int FP2_BOX_W = 80;
constexpr int FP2_BOX_H = 75;
constexpr int FP2_STRIDE_MAX = FP2_BOX_W + 8;       // strides 80, 82, ..., 88 elements
constexpr int FP2_MAX_CHUNKS = (8192 + FP2_TR - 1) / FP2_TR;
static_assert(FP2_MAX_CHUNKS <= FP_THREADS, "one thread per chunk box");
constexpr int FP2_FILL_BATCH = 2;
constexpr size_t FP2_SMEM_BYTES = (size_t)FP2_STRIDE_MAX * FP2_BOX_H * sizeof(float2);

template <bool HAS_MAPS, int MAPS_DTYPE>
__device__ __forceinline__ float4 fp2_quad(const float* vol, const MapRef& mref, int n, int gy, int gx, bool vec4,
                                           bool ok) {
  if (!ok) return make_float4(0.f, 0.f, 0.f, 0.f);
  if (vec4) {
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if ((unsigned)gy < (unsigned)n && (unsigned)gx < (unsigned)n) {
      const int off = gy * n + gx;
      v = __ldg(reinterpret_cast<const float4*>(vol + off));
      if (HAS_MAPS) {
        const float4 mv = map_at4<MAPS_DTYPE>(mref, off);
        v.x *= mv.x; v.y *= mv.y; v.z *= mv.z; v.w *= mv.w;
      }
    }
    return v;
  }
  return fp_load_item<HAS_MAPS, MAPS_DTYPE>(vol, mref, n, gy, gx, false);
}

template <int EPI, bool HAS_MAPS, int MAPS_DTYPE>
__global__ void __launch_bounds__(FP_THREADS, 4) fp_pair_kernel(FpArgs args) {
  extern __shared__ __align__(16) float2 z2[];  // [FP2_BOX_H][stride] elements (slice 0, slice 1)
  __shared__ double red_d[FP_TC / FP_LC];
  __shared__ short4 box_sh[FP2_MAX_CHUNKS];  // (bx0, by0, quads, rows) of every chunk's box
  __shared__ short2 quads_sh[FP2_BOX_H];

  const int n = args.n;
  const int band = blockIdx.x;
  const int ad = blockIdx.y;
  const int s0 = 2 * blockIdx.z;
  bool ok[2];
#pragma unroll
  for (int g = 0; g < 2; ++g) {
    const int s = s0 + g;
    ok[g] = s < args.n_slices && (args.active == nullptr || args.active[s] != 0);
  }
  if (!ok[0] && !ok[1]) return;  // the whole CTA
  const int a = ad / args.n_det;
  const int d = ad - a * args.n_det;

  const float* M = args.fp_matrix + 6 * a;
  const float m00 = M[0], m01 = M[1], m02 = M[2], m10 = M[3], m11 = M[4], m12 = M[5];
  const int sel = args.box_strides != nullptr ? min(max(args.box_strides[2 * a + 1], 0), 4) : 0;
  const int S = FP2_BOX_W + 2 * sel;  // row stride (elements), even

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int lc = lane & (FP_LC - 1);
  const int lr = lane / FP_LC;
  const int c0 = band * FP_TC;
  const int c = c0 + warp * FP_LC + lc;
  const int c_last = min(c0 + FP_TC, n) - 1;
  const bool vec4 = args.vec4 != 0;
  const bool swap = (lane & 4) != 0;  // lanes 4-7 of each store phase write their second pair first

  const float* vol[2];
  MapRef mref[2];
#pragma unroll
  for (int g = 0; g < 2; ++g) {
    const int s = ok[g] ? s0 + g : s0 + (ok[0] ? 0 : 1);
    vol[g] = args.vol + (int64_t)s * n * n;
    mref[g] = make_map_ref(args.maps, MAPS_DTYPE, args.maps_slice_stride, args.n_angles, args.n_det, n, s, a, d,
                           args.n_channels, args.chan_scale);
  }
  const float fc = (float)c;
  const float pxc = fmaf(m00, fc, m02);
  const float pyc = fmaf(m10, fc, m12);

  // box coordinates fit 16 bits: |x|, |y| < 1.5 n + 3 for n <= 8192
  if (tid * FP2_TR < n) {
    int bx0, bx1, by0, by1;
    chunk_box(m00, m01, m02, m10, m11, m12, c0, c_last, tid * FP2_TR, min((tid + 1) * FP2_TR, n) - 1, bx0, bx1, by0,
              by1);
    box_sh[tid] = make_short4((short)bx0, (short)by0, (short)((bx1 - bx0) / 4 + 1), (short)(by1 - by0 + 1));
  }
  __syncthreads();
  {
    const short4 b0 = box_sh[0];
    if (tid < b0.w && tid < FP2_BOX_H) {
      float px[4], py[4];
      chunk_corners(m00, m01, m02, m10, m11, m12, c0, c_last, 0, min(FP2_TR, n) - 1, px, py);
      quads_sh[tid] = fp_row_quads(px, py, b0.y + tid, b0.x, b0.z);
    }
  }
  __syncthreads();

  float acc0 = 0.f, acc1 = 0.f;
  for (int r0 = 0; r0 < n; r0 += FP2_TR) {
    const int r_last = min(r0 + FP2_TR, n) - 1;
    const short4 box = box_sh[r0 / FP2_TR];
    const int bx0 = box.x, by0 = box.y, q4 = box.z, bh = box.w;
    if (4 * q4 > FP2_BOX_W || bh > FP2_BOX_H) {  // cannot happen for valid matrices; never trap
      if (tid == 0) atomicExch(&g_box_overflow, 1);
      return;
    }

    const int items = q4 * bh;
    const unsigned magic = (1048576u + (unsigned)q4 - 1u) / (unsigned)q4;  // it / q4 as in fp_cta
    for (int base = tid; base < items; base += FP_THREADS * FP2_FILL_BATCH) {
      float4 v0[FP2_FILL_BATCH], v1[FP2_FILL_BATCH];
      int dst[FP2_FILL_BATCH];
#pragma unroll
      for (int k = 0; k < FP2_FILL_BATCH; ++k) {
        const int it = base + k * FP_THREADS;
        dst[k] = -1;
        v0[k] = v1[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (it < items) {
          const int rr = (int)(((unsigned)it * magic) >> 20);
          const int qq = it - rr * q4;
          const short2 qr = quads_sh[rr];
          if (qq >= qr.x && qq <= qr.y) {
            const int gy = by0 + rr, gx = bx0 + 4 * qq;
            dst[k] = rr * S + 4 * qq;
            v0[k] = fp2_quad<HAS_MAPS, MAPS_DTYPE>(vol[0], mref[0], n, gy, gx, vec4, ok[0]);
            v1[k] = fp2_quad<HAS_MAPS, MAPS_DTYPE>(vol[1], mref[1], n, gy, gx, vec4, ok[1]);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < FP2_FILL_BATCH; ++k) {
        if (dst[k] >= 0) {
          // elements 4q, 4q + 1 (lo) and 4q + 2, 4q + 3 (hi); the order of the two stores is
          // selected per lane so that both store instructions run with every lane active
          const float4 lo = make_float4(v0[k].x, v1[k].x, v0[k].y, v1[k].y);
          const float4 hi = make_float4(v0[k].z, v1[k].z, v0[k].w, v1[k].w);
          float4* q = reinterpret_cast<float4*>(z2 + dst[k]);
          const int f = swap ? 1 : 0;
          q[f] = swap ? hi : lo;
          q[1 - f] = swap ? lo : hi;
        }
      }
    }
    __syncthreads();

    if (r0 + FP2_TR < n) {
      const short4 nb = box_sh[r0 / FP2_TR + 1];
      if (tid < nb.w && tid < FP2_BOX_H) {
        float px[4], py[4];
        chunk_corners(m00, m01, m02, m10, m11, m12, c0, c_last, r0 + FP2_TR, min(r0 + 2 * FP2_TR, n) - 1, px, py);
        quads_sh[tid] = fp_row_quads(px, py, nb.y + tid, nb.x, nb.z);
      }
    }

    if (c <= c_last) {
      const int zoff = -by0 * S - bx0;
      float fr = (float)(r0 + lr);
      const int rem = r_last - r0 - lr;
      const int kmax = rem >= 0 ? rem / FP_LR + 1 : 0;
      if (kmax >= FP2_RPT) {
        // both slices' lerps in packed FP32x2 arithmetic, rounding like the scalar loop below
        // (a - b as fma(b, -1, a))
        const float2 neg1 = make_float2(-1.f, -1.f);
        float2 acc2 = make_float2(acc0, acc1);
#pragma unroll 4
        for (int k = 0; k < FP2_RPT; ++k) {
          const FloorSplit fx = floor_split(fmaf(m01, fr, pxc));
          const FloorSplit fy = floor_split(fmaf(m11, fr, pyc));
          const int q = fy.i * S + fx.i + zoff;
          const float2 t0 = z2[q], t1 = z2[q + 1], b0 = z2[q + S], b1 = z2[q + S + 1];
          const float2 fxx = make_float2(fx.f, fx.f), fyy = make_float2(fy.f, fy.f);
          const float2 top = __ffma2_rn(fxx, __ffma2_rn(t0, neg1, t1), t0);
          const float2 bot = __ffma2_rn(fxx, __ffma2_rn(b0, neg1, b1), b0);
          acc2 = __fadd2_rn(acc2, __ffma2_rn(fyy, __ffma2_rn(top, neg1, bot), top));
          fr += (float)FP_LR;
        }
        acc0 = acc2.x;
        acc1 = acc2.y;
      } else {
        for (int k = 0; k < kmax; ++k) {
          const FloorSplit fx = floor_split(fmaf(m01, fr, pxc));
          const FloorSplit fy = floor_split(fmaf(m11, fr, pyc));
          const int q = fy.i * S + fx.i + zoff;
          const float2 t0 = z2[q], t1 = z2[q + 1], b0 = z2[q + S], b1 = z2[q + S + 1];
          const float top0 = fmaf(fx.f, t1.x - t0.x, t0.x), bot0 = fmaf(fx.f, b1.x - b0.x, b0.x);
          const float top1 = fmaf(fx.f, t1.y - t0.y, t0.y), bot1 = fmaf(fx.f, b1.y - b0.y, b0.y);
          acc0 += fmaf(fy.f, bot0 - top0, top0);
          acc1 += fmaf(fy.f, bot1 - top1, top1);
          fr += (float)FP_LR;
        }
      }
    }
    __syncthreads();
  }

  const int n_bands = gridDim.x;
  const int n_ad = gridDim.y;
#pragma unroll
  for (int g = 0; g < 2; ++g) {
    if (!ok[g]) continue;  // uniform across the CTA
    const int s = s0 + g;
    float col = g == 0 ? acc0 : acc1;
    col += __shfl_xor_sync(0xffffffffu, col, 8);
    col += __shfl_xor_sync(0xffffffffu, col, 16);
    double part = 0.0, ptest = 0.0;
    if (lr == 0 && c <= c_last) {
      float total = col;
      if (args.weights != nullptr) total *= args.weights[a * args.n_det + d];
      const int64_t idx = (((int64_t)s * args.n_det + d) * args.n_angles + a) * n + c;
      part = fp_epilogue<EPI>(args, idx, total, &ptest);
    }
    if (EPI == FP_EPI_MLEM || EPI == FP_EPI_SIRT) {
      const int64_t slot = (int64_t)s * n_bands * n_ad + (int64_t)ad * n_bands + band;
      fp_write_partial(part, args.partials, slot, red_d, lane, warp, tid);
      if (args.partials_test != nullptr) fp_write_partial(ptest, args.partials_test, slot, red_d, lane, warp, tid);
    }
  }
}

// ------------------------------------------------------------------------------------------
// Back projection (reference iradon discretisation, optional maps x weights)
// ------------------------------------------------------------------------------------------
constexpr int BP_TJ = 32;                                // tile columns (one per lane)
constexpr int BP_TI = 64;                                // tile rows
constexpr int BP_THREADS = 256;
constexpr int BP_PPT = BP_TI / (BP_THREADS / 32);        // 8 pixels (rows warp, warp+8, ...) per thread
constexpr int BP_LINES = 32;                             // lines staged per chunk
constexpr int BP_KW = 80;                                // staged pairs per line (>= 74 needed)
constexpr float BP_EDGE_GUARD = 0.01f;

enum : int { LINE_FAST = 0, LINE_CHECKED = 1, LINE_EMPTY = 2 };

// One CTA of the back projection: pixel tile `tile` of slice `s`.
template <int EPI, bool SYM, int MAPS_DTYPE>
__device__ __forceinline__ void bp_cta(const BpArgs& args, const int tile, const int s) {
  __shared__ __align__(16) float2 pairs[BP_LINES][BP_KW];
  __shared__ float4 linfo[BP_LINES];  // cos, sin, offset (K - kbase), weight
  __shared__ int lkind[BP_LINES];
  __shared__ int lkbase[BP_LINES];
  __shared__ float2 linner[BP_LINES];  // checked lines: interior range of the FP32 coordinate

  const int n = args.n;
  if (args.active != nullptr && args.active[s] == 0) return;
  const int tiles_j = (n + BP_TJ - 1) / BP_TJ;
  const int ti = tile / tiles_j;
  const int tj = tile - ti * tiles_j;
  const int i0 = ti * BP_TI, j0 = tj * BP_TJ;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int j = j0 + lane;
  const int R = n / 2;      // iradon output radius (output_size // 2)
  const int K = n / 2;      // detector offset (img_shape // 2)
  const float t_left = (float)(-K), t_right = (float)(n - 1 - K);
  const int n_lines = args.n_det * args.n_angles;
  const float* sino = args.sino + (int64_t)s * n_lines * n;

  // full tile (also pixels beyond n, which are computed and discarded) so every thread's
  // lookup stays inside the staged range
  const float cj0 = (float)(j0 - R), cj1 = (float)(j0 + BP_TJ - 1 - R);
  const float ci0 = (float)(i0 - R), ci1 = (float)(i0 + BP_TI - 1 - R);
  const float fjR = (float)(j - R);
  float nfiR[BP_PPT];
#pragma unroll
  for (int k = 0; k < BP_PPT; ++k) nfiR[k] = -(float)(i0 + warp + 8 * k - R);

  float acc[BP_PPT];
#pragma unroll
  for (int k = 0; k < BP_PPT; ++k) acc[k] = 0.f;

  for (int l0 = 0; l0 < n_lines; l0 += BP_LINES) {
    // ---- stage up to BP_LINES lines: each warp fills 4 lines
    for (int ll = warp; ll < BP_LINES; ll += BP_THREADS / 32) {
      const int l = l0 + ll;
      if (l >= n_lines) break;
      const int d = l / args.n_angles;
      const int a = l - d * args.n_angles;
      const float cs = args.bp_trig[2 * a], sn = args.bp_trig[2 * a + 1];
      // t = (j - R) cos - (i - R) sin at the four corners
      const float t00 = fmaf(cj0, cs, -ci0 * sn), t01 = fmaf(cj1, cs, -ci0 * sn);
      const float t10 = fmaf(cj0, cs, -ci1 * sn), t11 = fmaf(cj1, cs, -ci1 * sn);
      const float tmin = fminf(fminf(t00, t01), fminf(t10, t11));
      const float tmax = fmaxf(fmaxf(t00, t01), fmaxf(t10, t11));
      int kind = LINE_FAST;
      if (tmax < t_left - BP_EDGE_GUARD || tmin > t_right + BP_EDGE_GUARD) {
        kind = LINE_EMPTY;
      } else if (tmin < t_left + BP_EDGE_GUARD || tmax > t_right - BP_EDGE_GUARD) {
        kind = LINE_CHECKED;
      }
      const int kbase = (int)floorf(tmin + (float)K) - 1;
      float w = 1.f;
      if (SYM && args.weights != nullptr) w = args.weights[a * args.n_det + d];
      if (!SYM && args.line_scale != nullptr) w = args.line_scale[a];
      const float* line = sino + ((int64_t)d * args.n_angles + a) * n;
      if (kind != LINE_EMPTY) {
        float v[3], vn[3];
#pragma unroll
        for (int q3 = 0; q3 < 3; ++q3) {
          const int kk = kbase + lane + 32 * q3;
          v[q3] = (kk >= 0 && kk < n) ? __ldg(line + kk) : 0.f;
          vn[q3] = (kk + 1 >= 0 && kk + 1 < n) ? __ldg(line + kk + 1) : 0.f;
        }
#pragma unroll
        for (int q3 = 0; q3 < 3; ++q3) {
          const int q = lane + 32 * q3;
          if (q < BP_KW) pairs[ll][q] = make_float2(w * v[q3], w * (vn[q3] - v[q3]));
        }
      }
      if (lane == 0) {
        linfo[ll] = make_float4(cs, sn, (float)(K - kbase), w);
        lkind[ll] = kind;
        lkbase[ll] = kbase;
        // the FP32 coordinate u = t + K - kbase of the accumulate loop is within ~1e-4 of its
        // exact value: pixels with u inside the detector by more than BP_EDGE_GUARD take the
        // fast lerp, only the others decide the edge in double precision
        linner[ll] = make_float2((float)(-kbase) + BP_EDGE_GUARD, (float)(n - 1 - kbase) - BP_EDGE_GUARD);
      }
    }
    __syncthreads();

    // ---- accumulate
    const int lines_here = min(BP_LINES, n_lines - l0);
    for (int ll = 0; ll < lines_here; ++ll) {
      const int kind = lkind[ll];
      if (kind == LINE_EMPTY) continue;
      const float4 inf = linfo[ll];
      const float base = fmaf(fjR, inf.x, inf.z);
      const float2* pr = pairs[ll];
      int a = 0, d = 0;
      if (SYM) {
        const int l = l0 + ll;
        d = l / args.n_angles;
        a = l - d * args.n_angles;
      }
      if (kind == LINE_FAST && !SYM) {
#pragma unroll
        for (int k = 0; k < BP_PPT; ++k) {
          const FloorSplit fs = floor_split(fmaf(nfiR[k], inf.y, base));
          const float2 p = pr[fs.i];
          acc[k] += fmaf(fs.f, p.y, p.x);
        }
        continue;
      }
      const float2 inner = linner[ll];
#pragma unroll
      for (int k = 0; k < BP_PPT; ++k) {
        const int i = i0 + warp + 8 * k;
        const float u = fmaf(nfiR[k], inf.y, base);
        const FloorSplit fs = floor_split(u);
        const float2 p = pr[fs.i];
        float v = fmaf(fs.f, p.y, p.x);
        if (kind == LINE_CHECKED && !(u > inner.x && u < inner.y)) {
          // np.interp(t, k - K, line, left=0, right=0) decided in double like numpy
          const double td = __dsub_rn(__dmul_rn((double)(j - R), (double)inf.x),
                                      __dmul_rn((double)(i - R), (double)inf.y));
          if (td < -(double)K || td > (double)(n - 1 - K)) {
            v = 0.f;
          } else {
            const double uk = td + (double)K;
            const double fl = floor(uk);
            const int kidx = (int)fl - lkbase[ll];
            const float2 pe = pr[min(max(kidx, 0), BP_KW - 1)];
            v = (float)((double)pe.x + (uk - fl) * (double)pe.y);
          }
        }
        if (SYM) {
          if (i < n && j < n) {
            const MapRef mr = make_map_ref(args.maps, MAPS_DTYPE, args.maps_slice_stride, args.n_angles, args.n_det, n,
                                           s, a, d, args.n_channels, args.chan_scale);
            v *= map_at<MAPS_DTYPE>(mr, (int64_t)i * n + j);
          }
        }
        acc[k] += v;
      }
    }
    __syncthreads();
  }

  if constexpr (EPI == BP_EPI_MLEM || EPI == BP_EPI_SIRT) {
    bp_epilogue_rows<EPI, BP_PPT>(args, s, i0 + warp, 8, j, acc);
  } else {
#pragma unroll
    for (int k = 0; k < BP_PPT; ++k) {
      const int i = i0 + warp + 8 * k;
      if (i < n && j < n) bp_epilogue<EPI>(args, s, i, j, acc[k]);
    }
  }
}

template <int EPI, bool SYM, int MAPS_DTYPE>
__global__ void __launch_bounds__(BP_THREADS, 4) bp_kernel(BpArgs args) {
  bp_cta<EPI, SYM, MAPS_DTYPE>(args, blockIdx.x, blockIdx.y);
}

// Back projection over groups of slices in one launch: group g's CTAs are (tile, slice),
// tile fastest.
template <int EPI, bool SYM, int MAPS_DTYPE>
__global__ void __launch_bounds__(BP_THREADS) bp_ragged_kernel(const BpArgs* __restrict__ groups,
                                                               const int64_t* __restrict__ start, int n_groups) {
  const int64_t cta = blockIdx.x;
  const int g = ragged_group(start, n_groups, cta);
  const BpArgs& a = groups[g];
  const int tiles = ((a.n + BP_TJ - 1) / BP_TJ) * ((a.n + BP_TI - 1) / BP_TI);
  const int64_t local = cta - start[g];
  bp_cta<EPI, SYM, MAPS_DTYPE>(a, (int)(local % tiles), (int)(local / tiles));
}

// ------------------------------------------------------------------------------------------
// Exact adjoint of the forward projection (gather form; no reference counterpart)
// bp[p] = sum_a sum_{(r,c)} w_a hat(col_in(r,c) - p_x) hat(row_in(r,c) - p_y) y[a][c] (* map[a][p])
// For a pixel p and angle a the candidate samples are the rotated-lattice points within
// distance < 1 (per axis) of p: r, c within +-2 of the inverse-rotated position.
// ------------------------------------------------------------------------------------------
template <bool HAS_MAPS, int MAPS_DTYPE>
__global__ void __launch_bounds__(256) bp_adjoint_kernel(BpArgs args) {
  const int n = args.n;
  const int64_t total = (int64_t)n * n;
  const int s = blockIdx.y;
  const int64_t pix = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= total) return;
  const int pi = (int)(pix / n), pj = (int)(pix - (int64_t)pi * n);
  const int n_lines = args.n_det * args.n_angles;
  const float* sino = args.sino + (int64_t)s * n_lines * n;
  double acc = 0.0;
  for (int l = 0; l < n_lines; ++l) {
    const int d = l / args.n_angles;
    const int a = l - d * args.n_angles;
    const float* M = args.fp_matrix + 6 * a;
    const float m00 = M[0], m01 = M[1], m02 = M[2], m10 = M[3], m11 = M[4], m12 = M[5];
    // invert the 2x2 part to find the lattice point nearest to p
    const double det = (double)m00 * m11 - (double)m01 * m10;
    const double dx = pj - (double)m02, dy = pi - (double)m12;
    const double cc = (m11 * dx - m01 * dy) / det;
    const double rr = (-m10 * dx + m00 * dy) / det;
    const int cb = (int)floor(cc), rb = (int)floor(rr);
    double lsum = 0.0;
    for (int r = rb - 2; r <= rb + 3; ++r) {
      if (r < 0 || r >= n) continue;
      for (int c = cb - 2; c <= cb + 3; ++c) {
        if (c < 0 || c >= n) continue;
        // same float arithmetic as the forward kernel's sample position
        const float px = sample_x(m00, m01, m02, (float)c, (float)r);
        const float py = sample_x(m10, m11, m12, (float)c, (float)r);
        const float hx = 1.f - fabsf(px - (float)pj);
        const float hy = 1.f - fabsf(py - (float)pi);
        if (hx > 0.f && hy > 0.f) lsum += (double)hx * hy * sino[((int64_t)d * args.n_angles + a) * n + c];
      }
    }
    float w = args.weights != nullptr ? args.weights[a * args.n_det + d] : 1.f;
    double contrib = lsum * w;
    if (HAS_MAPS) {
      const MapRef mr = make_map_ref(args.maps, MAPS_DTYPE, args.maps_slice_stride, args.n_angles, args.n_det, n, s, a, d,
                                     args.n_channels, args.chan_scale);
      contrib *= map_at<MAPS_DTYPE>(mr, pix);
    }
    acc += contrib;
  }
  bp_epilogue<BP_EPI_STORE>(args, s, pi, pj, (float)acc);
}

// ------------------------------------------------------------------------------------------
// Detector PSF: out[i] = sum_j in[clamp(i + (L-1)/2 - j)] * k[j] along each sinogram line (the
// reference pads with edge values, convolves with scipy 'same' and crops), followed by the same
// fused solver epilogue as the fp.  One CTA per line; args.vol holds the unconvolved sinogram.
// ------------------------------------------------------------------------------------------
constexpr int PSF_THREADS = 256;

template <int EPI>
__global__ void __launch_bounds__(PSF_THREADS) psf_kernel(FpArgs args, const float* __restrict__ k, int len) {
  extern __shared__ float line_sh[];
  __shared__ double red_d[PSF_THREADS / 32];
  const int n = args.n;
  const int64_t line = blockIdx.x;  // ((s * D + d) * A + a)
  const int s = (int)(line / ((int64_t)args.n_det * args.n_angles));
  if (args.active != nullptr && args.active[s] == 0) return;
  const float* in = args.vol + line * n;
  for (int i = threadIdx.x; i < n; i += PSF_THREADS) line_sh[i] = in[i];
  __syncthreads();
  const int p = (len - 1) / 2;
  double part = 0.0, ptest = 0.0;
  for (int i = threadIdx.x; i < n; i += PSF_THREADS) {
    float acc = 0.f;
    for (int j = 0; j < len; ++j) {
      int q = i + p - j;
      q = q < 0 ? 0 : (q >= n ? n - 1 : q);
      acc = fmaf(line_sh[q], __ldg(k + j), acc);
    }
    part += fp_epilogue<EPI>(args, line * n + i, acc, &ptest);
  }
  if (EPI == FP_EPI_MLEM || EPI == FP_EPI_SIRT) {
    // one partial per (detector, angle) line of the slice
    for (int which = 0; which < 2; ++which) {
      double* dst = which == 0 ? args.partials : args.partials_test;
      if (dst == nullptr) continue;  // uniform across the CTA
      double v = warp_sum_double(which == 0 ? part : ptest);
      __syncthreads();
      if ((threadIdx.x & 31) == 0) red_d[threadIdx.x >> 5] = v;
      __syncthreads();
      if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < PSF_THREADS / 32; ++w) t += red_d[w];
        dst[line] = t;
      }
    }
  }
}

void launch_psf(const FpArgs& a, const float* psf, int psf_len, cudaStream_t st) {
  const unsigned lines = (unsigned)((int64_t)a.n_slices * a.n_det * a.n_angles);
  const size_t smem = (size_t)a.n * sizeof(float);
  switch (a.epi) {
    case FP_EPI_MLEM: psf_kernel<FP_EPI_MLEM><<<lines, PSF_THREADS, smem, st>>>(a, psf, psf_len); break;
    case FP_EPI_SIRT: psf_kernel<FP_EPI_SIRT><<<lines, PSF_THREADS, smem, st>>>(a, psf, psf_len); break;
    case FP_EPI_PDHG: psf_kernel<FP_EPI_PDHG><<<lines, PSF_THREADS, smem, st>>>(a, psf, psf_len); break;
    default: psf_kernel<FP_EPI_STORE><<<lines, PSF_THREADS, smem, st>>>(a, psf, psf_len); break;
  }
}

// ------------------------------------------------------------------------------------------
// Launchers
// ------------------------------------------------------------------------------------------

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link needed)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess) {
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
  }
  return fn;
}

// 3-D tiled map over `images` row-major n x n images with a 96 x 104 box.
static bool make_box_map(CUtensorMap* map, const void* base, int n, int64_t images, bool bf16) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (enc == nullptr) return false;
  const uint64_t esz = bf16 ? 2 : 4;
  const cuuint64_t dims[3] = {(cuuint64_t)n, (cuuint64_t)n, (cuuint64_t)images};
  const cuuint64_t strides[2] = {(cuuint64_t)(n * esz), (cuuint64_t)((uint64_t)n * n * esz)};
  const cuuint32_t box[3] = {(cuuint32_t)FPT_BOX_W, (cuuint32_t)FPT_BOX_H, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = enc(map, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                         const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <int EPI, bool HAS_MAPS, int MAPS_DTYPE>
static bool launch_fp_tma_inst(const FpArgs& a, const dim3& grid, cudaStream_t st) {
  CUtensorMap tv, tm;
  std::memset(&tm, 0, sizeof(tm));
  if (!make_box_map(&tv, a.vol, a.n, a.n_slices, false)) return false;
  if (HAS_MAPS &&
      !make_box_map(&tm, a.maps, a.n, (int64_t)a.n_slices * a.n_angles * a.n_det, MAPS_DTYPE == CCT_DTYPE_BF16)) {
    return false;
  }
  const size_t smem = FPT_BOX_H * FPT_BOX_W * sizeof(float) +
                      (HAS_MAPS ? FPT_BOX_H * FPT_BOX_W * (MAPS_DTYPE == CCT_DTYPE_BF16 ? 2 : 4) : 0);
  if (!ensure_dynamic_smem<fp_tma_kernel<EPI, HAS_MAPS, MAPS_DTYPE>>((int)smem)) return false;
  fp_tma_kernel<EPI, HAS_MAPS, MAPS_DTYPE><<<grid, FP_THREADS, smem, st>>>(a, tv, tm);
  return launched_ok();
}

template <int EPI, bool HAS_MAPS, int MAPS_DTYPE>
static bool launch_fp_pair_inst(const FpArgs& a, cudaStream_t st) {
  const dim3 grid((a.n + FP_TC - 1) / FP_TC, a.n_angles * a.n_det, (a.n_slices + 1) / 2);
  if (!ensure_dynamic_smem<fp_pair_kernel<EPI, HAS_MAPS, MAPS_DTYPE>>((int)FP2_SMEM_BYTES)) return false;
  fp_pair_kernel<EPI, HAS_MAPS, MAPS_DTYPE><<<grid, FP_THREADS, FP2_SMEM_BYTES, st>>>(a);
  return launched_ok();
}

template <int EPI>
static bool launch_fp_pair(const FpArgs& a, cudaStream_t st) {
  if (a.maps == nullptr) return launch_fp_pair_inst<EPI, false, CCT_DTYPE_F32>(a, st);
  if (a.maps_dtype == CCT_DTYPE_BF16) return launch_fp_pair_inst<EPI, true, CCT_DTYPE_BF16>(a, st);
  if (a.maps_dtype == CCT_DTYPE_FIELDS_F32) return launch_fp_pair_inst<EPI, true, CCT_DTYPE_FIELDS_F32>(a, st);
  return launch_fp_pair_inst<EPI, true, CCT_DTYPE_F32>(a, st);
}

// 16-byte staging loads need a 16-byte aligned volume, maps at 16 (FP32) or 8 (BF16) bytes and
// map images that stay aligned (n % 4 == 0, slice stride a multiple of 4 elements)
bool fp_vec4_ok(const FpArgs& a) {
  const uintptr_t map_align = a.maps_dtype == CCT_DTYPE_BF16 ? 8 : 16;
  return (a.n % 4) == 0 && (reinterpret_cast<uintptr_t>(a.vol) % 16) == 0 &&
         (a.maps == nullptr || ((reinterpret_cast<uintptr_t>(a.maps) % map_align) == 0 && a.maps_slice_stride % 4 == 0));
}

template <int EPI>
static void launch_fp_epi(const FpArgs& a, cudaStream_t st) {
  const dim3 grid((a.n + FP_TC - 1) / FP_TC, a.n_angles * a.n_det, a.n_slices);
  // two slices per CTA: any n, maps stride and storage type; the plain kernel if refused
  if ((a.variant & CCT_VARIANT_FP_SLICES2) && a.n_slices >= 2) {
    FpArgs v = a;
    v.vec4 = fp_vec4_ok(a) ? 1 : 0;
    if (launch_fp_pair<EPI>(v, st)) return;
  }
  // TMA path: rows and images must be 16-byte multiples for both FP32 and BF16 boxes
  const int64_t dense = (int64_t)a.n_angles * a.n_det * a.n * a.n;
  const bool aligned = (a.n % 8) == 0 && (reinterpret_cast<uintptr_t>(a.vol) % 16) == 0 &&
                       (a.maps == nullptr || (reinterpret_cast<uintptr_t>(a.maps) % 16) == 0) &&
                       a.maps_slice_stride == dense && a.maps_dtype != CCT_DTYPE_FIELDS_F32;
  if (aligned && (a.variant & CCT_VARIANT_FP_TMA)) {
    bool ok;
    if (a.maps == nullptr) {
      ok = launch_fp_tma_inst<EPI, false, CCT_DTYPE_F32>(a, grid, st);
    } else if (a.maps_dtype == CCT_DTYPE_BF16) {
      ok = launch_fp_tma_inst<EPI, true, CCT_DTYPE_BF16>(a, grid, st);
    } else {
      ok = launch_fp_tma_inst<EPI, true, CCT_DTYPE_F32>(a, grid, st);
    }
    if (ok) return;
  }
  FpArgs v = a;
  v.vec4 = fp_vec4_ok(a) ? 1 : 0;
  if (a.maps == nullptr) {
    fp_kernel<EPI, false, CCT_DTYPE_F32><<<grid, FP_THREADS, 0, st>>>(v);
  } else if (a.maps_dtype == CCT_DTYPE_BF16) {
    fp_kernel<EPI, true, CCT_DTYPE_BF16><<<grid, FP_THREADS, 0, st>>>(v);
  } else if (a.maps_dtype == CCT_DTYPE_FIELDS_F32) {
    const dim3 fgrid(grid.x * a.n_channels, grid.y, a.n_slices / a.n_channels);
    fp_fields_kernel<EPI><<<fgrid, FP_THREADS, 0, st>>>(v);
  } else {
    fp_kernel<EPI, true, CCT_DTYPE_F32><<<grid, FP_THREADS, 0, st>>>(v);
  }
}

void launch_fp(const FpArgs& a, cudaStream_t st) {
  switch (a.epi) {
    case FP_EPI_MLEM: launch_fp_epi<FP_EPI_MLEM>(a, st); break;
    case FP_EPI_SIRT: launch_fp_epi<FP_EPI_SIRT>(a, st); break;
    case FP_EPI_PDHG: launch_fp_epi<FP_EPI_PDHG>(a, st); break;
    default: launch_fp_epi<FP_EPI_STORE>(a, st); break;
  }
}

template <int EPI>
static void launch_bp_epi(const BpArgs& a, cudaStream_t st) {
  const int tiles = ((a.n + BP_TJ - 1) / BP_TJ) * ((a.n + BP_TI - 1) / BP_TI);
  const dim3 grid(tiles, a.n_slices);
  const bool sym = a.mode == CCT_BP_SYMMETRIC;
  if (!sym) {
    bp_kernel<EPI, false, CCT_DTYPE_F32><<<grid, BP_THREADS, 0, st>>>(a);
  } else if (a.maps_dtype == CCT_DTYPE_BF16) {
    bp_kernel<EPI, true, CCT_DTYPE_BF16><<<grid, BP_THREADS, 0, st>>>(a);
  } else if (a.maps_dtype == CCT_DTYPE_FIELDS_F32) {
    bp_kernel<EPI, true, CCT_DTYPE_FIELDS_F32><<<grid, BP_THREADS, 0, st>>>(a);
  } else {
    bp_kernel<EPI, true, CCT_DTYPE_F32><<<grid, BP_THREADS, 0, st>>>(a);
  }
}

template <int EPI>
static void launch_fp_ragged_epi(const FpArgs* g, const int64_t* start, int ng, int64_t ctas, bool has_maps, int dt,
                                 cudaStream_t st) {
  const dim3 grid((unsigned)ctas);
  if (!has_maps) {
    fp_ragged_kernel<EPI, false, CCT_DTYPE_F32><<<grid, FP_THREADS, 0, st>>>(g, start, ng);
  } else if (dt == CCT_DTYPE_BF16) {
    fp_ragged_kernel<EPI, true, CCT_DTYPE_BF16><<<grid, FP_THREADS, 0, st>>>(g, start, ng);
  } else if (dt == CCT_DTYPE_FIELDS_F32) {
    fp_ragged_kernel<EPI, true, CCT_DTYPE_FIELDS_F32><<<grid, FP_THREADS, 0, st>>>(g, start, ng);
  } else {
    fp_ragged_kernel<EPI, true, CCT_DTYPE_F32><<<grid, FP_THREADS, 0, st>>>(g, start, ng);
  }
}

void launch_fp_ragged(const FpArgs* groups, const int64_t* start, int n_groups, int64_t ctas, int epi, bool has_maps,
                      int maps_dtype, cudaStream_t st) {
  if (epi == FP_EPI_SIRT) {
    launch_fp_ragged_epi<FP_EPI_SIRT>(groups, start, n_groups, ctas, has_maps, maps_dtype, st);
  } else {
    launch_fp_ragged_epi<FP_EPI_MLEM>(groups, start, n_groups, ctas, has_maps, maps_dtype, st);
  }
}

template <int EPI>
static void launch_bp_ragged_epi(const BpArgs* g, const int64_t* start, int ng, int64_t ctas, bool sym, int dt,
                                 cudaStream_t st) {
  const dim3 grid((unsigned)ctas);
  if (!sym) {
    bp_ragged_kernel<EPI, false, CCT_DTYPE_F32><<<grid, BP_THREADS, 0, st>>>(g, start, ng);
  } else if (dt == CCT_DTYPE_BF16) {
    bp_ragged_kernel<EPI, true, CCT_DTYPE_BF16><<<grid, BP_THREADS, 0, st>>>(g, start, ng);
  } else if (dt == CCT_DTYPE_FIELDS_F32) {
    bp_ragged_kernel<EPI, true, CCT_DTYPE_FIELDS_F32><<<grid, BP_THREADS, 0, st>>>(g, start, ng);
  } else {
    bp_ragged_kernel<EPI, true, CCT_DTYPE_F32><<<grid, BP_THREADS, 0, st>>>(g, start, ng);
  }
}

void launch_bp_ragged(const BpArgs* groups, const int64_t* start, int n_groups, int64_t ctas, int epi, bool sym,
                      int maps_dtype, cudaStream_t st) {
  if (epi == BP_EPI_SIRT) {
    launch_bp_ragged_epi<BP_EPI_SIRT>(groups, start, n_groups, ctas, sym, maps_dtype, st);
  } else {
    launch_bp_ragged_epi<BP_EPI_MLEM>(groups, start, n_groups, ctas, sym, maps_dtype, st);
  }
}

void launch_bp(const BpArgs& a, cudaStream_t st) {
  if (a.mode == CCT_BP_ADJOINT) {
    const dim3 grid((unsigned)(((int64_t)a.n * a.n + 255) / 256), a.n_slices);
    if (a.maps == nullptr) {
      bp_adjoint_kernel<false, CCT_DTYPE_F32><<<grid, 256, 0, st>>>(a);
    } else if (a.maps_dtype == CCT_DTYPE_BF16) {
      bp_adjoint_kernel<true, CCT_DTYPE_BF16><<<grid, 256, 0, st>>>(a);
    } else if (a.maps_dtype == CCT_DTYPE_FIELDS_F32) {
      bp_adjoint_kernel<true, CCT_DTYPE_FIELDS_F32><<<grid, 256, 0, st>>>(a);
    } else {
      bp_adjoint_kernel<true, CCT_DTYPE_F32><<<grid, 256, 0, st>>>(a);
    }
    return;
  }
  switch (a.epi) {
    case BP_EPI_MLEM: launch_bp_epi<BP_EPI_MLEM>(a, st); break;
    case BP_EPI_SIRT: launch_bp_epi<BP_EPI_SIRT>(a, st); break;
    case BP_EPI_PDHG: launch_bp_epi<BP_EPI_PDHG>(a, st); break;
    default: launch_bp_epi<BP_EPI_STORE>(a, st); break;
  }
}

}  // namespace cct

namespace cct {
int read_device_error(int clear, int* value) {
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_box_overflow, sizeof(int));
  if (e != cudaSuccess) return (int)e;
  int t = 0;
  e = cudaMemcpyFromSymbol(&t, g_tma_timeout, sizeof(int));
  if (e != cudaSuccess) return (int)e;
  if (clear) {
    const int zero = 0;
    e = cudaMemcpyToSymbol(g_box_overflow, &zero, sizeof(int));
    if (e != cudaSuccess) return (int)e;
    e = cudaMemcpyToSymbol(g_tma_timeout, &zero, sizeof(int));
    if (e != cudaSuccess) return (int)e;
  }
  *value = v | (t << 1);
  return 0;
}
}  // namespace cct
