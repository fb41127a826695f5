// Internal launch arguments and fused epilogues shared by the projection and solver kernels.
#pragma once

#include "cct_common.cuh"

namespace cct {

constexpr float EPS32 = 1.1920928955078125e-07f;  // np.finfo(np.float32).eps (corrct solvers.py:20)

// Sample position of output (col c, row r) under a radon inverse map; every kernel that
// needs the position of a forward-projection sample evaluates exactly this expression.
__device__ __forceinline__ float sample_x(float ma, float mb, float mc, float c, float r) {
  return fmaf(mb, r, fmaf(ma, c, mc));
}

enum FpEpilogue : int { FP_EPI_STORE = 0, FP_EPI_MLEM = 1, FP_EPI_SIRT = 2, FP_EPI_PDHG = 3 };
enum BpEpilogue : int { BP_EPI_STORE = 0, BP_EPI_MLEM = 1, BP_EPI_SIRT = 2, BP_EPI_PDHG = 3 };

struct FpArgs {
  int n, n_angles, n_det, n_slices, maps_dtype, epi, variant;
  int vec4;                    // 16-byte staging loads allowed (n % 4 == 0 and aligned pointers)
  int64_t maps_slice_stride;   // elements between consecutive slices' maps (field slices' fields)
  int n_channels;              // CCT_DTYPE_FIELDS_F32: channels per field slice
  const float* chan_scale;
  const float* fp_matrix;
  const float* weights;
  const float* vol;
  const void* maps;
  float* out;          // STORE: A x; MLEM: b / max(Ax + bg, eps); SIRT: (b - Ax - bg) * sigma; PDHG: dual p
  const float* b;
  const float* sigma;  // SIRT / PDHG
  float background;
  int has_background;
  double* partials;    // per-CTA residual partial sums (MLEM, SIRT)
  const int* active;
  const float* b_mask;       // data mask of the residual, or nullptr
  const float* b_test_mask;  // cross-validation mask, or nullptr
  double* partials_test;     // per-CTA test residual partials (with b_test_mask)
  const int* box_strides;    // [A][2] staged-box row-stride selectors per angle (speed only), or nullptr
};

struct BpArgs {
  int n, n_angles, n_det, n_slices, maps_dtype, mode, epi;
  int64_t maps_slice_stride;   // elements between consecutive slices' maps (field slices' fields)
  int n_channels;
  const float* chan_scale;
  const float* fp_matrix;
  const float* bp_trig;
  const float* weights;
  const float* line_scale;  // reference mode: per-angle intensity scaling of the lines
  const float* sino;
  const void* maps;
  float* out;              // STORE target
  // fused solver epilogues
  float* x;
  float* x_relax;
  const float* tau;
  int tau_shared;
  const float* x_mask;
  int mask_per_slice;      // x_mask is [S][n][n] instead of one [n][n] mask
  const float* tv_dual;    // PDHG: updated TV dual [S][2][n][n]
  float lower, upper;
  int has_lower, has_upper;
  const int* active;
};

// Fused forward-projection epilogue for one final value `ax` = (A x)[idx].
// Returns this element's contribution to the slice residual (FP64) and adds its contribution
// to the cross-validation residual to *test (with b_test_mask).
template <int EPI>
__device__ __forceinline__ double fp_epilogue(const FpArgs& a, int64_t idx, float ax, double* test) {
  if (EPI == FP_EPI_STORE) {
    a.out[idx] = ax;
    return 0.0;
  } else if (EPI == FP_EPI_MLEM) {
    // corrct solvers.py:787-796 and data_terms.py:720-742 (KL, sigma = 1); the masks scale the
    // residual only, the MLEM ratio is unmasked (solvers.py:797)
    const float bb = a.b[idx];
    const float proj = a.has_background ? ax + a.background : ax;
    const float clipped = fmaxf(proj, EPS32);
    a.out[idx] = bb / clipped;
    const double r = (double)clipped;
    const double sd = 4.0 * fmax((double)bb, 0.0);
    const double res = fabs((1.0 + r - sqrt((r - 1.0) * (r - 1.0) + sd)) * 0.5);
    if (a.b_test_mask != nullptr) *test += res * (double)fabsf(a.b_test_mask[idx]);
    return a.b_mask != nullptr ? res * (double)fabsf(a.b_mask[idx]) : res;
  } else if (EPI == FP_EPI_SIRT) {
    // corrct data_terms.py:136-161 (l2 residual), solvers.py:954-977; the masked residual drives
    // the update
    const float proj = a.has_background ? ax + a.background : ax;
    const float raw = a.b[idx] - proj;
    const float res = a.b_mask != nullptr ? raw * a.b_mask[idx] : raw;
    a.out[idx] = res * a.sigma[idx];
    if (a.b_test_mask != nullptr) {
      const double t = (double)(raw * a.b_test_mask[idx]);
      *test += t * t;
    }
    return (double)res * (double)res;
  } else {
    // PDHG dual update + KL prox (corrct data_terms.py:262-276, 682-692), then p *= b_mask
    // (solvers.py:1168-1169)
    const float proj = a.has_background ? ax + a.background : ax;
    const double sg = (double)a.sigma[idx];
    const double p = (double)a.out[idx] + (double)proj * sg;
    const double sd = 4.0 * sg * fmax((double)a.b[idx], 0.0);
    float pn = (float)((1.0 + p - sqrt((p - 1.0) * (p - 1.0) + sd)) * 0.5);
    if (a.b_mask != nullptr) pn *= a.b_mask[idx];
    a.out[idx] = pn;
    return 0.0;
  }
}

__device__ __forceinline__ float apply_limits(const BpArgs& a, float v) {
  // x.clip(lower, upper): numpy clip is min(max(v, lower), upper)
  if (a.has_lower) v = fmaxf(v, a.lower);
  if (a.has_upper) v = fminf(v, a.upper);
  return v;
}

// Fused back-projection epilogue for pixel (s, i, j) with back-projected value `v`.
template <int EPI>
__device__ __forceinline__ void bp_epilogue(const BpArgs& a, int s, int i, int j, float v) {
  const int64_t n2 = (int64_t)a.n * a.n;
  const int64_t pix = (int64_t)i * a.n + j;
  const int64_t idx = (int64_t)s * n2 + pix;
  if (EPI == BP_EPI_STORE) {
    a.out[idx] = v;
    return;
  }
  const float tau = a.tau[(a.tau_shared ? 0 : (int64_t)s * n2) + pix];
  float x = a.x[idx];
  if (EPI == BP_EPI_MLEM) {
    // x *= upd / tau  (corrct solvers.py:798-803); a pixel that no line reaches (tau = 0, which an
    // ordered subset of few angles can leave in the corners) keeps its value
    x = tau != 0.f ? x * (v / tau) : x;
  } else if (EPI == BP_EPI_SIRT) {
    // x += upd * tau  (corrct solvers.py:977)
    x = x + v * tau;
  } else {
    // PDHG primal step (corrct solvers.py:1179-1190): x_new = x - (A^T p - div q) * tau,
    // div with edge padding (operators.py:818-844)
    const float* q = a.tv_dual + (int64_t)s * 2 * n2;
    const float q0 = q[pix], q1 = q[n2 + pix];
    const float d0 = (i > 0) ? q0 - q[pix - a.n] : 0.f;
    const float d1 = (j > 0) ? q1 - q[n2 + pix - 1] : 0.f;
    const float upd = v - (d0 + d1);
    float xn = x - upd * tau;
    xn = apply_limits(a, xn);
    if (a.x_mask != nullptr) xn *= a.x_mask[a.mask_per_slice ? idx : pix];
    a.x_relax[idx] = xn + (xn - x);
    a.x[idx] = xn;
    return;
  }
  x = apply_limits(a, x);
  if (a.x_mask != nullptr) x *= a.x_mask[a.mask_per_slice ? idx : pix];
  a.x[idx] = x;
}

// The MLEM / SIRT epilogue of K pixels (s, i0 + di * k, j) of one thread: the loads of tau and x
// are issued before the first store of x, which the per-pixel form cannot do (a store to x
// may alias the next pixel's loads), so that a back projection of few lines does not wait for K
// memory round trips in a row.  Same arithmetic as bp_epilogue.
template <int EPI, int K>
__device__ __forceinline__ void bp_epilogue_rows(const BpArgs& a, int s, int i0, int di, int j, const float (&v)[K]) {
  static_assert(EPI == BP_EPI_MLEM || EPI == BP_EPI_SIRT, "MLEM and SIRT epilogues only");
  const int n = a.n;
  const int64_t n2 = (int64_t)n * n;
  const float* tau = a.tau + (a.tau_shared ? 0 : (int64_t)s * n2);
  float tv[K], xv[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int i = i0 + di * k;
    const int64_t pix = (int64_t)i * n + j;
    const bool in = i < n && j < n;
    tv[k] = in ? tau[pix] : 1.f;
    xv[k] = in ? a.x[(int64_t)s * n2 + pix] : 0.f;
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int i = i0 + di * k;
    if (i >= n || j >= n) continue;
    const int64_t pix = (int64_t)i * n + j;
    // MLEM: a pixel that no line reaches (tau = 0) keeps its value, as in bp_epilogue
    float x = EPI == BP_EPI_MLEM ? (tv[k] != 0.f ? xv[k] * (v[k] / tv[k]) : xv[k]) : xv[k] + v[k] * tv[k];
    x = apply_limits(a, x);
    if (a.x_mask != nullptr) x *= a.x_mask[a.mask_per_slice ? (int64_t)s * n2 + pix : pix];
    a.x[(int64_t)s * n2 + pix] = x;
  }
}

void launch_fp(const FpArgs& a, cudaStream_t st);
bool fp_vec4_ok(const FpArgs& a);  // may the fp staging use 16-byte loads for these pointers
// PSF convolution of finished sinogram lines (a.vol = input sinogram) with the fp epilogue EPI
void launch_psf(const FpArgs& a, const float* psf, int psf_len, cudaStream_t st);
int read_device_error(int clear, int* value);
void launch_bp(const BpArgs& a, cudaStream_t st);

// Ragged launches: one grid over groups of slices (tables in device memory, CTA offsets
// start[0..n_groups], start[n_groups] = total CTAs).  Every group shares the epilogue, the
// presence and the storage type of the maps (and, for bp, the mode).
void launch_fp_ragged(const FpArgs* groups, const int64_t* start, int n_groups, int64_t ctas, int epi, bool has_maps,
                      int maps_dtype, cudaStream_t st);
void launch_bp_ragged(const BpArgs* groups, const int64_t* start, int n_groups, int64_t ctas, int epi, bool sym,
                      int maps_dtype, cudaStream_t st);

struct ResidualGroup {
  const double* partials;
  int64_t per_slice;
  double* residuals;
  int* active;
  int* iterations;
  const double* tolerance;
  double* history;
  int history_len;
};
void launch_residual_ragged(const ResidualGroup* groups, const int64_t* slice_start, int n_groups, int64_t slices,
                            cudaStream_t st);

}  // namespace cct
