// Solver-side kernels of the XRF path: deterministic FP64 residual reductions with the
// per-slice stopping test, the PDHG TV dual update, and FP64 norms.

#include "cct_common.cuh"
#include "cct_internal.cuh"

namespace cct {

constexpr int RED_THREADS = 256;

__device__ __forceinline__ double block_sum_double(double v) {
  __shared__ double warp_part[RED_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum_double(v);
  if (lane == 0) warp_part[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (warp == 0) {
    t = lane < RED_THREADS / 32 ? warp_part[lane] : 0.0;
    t = warp_sum_double(t);
  }
  return t;  // valid in thread 0
}

// residual[s] = sum of the slice's partials (fixed order); counts the iteration and applies
// the reference's stopping rule `if tolerance > residual: break` (corrct solvers.py:787-791).
__global__ void __launch_bounds__(RED_THREADS) residual_step_kernel(const double* partials, int64_t per_slice,
                                                                    double* residuals, int* active, int* iterations,
                                                                    const double* tolerance, double* history,
                                                                    int history_len) {
  const int s = blockIdx.x;
  if (active[s] == 0) return;
  double v = 0.0;
  const double* p = partials + (int64_t)s * per_slice;
  for (int64_t k = threadIdx.x; k < per_slice; k += RED_THREADS) v += p[k];
  v = block_sum_double(v);
  if (threadIdx.x == 0) {
    residuals[s] = v;
    const int it = iterations[s];
    if (history != nullptr && it < history_len) history[(int64_t)s * history_len + it] = v;
    iterations[s] = it + 1;
    if (tolerance != nullptr && tolerance[s] > v) active[s] = 0;
  }
}

// PDHG TV dual: q += 0.5 grad(x_relax) (edge padding, corrct operators.py:796-816,
// regularizers.py:260-266), then q = q / max(|q|_2, lambda) * lambda (data_terms.py:549-555).
__global__ void __launch_bounds__(256) tv_dual_kernel(const float* x_relax, float* q, int n, float lam,
                                                      const int* active) {
  const int s = blockIdx.y;
  if (active != nullptr && active[s] == 0) return;
  const int64_t n2 = (int64_t)n * n;
  const int64_t pix = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= n2) return;
  const int i = (int)(pix / n), j = (int)(pix - (int64_t)i * n);
  const float* x = x_relax + (int64_t)s * n2;
  float* qs = q + (int64_t)s * 2 * n2;
  const float xc = x[pix];
  const float g0 = (i + 1 < n) ? x[pix + n] - xc : 0.f;
  const float g1 = (j + 1 < n) ? x[pix + 1] - xc : 0.f;
  float q0 = qs[pix] + 0.5f * g0;
  float q1 = qs[n2 + pix] + 0.5f * g1;
  const float nrm = sqrtf(q0 * q0 + q1 * q1);
  const float den = fmaxf(nrm, lam);
  q0 = q0 / den * lam;
  q1 = q1 / den * lam;
  qs[pix] = q0;
  qs[n2 + pix] = q1;
}

__global__ void __launch_bounds__(RED_THREADS) norm_partial_kernel(const float* v, int64_t count, int ord,
                                                                   double* partials, int blocks_per_slice) {
  const int s = blockIdx.y;
  const float* vs = v + (int64_t)s * count;
  double acc = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * RED_THREADS + threadIdx.x; k < count;
       k += (int64_t)blocks_per_slice * RED_THREADS) {
    const double e = (double)vs[k];
    acc += ord == 1 ? fabs(e) : e * e;
  }
  acc = block_sum_double(acc);
  if (threadIdx.x == 0) partials[(int64_t)s * blocks_per_slice + blockIdx.x] = acc;
}

__global__ void __launch_bounds__(RED_THREADS) norm_final_kernel(const double* partials, int blocks_per_slice,
                                                                 double* out) {
  const int s = blockIdx.x;
  double acc = 0.0;
  for (int k = threadIdx.x; k < blocks_per_slice; k += RED_THREADS) acc += partials[(int64_t)s * blocks_per_slice + k];
  acc = block_sum_double(acc);
  if (threadIdx.x == 0) out[s] = acc;
}

// Cross-validation residual of the iterate just projected (corrct solvers.py:783-785): the sum
// of the slice's test partials; recorded at the iteration index before residual_step_kernel
// counts the iteration.  No stopping test.
__global__ void __launch_bounds__(RED_THREADS) residual_test_kernel(const double* partials, int64_t per_slice,
                                                                    double* residuals, const int* active,
                                                                    const int* iterations, double* history,
                                                                    int history_len) {
  const int s = blockIdx.x;
  if (active[s] == 0) return;
  double v = 0.0;
  const double* p = partials + (int64_t)s * per_slice;
  for (int64_t k = threadIdx.x; k < per_slice; k += RED_THREADS) v += p[k];
  v = block_sum_double(v);
  if (threadIdx.x == 0) {
    residuals[s] = v;
    const int it = iterations[s];
    if (history != nullptr && it < history_len) history[(int64_t)s * history_len + it] = v;
  }
}

void launch_residual_test(const double* partials, int64_t per_slice, int n_slices, double* residuals,
                          const int* active, const int* iterations, double* history, int history_len,
                          cudaStream_t st) {
  residual_test_kernel<<<n_slices, RED_THREADS, 0, st>>>(partials, per_slice, residuals, active, iterations, history,
                                                          history_len);
}

// A 3-D volume solved as a stack of slices: the reference computes one residual norm over the
// whole volume, which for its additive norms (sum |r|, sum r^2) is the sum of the slice residuals.
// Runs after residual_step_kernel of the same iteration; one CTA, fixed summation order.
__global__ void __launch_bounds__(RED_THREADS) residual_joint_kernel(const double* residuals, int n_slices,
                                                                     int* active, const int* iterations,
                                                                     const double* tolerance, double* history,
                                                                     int history_len) {
  if (active[0] == 0) return;  // the volume met its tolerance at an earlier iteration
  double v = 0.0;
  for (int s = threadIdx.x; s < n_slices; s += RED_THREADS) v += residuals[s];
  v = block_sum_double(v);
  __shared__ int stop;
  if (threadIdx.x == 0) {
    const int it = iterations[0] - 1;
    if (history != nullptr && it >= 0 && it < history_len) history[it] = v;
    stop = (tolerance != nullptr && tolerance[0] > v) ? 1 : 0;
  }
  __syncthreads();
  if (stop)
    for (int s = threadIdx.x; s < n_slices; s += RED_THREADS) active[s] = 0;
}

void launch_residual_step(const double* partials, int64_t per_slice, int n_slices, double* residuals, int* active,
                          int* iterations, const double* tolerance, double* history, int history_len, int joint,
                          cudaStream_t st) {
  if (!joint) {
    residual_step_kernel<<<n_slices, RED_THREADS, 0, st>>>(partials, per_slice, residuals, active, iterations,
                                                            tolerance, history, history_len);
    return;
  }
  residual_step_kernel<<<n_slices, RED_THREADS, 0, st>>>(partials, per_slice, residuals, active, iterations,
                                                          nullptr, nullptr, 0);
  residual_joint_kernel<<<1, RED_THREADS, 0, st>>>(residuals, n_slices, active, iterations, tolerance, history,
                                                   history_len);
}

// residual_step_kernel over groups of slices in one launch (one CTA per slice of every group).
__global__ void __launch_bounds__(RED_THREADS) residual_ragged_kernel(const ResidualGroup* __restrict__ groups,
                                                                      const int64_t* __restrict__ start,
                                                                      int n_groups) {
  const int64_t gs = blockIdx.x;
  int lo = 0, hi = n_groups - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (start[mid] <= gs) lo = mid; else hi = mid - 1;
  }
  const ResidualGroup& g = groups[lo];
  const int s = (int)(gs - start[lo]);
  if (g.active[s] == 0) return;
  double v = 0.0;
  const double* p = g.partials + (int64_t)s * g.per_slice;
  for (int64_t k = threadIdx.x; k < g.per_slice; k += RED_THREADS) v += p[k];
  v = block_sum_double(v);
  if (threadIdx.x == 0) {
    g.residuals[s] = v;
    const int it = g.iterations[s];
    if (g.history != nullptr && it < g.history_len) g.history[(int64_t)s * g.history_len + it] = v;
    g.iterations[s] = it + 1;
    if (g.tolerance != nullptr && g.tolerance[s] > v) g.active[s] = 0;
  }
}

void launch_residual_ragged(const ResidualGroup* groups, const int64_t* slice_start, int n_groups, int64_t slices,
                            cudaStream_t st) {
  residual_ragged_kernel<<<(unsigned)slices, RED_THREADS, 0, st>>>(groups, slice_start, n_groups);
}

void launch_tv_dual(const float* x_relax, float* q, int n, int n_slices, float lam, const int* active,
                    cudaStream_t st) {
  const dim3 grid((unsigned)(((int64_t)n * n + 255) / 256), n_slices);
  tv_dual_kernel<<<grid, 256, 0, st>>>(x_relax, q, n, lam, active);
}

int norm_blocks_per_slice(int64_t count) {
  const int64_t b = (count + RED_THREADS * 8 - 1) / (RED_THREADS * 8);
  return (int)(b < 1 ? 1 : (b > 1024 ? 1024 : b));
}

void launch_norm(const float* v, int64_t count, int n_slices, int ord, double* out, double* partials,
                 cudaStream_t st) {
  const int bps = norm_blocks_per_slice(count);
  norm_partial_kernel<<<dim3(bps, n_slices), RED_THREADS, 0, st>>>(v, count, ord, partials, bps);
  norm_final_kernel<<<n_slices, RED_THREADS, 0, st>>>(partials, bps, out);
}

}  // namespace cct
