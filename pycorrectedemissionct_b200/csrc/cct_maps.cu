// Attenuation maps of the XRF path (sm_100a).
//
// The reference (corrct: src/corrct/_projector_backends.py:43-99) computes, per angle and
// direction, on the image zero-padded to P = n + 2e (e = ceil((ceil(sqrt(2) n) - n) / 2)):
//   U = rotate(V, -phi)                       (scikit-image bilinear, zero outside)
//   W[r] = sum_{k<r} U[k] + U[r]/2 + U[P-1]/2  (roll + cumsum of halves along rows)
//   L = rotate(W, +phi)[e:e+n, e:e+n]
//   factor = exp(-L)
// and AttenuationVolume (corrct: src/corrct/physics/attenuation.py:105-180) multiplies the
// incident factor by the mean over sub-angles of the emitted factor of every detector.
//
// Phase 1 (maps_scan_kernel): one thread per rotated-frame column c' of one rotation job
// walks r' = 0..P-1, sampling U only where the column crosses the image (elsewhere U is
// exactly 0), keeping the running sum in FP64, and writes W (FP32) to the workspace.
// Phase 2 (maps_resample_kernel): one thread per map pixel samples W of the incident job
// and of every emitted (detector, sub-angle) job at the rotated-back position, and writes
// exp(-L_in) * mean_k exp(-L_out,k) as FP32 or BF16.  Angles are processed in passes sized
// to the caller's workspace.

#include <algorithm>
#include <cmath>

#include "cct_common.cuh"
#include "cct_internal.cuh"

namespace cct {

struct MapsPass {
  int n, P, e, n_det, n_sub, has_in, has_out, maps_dtype, n_angles;
  int a0, na;                 // angles of this pass
  int jobs_per_angle;         // has_in + has_out * n_det * n_sub
  const double* rot_in;       // [A][2][6]
  const double* rot_out;      // [A][D][n_sub][2][6]
  const float* mu_in;         // [S][n][n]
  const float* mu_out;
  float* work;                // [S][na][jobs_per_angle][P][P]
  void* maps;                 // [S][A][D][n][n]
};

__device__ __forceinline__ const double* job_matrix(const MapsPass& p, int a, int job, int which) {
  // job 0 = incident (if has_in); then emitted jobs d * n_sub + k
  if (p.has_in) {
    if (job == 0) return p.rot_in + ((int64_t)a * 2 + which) * 6;
    job -= 1;
  }
  return p.rot_out + ((((int64_t)a * p.n_det * p.n_sub) + job) * 2 + which) * 6;
}

// Bilinear sample of an (h x w) FP32 image with zero outside (scikit-image constant mode).
__device__ __forceinline__ float bilin_zero(const float* img, int h, int w, float x, float y) {
  const FloorSplit fx = floor_split(x), fy = floor_split(y);
  const int x0 = fx.i, y0 = fy.i;
  const bool xin0 = x0 >= 0 && x0 < w, xin1 = x0 + 1 >= 0 && x0 + 1 < w;
  const bool yin0 = y0 >= 0 && y0 < h, yin1 = y0 + 1 >= 0 && y0 + 1 < h;
  const float v00 = (yin0 && xin0) ? __ldg(img + (int64_t)y0 * w + x0) : 0.f;
  const float v01 = (yin0 && xin1) ? __ldg(img + (int64_t)y0 * w + x0 + 1) : 0.f;
  const float v10 = (yin1 && xin0) ? __ldg(img + (int64_t)(y0 + 1) * w + x0) : 0.f;
  const float v11 = (yin1 && xin1) ? __ldg(img + (int64_t)(y0 + 1) * w + x0 + 1) : 0.f;
  const float top = fmaf(fx.f, v01 - v00, v00);
  const float bot = fmaf(fx.f, v11 - v10, v10);
  return fmaf(fy.f, bot - top, top);
}

// Range of r' (inclusive) where the column c' samples inside (-1, n) x (-1, n) of mu, widened
// by one row each side; outside it every bilinear tap is zero padding.
__device__ __forceinline__ void column_support(double ax, double bx, double ay, double by, int n, int P,
                                               int* lo, int* hi) {
  double tlo = -1e300, thi = 1e300;
  const double lim0 = -1.0, lim1 = (double)n;
  // x(r) = ax + r bx in (lim0, lim1)
  if (fabs(bx) < 1e-12) {
    if (!(ax > lim0 && ax < lim1)) { *lo = 1; *hi = 0; return; }
  } else {
    double t0 = (lim0 - ax) / bx, t1 = (lim1 - ax) / bx;
    if (t0 > t1) { double t = t0; t0 = t1; t1 = t; }
    tlo = fmax(tlo, t0); thi = fmin(thi, t1);
  }
  if (fabs(by) < 1e-12) {
    if (!(ay > lim0 && ay < lim1)) { *lo = 1; *hi = 0; return; }
  } else {
    double t0 = (lim0 - ay) / by, t1 = (lim1 - ay) / by;
    if (t0 > t1) { double t = t0; t0 = t1; t1 = t; }
    tlo = fmax(tlo, t0); thi = fmin(thi, t1);
  }
  if (tlo > thi) { *lo = 1; *hi = 0; return; }
  *lo = max(0, (int)floor(tlo) - 1);
  *hi = min(P - 1, (int)ceil(thi) + 1);
}

__global__ void __launch_bounds__(128) maps_scan_kernel(MapsPass p) {
  const int P = p.P, n = p.n;
  const int cpr = blockIdx.x * blockDim.x + threadIdx.x;  // rotated-frame column c'
  const int job_lin = blockIdx.y;                          // (angle in pass, job)
  const int s = blockIdx.z;
  if (cpr >= P) return;
  const int ai = job_lin / p.jobs_per_angle;
  const int job = job_lin - ai * p.jobs_per_angle;
  const int a = p.a0 + ai;
  const double* Md = job_matrix(p, a, job, 0);  // rotate(-phi)
  const bool incident = p.has_in && job == 0;
  const float* mu = (incident ? p.mu_in : p.mu_out) + (int64_t)s * n * n;
  // mu coordinates = padded coordinates - e
  const float m00 = (float)Md[0], m01 = (float)Md[1], m02 = (float)(Md[2] - p.e);
  const float m10 = (float)Md[3], m11 = (float)Md[4], m12 = (float)(Md[5] - p.e);
  int lo, hi;
  column_support(Md[0] * cpr + Md[2] - p.e, Md[1], Md[3] * cpr + Md[5] - p.e, Md[4], n, P, &lo, &hi);
  const float fc = (float)cpr;
  const float xc = fmaf(m00, fc, m02), yc = fmaf(m10, fc, m12);
  float* W = p.work + (((int64_t)s * p.na + ai) * p.jobs_per_angle + job) * (int64_t)P * P + cpr;

  // wrap-around term U[P-1] / 2 of roll + cumsum
  double wrap = 0.0;
  if (P - 1 >= lo && P - 1 <= hi) {
    const float fr = (float)(P - 1);
    wrap = 0.5 * (double)bilin_zero(mu, n, n, fmaf(m01, fr, xc), fmaf(m11, fr, yc));
  }
  double acc = 0.0;
  for (int r = 0; r < P; ++r) {
    float u = 0.f;
    if (r >= lo && r <= hi) {
      const float fr = (float)r;
      u = bilin_zero(mu, n, n, fmaf(m01, fr, xc), fmaf(m11, fr, yc));
    }
    W[(int64_t)r * P] = (float)(acc + 0.5 * (double)u + wrap);
    acc += (double)u;
  }
}

__global__ void __launch_bounds__(256) maps_resample_kernel(MapsPass p) {
  const int n = p.n, P = p.P;
  const int64_t pix = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int ai = blockIdx.y;
  const int s = blockIdx.z;
  if (pix >= (int64_t)n * n) return;
  const int i = (int)(pix / n), j = (int)(pix - (int64_t)i * n);
  const int a = p.a0 + ai;
  const float X = (float)(j + p.e), Y = (float)(i + p.e);  // padded coordinates of the pixel
  const float* wbase = p.work + ((int64_t)s * p.na + ai) * p.jobs_per_angle * (int64_t)P * P;

  auto sample_job = [&](int job) -> float {
    const double* Mb = job_matrix(p, a, job, 1);  // rotate(+phi)
    const float x = fmaf((float)Mb[1], Y, fmaf((float)Mb[0], X, (float)Mb[2]));
    const float y = fmaf((float)Mb[4], Y, fmaf((float)Mb[3], X, (float)Mb[5]));
    return bilin_zero(wbase + (int64_t)job * P * P, P, P, x, y);
  };

  if (p.maps_dtype == CCT_DTYPE_FIELDS_F32) {
    // line-integral fields: plane 0 = L_in, plane 1 + d = L_out of detector d (n_sub == 1)
    float* fo = reinterpret_cast<float*>(p.maps) + ((int64_t)s * p.n_angles + a) * (1 + p.n_det) * (int64_t)n * n + pix;
    fo[0] = p.has_in ? sample_job(0) : 0.f;
    for (int d = 0; d < p.n_det; ++d)
      fo[(int64_t)(1 + d) * n * n] = p.has_out ? sample_job((p.has_in ? 1 : 0) + d) : 0.f;
    return;
  }
  float f_in = 1.f;
  int job = 0;
  if (p.has_in) {
    f_in = expf(-sample_job(0));
    job = 1;
  }
  for (int d = 0; d < p.n_det; ++d) {
    float f = f_in;
    if (p.has_out) {
      float sum = 0.f;
      for (int k = 0; k < p.n_sub; ++k) sum += expf(-sample_job(job + d * p.n_sub + k));
      f *= sum / (float)p.n_sub;
    }
    const int64_t off = (((int64_t)s * p.n_angles + a) * p.n_det + d) * (int64_t)n * n + pix;
    if (p.maps_dtype == CCT_DTYPE_BF16) {
      reinterpret_cast<__nv_bfloat16*>(p.maps)[off] = __float2bfloat16_rn(f);
    } else {
      reinterpret_cast<float*>(p.maps)[off] = f;
    }
  }
}

int padded_edge(int n) {
  // edges = ceil((ceil(sqrt(2 n^2)) - n) / 2)  (corrct: src/corrct/_projector_backends.py:75-77)
  const double min_size = ceil(sqrt(2.0 * (double)n * (double)n));
  return (int)ceil((min_size - n) / 2.0);
}

int64_t maps_bytes_per_angle(const cct_maps_desc* d) {
  const int e = padded_edge(d->n);
  const int64_t P = d->n + 2 * e;
  const int64_t jobs = (d->has_in ? 1 : 0) + (d->has_out ? (int64_t)d->n_det * d->n_sub : 0);
  return jobs * P * P * (int64_t)sizeof(float) * d->n_slices;
}

int launch_maps(const cct_maps_desc* d, const float* mu_in, const float* mu_out, void* maps, void* work,
                size_t work_bytes, cudaStream_t st) {
  const int e = padded_edge(d->n);
  const int P = d->n + 2 * e;
  const int64_t per_angle = maps_bytes_per_angle(d);
  int per_pass = (int)std::min<int64_t>((int64_t)work_bytes / per_angle, (int64_t)d->n_angles);
  if (per_pass < 1) return CCT_ERR_VALUE;
  MapsPass p;
  p.n = d->n; p.P = P; p.e = e; p.n_det = d->n_det; p.n_sub = d->n_sub;
  p.has_in = d->has_in; p.has_out = d->has_out; p.maps_dtype = d->maps_dtype; p.n_angles = d->n_angles;
  p.jobs_per_angle = (d->has_in ? 1 : 0) + (d->has_out ? d->n_det * d->n_sub : 0);
  p.rot_in = d->rot_in; p.rot_out = d->rot_out; p.mu_in = mu_in; p.mu_out = mu_out;
  p.work = reinterpret_cast<float*>(work); p.maps = maps;
  for (int a0 = 0; a0 < d->n_angles; a0 += per_pass) {
    p.a0 = a0;
    p.na = std::min(per_pass, d->n_angles - a0);
    const dim3 g1((P + 127) / 128, p.na * p.jobs_per_angle, d->n_slices);
    maps_scan_kernel<<<g1, 128, 0, st>>>(p);
    const dim3 g2((unsigned)(((int64_t)d->n * d->n + 255) / 256), p.na, d->n_slices);
    maps_resample_kernel<<<g2, 256, 0, st>>>(p);
  }
  return CCT_OK;
}

}  // namespace cct
