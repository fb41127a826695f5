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
// exactly 0; where all four taps are inside the image, without per-tap tests), keeping the
// running sum in FP64, and writes W (FP32) to the workspace.
// Phase 2 (maps_resample_kernel): one thread per map pixel samples W of the incident job
// and of every emitted (detector, sub-angle) job at the rotated-back position, and writes
// exp(-L_in) * mean_k exp(-L_out,k) as FP32 or BF16.  Angles are processed in passes sized
// to the caller's workspace.
// Half-turn pairs: for angles phi and phi + pi every rotation of the second is the first's turned
// by 180 degrees about the frame centre, a permutation of the lattice.  Its W at the first's
// (r', c') is then K[c'] - W[r'][c'] with the per-column constant K = sum U + U[0]/2 + U[P-1]/2,
// and its rotate-back samples sit at the same positions; one scan and one resample per direction
// give both angles' maps.

#include <algorithm>
#include <cmath>

#include "cct_common.cuh"
#include "cct_internal.cuh"

namespace cct {

struct MapsPass {
  int n, P, e, n_det, n_sub, has_in, has_out, maps_dtype, n_angles;
  int a0, na;                 // first entry (first quad with quads) and scanned entries of this pass
  int n_entries;              // entries of `pairs` (angles without)
  int jobs_per_angle;         // has_in + has_out * n_det * n_sub
  const double* rot_in;       // [A][2][6]
  const double* rot_out;      // [A][D][n_sub][2][6]
  const int* pairs;           // [entries][2] (angle, partner) or NULL
  const int* quads;           // [quads][6] (entry, entry', emitted source of the 4 angles) or NULL
  float emitted_scale;        // quads: mu_out = emitted_scale * mu_in
  const float* mu_in;         // [S][n][n]
  const float* mu_out;
  const float* mu_in_t;       // [S][n][n] transposed copies (mu_t[s][x][y] = mu[s][y][x]) or NULL
  const float* mu_out_t;
  float* work;                // [S][na][jobs_per_angle][P][P]
  float* kcol;                // [S][na][jobs_per_angle][P] per-column constants of the partner scans
  void* maps;                 // [S][A][D][n][n]
};

// Entry scanned in slot ai of the pass: with quads, slots 2q and 2q + 1 are quad (a0 + q)'s two
// entries (a0 counts quads); otherwise slot ai is entry a0 + ai.
__device__ __forceinline__ int slot_entry(const MapsPass& p, int ai) {
  if (p.quads == nullptr) return p.a0 + ai;
  return p.quads[6 * (p.a0 + (ai >> 1)) + (ai & 1)];
}

// Angle of entry e and its half-turn partner (-1: none); a = -1 for an out-of-range entry.
__device__ __forceinline__ void entry_angles(const MapsPass& p, int e, int* a, int* b) {
  if (e < 0 || e >= p.n_entries) {
    *a = *b = -1;
    return;
  }
  if (p.pairs == nullptr) {
    *a = e;
    *b = -1;
    return;
  }
  const int aa = p.pairs[2 * e], bb = p.pairs[2 * e + 1];
  *a = (aa >= 0 && aa < p.n_angles) ? aa : -1;
  *b = (bb >= 0 && bb < p.n_angles && bb != aa) ? bb : -1;
}

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

// Bilinear sample whose four taps are known to lie inside the (w x hgt) image.  The clamps are
// no-ops for such coordinates; they only keep every access in bounds.  Same arithmetic as
// bilin_zero.
__device__ __forceinline__ float bilin_inside(const float* img, int w, int hgt, float x, float y) {
  const FloorSplit fx = floor_split(x), fy = floor_split(y);
  const int x0 = min(max(fx.i, 0), w - 2), y0 = min(max(fy.i, 0), hgt - 2);
  const float* q = img + (int64_t)y0 * w + x0;
  const float v00 = __ldg(q), v01 = __ldg(q + 1), v10 = __ldg(q + w), v11 = __ldg(q + w + 1);
  const float top = fmaf(fx.f, v01 - v00, v00);
  const float bot = fmaf(fx.f, v11 - v10, v10);
  return fmaf(fy.f, bot - top, top);
}

// The same two samplers on an n x n image whose element (y, x) sits at y * sy + x * sx: row-major
// (sy, sx) = (n, 1) or transposed (1, n).  The taps and the arithmetic are those of bilin_zero /
// bilin_inside, so both layouts give bit-identical samples; the layout only decides which lanes
// of a warp share memory sectors.
__device__ __forceinline__ float bilin_zero_mu(const float* img, int n, int sy, int sx, float x, float y) {
  const FloorSplit fx = floor_split(x), fy = floor_split(y);
  const int x0 = fx.i, y0 = fy.i;
  const bool xin0 = x0 >= 0 && x0 < n, xin1 = x0 + 1 >= 0 && x0 + 1 < n;
  const bool yin0 = y0 >= 0 && y0 < n, yin1 = y0 + 1 >= 0 && y0 + 1 < n;
  const int64_t q = (int64_t)y0 * sy + (int64_t)x0 * sx;
  const float v00 = (yin0 && xin0) ? __ldg(img + q) : 0.f;
  const float v01 = (yin0 && xin1) ? __ldg(img + q + sx) : 0.f;
  const float v10 = (yin1 && xin0) ? __ldg(img + q + sy) : 0.f;
  const float v11 = (yin1 && xin1) ? __ldg(img + q + sx + sy) : 0.f;
  const float top = fmaf(fx.f, v01 - v00, v00);
  const float bot = fmaf(fx.f, v11 - v10, v10);
  return fmaf(fy.f, bot - top, top);
}

__device__ __forceinline__ float bilin_inside_mu(const float* img, int n, int sy, int sx, float x, float y) {
  const FloorSplit fx = floor_split(x), fy = floor_split(y);
  const int x0 = min(max(fx.i, 0), n - 2), y0 = min(max(fy.i, 0), n - 2);
  const float* q = img + (y0 * sy + x0 * sx);  // < n * n
  const float v00 = __ldg(q), v01 = __ldg(q + sx), v10 = __ldg(q + sy), v11 = __ldg(q + sx + sy);
  const float top = fmaf(fx.f, v01 - v00, v00);
  const float bot = fmaf(fx.f, v11 - v10, v10);
  return fmaf(fy.f, bot - top, top);
}

// Bilinear sample of a (P x P) image with zero outside: one range test picks the unchecked
// four-tap load for interior coordinates, bilin_zero otherwise.
__device__ __forceinline__ float bilin_square(const float* img, int P, float x, float y) {
  const FloorSplit fx = floor_split(x), fy = floor_split(y);
  if ((unsigned)fx.i < (unsigned)(P - 1) && (unsigned)fy.i < (unsigned)(P - 1)) {
    const float* q = img + (int64_t)fy.i * P + fx.i;
    const float v00 = __ldg(q), v01 = __ldg(q + 1), v10 = __ldg(q + P), v11 = __ldg(q + P + 1);
    const float top = fmaf(fx.f, v01 - v00, v00);
    const float bot = fmaf(fx.f, v11 - v10, v10);
    return fmaf(fy.f, bot - top, top);
  }
  return bilin_zero(img, P, P, x, y);
}

// Bilinear samples at (x, y) of a (P x P) image W and of the partner field K[c] - W[r][c]
// (zero outside the frame for both).  *La is bilin_square(W) exactly.  Inside the frame the
// partner's sample is the x-interpolated column constant minus *La (bilinear interpolation is
// linear and K does not vary along rows); at the frame edge, where the partner field is zero
// outside, its four taps are interpolated.
__device__ __forceinline__ void bilin_square_pair(const float* img, const float* K, int P, float x, float y,
                                                  float* La, float* Lb) {
  const FloorSplit fx = floor_split(x), fy = floor_split(y);
  const int x0 = fx.i, y0 = fy.i;
  float v00, v01, v10, v11, u00, u01, u10, u11;
  if ((unsigned)x0 < (unsigned)(P - 1) && (unsigned)y0 < (unsigned)(P - 1)) {
    const float* q = img + (int64_t)y0 * P + x0;
    v00 = __ldg(q); v01 = __ldg(q + 1); v10 = __ldg(q + P); v11 = __ldg(q + P + 1);
    const float k0 = __ldg(K + x0), k1 = __ldg(K + x0 + 1);
    const float top = fmaf(fx.f, v01 - v00, v00);
    const float bot = fmaf(fx.f, v11 - v10, v10);
    *La = fmaf(fy.f, bot - top, top);
    *Lb = fmaf(fx.f, k1 - k0, k0) - *La;
    return;
  } else {
    const bool xin0 = x0 >= 0 && x0 < P, xin1 = x0 + 1 >= 0 && x0 + 1 < P;
    const bool yin0 = y0 >= 0 && y0 < P, yin1 = y0 + 1 >= 0 && y0 + 1 < P;
    const float k0 = xin0 ? __ldg(K + x0) : 0.f, k1 = xin1 ? __ldg(K + x0 + 1) : 0.f;
    v00 = (yin0 && xin0) ? __ldg(img + (int64_t)y0 * P + x0) : 0.f;
    v01 = (yin0 && xin1) ? __ldg(img + (int64_t)y0 * P + x0 + 1) : 0.f;
    v10 = (yin1 && xin0) ? __ldg(img + (int64_t)(y0 + 1) * P + x0) : 0.f;
    v11 = (yin1 && xin1) ? __ldg(img + (int64_t)(y0 + 1) * P + x0 + 1) : 0.f;
    u00 = (yin0 && xin0) ? k0 - v00 : 0.f;
    u01 = (yin0 && xin1) ? k1 - v01 : 0.f;
    u10 = (yin1 && xin0) ? k0 - v10 : 0.f;
    u11 = (yin1 && xin1) ? k1 - v11 : 0.f;
  }
  const float top = fmaf(fx.f, v01 - v00, v00);
  const float bot = fmaf(fx.f, v11 - v10, v10);
  *La = fmaf(fy.f, bot - top, top);
  const float topb = fmaf(fx.f, u01 - u00, u00);
  const float botb = fmaf(fx.f, u11 - u10, u10);
  *Lb = fmaf(fy.f, botb - topb, topb);
}

// Integer r in [*lo, *hi] with x(r) = ax + r bx and y(r) = ay + r by both in [lim0, lim1]
// (exact arithmetic), clipped to [0, P - 1]; *lo > *hi when there is none.
__device__ __forceinline__ void column_inside(double ax, double bx, double ay, double by, double lim0, double lim1,
                                              int P, int* lo, int* hi) {
  double tlo = -1e300, thi = 1e300;
  if (fabs(bx) < 1e-12) {
    if (!(ax >= lim0 && ax <= lim1)) { *lo = 1; *hi = 0; return; }
  } else {
    double t0 = (lim0 - ax) / bx, t1 = (lim1 - ax) / bx;
    if (t0 > t1) { double t = t0; t0 = t1; t1 = t; }
    tlo = fmax(tlo, t0); thi = fmin(thi, t1);
  }
  if (fabs(by) < 1e-12) {
    if (!(ay >= lim0 && ay <= lim1)) { *lo = 1; *hi = 0; return; }
  } else {
    double t0 = (lim0 - ay) / by, t1 = (lim1 - ay) / by;
    if (t0 > t1) { double t = t0; t0 = t1; t1 = t; }
    tlo = fmax(tlo, t0); thi = fmin(thi, t1);
  }
  if (tlo > thi) { *lo = 1; *hi = 0; return; }
  *lo = (int)fmax(0.0, ceil(tlo));
  *hi = (int)fmin((double)(P - 1), floor(thi));
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

// One thread per column; the 32 columns of a warp walk the rows in lockstep (coalesced W
// stores), with warp-uniform row ranges: no lane samples before the warp's first support row or
// after its last, and rows where every lane's four taps are inside mu skip the per-tap tests.
template <bool PAIRS>
__global__ void __launch_bounds__(128) maps_scan_kernel(MapsPass p) {
  const int P = p.P, n = p.n;
  const int cpr_raw = blockIdx.x * blockDim.x + threadIdx.x;  // rotated-frame column c'
  const bool valid = cpr_raw < P;
  const int cpr = valid ? cpr_raw : P - 1;  // lanes past the frame shadow the last column, store nothing
  const int job_lin = blockIdx.y;           // (angle in pass, job)
  const int s = blockIdx.z;
  const int ai = job_lin / p.jobs_per_angle;
  const int job = job_lin - ai * p.jobs_per_angle;
  int a, b;
  entry_angles(p, slot_entry(p, ai), &a, &b);
  if (a < 0) return;  // the whole CTA
  const double* Md = job_matrix(p, a, job, 0);  // rotate(-phi)
  const bool incident = p.has_in && job == 0;
  // the lanes of a warp step along (m00, m10) in mu: where that is closer to y than to x, the
  // transposed copy (if given) puts neighbouring lanes in neighbouring memory
  const float* mu_t = incident ? p.mu_in_t : p.mu_out_t;
  const bool tr = mu_t != nullptr && fabs(Md[3]) > fabs(Md[0]);
  const float* mu = (tr ? mu_t : (incident ? p.mu_in : p.mu_out)) + (int64_t)s * n * n;
  const int sy = tr ? 1 : n, sx = tr ? n : 1;  // element (y, x) of mu at y * sy + x * sx
  // mu coordinates = padded coordinates - e
  const float m00 = (float)Md[0], m01 = (float)Md[1], m02 = (float)(Md[2] - p.e);
  const float m10 = (float)Md[3], m11 = (float)Md[4], m12 = (float)(Md[5] - p.e);
  const double ax = Md[0] * cpr + Md[2] - p.e, ay = Md[3] * cpr + Md[5] - p.e;
  int lo, hi;
  column_support(ax, Md[1], ay, Md[4], n, P, &lo, &hi);
  if (lo > hi) { lo = P; hi = -1; }
  // rows whose four taps all lie inside mu, with a 0.01-pixel margin against the FP32
  // evaluation of the coordinates below
  int ilo = P, ihi = -1;
  if (n >= 2) column_inside(ax, Md[1], ay, Md[4], 0.01, (double)n - 1.01, P, &ilo, &ihi);
  ilo = max(ilo, lo);
  ihi = min(ihi, hi);
  if (ilo > ihi) { ilo = P; ihi = -1; }
  int wlo = lo, whi = hi, wilo = ilo, wihi = ihi;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    wlo = min(wlo, __shfl_xor_sync(0xffffffffu, wlo, o));
    whi = max(whi, __shfl_xor_sync(0xffffffffu, whi, o));
    wilo = max(wilo, __shfl_xor_sync(0xffffffffu, wilo, o));
    wihi = min(wihi, __shfl_xor_sync(0xffffffffu, wihi, o));
  }
  if (wilo > wihi) { wilo = whi + 1; wihi = whi; }  // no row is inside for every lane
  const float fc = (float)cpr;
  const float xc = fmaf(m00, fc, m02), yc = fmaf(m10, fc, m12);
  float* W = p.work + (((int64_t)s * p.na + ai) * p.jobs_per_angle + job) * (int64_t)P * P + cpr;

  // wrap-around term U[P-1] / 2 of roll + cumsum
  double wrap = 0.0;
  if (P - 1 >= lo && P - 1 <= hi) {
    const float fr = (float)(P - 1);
    wrap = 0.5 * (double)bilin_zero_mu(mu, n, sy, sx, fmaf(m01, fr, xc), fmaf(m11, fr, yc));
  }
  // W[r] = acc + U[r]/2 + wrap with acc = sum_{k<r} U[k] (FP64); U = 0 outside [lo, hi].  Only
  // the warp's rows [wlo, whi] are stored: outside them W is constant per column and the
  // resample, whose positions all map back into the image, never reads it there
  // (tests/test_host.py::test_maps_resample_reads_only_scanned_rows mirrors that arithmetic).
  double acc = 0.0;
  int r = wlo;
  for (; r < wilo; ++r) {
    const float fr = (float)r;
    const float u = (r >= lo && r <= hi) ? bilin_zero_mu(mu, n, sy, sx, fmaf(m01, fr, xc), fmaf(m11, fr, yc)) : 0.f;
    if (valid) W[(int64_t)r * P] = (float)(acc + 0.5 * (double)u + wrap);
    acc += (double)u;
  }
  for (; r + 3 <= wihi; r += 4) {
    float u[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float fr = (float)(r + k);
      u[k] = bilin_inside_mu(mu, n, sy, sx, fmaf(m01, fr, xc), fmaf(m11, fr, yc));
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (valid) W[(int64_t)(r + k) * P] = (float)(acc + 0.5 * (double)u[k] + wrap);
      acc += (double)u[k];
    }
  }
  for (; r <= wihi; ++r) {
    const float fr = (float)r;
    const float u = bilin_inside_mu(mu, n, sy, sx, fmaf(m01, fr, xc), fmaf(m11, fr, yc));
    if (valid) W[(int64_t)r * P] = (float)(acc + 0.5 * (double)u + wrap);
    acc += (double)u;
  }
  for (; r <= whi; ++r) {
    const float fr = (float)r;
    const float u = (r >= lo && r <= hi) ? bilin_zero_mu(mu, n, sy, sx, fmaf(m01, fr, xc), fmaf(m11, fr, yc)) : 0.f;
    if (valid) W[(int64_t)r * P] = (float)(acc + 0.5 * (double)u + wrap);
    acc += (double)u;
  }
  if (PAIRS && b >= 0 && valid) {
    // the partner angle (phi + pi) rotates by a half turn more: its frame is this one turned
    // about the centre, and its W at this frame's (r', c') is K[c'] - W[r'][c'] with
    // K = sum_k U[k] + U[0]/2 + U[P-1]/2 (the reverse roll + cumsum of the same column)
    double first = 0.0;
    if (0 >= lo && 0 <= hi) first = 0.5 * (double)bilin_zero_mu(mu, n, sy, sx, xc, yc);
    p.kcol[(((int64_t)s * p.na + ai) * p.jobs_per_angle + job) * P + cpr] = (float)(acc + first + wrap);
  }
}

// One CTA = a 32 x 32 pixel tile of one (slice, angle); thread t owns the four pixels
// (x, y + 8k), k < 4, so that each warp instruction covers an 8-wide, 4-tall block whose taps
// fall in a compact patch of the rotated frame.  The rotate(+phi) matrices of the angle's jobs
// are converted to FP32 once per CTA into shared memory.
constexpr int RS_TILE = 32;
constexpr int RS_PIX = 4;

template <bool PAIRS>
__global__ void __launch_bounds__(256, PAIRS ? 5 : 1) maps_resample_kernel(MapsPass p) {
  extern __shared__ float rs_mats[];  // [jobs_per_angle][6]
  const int n = p.n, P = p.P;
  const int ai = blockIdx.y;
  const int s = blockIdx.z;
  int a, b;
  entry_angles(p, p.a0 + ai, &a, &b);
  if (a < 0) return;  // the whole CTA
  const bool paired = PAIRS && b >= 0;
  const int J = p.jobs_per_angle;
  for (int t = threadIdx.x; t < 6 * J; t += blockDim.x) {
    const int job = t / 6;
    rs_mats[t] = (float)job_matrix(p, a, job, 1)[t - job * 6];
  }
  __syncthreads();
  const int tiles_x = (n + RS_TILE - 1) / RS_TILE;
  const int ty = blockIdx.x / tiles_x, tx = blockIdx.x - ty * tiles_x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = tx * RS_TILE + (warp & 3) * 8 + (lane & 7);
  const int i0 = ty * RS_TILE + (warp >> 2) * 4 + (lane >> 3);
  if (j >= n || i0 >= n) return;
  const float X = (float)(j + p.e);  // padded coordinates of the pixels
  const float* wbase = p.work + ((int64_t)s * p.na + ai) * J * (int64_t)P * P;
  const int64_t n2 = (int64_t)n * n;

  const float* kbase = p.kcol + ((int64_t)s * p.na + ai) * J * (int64_t)P;

  // L of job `job` at the four pixels, and with a partner its L at the same pixels (pixels
  // past the image edge are sampled, in bounds, and not stored)
  auto sample4 = [&](int job, float* L, float* Lb) {
    const float* m = rs_mats + job * 6;
    const float* w = wbase + (int64_t)job * P * P;
    const float* kc = kbase + (int64_t)job * P;
#pragma unroll
    for (int k = 0; k < RS_PIX; ++k) {
      const float Y = (float)(i0 + 8 * k + p.e);
      const float x = fmaf(m[1], Y, fmaf(m[0], X, m[2]));
      const float y = fmaf(m[4], Y, fmaf(m[3], X, m[5]));
      if (PAIRS && paired) {
        bilin_square_pair(w, kc, P, x, y, &L[k], &Lb[k]);
      } else {
        L[k] = bilin_square(w, P, x, y);
      }
    }
  };
  auto store4 = [&](int64_t plane, const float* v) {
#pragma unroll
    for (int k = 0; k < RS_PIX; ++k) {
      const int i = i0 + 8 * k;
      if (i >= n) break;
      const int64_t off = plane * n2 + (int64_t)i * n + j;
      if (p.maps_dtype == CCT_DTYPE_BF16) {
        reinterpret_cast<__nv_bfloat16*>(p.maps)[off] = __float2bfloat16_rn(v[k]);
      } else {
        reinterpret_cast<float*>(p.maps)[off] = v[k];
      }
    }
  };

  float L[RS_PIX], Lb[RS_PIX];
  if (p.maps_dtype == CCT_DTYPE_FIELDS_F32) {
    // line-integral fields: plane 0 = L_in, plane 1 + d = L_out of detector d (n_sub == 1)
    const int64_t plane0 = ((int64_t)s * p.n_angles + a) * (1 + p.n_det);
    const int64_t plane0b = ((int64_t)s * p.n_angles + b) * (1 + p.n_det);
    if (p.has_in) {
      sample4(0, L, Lb);
    } else {
#pragma unroll
      for (int k = 0; k < RS_PIX; ++k) L[k] = Lb[k] = 0.f;
    }
    store4(plane0, L);
    if (paired) store4(plane0b, Lb);
    for (int d = 0; d < p.n_det; ++d) {
      if (p.has_out) {
        sample4((p.has_in ? 1 : 0) + d, L, Lb);
      } else {
#pragma unroll
        for (int k = 0; k < RS_PIX; ++k) L[k] = Lb[k] = 0.f;
      }
      store4(plane0 + 1 + d, L);
      if (paired) store4(plane0b + 1 + d, Lb);
    }
    return;
  }
  float f_in[RS_PIX], f_inb[RS_PIX];
  int job = 0;
  if (p.has_in) {
    sample4(0, L, Lb);
#pragma unroll
    for (int k = 0; k < RS_PIX; ++k) {
      f_in[k] = __expf(-L[k]);
      f_inb[k] = paired ? __expf(-Lb[k]) : 1.f;
    }
    job = 1;
  } else {
#pragma unroll
    for (int k = 0; k < RS_PIX; ++k) f_in[k] = f_inb[k] = 1.f;
  }
  for (int d = 0; d < p.n_det; ++d) {
    float f[RS_PIX], fb[RS_PIX];
#pragma unroll
    for (int k = 0; k < RS_PIX; ++k) {
      f[k] = f_in[k];
      fb[k] = f_inb[k];
    }
    if (p.has_out) {
      float sum[RS_PIX] = {0.f, 0.f, 0.f, 0.f}, sumb[RS_PIX] = {0.f, 0.f, 0.f, 0.f};
      for (int q = 0; q < p.n_sub; ++q) {
        sample4(job + d * p.n_sub + q, L, Lb);
#pragma unroll
        for (int k = 0; k < RS_PIX; ++k) {
          sum[k] += __expf(-L[k]);
          if (paired) sumb[k] += __expf(-Lb[k]);
        }
      }
      if (p.n_sub == 1) {
#pragma unroll
        for (int k = 0; k < RS_PIX; ++k) {
          f[k] *= sum[k];
          fb[k] *= sumb[k];
        }
      } else {
        const float ns = (float)p.n_sub;
#pragma unroll
        for (int k = 0; k < RS_PIX; ++k) {
          f[k] *= sum[k] / ns;
          fb[k] *= sumb[k] / ns;
        }
      }
    }
    store4(((int64_t)s * p.n_angles + a) * p.n_det + d, f);
    if (paired) store4(((int64_t)s * p.n_angles + b) * p.n_det + d, fb);
  }
}

// Quarter-turn quads (one point detector whose emitted direction is the incident direction of
// another angle of the set, mu_out = emitted_scale * mu_in): the pass scanned only incident
// fields, two per quad (slots 2q, 2q + 1), each a half-turn pair of angles.  At every pixel the two
// pair samples give the incident line integrals L[0..3] of the quad's four angles (entry e's angle
// and partner, entry e''s angle and partner); the map of angle k is
// exp(-L[k]) * exp(-emitted_scale * L[src[k]]), src[k] naming which of the four angles the
// emitted direction of angle k is (its rotation angle differs from the reference's emitted angle
// only by the float32 rounding of the angles, like a half-turn partner's).  Four maps from two
// gathers per pixel, where the per-pair resample needs two gathers for two maps.
__global__ void __launch_bounds__(256, 5) maps_resample_quad_kernel(MapsPass p) {
  __shared__ float qm[2][6];  // rotate(+phi) matrices of the two entries' angles
  __shared__ int qa[4];       // the four angles
  __shared__ int qs[4];       // emitted sources
  const int n = p.n, P = p.P;
  const int qi = blockIdx.y;
  const int s = blockIdx.z;
  const int* row = p.quads + 6 * (p.a0 + qi);
  if (threadIdx.x < 2) {
    int a, b;
    entry_angles(p, slot_entry(p, 2 * qi + threadIdx.x), &a, &b);
    qa[2 * threadIdx.x] = a;
    qa[2 * threadIdx.x + 1] = b;
  }
  if (threadIdx.x >= 32 && threadIdx.x < 36) qs[threadIdx.x - 32] = row[2 + threadIdx.x - 32];
  __syncthreads();
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 4; ++k) ok = ok && qa[k] >= 0 && qs[k] >= 0 && qs[k] < 4;
  if (!ok) return;  // the whole CTA (only complete quads are valid)
  if (threadIdx.x < 12) {
    const int w = threadIdx.x / 6;
    qm[w][threadIdx.x - 6 * w] = (float)job_matrix(p, qa[2 * w], 0, 1)[threadIdx.x - 6 * w];
  }
  __syncthreads();
  const int tiles_x = (n + RS_TILE - 1) / RS_TILE;
  const int ty = blockIdx.x / tiles_x, tx = blockIdx.x - ty * tiles_x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = tx * RS_TILE + (warp & 3) * 8 + (lane & 7);
  const int i0 = ty * RS_TILE + (warp >> 2) * 4 + (lane >> 3);
  if (j >= n || i0 >= n) return;
  const float X = (float)(j + p.e);
  const int64_t n2 = (int64_t)n * n;
  const float sc = p.emitted_scale;
  float L[4][RS_PIX];
#pragma unroll
  for (int w = 0; w < 2; ++w) {
    const float* m = qm[w];
    const int slot = 2 * qi + w;
    const float* wf = p.work + ((int64_t)s * p.na + slot) * (int64_t)P * P;
    const float* kc = p.kcol + ((int64_t)s * p.na + slot) * (int64_t)P;
#pragma unroll
    for (int k = 0; k < RS_PIX; ++k) {
      const float Y = (float)(i0 + 8 * k + p.e);
      const float x = fmaf(m[1], Y, fmaf(m[0], X, m[2]));
      const float y = fmaf(m[4], Y, fmaf(m[3], X, m[5]));
      bilin_square_pair(wf, kc, P, x, y, &L[2 * w][k], &L[2 * w + 1][k]);
    }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int src = qs[q];
    const int64_t plane = (int64_t)s * p.n_angles + qa[q];  // n_det == 1
#pragma unroll
    for (int k = 0; k < RS_PIX; ++k) {
      const int i = i0 + 8 * k;
      if (i >= n) break;
      const float le = src == 0 ? L[0][k] : (src == 1 ? L[1][k] : (src == 2 ? L[2][k] : L[3][k]));
      const float v = __expf(-L[q][k]) * __expf(-sc * le);
      const int64_t off = plane * n2 + (int64_t)i * n + j;
      if (p.maps_dtype == CCT_DTYPE_BF16) {
        reinterpret_cast<__nv_bfloat16*>(p.maps)[off] = __float2bfloat16_rn(v);
      } else {
        reinterpret_cast<float*>(p.maps)[off] = v;
      }
    }
  }
}

int padded_edge(int n) {
  // edges = ceil((ceil(sqrt(2 n^2)) - n) / 2)  (corrct: src/corrct/_projector_backends.py:75-77)
  const double min_size = ceil(sqrt(2.0 * (double)n * (double)n));
  return (int)ceil((min_size - n) / 2.0);
}

// mu_t[s][x][y] = mu[s][y][x] for the scan's transposed reads (32 x 32 tiles through shared
// memory, coalesced on both sides).
__global__ void __launch_bounds__(256) maps_transpose_kernel(const float* __restrict__ src, float* __restrict__ dst,
                                                             int n) {
  __shared__ float t[32][33];
  const int64_t off = (int64_t)blockIdx.z * n * n;
  const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int y = y0 + k, x = x0 + threadIdx.x;
    if (y < n && x < n) t[k][threadIdx.x] = src[off + (int64_t)y * n + x];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int x = x0 + k, y = y0 + threadIdx.x;
    if (x < n && y < n) dst[off + (int64_t)x * n + y] = t[threadIdx.x][k];
  }
}

static size_t transposed_bytes(const cct_maps_desc* d) {
  const size_t b = (size_t)d->n * d->n * sizeof(float) * d->n_slices;
  return (b + 255) & ~(size_t)255;
}

static void launch_transpose(const float* src, float* dst, int n, int slices, cudaStream_t st) {
  const int t = (n + 31) / 32;
  maps_transpose_kernel<<<dim3(t, t, slices), dim3(32, 8), 0, st>>>(src, dst, n);
}

// Entries per pass and whether the workspace also holds `copies` transposed copies of mu at its
// start: they are used when, after them, at least half the entries of a pass without them fit.
static int plan_pass(const cct_maps_desc* d, size_t work_bytes, int64_t per_entry, int entries, int copies,
                     size_t* prefix) {
  const int64_t plain = std::min<int64_t>((int64_t)work_bytes / per_entry, entries);
  const size_t tb = (size_t)copies * transposed_bytes(d);
  const int64_t with_t = work_bytes > tb ? std::min<int64_t>((int64_t)(work_bytes - tb) / per_entry, entries) : 0;
  if (copies > 0 && with_t >= 1 && 2 * with_t >= plain) {
    *prefix = tb;
    return (int)with_t;
  }
  *prefix = 0;
  return (int)plain;
}

int64_t maps_bytes_per_angle(const cct_maps_desc* d) {
  const int e = padded_edge(d->n);
  const int64_t P = d->n + 2 * e;
  const int64_t jobs = (d->has_in ? 1 : 0) + (d->has_out ? (int64_t)d->n_det * d->n_sub : 0);
  return jobs * (P * P + P) * (int64_t)sizeof(float) * d->n_slices;  // W planes + partner constants
}

// Quarter-turn quads: per pass, the incident fields of 2 entries per quad (one job each, so a quad
// takes the workspace of one entry with incident and emitted jobs), then one quad resample.
static int launch_maps_quads(const cct_maps_desc* d, const float* mu_in, void* maps, void* work, size_t work_bytes,
                             cudaStream_t st) {
  const int e = padded_edge(d->n);
  const int P = d->n + 2 * e;
  const int64_t per_quad = 2 * ((int64_t)P * P + P) * (int64_t)sizeof(float) * d->n_slices;
  size_t prefix = 0;
  int per_pass = plan_pass(d, work_bytes, per_quad, d->n_quads, 1, &prefix);
  if (per_pass < 1) return CCT_ERR_VALUE;
  per_pass = std::min(per_pass, 65535 / 2);
  MapsPass p;
  p.mu_in_t = p.mu_out_t = nullptr;
  if (prefix > 0) {
    p.mu_in_t = reinterpret_cast<float*>(work);
    launch_transpose(mu_in, const_cast<float*>(p.mu_in_t), d->n, d->n_slices, st);
    work = reinterpret_cast<char*>(work) + prefix;
  }
  p.n = d->n; p.P = P; p.e = e; p.n_det = 1; p.n_sub = 1;
  p.has_in = 1; p.has_out = 0; p.maps_dtype = d->maps_dtype; p.n_angles = d->n_angles;
  p.jobs_per_angle = 1;
  p.rot_in = d->rot_in; p.rot_out = d->rot_out; p.pairs = d->pairs; p.mu_in = mu_in; p.mu_out = nullptr;
  p.quads = d->quads; p.emitted_scale = d->emitted_scale; p.n_entries = d->n_entries;
  p.work = reinterpret_cast<float*>(work); p.maps = maps;
  p.kcol = p.work + (int64_t)2 * per_pass * (int64_t)P * P * d->n_slices;
  const int tiles = (d->n + RS_TILE - 1) / RS_TILE;
  for (int q0 = 0; q0 < d->n_quads; q0 += per_pass) {
    const int nq = std::min(per_pass, d->n_quads - q0);
    p.a0 = q0;
    p.na = 2 * nq;
    maps_scan_kernel<true><<<dim3((P + 127) / 128, p.na, d->n_slices), 128, 0, st>>>(p);
    maps_resample_quad_kernel<<<dim3((unsigned)(tiles * tiles), nq, d->n_slices), 256, 0, st>>>(p);
  }
  return CCT_OK;
}

int launch_maps(const cct_maps_desc* d, const float* mu_in, const float* mu_out, void* maps, void* work,
                size_t work_bytes, cudaStream_t st) {
  const int e = padded_edge(d->n);
  const int P = d->n + 2 * e;
  const int64_t per_angle = maps_bytes_per_angle(d);
  const int entries = d->pairs != nullptr ? d->n_entries : d->n_angles;
  if (entries < 1 || entries > d->n_angles) return CCT_ERR_VALUE;
  if (d->quads != nullptr) return launch_maps_quads(d, mu_in, maps, work, work_bytes, st);
  // transposed copies of mu_in and of a distinct mu_out
  const bool out_own = d->has_out && (!d->has_in || mu_out != mu_in);
  const int copies = (d->has_in ? 1 : 0) + (out_own ? 1 : 0);
  size_t prefix = 0;
  int per_pass = plan_pass(d, work_bytes, per_angle, entries, copies, &prefix);
  if (per_pass < 1) return CCT_ERR_VALUE;
  // the scan grid's y dimension is entries x jobs (at most 65535): small slices with a large
  // workspace take more passes instead
  const int jobs = (d->has_in ? 1 : 0) + (d->has_out ? d->n_det * d->n_sub : 0);
  per_pass = std::max(1, std::min(per_pass, 65535 / std::max(1, jobs)));
  if ((int64_t)jobs > 65535) return CCT_ERR_VALUE;
  MapsPass p;
  p.mu_in_t = p.mu_out_t = nullptr;
  if (prefix > 0) {
    float* t = reinterpret_cast<float*>(work);
    const size_t tb = transposed_bytes(d);
    if (d->has_in) {
      launch_transpose(mu_in, t, d->n, d->n_slices, st);
      p.mu_in_t = t;
      t = reinterpret_cast<float*>(reinterpret_cast<char*>(t) + tb);
    }
    if (out_own) {
      launch_transpose(mu_out, t, d->n, d->n_slices, st);
      p.mu_out_t = t;
    } else if (d->has_out) {
      p.mu_out_t = p.mu_in_t;
    }
    work = reinterpret_cast<char*>(work) + prefix;
  }
  p.n = d->n; p.P = P; p.e = e; p.n_det = d->n_det; p.n_sub = d->n_sub;
  p.has_in = d->has_in; p.has_out = d->has_out; p.maps_dtype = d->maps_dtype; p.n_angles = d->n_angles;
  p.jobs_per_angle = (d->has_in ? 1 : 0) + (d->has_out ? d->n_det * d->n_sub : 0);
  p.rot_in = d->rot_in; p.rot_out = d->rot_out; p.pairs = d->pairs; p.mu_in = mu_in; p.mu_out = mu_out;
  p.quads = nullptr; p.emitted_scale = 0.f; p.n_entries = entries;
  p.work = reinterpret_cast<float*>(work); p.maps = maps;
  p.kcol = p.work + (int64_t)per_pass * p.jobs_per_angle * (int64_t)P * P * d->n_slices;
  for (int a0 = 0; a0 < entries; a0 += per_pass) {
    p.a0 = a0;
    p.na = std::min(per_pass, entries - a0);
    const dim3 g1((P + 127) / 128, p.na * p.jobs_per_angle, d->n_slices);
    if (p.pairs != nullptr) {
      maps_scan_kernel<true><<<g1, 128, 0, st>>>(p);
    } else {
      maps_scan_kernel<false><<<g1, 128, 0, st>>>(p);
    }
    const int tiles = (d->n + RS_TILE - 1) / RS_TILE;
    const dim3 g2((unsigned)(tiles * tiles), p.na, d->n_slices);
    const size_t smem = 6 * p.jobs_per_angle * sizeof(float);
    if (p.pairs != nullptr) {
      maps_resample_kernel<true><<<g2, 256, smem, st>>>(p);
    } else {
      maps_resample_kernel<false><<<g2, 256, smem, st>>>(p);
    }
  }
  return CCT_OK;
}

}  // namespace cct
