/*
 * corrct_b200 — C ABI of the B200 (sm_100a) attenuation-corrected XRF projection path.
 *
 * Every entry point takes plain device pointers, sizes, and a CUDA stream handle
 * (a cudaStream_t passed as void*; NULL = legacy default stream).  The caller owns
 * every buffer; the library never allocates or frees device memory on these paths
 * (scratch space is passed in as a workspace).  Calls are stream-ordered, return an
 * int status (CCT_OK = 0), and keep no hidden state other than the thread-local
 * message returned by cct_last_error().
 *
 * Layouts (row-major, C order, n = volume side = detector width):
 *   volume     [S][n][n]            float32
 *   sinogram   [S][D][A][n]         float32   (S slices, D detectors, A angles)
 *   maps       [S][A][D][n][n]      float32 or bfloat16
 * which per slice are the reference's own shapes: volume (n, n) and sinogram
 * (n_det, A, n) (corrct: src/corrct/projectors.py:591-594), maps (A, n_det, n, n)
 * (corrct: src/corrct/physics/attenuation.py:134).
 */
#ifndef CORRCT_B200_H
#define CORRCT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CCT_ABI_VERSION 7

/* Status codes. */
#define CCT_OK 0
#define CCT_ERR_VALUE 1       /* bad shape, geometry or argument (Python: ValueError) */
#define CCT_ERR_CUDA 2        /* CUDA runtime error (Python: RuntimeError) */
#define CCT_ERR_UNSUPPORTED 3 /* valid but unsupported combination (Python: NotImplementedError) */

/* Map storage types. */
#define CCT_DTYPE_F32 0
#define CCT_DTYPE_BF16 1
#define CCT_DTYPE_FIELDS_F32 2 /* line-integral fields instead of maps: [S/C][A][1 + D][n][n] float32 with
                                  plane 0 = L_in and plane 1 + d = L_out of detector d for the emitted
                                  attenuation of the slice's first channel; channel c of a slice uses the
                                  map exp(-(L_in + channel_scale[c] * L_out)).  Slices are channel-major
                                  within a field slice (slice s = field slice s / C, channel s % C).  For
                                  fluorescence channels whose emitted attenuation is a multiple of one
                                  volume (mu_out,c = s_c * mu_out) the line integrals are linear in mu
                                  (corrct: src/corrct/_projector_backends.py:43-99 is linear up to the
                                  exp), so C channels need two fields instead of C maps. */

/* Back-projection modes. */
#define CCT_BP_REFERENCE 0 /* scikit-image iradon discretisation, no maps, no weights
                              (corrct: src/corrct/projectors.py:619-622, _projector_backends.py:335-359) */
#define CCT_BP_SYMMETRIC 1 /* iradon discretisation x weights x maps
                              (corrct: src/corrct/projectors.py:533-568, 608-618) */
#define CCT_BP_ADJOINT 2   /* exact transpose of cct_fp (no reference counterpart) */

/* Kernel variants (results are identical; only the speed differs). */
#define CCT_VARIANT_FP_TMA 1 /* forward projection stages its boxes with TMA bulk tensor copies
                                (needs n % 8 == 0; otherwise the load/store staging is used) */
#define CCT_VARIANT_FP_SLICES2 2 /* forward projection: one CTA per two slices of the batch (shared
                                    sample coordinates, one 8-byte shared load per tap for both) */

/* Geometry of a batch of slices that share n, the angles and the detectors. */
typedef struct cct_xrf_desc {
  int32_t n;          /* square volume side and detector width in pixels (>= 2) */
  int32_t n_angles;   /* A >= 1 */
  int32_t n_det;      /* D >= 1 fluorescence detectors (maps per angle) */
  int32_t n_slices;   /* S >= 1 */
  int32_t maps_dtype; /* CCT_DTYPE_F32 or CCT_DTYPE_BF16 */
  int32_t variant;    /* kernel variant chosen by the autotuner: CCT_VARIANT_* flags, 0 = default */
  const float* fp_matrix; /* device [A][6]: per-angle inverse map of scikit-image radon,
                             (M00, M01, M02, M10, M11, M12): col_in = M00*c + M01*r + M02,
                             row_in = M10*c + M11*r + M12, entries as radon builds them in float32 */
  const float* bp_trig;   /* device [A][2]: (cos, sin) of each angle as iradon evaluates them (float32) */
  const float* weights;   /* device [A][D]: w_det[d] * w_angle[a][d] * intensity[a], or NULL for all ones */
  const float* line_scale; /* device [A]: projection intensities applied by the reference-mode back
                              projection (corrct: src/corrct/projectors.py:336-337), or NULL */
  const float* psf;       /* device [psf_len]: detector point-spread function applied after the forward
                             projection (corrct: src/corrct/projectors.py:199-203, 317-320,
                             operators.py:480-483: edge-padded 'same' convolution along the detector;
                             the back projection ignores it, as the reference's default is_symm=False
                             makes its adjoint the identity), or NULL */
  int32_t psf_len;
  int32_t n_channels;        /* CCT_DTYPE_FIELDS_F32: channels per field slice (n_slices % n_channels == 0) */
  int64_t maps_slice_stride; /* elements between the maps (or fields) of consecutive slices (field
                                slices); 0 = dense (n_angles * n_det * n * n, or n_angles * (1 + n_det)
                                * n * n for fields).  Lets a call read an angle range of a larger array. */
  const float* channel_scale; /* device [n_channels]: s_c of CCT_DTYPE_FIELDS_F32 */
  const int32_t* fp_box_strides; /* device [A][2] or NULL (all 0): per angle, row-stride selectors of the
                                    forward projection's staged box: column 1 for two slices per CTA
                                    (stride 80 + 2v elements, v in 0..4; column 0 is reserved, 0),
                                    chosen on the host to spread the angle's bilinear taps over the
                                    shared-memory banks.  Speed only: any values give the same
                                    results. */
} cct_xrf_desc;

/* Library identity. */
int cct_abi_version(void);
const char* cct_last_error(void);

/* Kernels never trap: an internal bound that valid inputs cannot exceed raises a device flag
   instead.  *value = the flag (0 = clean); clear != 0 resets it.  Synchronous. */
int cct_device_error(int32_t clear, int32_t* value);

/*
 * Forward projection.  maps == NULL: uncorrected projection (D must be 1), the
 * scikit-image backend's fp (corrct: src/corrct/_projector_backends.py:312-333).
 * maps != NULL: attenuated projection sino[s][d][a] = w[a][d] * radon_a(vol[s] * maps[s][a][d])
 * (corrct: src/corrct/projectors.py:502-531, 570-596).
 */
int cct_fp(const cct_xrf_desc* desc, const float* vol, const void* maps, float* sino, void* stream);

/*
 * Back projection, mode = CCT_BP_*.  Replaces ProjectorAttenuationXRF.bp / bp_angle
 * (corrct: src/corrct/projectors.py:533-568, 598-622) and ProjectorBackendSKimage.bp
 * (corrct: src/corrct/_projector_backends.py:335-359).  maps may be NULL for
 * CCT_BP_REFERENCE and CCT_BP_ADJOINT (uncorrected transpose).
 */
int cct_bp(const cct_xrf_desc* desc, int32_t mode, const float* sino, const void* maps, float* vol,
           void* stream);

/* ---------------------------------------------------------------------------------------------
 * Attenuation maps: maps[s][a][d] = exp(-L_in(theta_a)) * mean_k exp(-L_out(theta_a + phi_d + s_k)),
 * with L the reference's pad / rotate / half-voxel cumulative sum / rotate-back line integral
 * (corrct: src/corrct/_projector_backends.py:43-99, src/corrct/physics/attenuation.py:105-180).
 * ------------------------------------------------------------------------------------------- */
typedef struct cct_maps_desc {
  int32_t n;          /* volume side */
  int32_t n_angles;   /* A */
  int32_t n_det;      /* D */
  int32_t n_slices;   /* S */
  int32_t n_sub;      /* emitted sub-angles per detector (>= 1) */
  int32_t maps_dtype; /* CCT_DTYPE_F32 or CCT_DTYPE_BF16 */
  int32_t has_in;     /* incident attenuation present */
  int32_t has_out;    /* emitted attenuation present */
  const double* rot_in;  /* device [A][2][6]: scikit-image rotate inverse maps of the padded image,
                            [0] = rotate(-phi), [1] = rotate(+phi), same entry order as fp_matrix */
  const double* rot_out; /* device [A][D][n_sub][2][6], emitted directions (phi includes + pi) */
  const int32_t* pairs;  /* device [n_entries][2] (angle, partner), or NULL (every angle on its own).
                            Each entry computes the maps of `angle` and, when partner >= 0, of the
                            angle `partner` = angle + pi (to float32 rounding) from the same
                            rotations: the half turn of the rotated frame is a permutation of its
                            lattice and the partner's scans are the reverse scans, so one rotation
                            per direction serves both angles.  Every angle must appear once; out of
                            range indices are skipped. */
  int32_t n_entries;     /* entries of `pairs` (ignored when pairs is NULL) */
  int32_t reserved;
  const int32_t* quads;  /* device [n_quads][6], or NULL.  Quarter-turn quads for one point detector
                            whose emitted direction (angle + detector angle + pi) is, for every
                            angle, the incident direction of another angle of the set, with
                            mu_out = emitted_scale * mu_in: row (e, e', s0, s1, s2, s3) names two
                            `pairs` entries, whose angles and partners are the quad's four angles
                            k = 0..3 (e's angle, e's partner, e''s angle, e''s partner), and s_k, the
                            one among them whose incident direction is angle k's emitted direction.
                            Only incident fields are scanned (two per quad) and the map of angle k
                            is exp(-L_in(k)) * exp(-emitted_scale * L_in(s_k)) (the emitted rotation
                            then differs from the reference's by the float32 rounding of the angles,
                            as a half-turn partner's does).  Needs pairs, n_det == n_sub == 1,
                            has_in and has_out set, F32 or BF16 maps; mu_out is not read.
                            Every pairs entry must be in exactly one quad. */
  int32_t n_quads;
  float emitted_scale;   /* quads: mu_out / mu_in (>= 0) */
} cct_maps_desc;

/* Workspace bytes needed to process `angles_per_pass` angles (entries, with pairs) per pass (>= 1). */
int cct_maps_workspace_size(const cct_maps_desc* desc, int32_t angles_per_pass, size_t* bytes);

/* Compute maps.  mu_in / mu_out: device [S][n][n] float32 (NULL when absent).  The number of
   angles per pass is the largest that fits in workspace_bytes.  When the workspace also holds
   transposed copies of mu_in and mu_out (n * n * S floats each, 256-byte rounded) beside at least
   half of that many entries, their start of the workspace holds those copies, which the column
   scans read at angles whose columns run closer to y than to x (same results, coalesced loads).
   maps_dtype = CCT_DTYPE_FIELDS_F32
   writes the line-integral fields [S][A][1 + D][n][n] (L_in, then L_out per detector; zero for an
   absent volume; needs n_sub == 1) instead of maps. */
int cct_compute_maps(const cct_maps_desc* desc, const float* mu_in, const float* mu_out, void* maps,
                     void* workspace, size_t workspace_bytes, void* stream);

/* Same maps as cct_compute_maps, computed without any device allocation: the scratch is a
   32 MiB array in the library's static device memory.  No counterpart in the reference; it is
   for callers that cannot allocate device memory (a pool allocator owns it all, a plugin host
   forbids cudaMalloc in its callbacks, or cudaMalloc's implicit synchronisation is not allowed).
   Calls whose one-angle pass needs more than 32 MiB return CCT_ERR_VALUE.  The first call on a
   device looks up the array's device address (cudaGetSymbolAddress), so make that first call
   before any stream capture; the address is kept for the life of the process's CUDA context on
   that device (after a cudaDeviceReset the library must be reloaded).  All calls share the array:
   calls that overlap on the GPU race. */
int cct_compute_maps_noalloc(const cct_maps_desc* desc, const float* mu_in, const float* mu_out, void* maps,
                             void* stream);

/* ---------------------------------------------------------------------------------------------
 * Device-resident solver steps for a batch of slices (update equations of corrct's MLEM,
 * SIRT and PDHG: src/corrct/solvers.py:688-805, 867-984, 1060-1206).
 * ------------------------------------------------------------------------------------------- */
typedef struct cct_solver_state {
  float* x;              /* [S][n][n] iterate, updated in place */
  float* x_relax;        /* [S][n][n] PDHG over-relaxed iterate (NULL otherwise) */
  const float* b;        /* [S][D][A][n] data */
  const float* tau;      /* [S][n][n], or [n][n] when tau_shared (MLEM: A^T 1; SIRT/PDHG: scaling) */
  const float* sigma;    /* [S][D][A][n] SIRT/PDHG data-space scaling, NULL for MLEM */
  float* sino_buf;       /* [S][D][A][n] workspace (MLEM ratio, SIRT residual, PDHG dual) */
  float* vol_buf;        /* [S][n][n] workspace */
  float* tv_dual;        /* [S][2][n][n] PDHG TV dual (NULL otherwise) */
  double* partials;      /* workspace, cct_solver_partials_count() doubles */
  double* residuals;     /* [S] residual norm of the last evaluated iterate */
  int32_t* active;       /* [S] 1 while a slice iterates, 0 once it met its tolerance */
  int32_t* iterations;   /* [S] iterations performed (counted like SolutionInfo.iterations) */
  const double* tolerance; /* [S] stop when tolerance > residual; NULL = never stop early */
  const float* x_mask;   /* [n][n] solution mask shared by all slices, or NULL */
  float lower_limit;
  float upper_limit;
  int32_t has_lower;
  int32_t has_upper;
  float background;      /* data background added to A x (0 with has_background = 0) */
  int32_t has_background;
  float tv_lambda;       /* PDHG isotropic TV weight */
  int32_t tau_shared;
  float* sino_tmp;       /* [S][D][A][n] workspace, required by PDHG when desc->psf is set */
  double* residual_history; /* [S][history_len] residual of every iteration (SolutionInfo.residuals), or NULL */
  int32_t history_len;
  int32_t x_mask_per_slice; /* 1: x_mask is [S][n][n] (a 3-D volume mask); 0: one [n][n] mask */
  int32_t joint_stop;    /* 1: the S slices are one 3-D volume: one residual (the sum over slices, which
                            is the reference's norm of the whole volume's residual) is compared with
                            tolerance[0] and all slices stop together; its history is row 0 of
                            residual_history.  0: every slice has its own stopping test. */
  const float* b_mask;      /* [S][D][A][n] data mask (corrct: solvers.py:497-508, 731-736, 788, 1168-1169):
                               masks the residual (its norm, SIRT's update) and PDHG's dual; NULL = none */
  const float* b_test_mask; /* [S][D][A][n] cross-validation mask (solvers.py:333-343, 783-785): the test
                               residual of every iterate is reduced separately by MLEM and SIRT; PDHG
                               takes NULL; NULL = none */
  double* partials_test;    /* like partials; required with b_test_mask */
  double* residuals_test;   /* [S] test residual of the last evaluated iterate */
  double* history_test;     /* [S][history_len] test residuals (SolutionInfo.residuals_cv), or NULL */
} cct_solver_state;

/* Number of doubles the `partials` workspace must hold. */
int cct_solver_partials_count(const cct_xrf_desc* desc, int64_t* count);

/* One MLEM iteration with the KL residual stopping test (corrct: src/corrct/solvers.py:777-803).
   Equivalent to cct_mlem_fp followed by cct_mlem_update. */
int cct_mlem_step(const cct_xrf_desc* desc, const void* maps, cct_solver_state* st, void* stream);

/* First half of an MLEM iteration: attenuated fp of x with the fused epilogue
   ratio = b / max(Ax + bg, eps) into sino_buf, the FP64 KL residual, the iteration count and
   the stopping test (corrct: src/corrct/solvers.py:779-796). */
int cct_mlem_fp(const cct_xrf_desc* desc, const void* maps, cct_solver_state* st, void* stream);

/* Second half: x *= A^T(ratio) / tau, clip, mask, for slices still active
   (corrct: src/corrct/solvers.py:798-803). */
int cct_mlem_update(const cct_xrf_desc* desc, cct_solver_state* st, void* stream);

/* One SIRT iteration with the l2 residual (corrct: src/corrct/solvers.py:951-982). */
int cct_sirt_step(const cct_xrf_desc* desc, const void* maps, int32_t bp_mode, cct_solver_state* st,
                  void* stream);

/* One PDHG iteration, KL data term + isotropic TV2D (corrct: src/corrct/solvers.py:1165-1206). */
int cct_pdhg_step(const cct_xrf_desc* desc, const void* maps, int32_t bp_mode, cct_solver_state* st,
                  void* stream);

/* Norms in FP64 per slice: out[s] = sum |v| (ord 1) or sum v^2 (ord 2) over `count` elements of
   slice s of v (slices `count` apart).  Replaces np.linalg.norm on solver arrays. */
int cct_reduce_norm(const float* v, int64_t count, int32_t n_slices, int32_t ord, double* out,
                    double* partials, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Ragged batches: one launch per operator over groups of slices that differ in size, angle
 * count, detectors and buffers.  Each group is a uniform batch with its own cct_xrf_desc, maps
 * and cct_solver_state (as for cct_mlem_step / cct_sirt_step); one cct_ragged_step is one
 * iteration of every group (fp with the fused epilogue, residuals and stopping tests, bp with
 * the fused update): three launches for all groups instead of three per group.  No reference
 * counterpart: the reference solves one slice per call; the per-slice arithmetic is that of
 * cct_mlem_step (corrct: src/corrct/solvers.py:777-803) and cct_sirt_step (:951-982).
 * ------------------------------------------------------------------------------------------- */
#define CCT_METHOD_MLEM 0
#define CCT_METHOD_SIRT 1

typedef struct cct_ragged_plan cct_ragged_plan; /* opaque host object */

/* Device workspace bytes for a plan of n_groups groups (256-byte aligned tables). */
int cct_ragged_workspace_size(int32_t n_groups, size_t* bytes);

/* Build a plan: validates every group (one maps type for all, no PSF, per-slice stopping; MLEM
   uses the reference back projection, SIRT REFERENCE or SYMMETRIC) and copies the launch tables
   into `workspace` on `stream`.  The plan holds the groups' pointers: it stays valid while their
   buffers and the workspace live.  maps[g] may be NULL (uncorrected, n_det == 1) for all groups
   or for none. */
int cct_ragged_plan_create(int32_t method, int32_t bp_mode, int32_t n_groups, const cct_xrf_desc* descs,
                           const void* const* maps, const cct_solver_state* states, void* workspace,
                           size_t workspace_bytes, cct_ragged_plan** plan, void* stream);

/* One iteration of every group (stream-ordered). */
int cct_ragged_step(const cct_ragged_plan* plan, void* stream);

int cct_ragged_plan_destroy(cct_ragged_plan* plan);

/* ---------------------------------------------------------------------------------------------
 * Learned warm start (no reference counterpart): a small convolutional encoder-decoder whose
 * 3x3 convolutions run as implicit GEMMs on tcgen05 tensor cores (BF16 in, FP32 accumulate in
 * TMEM).  Activations are NHWC bfloat16 with channel counts that are multiples of 16; weights are
 * [cout][3][3][cin] bfloat16; padding is 1 (same size), stride 1.  Its output is only an initial
 * guess x0 for the reference's MLEM (corrct: src/corrct/solvers.py:747-752 accepts x0).
 * ------------------------------------------------------------------------------------------- */
typedef struct cct_conv_desc {
  int32_t batch;
  int32_t height;
  int32_t width;
  int32_t cin;  /* power of two in [16, 512] */
  int32_t cout; /* multiple of 16 in [16, 512] */
} cct_conv_desc;

/* y = act(conv3x3(x, w) + bias); act = ReLU when relu != 0; bias may be NULL.  With x = dy and
   w = the flipped weights of cct_net_flip_weights this is the data gradient of a convolution. */
int cct_conv3x3_fwd(const cct_conv_desc* desc, const void* x, const void* w, const float* bias, int32_t relu,
                    void* y, void* stream);

/* dw[co][tap][ci] += sum over pixels of dy[p][co] * x[p + tap][ci] (FP32, caller zeroes dw). */
int cct_conv3x3_wgrad(const cct_conv_desc* desc, const void* x, const void* dy, float* dw, void* stream);

/* [cout][3][3][cin] -> [cin][3][3][cout] with the 3x3 taps reversed (data-gradient weights). */
int cct_net_flip_weights(const void* w, void* w_flipped, int32_t cin, int32_t cout, void* stream);

/* dx = dy where y > 0 else 0 (bf16, `count` elements). */
int cct_net_relu_bwd(const void* y, const void* dy, void* dx, int64_t count, void* stream);

/* 2x2 average pooling of NHWC x (height, width even); backward != 0: adjoint from the pooled
   gradient x to the full-resolution gradient y. */
int cct_net_avgpool2(const void* x, void* y, int32_t batch, int32_t height, int32_t width, int32_t channels,
                     int32_t backward, void* stream);

/* nearest 2x upsampling of NHWC x (height, width = the small size); backward != 0: adjoint
   (sum of the 4 children) from the large gradient x to the small gradient y. */
int cct_net_upsample2(const void* x, void* y, int32_t batch, int32_t height, int32_t width, int32_t channels,
                      int32_t backward, void* stream);

/* out = a + b (bf16, `count` elements). */
int cct_net_add(const void* a, const void* b, void* out, int64_t count, void* stream);

/* db[c] += sum over pixels of dy[p][c] (FP32, caller zeroes db). */
int cct_net_bias_grad(const void* dy, float* db, int64_t pixels, int32_t channels, void* stream);

/* Mean squared error of channel 0 of pred (NHWC) against target [pixels] (FP32):
   *loss += mean (pred - target)^2 (FP64), grad (NHWC bf16) = d loss / d pred. */
int cct_net_mse(const void* pred, const float* target, void* grad, double* loss, int64_t pixels, int32_t channels,
                void* stream);

/* One Adam step on FP32 master parameters p with gradient g and moments m, v (step >= 1, bias
   corrected); p_bf16 (may be NULL) receives the bfloat16 copy used by the convolutions. */
int cct_net_adam(float* p, const float* g, float* m, float* v, void* p_bf16, int64_t count, float lr, float beta1,
                 float beta2, float eps, int32_t step, void* stream);

/* NHWC bf16 network input from n_src FP32 planar images of `pixels` values each (device array of
   device pointers); every value is divided by its slice's slice_scale[p / slice_pixels]
   (slice_scale may be NULL); channels beyond n_src are zero. */
int cct_net_pack_nhwc(const float* const* src, int32_t n_src, void* dst, int64_t pixels, int32_t channels,
                      const float* slice_scale, int64_t slice_pixels, void* stream);

/* Warm start from the head output v = src[p][0] with s = slice_scale[p / slice_pixels] (1 if NULL):
   mode 0 (additive):       out[p] = max(base[p] + s * v, floor_value)
   mode 1 (multiplicative): out[p] = max((base[p] + s * floor_value) * exp(v) - s * floor_value, floor_value)
   (base may be NULL). */
int cct_net_unpack_c0(const void* src, int32_t channels, const float* base, const float* slice_scale,
                      int64_t slice_pixels, int32_t mode, float floor_value, float* out, int64_t pixels, void* stream);

/* out[i] = a[i] / b[i % b_count] (FP32; b broadcast over slices), e.g. A^T b / A^T 1. */
int cct_net_ratio(const float* a, const float* b, float* out, int64_t count, int64_t b_count, void* stream);

/* Network kernels never trap: a tensor-core wait that exceeds its bound raises a flag instead.
   *value = the flag; clear != 0 resets it.  Synchronous. */
int cct_net_timeout(int32_t clear, int32_t* value);

/* ---------------------------------------------------------------------------------------------
 * Synthetic data: the noise model of corrct's testing.add_noise (corrct: src/corrct/testing.py:
 * 266-320) on device arrays.  Random numbers are counter based (Philox-4x32-10 keyed by `seed`):
 * every element's draws depend only on the seed and the element index, so results are
 * reproducible for any launch, and agree with the reference in distribution (numpy's generator
 * is a different stream).
 * ------------------------------------------------------------------------------------------- */
typedef struct cct_noise_desc {
  double num_photons;          /* photons for an image value of 1.0 */
  double detection_efficiency; /* scales the photons (the reference passes the detector solid angle) */
  double background_avg;       /* used when has_background: noisy += photons * eff * |N(avg, std)| */
  double background_std;
  double readout_std;          /* used when has_readout: noisy += N(0, readout_std) after the counts */
  uint64_t seed;
  int32_t add_poisson;         /* noisy = Poisson(noisy) (after the background) */
  int32_t has_background;
  int32_t has_readout;
  int32_t reserved;
} cct_noise_desc;

/* Doubles the `partials` workspace of cct_add_noise must hold. */
int cct_noise_partials_count(int64_t* count);

/* clean_scaled[i] = (float)(photons * eff) * clean[i] (may be NULL), noisy as described above,
   *background = mean(noisy - clean_scaled) before the Poisson draw (FP64, device).  flags: two
   int32 that the caller zeroes; flags[0] != 0 when a Poisson mean was negative, NaN or too large
   (those elements become NaN; numpy raises ValueError), flags[1] != 0 when a draw hit its
   iteration bound (returns the rounded mean; not reachable in practice). */
int cct_add_noise(const cct_noise_desc* desc, const float* clean, int64_t count, float* noisy, float* clean_scaled,
                  double* partials, double* background, int32_t* flags, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CORRCT_B200_H */
