// C ABI entry points: argument validation, status codes, launches.

#include <cstring>
#include <string>
#include <vector>

#include "cct_common.cuh"
#include "cct_internal.cuh"

namespace cct {
int launch_maps(const cct_maps_desc* d, const float* mu_in, const float* mu_out, void* maps, void* work,
                size_t work_bytes, cudaStream_t st);
int64_t maps_bytes_per_angle(const cct_maps_desc* d);
void launch_residual_step(const double* partials, int64_t per_slice, int n_slices, double* residuals, int* active,
                          int* iterations, const double* tolerance, double* history, int history_len, int joint,
                          cudaStream_t st);
void launch_tv_dual(const float* x_relax, float* q, int n, int n_slices, float lam, const int* active,
                    cudaStream_t st);
void launch_residual_test(const double* partials, int64_t per_slice, int n_slices, double* residuals,
                          const int* active, const int* iterations, double* history, int history_len,
                          cudaStream_t st);
void launch_norm(const float* v, int64_t count, int n_slices, int ord, double* out, double* partials,
                 cudaStream_t st);
}  // namespace cct

static thread_local std::string g_last_error;

void cct_set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }

static int check_launch() {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    cct_set_last_error(cudaGetErrorString(e));
    return CCT_ERR_CUDA;
  }
  return CCT_OK;
}

static int64_t dense_maps_stride(const cct_xrf_desc* d) {
  const int64_t planes = d->maps_dtype == CCT_DTYPE_FIELDS_F32 ? 1 + d->n_det : d->n_det;
  return (int64_t)d->n_angles * planes * d->n * d->n;
}

static int validate_desc(const cct_xrf_desc* d) {
  CCT_REQUIRE(d != nullptr, "descriptor is NULL");
  CCT_REQUIRE(d->n >= 2 && d->n <= 8192, "volume side n must be in [2, 8192]");
  CCT_REQUIRE(d->n_angles >= 1 && d->n_det >= 1 && d->n_slices >= 1, "n_angles, n_det and n_slices must be >= 1");
  CCT_REQUIRE((int64_t)d->n_angles * d->n_det <= 65535, "n_angles * n_det must be <= 65535");
  CCT_REQUIRE(d->n_slices <= 65535, "n_slices must be <= 65535");
  CCT_REQUIRE(d->maps_dtype == CCT_DTYPE_F32 || d->maps_dtype == CCT_DTYPE_BF16 || d->maps_dtype == CCT_DTYPE_FIELDS_F32,
              "maps_dtype must be F32, BF16 or FIELDS_F32");
  CCT_REQUIRE(d->maps_dtype != CCT_DTYPE_FIELDS_F32 ||
                  (d->n_channels >= 1 && d->channel_scale != nullptr && d->n_slices % d->n_channels == 0),
              "fields need n_channels >= 1 dividing n_slices and channel_scale");
  CCT_REQUIRE(d->fp_matrix != nullptr && d->bp_trig != nullptr, "fp_matrix and bp_trig are required");
  CCT_REQUIRE(d->psf == nullptr || (d->psf_len >= 1 && d->psf_len <= 1024), "psf_len must be in [1, 1024]");
  CCT_REQUIRE(d->maps_slice_stride >= 0, "maps_slice_stride must be >= 0");
  CCT_REQUIRE(d->maps_slice_stride == 0 || d->maps_slice_stride >= dense_maps_stride(d),
              "maps_slice_stride must be 0 or at least one slice's maps (fields)");
  return CCT_OK;
}

static int64_t maps_stride(const cct_xrf_desc* d) {
  return d->maps_slice_stride > 0 ? d->maps_slice_stride : dense_maps_stride(d);
}

static cct::FpArgs make_fp_args(const cct_xrf_desc* d, const float* vol, const void* maps, float* out) {
  cct::FpArgs a;
  std::memset(&a, 0, sizeof(a));
  a.n = d->n; a.n_angles = d->n_angles; a.n_det = d->n_det; a.n_slices = d->n_slices;
  a.maps_dtype = d->maps_dtype; a.epi = cct::FP_EPI_STORE; a.variant = d->variant;
  a.fp_matrix = d->fp_matrix; a.weights = d->weights; a.vol = vol; a.maps = maps; a.out = out;
  a.maps_slice_stride = maps_stride(d);
  a.n_channels = d->n_channels > 0 ? d->n_channels : 1;
  a.chan_scale = d->channel_scale;
  a.box_strides = d->fp_box_strides;
  return a;
}

static cct::BpArgs make_bp_args(const cct_xrf_desc* d, int mode, const float* sino, const void* maps, float* out) {
  cct::BpArgs a;
  std::memset(&a, 0, sizeof(a));
  a.n = d->n; a.n_angles = d->n_angles; a.n_det = d->n_det; a.n_slices = d->n_slices;
  a.maps_dtype = d->maps_dtype; a.mode = mode; a.epi = cct::BP_EPI_STORE;
  a.fp_matrix = d->fp_matrix; a.bp_trig = d->bp_trig; a.weights = d->weights; a.line_scale = d->line_scale;
  a.sino = sino; a.maps = maps; a.out = out;
  a.maps_slice_stride = maps_stride(d);
  a.n_channels = d->n_channels > 0 ? d->n_channels : 1;
  a.chan_scale = d->channel_scale;
  return a;
}

extern "C" {

int cct_abi_version(void) { return CCT_ABI_VERSION; }

const char* cct_last_error(void) { return g_last_error.c_str(); }

int cct_fp(const cct_xrf_desc* desc, const float* vol, const void* maps, float* sino, void* stream) {
  int rc = validate_desc(desc);
  if (rc != CCT_OK) return rc;
  CCT_REQUIRE(vol != nullptr && sino != nullptr, "vol and sino are required");
  CCT_REQUIRE(maps != nullptr || desc->n_det == 1, "an uncorrected projection (maps == NULL) needs n_det == 1");
  cct::FpArgs a = make_fp_args(desc, vol, maps, sino);
  cct::launch_fp(a, reinterpret_cast<cudaStream_t>(stream));
  if (desc->psf != nullptr) {
    // in place: each CTA stages its whole line before writing it back
    cct::FpArgs p = make_fp_args(desc, sino, maps, sino);
    cct::launch_psf(p, desc->psf, desc->psf_len, reinterpret_cast<cudaStream_t>(stream));
  }
  return check_launch();
}

int cct_bp(const cct_xrf_desc* desc, int32_t mode, const float* sino, const void* maps, float* vol, void* stream) {
  int rc = validate_desc(desc);
  if (rc != CCT_OK) return rc;
  CCT_REQUIRE(sino != nullptr && vol != nullptr, "sino and vol are required");
  CCT_REQUIRE(mode == CCT_BP_REFERENCE || mode == CCT_BP_SYMMETRIC || mode == CCT_BP_ADJOINT, "unknown bp mode");
  CCT_REQUIRE(mode != CCT_BP_SYMMETRIC || maps != nullptr, "the symmetric back projection needs maps");
  CCT_REQUIRE(!(mode == CCT_BP_ADJOINT && maps == nullptr && desc->n_det != 1),
              "an uncorrected adjoint (maps == NULL) needs n_det == 1");
  cct::BpArgs a = make_bp_args(desc, mode, sino, maps, vol);
  cct::launch_bp(a, reinterpret_cast<cudaStream_t>(stream));
  return check_launch();
}

// Quarter-turn quads (cct_maps_desc.quads): the combinations they need (the table itself is device
// memory; the kernels skip rows that name entries out of range).
static int validate_quads(const cct_maps_desc* d) {
  if (d->quads == nullptr) return CCT_OK;
  CCT_REQUIRE(d->pairs != nullptr && d->n_det == 1 && d->n_sub == 1 && d->has_in && d->has_out,
              "quads need half-turn pairs, one point detector, and incident and emitted attenuation");
  CCT_REQUIRE(d->maps_dtype == CCT_DTYPE_F32 || d->maps_dtype == CCT_DTYPE_BF16, "quads need F32 or BF16 maps");
  CCT_REQUIRE(d->n_quads >= 1 && 2 * (int64_t)d->n_quads == d->n_entries, "quads must cover every pairs entry once");
  CCT_REQUIRE(d->emitted_scale >= 0.f, "emitted_scale must be >= 0");
  return CCT_OK;
}

int cct_maps_workspace_size(const cct_maps_desc* desc, int32_t angles_per_pass, size_t* bytes) {
  CCT_REQUIRE(desc != nullptr && bytes != nullptr, "descriptor and bytes are required");
  CCT_REQUIRE(desc->n >= 2 && desc->n <= 8192, "volume side n must be in [2, 8192]");
  CCT_REQUIRE(desc->n_angles >= 1 && desc->n_det >= 1 && desc->n_slices >= 1 && desc->n_sub >= 1,
              "n_angles, n_det, n_slices and n_sub must be >= 1");
  CCT_REQUIRE(angles_per_pass >= 1, "angles_per_pass must be >= 1");
  CCT_REQUIRE(desc->has_in || desc->has_out, "No attenuation volumes were given.");
  CCT_REQUIRE(desc->pairs == nullptr || (desc->n_entries >= 1 && desc->n_entries <= desc->n_angles),
              "n_entries must be in [1, n_angles] when pairs are given");
  *bytes = (size_t)cct::maps_bytes_per_angle(desc) * (size_t)angles_per_pass;
  return CCT_OK;
}

int cct_compute_maps(const cct_maps_desc* desc, const float* mu_in, const float* mu_out, void* maps,
                     void* workspace, size_t workspace_bytes, void* stream) {
  size_t need = 0;
  int rc = cct_maps_workspace_size(desc, 1, &need);
  if (rc != CCT_OK) return rc;
  CCT_REQUIRE(desc->maps_dtype == CCT_DTYPE_F32 || desc->maps_dtype == CCT_DTYPE_BF16 ||
                  desc->maps_dtype == CCT_DTYPE_FIELDS_F32,
              "maps_dtype must be F32, BF16 or FIELDS_F32");
  CCT_REQUIRE(desc->maps_dtype != CCT_DTYPE_FIELDS_F32 || desc->n_sub == 1,
              "line-integral fields need one emitted direction per detector (n_sub == 1)");
  CCT_REQUIRE(!desc->has_in || (mu_in != nullptr && desc->rot_in != nullptr), "incident volume or matrices missing");
  rc = validate_quads(desc);
  if (rc != CCT_OK) return rc;
  CCT_REQUIRE(!desc->has_out || desc->quads != nullptr || (mu_out != nullptr && desc->rot_out != nullptr),
              "emitted volume or matrices missing");
  CCT_REQUIRE(maps != nullptr && workspace != nullptr, "maps and workspace are required");
  CCT_REQUIRE(workspace_bytes >= need, "workspace smaller than one angle pass (cct_maps_workspace_size)");
  CCT_REQUIRE(desc->n_angles <= 65535 && desc->n_slices <= 65535, "too many angles or slices");
  CCT_REQUIRE((int64_t)(desc->has_in ? 1 : 0) + (desc->has_out ? (int64_t)desc->n_det * desc->n_sub : 0) <= 65535,
              "too many emitted directions (n_det * n_sub) per angle");
  rc = cct::launch_maps(desc, mu_in, mu_out, maps, workspace, workspace_bytes, reinterpret_cast<cudaStream_t>(stream));
  if (rc != CCT_OK) return rc;
  return check_launch();
}

int cct_device_error(int32_t clear, int32_t* value) {
  CCT_REQUIRE(value != nullptr, "value is required");
  int v = 0;
  const int e = cct::read_device_error(clear, &v);
  if (e != 0) {
    cct_set_last_error(cudaGetErrorString((cudaError_t)e));
    return CCT_ERR_CUDA;
  }
  *value = v;
  return CCT_OK;
}

int cct_solver_partials_count(const cct_xrf_desc* desc, int64_t* count) {
  int rc = validate_desc(desc);
  if (rc != CCT_OK) return rc;
  CCT_REQUIRE(count != nullptr, "count is required");
  const int64_t bands = (desc->n + 63) / 64;
  *count = (int64_t)desc->n_slices * bands * desc->n_angles * desc->n_det;
  return CCT_OK;
}

static int validate_state(const cct_xrf_desc* d, const cct_solver_state* st) {
  CCT_REQUIRE(st != nullptr, "solver state is NULL");
  CCT_REQUIRE(st->x && st->b && st->tau && st->sino_buf && st->partials && st->residuals && st->active &&
                  st->iterations,
              "solver state is missing a required buffer");
  CCT_REQUIRE(st->b_test_mask == nullptr || (st->partials_test != nullptr && st->residuals_test != nullptr),
              "b_test_mask needs partials_test and residuals_test");
  (void)d;
  return CCT_OK;
}

static cct::BpArgs make_solver_bp(const cct_xrf_desc* d, int mode, const void* maps, const cct_solver_state* st,
                                  int epi) {
  cct::BpArgs a = make_bp_args(d, mode, st->sino_buf, maps, st->vol_buf);
  a.epi = epi;
  a.x = st->x; a.x_relax = st->x_relax; a.tau = st->tau; a.tau_shared = st->tau_shared;
  a.x_mask = st->x_mask; a.mask_per_slice = st->x_mask_per_slice; a.tv_dual = st->tv_dual;
  a.lower = st->lower_limit; a.upper = st->upper_limit; a.has_lower = st->has_lower; a.has_upper = st->has_upper;
  a.active = st->active;
  return a;
}

int cct_mlem_fp(const cct_xrf_desc* desc, const void* maps, cct_solver_state* st, void* stream) {
  int rc = validate_desc(desc);
  if (rc != CCT_OK) return rc;
  rc = validate_state(desc, st);
  if (rc != CCT_OK) return rc;
  CCT_REQUIRE(maps != nullptr || desc->n_det == 1, "an uncorrected MLEM (maps == NULL) needs n_det == 1");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cct::FpArgs f = make_fp_args(desc, st->x, maps, st->sino_buf);
  f.epi = cct::FP_EPI_MLEM; f.b = st->b; f.background = st->background; f.has_background = st->has_background;
  f.partials = st->partials; f.active = st->active;
  f.b_mask = st->b_mask; f.b_test_mask = st->b_test_mask;
  f.partials_test = st->b_test_mask != nullptr ? st->partials_test : nullptr;
  int64_t per_slice = 0;
  if (desc->psf == nullptr) {
    cct::launch_fp(f, s);
    cct_solver_partials_count(desc, &per_slice);
    per_slice /= desc->n_slices;
  } else {
    // A x into sino_buf, then the PSF with the MLEM epilogue in place (one partial per line)
    cct::FpArgs raw = make_fp_args(desc, st->x, maps, st->sino_buf);
    raw.active = st->active;
    cct::launch_fp(raw, s);
    f.vol = st->sino_buf;
    cct::launch_psf(f, desc->psf, desc->psf_len, s);
    per_slice = (int64_t)desc->n_det * desc->n_angles;
  }
  if (st->b_test_mask != nullptr)
    cct::launch_residual_test(st->partials_test, per_slice, desc->n_slices, st->residuals_test, st->active,
                              st->iterations, st->history_test, st->history_len, s);
  cct::launch_residual_step(st->partials, per_slice, desc->n_slices, st->residuals, st->active, st->iterations,
                            st->tolerance, st->residual_history, st->history_len, st->joint_stop, s);
  return check_launch();
}

int cct_mlem_update(const cct_xrf_desc* desc, cct_solver_state* st, void* stream) {
  int rc = validate_desc(desc);
  if (rc != CCT_OK) return rc;
  rc = validate_state(desc, st);
  if (rc != CCT_OK) return rc;
  // the reference's default XRF back projection ignores maps and weights (projectors.py:619-622)
  cct::BpArgs b = make_solver_bp(desc, CCT_BP_REFERENCE, nullptr, st, cct::BP_EPI_MLEM);
  cct::launch_bp(b, reinterpret_cast<cudaStream_t>(stream));
  return check_launch();
}

int cct_mlem_step(const cct_xrf_desc* desc, const void* maps, cct_solver_state* st, void* stream) {
  const int rc = cct_mlem_fp(desc, maps, st, stream);
  if (rc != CCT_OK) return rc;
  return cct_mlem_update(desc, st, stream);
}

int cct_sirt_step(const cct_xrf_desc* desc, const void* maps, int32_t bp_mode, cct_solver_state* st, void* stream) {
  int rc = validate_desc(desc);
  if (rc != CCT_OK) return rc;
  rc = validate_state(desc, st);
  if (rc != CCT_OK) return rc;
  CCT_REQUIRE(st->sigma != nullptr, "SIRT needs sigma");
  CCT_REQUIRE(bp_mode == CCT_BP_REFERENCE || bp_mode == CCT_BP_SYMMETRIC, "SIRT bp_mode must be REFERENCE or SYMMETRIC");
  CCT_REQUIRE(bp_mode != CCT_BP_SYMMETRIC || maps != nullptr, "the symmetric back projection needs maps");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cct::FpArgs f = make_fp_args(desc, st->x, maps, st->sino_buf);
  f.epi = cct::FP_EPI_SIRT; f.b = st->b; f.sigma = st->sigma; f.background = st->background;
  f.has_background = st->has_background; f.partials = st->partials; f.active = st->active;
  f.b_mask = st->b_mask; f.b_test_mask = st->b_test_mask;
  f.partials_test = st->b_test_mask != nullptr ? st->partials_test : nullptr;
  int64_t per_slice = 0;
  if (desc->psf == nullptr) {
    cct::launch_fp(f, s);
    cct_solver_partials_count(desc, &per_slice);
    per_slice /= desc->n_slices;
  } else {
    cct::FpArgs raw = make_fp_args(desc, st->x, maps, st->sino_buf);
    raw.active = st->active;
    cct::launch_fp(raw, s);
    f.vol = st->sino_buf;
    cct::launch_psf(f, desc->psf, desc->psf_len, s);
    per_slice = (int64_t)desc->n_det * desc->n_angles;
  }
  if (st->b_test_mask != nullptr)
    cct::launch_residual_test(st->partials_test, per_slice, desc->n_slices, st->residuals_test, st->active,
                              st->iterations, st->history_test, st->history_len, s);
  cct::launch_residual_step(st->partials, per_slice, desc->n_slices, st->residuals, st->active, st->iterations,
                            st->tolerance, st->residual_history, st->history_len, st->joint_stop, s);
  cct::BpArgs b = make_solver_bp(desc, bp_mode, maps, st, cct::BP_EPI_SIRT);
  cct::launch_bp(b, s);
  return check_launch();
}

int cct_pdhg_step(const cct_xrf_desc* desc, const void* maps, int32_t bp_mode, cct_solver_state* st, void* stream) {
  int rc = validate_desc(desc);
  if (rc != CCT_OK) return rc;
  rc = validate_state(desc, st);
  if (rc != CCT_OK) return rc;
  CCT_REQUIRE(st->sigma != nullptr && st->x_relax != nullptr && st->tv_dual != nullptr,
              "PDHG needs sigma, x_relax and tv_dual");
  CCT_REQUIRE(st->vol_buf != nullptr, "PDHG needs vol_buf");
  CCT_REQUIRE(bp_mode == CCT_BP_REFERENCE || bp_mode == CCT_BP_SYMMETRIC, "PDHG bp_mode must be REFERENCE or SYMMETRIC");
  CCT_REQUIRE(bp_mode != CCT_BP_SYMMETRIC || maps != nullptr, "the symmetric back projection needs maps");
  CCT_REQUIRE(st->b_test_mask == nullptr, "the PDHG step keeps no test residual (b_test_mask must be NULL)");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cct::FpArgs f = make_fp_args(desc, st->x_relax, maps, st->sino_buf);
  f.epi = cct::FP_EPI_PDHG; f.b = st->b; f.sigma = st->sigma; f.background = st->background;
  f.has_background = st->has_background; f.active = st->active; f.b_mask = st->b_mask;
  if (desc->psf == nullptr) {
    cct::launch_fp(f, s);
  } else {
    CCT_REQUIRE(st->sino_tmp != nullptr, "PDHG with a PSF needs sino_tmp");
    cct::FpArgs raw = make_fp_args(desc, st->x_relax, maps, st->sino_tmp);
    raw.active = st->active;
    cct::launch_fp(raw, s);
    f.vol = st->sino_tmp;
    cct::launch_psf(f, desc->psf, desc->psf_len, s);
  }
  cct::launch_tv_dual(st->x_relax, st->tv_dual, desc->n, desc->n_slices, st->tv_lambda, st->active, s);
  cct::BpArgs b = make_solver_bp(desc, bp_mode, maps, st, cct::BP_EPI_PDHG);
  cct::launch_bp(b, s);
  return check_launch();
}

// ---------------------------------------------------------------------------------------------
// Ragged batches
// ---------------------------------------------------------------------------------------------
}  // extern "C"

struct cct_ragged_plan {
  int method = 0, bp_mode = 0, n_groups = 0, maps_dtype = 0;
  bool has_maps = false;
  int64_t fp_ctas = 0, bp_ctas = 0, slices = 0;
  const cct::FpArgs* d_fp = nullptr;
  const cct::BpArgs* d_bp = nullptr;
  const cct::ResidualGroup* d_res = nullptr;
  const int64_t* d_fp_start = nullptr;
  const int64_t* d_bp_start = nullptr;
  const int64_t* d_res_start = nullptr;
  std::vector<unsigned char> host;  // the tables as copied to the workspace
};

// Workspace layout: FpArgs[G], BpArgs[G], ResidualGroup[G], then three int64 offset tables of
// G + 1 entries, each part 256-byte aligned.
static size_t ragged_layout(int g, size_t off[7]) {
  auto up = [](size_t v) { return (v + 255) & ~(size_t)255; };
  size_t o = 0;
  off[0] = o; o = up(o + sizeof(cct::FpArgs) * g);
  off[1] = o; o = up(o + sizeof(cct::BpArgs) * g);
  off[2] = o; o = up(o + sizeof(cct::ResidualGroup) * g);
  off[3] = o; o = up(o + sizeof(int64_t) * (g + 1));
  off[4] = o; o = up(o + sizeof(int64_t) * (g + 1));
  off[5] = o; o = up(o + sizeof(int64_t) * (g + 1));
  off[6] = o;
  return o;
}

extern "C" {

int cct_ragged_workspace_size(int32_t n_groups, size_t* bytes) {
  CCT_REQUIRE(bytes != nullptr, "bytes is required");
  CCT_REQUIRE(n_groups >= 1 && n_groups <= (1 << 20), "n_groups must be in [1, 2^20]");
  size_t off[7];
  *bytes = ragged_layout(n_groups, off);
  return CCT_OK;
}

int cct_ragged_plan_create(int32_t method, int32_t bp_mode, int32_t n_groups, const cct_xrf_desc* descs,
                           const void* const* maps, const cct_solver_state* states, void* workspace,
                           size_t workspace_bytes, cct_ragged_plan** plan, void* stream) {
  CCT_REQUIRE(plan != nullptr && descs != nullptr && maps != nullptr && states != nullptr && workspace != nullptr,
              "descs, maps, states, workspace and plan are required");
  *plan = nullptr;
  CCT_REQUIRE(method == CCT_METHOD_MLEM || method == CCT_METHOD_SIRT, "method must be CCT_METHOD_MLEM or CCT_METHOD_SIRT");
  CCT_REQUIRE(bp_mode == CCT_BP_REFERENCE || (method == CCT_METHOD_SIRT && bp_mode == CCT_BP_SYMMETRIC),
              "bp_mode must be REFERENCE (or SYMMETRIC for SIRT)");
  size_t off[7];
  int rc = cct_ragged_workspace_size(n_groups, &off[6]);
  if (rc != CCT_OK) return rc;
  const size_t need = ragged_layout(n_groups, off);
  CCT_REQUIRE(workspace_bytes >= need, "workspace is smaller than cct_ragged_workspace_size()");
  CCT_REQUIRE(reinterpret_cast<uintptr_t>(workspace) % 256 == 0, "workspace must be 256-byte aligned");

  cct_ragged_plan* p = new cct_ragged_plan();
  p->method = method;
  p->bp_mode = bp_mode;
  p->n_groups = n_groups;
  p->has_maps = maps[0] != nullptr;
  p->maps_dtype = descs[0].maps_dtype;
  p->host.assign(need, 0);
  auto* fp = reinterpret_cast<cct::FpArgs*>(p->host.data() + off[0]);
  auto* bp = reinterpret_cast<cct::BpArgs*>(p->host.data() + off[1]);
  auto* res = reinterpret_cast<cct::ResidualGroup*>(p->host.data() + off[2]);
  auto* fps = reinterpret_cast<int64_t*>(p->host.data() + off[3]);
  auto* bps = reinterpret_cast<int64_t*>(p->host.data() + off[4]);
  auto* rss = reinterpret_cast<int64_t*>(p->host.data() + off[5]);
  auto fail = [&](int code) {
    delete p;
    return code;
  };
  fps[0] = bps[0] = rss[0] = 0;
  for (int g = 0; g < n_groups; ++g) {
    const cct_xrf_desc* d = descs + g;
    const cct_solver_state* st = states + g;
    if ((rc = validate_desc(d)) != CCT_OK) return fail(rc);
    if ((rc = validate_state(d, st)) != CCT_OK) return fail(rc);
    if (d->psf != nullptr || st->joint_stop || st->b_test_mask != nullptr || d->maps_dtype != p->maps_dtype ||
        (maps[g] != nullptr) != p->has_maps) {
      cct_set_last_error("ragged groups need one maps type, no PSF, no test mask and per-slice stopping");
      return fail(CCT_ERR_UNSUPPORTED);
    }
    if (maps[g] == nullptr && d->n_det != 1) {
      cct_set_last_error("a group without maps needs n_det == 1");
      return fail(CCT_ERR_VALUE);
    }
    if (method == CCT_METHOD_SIRT && st->sigma == nullptr) {
      cct_set_last_error("SIRT needs sigma in every group");
      return fail(CCT_ERR_VALUE);
    }
    if (bp_mode == CCT_BP_SYMMETRIC && maps[g] == nullptr) {
      cct_set_last_error("the symmetric back projection needs maps");
      return fail(CCT_ERR_VALUE);
    }
    cct::FpArgs f = make_fp_args(d, st->x, maps[g], st->sino_buf);
    f.epi = method == CCT_METHOD_SIRT ? cct::FP_EPI_SIRT : cct::FP_EPI_MLEM;
    f.b = st->b; f.sigma = st->sigma; f.background = st->background; f.has_background = st->has_background;
    f.partials = st->partials; f.active = st->active;
    f.b_mask = st->b_mask;
    f.vec4 = cct::fp_vec4_ok(f) ? 1 : 0;
    fp[g] = f;
    bp[g] = make_solver_bp(d, method == CCT_METHOD_SIRT ? bp_mode : CCT_BP_REFERENCE,
                           method == CCT_METHOD_SIRT ? maps[g] : nullptr, st,
                           method == CCT_METHOD_SIRT ? cct::BP_EPI_SIRT : cct::BP_EPI_MLEM);
    const int64_t bands = (d->n + 63) / 64;
    const int64_t per_slice = bands * d->n_angles * d->n_det;
    res[g] = cct::ResidualGroup{st->partials, per_slice, st->residuals, st->active, st->iterations, st->tolerance,
                                st->residual_history, st->history_len};
    const int64_t tiles = (int64_t)((d->n + 31) / 32) * ((d->n + 63) / 64);
    fps[g + 1] = fps[g] + per_slice * d->n_slices;
    bps[g + 1] = bps[g] + tiles * d->n_slices;
    rss[g + 1] = rss[g] + d->n_slices;
  }
  p->fp_ctas = fps[n_groups];
  p->bp_ctas = bps[n_groups];
  p->slices = rss[n_groups];
  if (p->fp_ctas > 0x7fffffffLL || p->bp_ctas > 0x7fffffffLL || p->slices > 0x7fffffffLL) {
    cct_set_last_error("a ragged batch may hold at most 2^31 - 1 CTAs per launch");
    return fail(CCT_ERR_VALUE);
  }
  unsigned char* w = reinterpret_cast<unsigned char*>(workspace);
  p->d_fp = reinterpret_cast<const cct::FpArgs*>(w + off[0]);
  p->d_bp = reinterpret_cast<const cct::BpArgs*>(w + off[1]);
  p->d_res = reinterpret_cast<const cct::ResidualGroup*>(w + off[2]);
  p->d_fp_start = reinterpret_cast<const int64_t*>(w + off[3]);
  p->d_bp_start = reinterpret_cast<const int64_t*>(w + off[4]);
  p->d_res_start = reinterpret_cast<const int64_t*>(w + off[5]);
  const cudaError_t e = cudaMemcpyAsync(workspace, p->host.data(), need, cudaMemcpyHostToDevice,
                                        reinterpret_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    cct_set_last_error(cudaGetErrorString(e));
    return fail(CCT_ERR_CUDA);
  }
  *plan = p;
  return CCT_OK;
}

int cct_ragged_step(const cct_ragged_plan* plan, void* stream) {
  CCT_REQUIRE(plan != nullptr, "plan is NULL");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const bool sirt = plan->method == CCT_METHOD_SIRT;
  cct::launch_fp_ragged(plan->d_fp, plan->d_fp_start, plan->n_groups, plan->fp_ctas,
                        sirt ? cct::FP_EPI_SIRT : cct::FP_EPI_MLEM, plan->has_maps, plan->maps_dtype, s);
  cct::launch_residual_ragged(plan->d_res, plan->d_res_start, plan->n_groups, plan->slices, s);
  cct::launch_bp_ragged(plan->d_bp, plan->d_bp_start, plan->n_groups, plan->bp_ctas,
                        sirt ? cct::BP_EPI_SIRT : cct::BP_EPI_MLEM, plan->bp_mode == CCT_BP_SYMMETRIC,
                        plan->maps_dtype, s);
  return check_launch();
}

int cct_ragged_plan_destroy(cct_ragged_plan* plan) {
  delete plan;
  return CCT_OK;
}

int cct_reduce_norm(const float* v, int64_t count, int32_t n_slices, int32_t ord, double* out, double* partials,
                    void* stream) {
  CCT_REQUIRE(v != nullptr && out != nullptr && partials != nullptr, "v, out and partials are required");
  CCT_REQUIRE(count >= 1 && n_slices >= 1 && n_slices <= 65535, "count and n_slices must be >= 1");
  CCT_REQUIRE(ord == 1 || ord == 2, "ord must be 1 or 2");
  cct::launch_norm(v, count, n_slices, ord, out, partials, reinterpret_cast<cudaStream_t>(stream));
  return check_launch();
}

}  // extern "C"
