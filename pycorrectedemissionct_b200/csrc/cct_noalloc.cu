// Attenuation maps without any device allocation.
//
// cct_compute_maps() needs a caller-provided workspace for the rotated-frame line
// integrals.  Some callers cannot provide one: a host application whose device memory is
// entirely pre-reserved by its own pool allocator, a plugin that is not allowed to call
// cudaMalloc from its callbacks, or code that must not trigger the implicit device
// synchronisation of cudaMalloc/cudaFree in a latency-critical loop.  For them,
// cct_compute_maps_noalloc() runs the same two-phase computation on a fixed scratch array
// that lives in the library's own static device memory.
//
// Limits and rules of the scratch:
// * it holds CCT_NOALLOC_SCRATCH_BYTES (32 MiB); one pass over angles needs
//   (incident + emitted jobs) x P^2 x 4 bytes x slices for one angle, with P the padded
//   side; calls that do not fit one angle are rejected with CCT_ERR_VALUE;
// * every GPU that loads this library reserves the array until the process exits;
// * all calls share it and it keeps the last call's contents; phase 1 rewrites every
//   element that phase 2 reads before reading it, so nothing has to start at zero;
// * calls whose work overlaps on the GPU (different streams, or different host threads
//   without ordering) race on the array and must be serialised by the caller.

#include <mutex>

#include "cct_common.cuh"
#include "cct_internal.cuh"

namespace cct {
int launch_maps(const cct_maps_desc* d, const float* mu_in, const float* mu_out, void* maps, void* work,
                size_t work_bytes, cudaStream_t st);
int64_t maps_bytes_per_angle(const cct_maps_desc* d);
}  // namespace cct

#define CCT_NOALLOC_SCRATCH_BYTES (32u << 20)
#define CCT_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char g_noalloc_scratch[CCT_NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch per device.  In host code the array's name is only a
// host-side stand-in, so the kernels get the address that cudaGetSymbolAddress returns
// with the device current.
static void* g_noalloc_ptr[CCT_NOALLOC_MAX_DEVICES];
static std::mutex g_noalloc_lock;

static int noalloc_scratch(void** out) {
  int dev = -1;
  CCT_CUDA_TRY(cudaGetDevice(&dev));
  CCT_REQUIRE(dev >= 0 && dev < CCT_NOALLOC_MAX_DEVICES, "device ordinal out of range for the no-alloc scratch");
  std::lock_guard<std::mutex> guard(g_noalloc_lock);
  if (g_noalloc_ptr[dev] == nullptr) {
    void* p = nullptr;
    CCT_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return CCT_OK;
}

extern "C" int cct_compute_maps_noalloc(const cct_maps_desc* desc, const float* mu_in, const float* mu_out,
                                        void* maps, void* stream) {
  size_t need = 0;
  int rc = cct_maps_workspace_size(desc, 1, &need);
  if (rc != CCT_OK) return rc;
  if (need > (size_t)CCT_NOALLOC_SCRATCH_BYTES) {
    cct_set_last_error(
        "cct_compute_maps_noalloc: one angle of this batch needs more than the 32 MiB static scratch "
        "(use fewer slices per call, or cct_compute_maps with a workspace)");
    return CCT_ERR_VALUE;
  }
  CCT_REQUIRE(desc->maps_dtype == CCT_DTYPE_F32 || desc->maps_dtype == CCT_DTYPE_BF16,
              "maps_dtype must be F32 or BF16");
  CCT_REQUIRE(!desc->has_in || (mu_in != nullptr && desc->rot_in != nullptr), "incident volume or matrices missing");
  CCT_REQUIRE(desc->quads == nullptr, "cct_compute_maps_noalloc computes every direction on its own (quads = NULL)");
  CCT_REQUIRE(!desc->has_out || (mu_out != nullptr && desc->rot_out != nullptr), "emitted volume or matrices missing");
  CCT_REQUIRE(maps != nullptr, "maps is required");
  CCT_REQUIRE(desc->n_angles <= 65535 && desc->n_slices <= 65535, "too many angles or slices");
  void* scratch = nullptr;
  rc = noalloc_scratch(&scratch);
  if (rc != CCT_OK) return rc;
  rc = cct::launch_maps(desc, mu_in, mu_out, maps, scratch, CCT_NOALLOC_SCRATCH_BYTES,
                        reinterpret_cast<cudaStream_t>(stream));
  if (rc != CCT_OK) return rc;
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    cct_set_last_error(cudaGetErrorString(e));
    return CCT_ERR_CUDA;
  }
  return CCT_OK;
}
