// pert_noalloc.cu -- abcmb_pert_forward without a caller-provided workspace.
//
// Some callers cannot allocate device memory at all: code that runs inside a
// framework that owns every device byte (an XLA custom call registered
// without a workspace operand, an embedding host with a fixed device-memory
// budget, a plugin that must not change the process's allocation pattern).
// This entry point runs the same perturbation kernels as
// abcmb_pert_forward, with the scratch they need (the start-time grids of
// get_starting_time and the work-queue counter) in a file-scope device array
// instead of a caller workspace.
//
// Limits and rules, stated in include/abcmb_b200.h as well:
//  - at most ABCMB_PERT_NOALLOC_MAX_COSMO cosmologies per call; larger calls
//    are rejected with ABCMB_ERR_WORKSPACE and a message;
//  - the array exists once per device that loads the library and stays
//    allocated until the process exits;
//  - every call on a device shares the array (it keeps the last call's
//    contents; the queue counter is cleared at the start of every call), so
//    calls whose kernels overlap on the GPU (different streams, no ordering
//    between them) race and must not be issued;
//  - the first call on a device looks up the array's device address (with
//    that device current); make that first call before any stream capture.
//  - no cudaMalloc, cudaFree or allocating library routine is called.
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace abcmb {
int64_t pert_workspace_bytes(int n_cosmo);
cudaError_t launch_pert(int n_cosmo, const abcmb_cosmo* cosmo, const double* tables, const double* kbuf,
                        int n_items, const int32_t* items, const abcmb_pert_settings& s, double* pt,
                        abcmb_kstat* kstat, void* ws, cudaStream_t stream, int warps_per_block, int* grid_out);
void set_last_error(const std::string& msg);
int pert_warps_per_block();
void set_last_pert_grid(int grid);
}  // namespace abcmb

// queue counter (256 B) + lna1 (256 B for <= 32 cosmologies) + two start grids
// of 10000 doubles per cosmology: 512 + 2 * 8 * 80000 B = 1,280,512 B for 8.
#define ABCMB_NOALLOC_SCRATCH_BYTES (512 + 2 * ABCMB_PERT_NOALLOC_MAX_COSMO * 80000)

static __device__ __align__(256) unsigned char g_pert_scratch[ABCMB_NOALLOC_SCRATCH_BYTES];

namespace {
std::mutex g_noalloc_mu;
std::vector<void*> g_noalloc_addr;   // per device, filled on the first call on that device
}  // namespace

extern "C" int abcmb_pert_forward_noalloc(int n_cosmo, const abcmb_cosmo* cosmo_dev, const double* tables_dev,
                                          const double* k_dev, int n_items, const int32_t* items_dev,
                                          const abcmb_pert_settings* settings, double* pt_dev,
                                          abcmb_kstat* kstat_dev, void* stream) {
  if (n_cosmo <= 0 || n_items < 0 || !cosmo_dev || !tables_dev || !k_dev || !settings || !pt_dev || !kstat_dev) {
    abcmb::set_last_error("abcmb_pert_forward_noalloc: null argument");
    return ABCMB_ERR_ARG;
  }
  if (n_cosmo > ABCMB_PERT_NOALLOC_MAX_COSMO ||
      abcmb::pert_workspace_bytes(n_cosmo) > (int64_t)ABCMB_NOALLOC_SCRATCH_BYTES) {
    abcmb::set_last_error("abcmb_pert_forward_noalloc: " + std::to_string(n_cosmo) +
                          " cosmologies exceed the static scratch limit of " +
                          std::to_string(ABCMB_PERT_NOALLOC_MAX_COSMO) +
                          "; split the call or use abcmb_pert_forward with a workspace");
    return ABCMB_ERR_WORKSPACE;
  }
  if (settings->max_ny <= 0 || settings->n_save < 2 || settings->max_steps <= 0) {
    abcmb::set_last_error("abcmb_pert_forward_noalloc: settings.max_ny / n_save / max_steps");
    return ABCMB_ERR_ARG;
  }
  if (n_items == 0) return ABCMB_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    abcmb::set_last_error(std::string("abcmb_pert_forward_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
    return ABCMB_ERR_CUDA;
  }
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if ((int)g_noalloc_addr.size() <= dev) g_noalloc_addr.resize(dev + 1, nullptr);
    if (!g_noalloc_addr[dev]) {
      // host code must not use g_pert_scratch directly: its name here is a
      // host-side stand-in, not the device address
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_pert_scratch);
      if (e != cudaSuccess || !p) {
        abcmb::set_last_error(std::string("abcmb_pert_forward_noalloc: cudaGetSymbolAddress: ") +
                              cudaGetErrorString(e));
        return ABCMB_ERR_CUDA;
      }
      g_noalloc_addr[dev] = p;
    }
    scratch = g_noalloc_addr[dev];
  }
  int grid = 0;
  e = abcmb::launch_pert(n_cosmo, cosmo_dev, tables_dev, k_dev, n_items, items_dev, *settings, pt_dev, kstat_dev,
                         scratch, static_cast<cudaStream_t>(stream), abcmb::pert_warps_per_block(), &grid);
  abcmb::set_last_pert_grid(grid);
  if (e != cudaSuccess) {
    abcmb::set_last_error(std::string("abcmb_pert_forward_noalloc: ") + cudaGetErrorString(e));
    return ABCMB_ERR_CUDA;
  }
  return ABCMB_OK;
}
