// nb_density_noalloc: the density operator (nb_density) for callers that cannot allocate device
// memory, e.g. code running inside a host framework whose device allocator it does not own, or a
// pre-planned run that must not allocate once set up.  It needs no context (nb_create allocates)
// and calls no cudaMalloc, cudaFree or allocating library routine.
//
// Its only scratch, the packed (x, y, z) positions the density kernel reads, lives in the
// file-scope array below, of a fixed maximum of NB_NOALLOC_MAX_N particles (8 MiB).  Every GPU
// that loads the library holds that array until the process exits.  All calls share it and it
// keeps the last call's contents; each call overwrites the first n entries before reading them,
// so nothing needs clearing, but calls that overlap on the GPU (different streams, or different
// host threads on the same device) race on it and must be serialised by the caller.
#include <cstdio>
#include <mutex>

#include "../../include/nebula_b200.h"
#include "common.cuh"
#include "sph.cuh"

namespace {

static __device__ __align__(256) double4 g_noalloc_pos[NB_NOALLOC_MAX_N];

// Device address of g_noalloc_pos on each device, looked up once per device.  In host code the
// symbol's name is only a host-side stand-in: a kernel handed &g_noalloc_pos would read the wrong
// memory, so the address comes from cudaGetSymbolAddress with that device current.
constexpr int kMaxDevices = 64;
double4* g_addr[kMaxDevices] = {nullptr};
std::mutex g_mutex;

int scratch_for_current_device(double4** out, char* msg, size_t msg_len) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    std::snprintf(msg, msg_len, "nb_density_noalloc: no usable current device (%s)",
                  cudaGetErrorString(e));
    return -2;
  }
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_pos);
    if (e != cudaSuccess || !p) {
      std::snprintf(msg, msg_len, "nb_density_noalloc: cudaGetSymbolAddress failed: %s",
                    cudaGetErrorString(e));
      return -2;
    }
    g_addr[dev] = (double4*)p;
  }
  *out = g_addr[dev];
  return 0;
}

thread_local char g_msg[256] = {0};

}  // namespace

extern "C" {

const char* nb_noalloc_last_error(void) { return g_msg; }

int nb_density_noalloc(int64_t n, const double* pos, const double* mass, const double* h_start,
                       const double* h_search, const int64_t* offset, const int64_t* index,
                       int64_t nrows, const int64_t* rows, int kernel_id, double eta, double tol,
                       double h_max, double* h_out, double* rho, double* omega, int64_t* iters,
                       int64_t* flags, void* stream) {
  g_msg[0] = 0;
  if (n < 0 || n > NB_NOALLOC_MAX_N) {
    std::snprintf(g_msg, sizeof(g_msg),
                  "nb_density_noalloc: n = %lld particles is beyond the fixed scratch of %d",
                  (long long)n, (int)NB_NOALLOC_MAX_N);
    return NB_ERR_INPUT;
  }
  if (rows && (nrows < 0 || nrows > n)) {
    std::snprintf(g_msg, sizeof(g_msg),
                  "nb_density_noalloc: nrows = %lld rows of n = %lld particles (must be 0..n)",
                  (long long)nrows, (long long)n);
    return NB_ERR_INPUT;
  }
  if (kernel_id != 0 && kernel_id != 1) {
    std::snprintf(g_msg, sizeof(g_msg), "nb_density_noalloc: kernel_id must be 0 or 1");
    return NB_ERR_INPUT;
  }
  if (n == 0) return 0;
  double4* scratch = nullptr;
  int r = scratch_for_current_device(&scratch, g_msg, sizeof(g_msg));
  if (r != 0) return r;
  cudaStream_t st = (cudaStream_t)stream;
  nbk::pack_pos(n, pos, nullptr, scratch, st);
  double cn = kernel_id == 0 ? 1.0 / M_PI : 495.0 / (256.0 * M_PI);
  nbk::DensityParams dp{kernel_id, cn, eta, tol, h_max};
  nbk::launch_density64<int64_t>(rows ? nrows : n, rows, scratch, mass, h_start, h_search, offset,
                                 index, dp, nullptr, h_out, rho, omega, iters, flags, nullptr, st);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::snprintf(g_msg, sizeof(g_msg), "nb_density_noalloc: launch failed: %s",
                  cudaGetErrorString(e));
    return -2;
  }
  return 0;
}

}  // extern "C"
