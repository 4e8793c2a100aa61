// Shared device helpers for the sm_100a SPH step.
//
// Error handling never traps on the device: kernels record the first problem in a device error
// word (atomicCAS from 0) and the host maps it to the reference's exception types.  Every loop
// over data-dependent work has a fixed bound.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define NB_THREADS 256

namespace nbk {

// error codes written to the device error word (0 = ok)
enum : int {
  ERR_OK = 0,
  ERR_LIST_OVERFLOW = 1,     // a neighbour list longer than the space reserved for it
  ERR_TRAVERSAL_STACK = 2,   // tree traversal stack exhausted (never expected: depth-bounded)
  ERR_BAD_INDEX = 3,         // an index outside [0, n)
  ERR_NONPOSITIVE_U = 4,     // u <= 0 where the equation of state needs it
  ERR_LEVEL = 5,             // a level beyond K_MAX
  ERR_LIMITER = 6,           // the level limiter did not settle within its sweep bound
  ERR_DT = 7,                // a wanted time step that is not positive
  ERR_EOS_RANGE = 8,         // u outside the gas + radiation EOS bracket [1, 1e13] K
  ERR_EOS_CONVERGE = 9,      // the gas + radiation temperature did not converge
};

__device__ __forceinline__ void set_error(int* err, int code) {
  if (err) atomicCAS(err, 0, code);
}

// Kernel shapes f(q), f'(q): cubic spline (kid 0, C = 1/pi) and Wendland C4 (kid 1,
// C = 495/(256 pi)), support q < 2 (reference physics/kernels.py:26-51, sim/kernels_nb.py:16-43).
template <typename R>
__device__ __forceinline__ R kernel_f(R q, int kid) {
  if (q >= R(2)) return R(0);
  if (kid == 0) {
    if (q < R(1)) return R(1) - R(1.5) * q * q + R(0.75) * q * q * q;
    R t = R(2) - q;
    return R(0.25) * t * t * t;
  }
  R x = R(1) - R(0.5) * q;
  R x2 = x * x;
  return x2 * x2 * x2 * (R(35.0 / 12.0) * q * q + R(3) * q + R(1));
}

template <typename R>
__device__ __forceinline__ R kernel_df(R q, int kid) {
  if (q >= R(2)) return R(0);
  if (kid == 0) {
    if (q < R(1)) return R(-3) * q + R(2.25) * q * q;
    R t = R(2) - q;
    return R(-0.75) * t * t;
  }
  R x = R(1) - R(0.5) * q;
  R x2 = x * x;
  return R(-7.0 / 3.0) * q * x2 * x2 * x * (R(5) * q + R(2));
}

// FP64 arithmetic that must round exactly like the reference's (no fused multiply-add): the
// neighbour-list distance test r^2 < (2h)^2 is compared bit for bit.
__device__ __forceinline__ double d2_exact(double dx, double dy, double dz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// List entries are read once per pass: load them with the streaming hint (evict first), so they
// do not push the gathered neighbour records out of L2.
template <typename I>
__device__ __forceinline__ I ld_stream(const I* p) {
  if constexpr (sizeof(I) == 4)
    return (I)__ldcs(reinterpret_cast<const int*>(p));
  else
    return (I)__ldcs(reinterpret_cast<const long long*>(p));
}

// Kahan-compensated accumulator for the FP32 pair sums.
struct Kahan {
  float s, c;
  __device__ __forceinline__ Kahan() : s(0.f), c(0.f) {}
  __device__ __forceinline__ void add(float v) {
    float y = __fsub_rn(v, c);
    float t = __fadd_rn(s, y);
    c = __fsub_rn(__fsub_rn(t, s), y);
    s = t;
  }
};

// Launches of this library's own kernels (read through nb_launch_count).
extern unsigned long long g_launch_count;
inline int count_launch() {
  __atomic_add_fetch(&g_launch_count, 1ull, __ATOMIC_RELAXED);
  return 0;
}

// Host waits on a stream (read through nb_sync_count): each is a round trip that leaves the GPU
// idle until the host launches again.
extern unsigned long long g_sync_count;
inline cudaError_t host_sync(cudaStream_t st) {
  __atomic_add_fetch(&g_sync_count, 1ull, __ATOMIC_RELAXED);
  return cudaStreamSynchronize(st);
}

inline unsigned grid_for(int64_t n, int threads = NB_THREADS) {
  int64_t b = (n + threads - 1) / threads;
  return (unsigned)(b > 0 ? b : 1);
}

}  // namespace nbk
