// Parameters and launchers of the SPH pair passes (sph.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace nbk {

struct DensityParams {
  int kid;
  double cnorm, eta, tol, h_max;
  const float* massf = nullptr;  // FP32 form: neighbour masses as floats (sorted order), or null
};

struct ForceParams {
  int kid;
  double cnorm;
  int use_sph;    // pressure force, P dV work, viscosity, conductivity
  int use_visc;
  int use_cond;
  int cond_signal;
  double beta, alpha_u;
  int use_disc;   // disc viscosity (Lodato-Price AV form on every pair)
  double disc_alpha_av;
  int tighten;    // skip list entries with r >= 2 max(h_a, h_b)
};

struct ForceOut {
  double* acc = nullptr;    // (rows, 3)
  double* dudt = nullptr;
  double* vsig = nullptr;
  double* vheat = nullptr;
  double* cheat = nullptr;
  double* dacc = nullptr;   // disc viscosity acceleration (rows, 3)
  double* ddudt = nullptr;  // disc viscosity heating
  int64_t* pairs = nullptr; // interacting pairs per row
};

template <typename I>
void launch_density64(int64_t nrows, const int64_t* rows, const double4* pos, const double* mass,
                      const double* h_start, const double* h_search, const int64_t* off,
                      const I* idx, DensityParams prm, const int32_t* out_map, double* h_out,
                      double* rho, double* omega, int64_t* iters, int64_t* flags, int64_t* work,
                      cudaStream_t st);
template <typename I>
void launch_density32(int64_t nrows, const int64_t* rows, const float4* pos, const double* box6,
                      const double* mass, const double* h_start, const double* h_search,
                      const int64_t* off, const I* idx, DensityParams prm, const int32_t* out_map,
                      double* h_out, double* rho, double* omega, int64_t* iters, int64_t* flags,
                      int64_t* work, cudaStream_t st);
template <typename I>
void launch_forces64(int64_t nrows, const int64_t* rows, const double4* pos, const double4* vm,
                     const double4* hydro, const double4* aux, const int64_t* off, const I* idx,
                     ForceParams prm, const int32_t* out_map, ForceOut out, cudaStream_t st);
template <typename I>
void launch_forces32(int64_t nrows, const int64_t* rows, const float4* pos, const double* box6,
                     const float4* vm, const float4* hydro, const float4* aux,
                     const int64_t* off, const I* idx, ForceParams prm, const int32_t* out_map,
                     ForceOut out, cudaStream_t st);

void pack_pos(int64_t n, const double* pos, const double* w, double4* out, cudaStream_t st);
void pack4(int64_t n, const double* a, const double* b, const double* c, const double* d,
           double4* out, cudaStream_t st);
void pack_vm(int64_t n, const double* vel, const double* m, double4* out, cudaStream_t st);

}  // namespace nbk
