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
  // velocity reconstruction in the viscosity (physics/viscosity.py:116-158): the velocity
  // gradients of every particle the pass reads, 9 per particle (row-major dv^i/dx^j) in the
  // pass's index space, double for the FP64 form and float for the FP32 form
  int use_recon = 0;
  int closeness = 1;
  int gate = 2;   // 0 both jumps approaching, 1 reconstructed jump only, 2 min-mod
  double eta_crit = 0.0, eta_fold = 0.2;
  const double* gv64 = nullptr;
  const float* gv32 = nullptr;
  // the rows' interacting entries for the level limiter (self included, list order) into tidx
  // (the lists' layout) and their counts into tcnt (row order); the FP32 form decides entries
  // within 1e-5 of the boundary from the sorted FP64 (x, y, z, h) in pos64
  int32_t* tidx = nullptr;
  int32_t* tcnt = nullptr;
  const double4* pos64 = nullptr;
};

// Corrected velocity (and acceleration) gradients, sim/sph.py:693-902.
struct GradParams {
  int kid;
  double cnorm;
  int tighten;    // only list entries with r < 2 max(h_a, h_b) (the tightened lists)
  const uint8_t* mask = nullptr;  // with rows == null: only particles whose mask (caller order,
                                  // through out_map) is set
};
struct GradOut {
  double* div = nullptr;    // div v, |curl v|, d(div v)/dt at the output index (needs acc)
  double* curl = nullptr;
  double* ddiv = nullptr;
  double* gv = nullptr;     // 9 per particle at the pass's own index
  // Cullen-Dehnen update of alpha at the output index (physics/viscosity.py:83-113), from the
  // row's c_s and h (caller order) over dt, or over (n_end - n_beg) tick when n_beg is set
  double* alpha = nullptr;
  const double* cs = nullptr;
  const double* h = nullptr;
  double dt = 0.0, tick = 0.0;
  const int64_t *n_beg = nullptr, *n_end = nullptr;
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

template <typename I>
void launch_gradients(int64_t nrows, const int64_t* rows, const double4* pos, const double4* vm,
                      const double4* hydro, const double4* acc, const int64_t* off, const I* idx,
                      GradParams prm, const int32_t* out_map, GradOut out, cudaStream_t st);

// The switch and the reconstruction's gradients of one step in one pass over the sorted lists:
// gv (sorted) for the particles of live_mask (caller order; null = all) when recon, over their
// untightened lists when recon_full; the switch's alpha update for the rows of row_sorted
// (sorted mask; null = no switch) with acc (sorted previous accelerations).
void launch_shock_gradients(int64_t n, const double4* pos, const double4* vm,
                            const double4* hydro, const double4* acc, const int64_t* off,
                            const int32_t* idx, int kid, double cnorm, int recon, int recon_full,
                            const uint8_t* live_mask, const uint8_t* row_sorted,
                            const int32_t* perm, GradOut out, cudaStream_t st);

void pack_pos(int64_t n, const double* pos, const double* w, double4* out, cudaStream_t st);
void pack4(int64_t n, const double* a, const double* b, const double* c, const double* d,
           double4* out, cudaStream_t st);
void pack_vm(int64_t n, const double* vel, const double* m, double4* out, cudaStream_t st);

}  // namespace nbk
