// Step runtime entry points shared between engine.cu, steps.cu and capi.cu.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/nebula_b200.h"
#include "engine.cuh"

namespace nbk {

constexpr int K_MAX = 40;

// How a hydro pass advances the viscosity switch and where the reconstruction's gradients come
// from: switch_on for a step (not the initialisation) with its length dt, or per row
// (n_end - n_beg) tick in block steps; recon_full: gradients of the touched particles over
// their untightened lists (block steps) instead of every particle over its interacting pairs.
struct ShockStep {
  int switch_on = 0;
  double dt = 0.0;
  const int64_t* n_beg = nullptr;
  const int64_t* n_end = nullptr;
  double tick = 0.0;
  int recon_full = 0;
  int want_tight = 0;  // block steps: the force pass also writes the rows' interacting entries
  // the touched set holds every list entry of the rows (marked on the lists the force pass
  // walks), so the force pass reads records of touched particles only
  int touched_covers_lists = 0;
};

// rows_mask / first_fail: the rows' mask and the first reuse test's outcome when
// reuse_first_test ran on it already (first_fail -1: neither)
int compute_density(Engine& E, int64_t n, const double* x, const double* mass, double* h,
                    double* rho, double* omega, int64_t nrows, const int64_t* rows,
                    const nb_params* prm, int64_t* builds, int64_t* reuses, cudaStream_t st,
                    const uint8_t* rows_mask = nullptr, int first_fail = -1);
int reuse_first_test(Engine& E, int64_t n, const double* x, const double* hg_in,
                     const uint8_t* mask, int* fail, cudaStream_t st);
// out = the indices of mask's set entries, ascending; count read on the host (with W.d_i64[1]
// into *also when given)
int select_mask(Engine& E, int64_t n, const uint8_t* mask, int64_t* out, int64_t* count,
                cudaStream_t st, int64_t* also = nullptr);
int engine_forces(Engine& E, nb_state* s, const double* vel, const double* u, int64_t nrows,
                  const int64_t* rows, const nb_params* prm, const uint8_t* touched,
                  const ShockStep& sk, cudaStream_t st);

int hydro_rows(Engine& E, nb_state* s, const nb_params* prm, int64_t nrows, const int64_t* rows,
               const double* vel, const double* u, cudaStream_t st,
               const ShockStep& sk = ShockStep{});
int coupled_initialise(Engine& E, nb_state* s, const nb_params* prm, cudaStream_t st);
int coupled_step(Engine& E, nb_state* s, const nb_params* prm, double dt, cudaStream_t st);
int coupled_stable_dt(Engine& E, nb_state* s, const nb_params* prm, double* dt, cudaStream_t st);
int block_initialise(Engine& E, nb_state* s, const nb_params* prm, cudaStream_t st);
// with v_eval_out (n x 3) and u_eval_out (n): stops after the closing kicks (the first half of a
// split step) and leaves the evaluation's velocities and energies there
int block_advance(Engine& E, nb_state* s, const nb_params* prm, int64_t* rows_out,
                  cudaStream_t st, double* v_eval_out = nullptr, double* u_eval_out = nullptr);
int block_finish(Engine& E, nb_state* s, const nb_params* prm, int64_t nrows, const int64_t* rows,
                 int redo, const double* v_eval, const double* u_eval, cudaStream_t st);
int block_wake_doomed(Engine& E, nb_state* s, int64_t nrows, const int64_t* rows,
                      const uint8_t* doomed, cudaStream_t st);
int block_land(Engine& E, nb_state* s, const nb_params* prm, cudaStream_t st);

// launchers of engine.cu kernels used by steps.cu
int mark_rows(Engine& E, int64_t nrows, const int64_t* rows, int tight, const double* x,
              const double* h, uint8_t* mark, cudaStream_t st);
// rows as ascending sorted positions in E.ws.rows_s (count ns) and E.ws.pk0 = sorted (x, h)
int sorted_rows(Engine& E, int64_t nrows, const int64_t* rows, int64_t* ns, cudaStream_t st);
int sorted_rows_and_pack(Engine& E, int64_t nrows, const int64_t* rows, const double* x,
                         const double* h, int64_t* ns, cudaStream_t st);
// checks read at the next host synchronisation (see Workspace::pend_*)
int pending_enqueue(Engine& E, cudaStream_t st);
int pending_finish(Engine& E, cudaStream_t st);
int pending_flush(Engine& E, cudaStream_t st);
void mask_and_not(int64_t n, const uint8_t* a, const uint8_t* b, uint8_t* out, cudaStream_t st);
void mask_or(int64_t n, const uint8_t* a, uint8_t* b, cudaStream_t st);

}  // namespace nbk
