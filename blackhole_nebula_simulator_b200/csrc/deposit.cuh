// Launchers of the particle -> grid deposition kernels (deposit.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace nbk {

constexpr int DEP_FIELDS = 6;  // m, m T, m T^4, m vx, m vy, m vz per cell

struct LogGeom {
  double r_min, dlnr, dth, dph;
  int nr, nth, nph;
  const double *sth, *cth, *dcth, *cph, *sph;  // theta / phi cell-centre tables
};

void launch_deposit_log(int64_t n, const double* x, const double* h, const double* m,
                        const double* t, const double* v, const LogGeom& g, int kid,
                        double* acc, double* outside, unsigned long long* n_tri,
                        cudaStream_t st);
void launch_deposit_box(int64_t n, const double* x, const double* h, const double* m,
                        const double* t, const double* v, double x0, double y0, double z0,
                        double dx, int nb, int kid, double* acc, double* outside,
                        unsigned long long* n_tri, cudaStream_t st);
void launch_grid_finish(int64_t ncell, const double* acc, const double* vol, int64_t per,
                        double* mass, float* rho, float* t_mass, float* t_em, float* vel,
                        cudaStream_t st);
// sums2: two device doubles (fine and coarse mass), zeroed by the caller
void launch_refine_sums(const double* acc_c, const double* vol_c, int nrc, int nthc, int nphc,
                        const double* vol_f, int nr, int nth, int nph, int cr, int ct, int cp,
                        double* out, double* sums2, cudaStream_t st);

// spatial order of the particles (grid_kind 0: log grid g, 1: box): keys and identity indices
void launch_deposit_keys(int64_t n, const double* x, int grid_kind, const LogGeom& g, double x0,
                         double y0, double z0, double dx, int nb, unsigned long long* keys,
                         int32_t* idx, cudaStream_t st);
// out (9 n doubles): x (3n), h, m, t, v (3n) gathered in idx order
void launch_deposit_gather(int64_t n, const int32_t* idx, const double* x, const double* h,
                           const double* m, const double* t, const double* v, double* out,
                           cudaStream_t st);

}  // namespace nbk
