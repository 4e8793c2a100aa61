// Launchers of the GN gravity kernels (gravity.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

namespace nbk {

constexpr double GLF_TOL = 1e-15;
constexpr int GLF_MAX_ITER = 10;
constexpr double GLF_R_MIN = 2.5;

// (This header is compiled without fused multiply-add, so every expression rounds like the
// reference's; integer powers are formed as Numba forms them: r^4 = (r^2)^2, r^5 = r^4 r.)
__device__ __forceinline__ void gn_dh_dx(const double x[3], const double p[3], double g[3]) {
  double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  double r2 = r * r, r3 = r2 * r, r4 = r2 * r2, r5 = r4 * r;
  double c = -2.0 * (r - 2.0) / r4;
  double da = 2.0 / r2;
  double dc = (6.0 * r - 16.0) / r5;
  double px = p[0] * x[0] + p[1] * x[1] + p[2] * x[2];
  double pp = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
  double radial = (0.5 * da * pp + 0.5 * dc * px * px) / r + 1.0 / r3;
  for (int k = 0; k < 3; ++k) g[k] = radial * x[k] + c * px * p[k];
}

__device__ __forceinline__ void gn_dh_dp(const double x[3], const double p[3], double v[3]) {
  double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  double r2 = r * r;
  double a = (r - 2.0) / r;
  double c = -2.0 * (r - 2.0) / (r2 * r2);
  double cpx = c * (p[0] * x[0] + p[1] * x[1] + p[2] * x[2]);
  for (int k = 0; k < 3; ++k) v[k] = a * p[k] + cpx * x[k];
}

__device__ __forceinline__ bool glf_converged(const double nw[3], const double old[3]) {
  double d = (nw[0] - old[0]) * (nw[0] - old[0]) + (nw[1] - old[1]) * (nw[1] - old[1]) +
             (nw[2] - old[2]) * (nw[2] - old[2]);
  return d <= GLF_TOL * GLF_TOL * (nw[0] * nw[0] + nw[1] * nw[1] + nw[2] * nw[2]);
}

// One step: p_half = p - dt/2 dH/dx(x, p_half) (fixed point); x1 = x + dt/2 [dH/dp(x, p_half) +
// dH/dp(x1, p_half)] (fixed point); p1 = p_half - dt/2 dH/dx(x1, p_half).  Returns iterations, or
// -1 / -2 (a stage did not converge in 10 iterations), -3 (r <= 2.5).
__device__ __forceinline__ int glf_one(const double x[3], const double p[3], double dt, double xo[3], double po[3]) {
  for (int k = 0; k < 3; ++k) {
    xo[k] = x[k];
    po[k] = p[k];
  }
  if (x[0] * x[0] + x[1] * x[1] + x[2] * x[2] <= GLF_R_MIN * GLF_R_MIN) return -3;
  double half = 0.5 * dt;
  int iters = 0;
  double hp[3] = {p[0], p[1], p[2]}, g[3], nw[3];
  bool ok = false;
  for (int it = 0; it < GLF_MAX_ITER; ++it) {
    gn_dh_dx(x, hp, g);
    for (int k = 0; k < 3; ++k) nw[k] = p[k] - half * g[k];
    iters += 1;
    ok = glf_converged(nw, hp);
    for (int k = 0; k < 3; ++k) hp[k] = nw[k];
    if (ok) break;
  }
  if (!ok) return -1;
  double v[3], w[3], y[3];
  gn_dh_dp(x, hp, v);
  for (int k = 0; k < 3; ++k) y[k] = x[k] + dt * v[k];
  ok = false;
  for (int it = 0; it < GLF_MAX_ITER; ++it) {
    gn_dh_dp(y, hp, w);
    for (int k = 0; k < 3; ++k) nw[k] = x[k] + half * (v[k] + w[k]);
    iters += 1;
    ok = glf_converged(nw, y);
    for (int k = 0; k < 3; ++k) y[k] = nw[k];
    if (ok) break;
  }
  if (!ok) return -2;
  gn_dh_dx(y, hp, g);
  for (int k = 0; k < 3; ++k) {
    xo[k] = y[k];
    po[k] = hp[k] - half * g[k];
  }
  return iters;
}


void launch_glf(int64_t n, const double* x, const double* p, const double* dt, double dt_scalar,
                double* xo, double* po, int64_t* iters, cudaStream_t st);
void launch_integrate_orbit(int norb, const double* state0, double dt_max, double eta,
                            int64_t n_end, int64_t max_records, double* t_out, double* s_out,
                            int64_t* it_out, int64_t* nrec, cudaStream_t st);
void launch_v_from_p(int64_t n, const double* x, const double* p, double* v, cudaStream_t st);
void launch_p_from_v(int64_t n, const double* x, const double* v, double* p, cudaStream_t st);
int ledger_blocks(int64_t n);
void launch_ledger(int64_t n, const double* x, const double* p, const double* u, const double* m,
                   double* part, double* out, cudaStream_t st);

}  // namespace nbk
