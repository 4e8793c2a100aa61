// Equations of state of the reference (sim/hydro.py:121-139, physics/eos.py): the ideal gas, the
// radiation limit and gas + radiation in local thermodynamic equilibrium,
//     u = 3 k T / (2 mu m_p) + a T^4 / rho,     P = rho k T / (mu m_p) + a T^4 / 3,
//     beta = P_gas / P,  Gamma_1 = beta + (4 - 3 beta)^2 (gamma - 1) / (beta + 12 (gamma - 1)(1 - beta))
//     with gamma = 5/3,  c_s = sqrt(Gamma_1 P / rho),
// T from (rho, u) by the reference's Newton iteration on log T inside a bisection bracket
// [1, 1e13] K narrowed every iteration, tolerance 1e-12, at most 200 iterations
// (sim/fastphys.py:45-72, _gasrad_t_kernel).  Physical (SI) units inside the T-solve.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/nebula_b200.h"
#include "common.cuh"

namespace nbk {

struct EosParams {
  int kind;         // 0 ideal, 1 gas + radiation, 2 radiation limit
  double gamma;     // ideal gas
  double rho_si;    // kg/m^3 per code density
  double u_si;      // J/kg per code specific energy (c^2)
  double a1;        // 3 k / (2 mu m_p)  [J/(kg K)]
  double kb_mu;     // k / (mu m_p)
  double a_rad;     // radiation constant [J m^-3 K^-4]
};

constexpr double EOS_LT_MIN = 0.0;                   // log(1 K)
constexpr double EOS_LT_MAX = 29.933606208922594;    // log(1e13 K)
constexpr double EOS_TOL = 1e-12;
constexpr int EOS_MAX_ITER = 200;

// T [K] from rho [kg/m^3] and u [J/kg]; status 1 = u outside u(1 K)..u(1e13 K), 2 = no convergence
__device__ __forceinline__ double gasrad_temperature(double r, double uu, double a1, double a_rad,
                                                     int* status) {
  const double t_min = 1.0, t_max = 1e13;
  const double u_lo = a1 * t_min + a_rad * (t_min * t_min * t_min * t_min) / r;
  const double t2m = t_max * t_max;
  const double u_hi = a1 * t_max + a_rad * (t2m * t2m) / r;
  if (uu < u_lo || uu > u_hi) {
    *status = 1;
    return 0.0;
  }
  double lo = EOS_LT_MIN, hi = EOS_LT_MAX;
  double t0 = fmin(uu / a1, pow(uu * r / a_rad, 0.25));
  double lt = log(fmin(fmax(t0, t_min), t_max));
  *status = 2;
  for (int it = 0; it < EOS_MAX_ITER; ++it) {
    double t = exp(lt);
    double t2 = t * t;
    double t4 = t2 * t2;
    double f = a1 * t + a_rad * t4 / r - uu;
    double dfdl = a1 * t + 4.0 * a_rad * t4 / r;
    if (f < 0) lo = lt;
    if (f > 0) hi = lt;
    double nw = lt - f / dfdl;
    if (nw <= lo || nw >= hi || !isfinite(nw)) nw = 0.5 * (lo + hi);
    double step = fabs(nw - lt);
    lt = nw;
    if (step < EOS_TOL) {
      *status = 0;
      break;
    }
  }
  return exp(lt);
}

// P (code), c_s (c) and, for gas + radiation, T [K] and beta_gas of one particle
__device__ __forceinline__ void eos_point(const EosParams& ep, double rho, double u, double& P,
                                          double& cs, double& T, double& beta, int* err) {
  if (ep.kind == 1) {
    const double rho_si = rho * ep.rho_si;
    int status = 0;
    T = gasrad_temperature(rho_si, u * ep.u_si, ep.a1, ep.a_rad, &status);
    if (status == 1) set_error(err, ERR_EOS_RANGE);
    if (status == 2) set_error(err, ERR_EOS_CONVERGE);
    const double t2 = T * T;
    const double p_gas = rho_si * ep.kb_mu * T;
    const double p_rad = ep.a_rad * (t2 * t2) / 3.0;
    beta = p_gas / (p_gas + p_rad);
    P = (p_gas + p_rad) / (ep.rho_si * ep.u_si);
    const double g = 5.0 / 3.0 - 1.0;
    const double g1 = beta + (4.0 - 3.0 * beta) * (4.0 - 3.0 * beta) * g / (beta + 12.0 * g * (1.0 - beta));
    cs = sqrt(g1 * P / rho);
  } else if (ep.kind == 2) {
    P = rho * u / 3.0;
    cs = sqrt(4.0 * u / 9.0);
    T = 0.0;
    beta = 0.0;
  } else {
    P = (ep.gamma - 1.0) * rho * u;
    cs = sqrt(ep.gamma * (ep.gamma - 1.0) * u);
    T = 0.0;
    beta = 1.0;
  }
}

EosParams eos_of(const nb_params* prm);  // engine.cu

}  // namespace nbk
