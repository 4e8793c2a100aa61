// Cooling laws (device functions shared by the cooling and step kernels).
//
// beta-cooling (reference physics/cooling.py:23-40; Gammie 2001): u relaxes exactly toward the
// floor, u_new = u_f + (u - u_f) exp(-dt / t_cool), t_cool = beta r^(3/2).
//
// Bremsstrahlung (this project's law; the reference has no bremsstrahlung cooling): optically
// thin free-free emission eps = C_ff g_B T^(1/2) (1 + a T) n_e sum n_i Z_i^2 (Rybicki & Lightman
// 1979, Eq. 5.15b, with the relativistic factor 1 + 4.4e-10 T) on an ideal gas T = tfac u.  At
// fixed rho, arctan(sqrt(a T)) falls linearly in time by kappa rho dt, so the update is exact;
// gas at or below the floor temperature does not cool, gas that would cool past it stops there.
#pragma once
#include <cuda_runtime.h>

namespace nbk {

struct BremsParams {
  double tfac;     // T [K] per code u
  double b;        // sqrt(a), a = 4.4e-10 1/K
  double kappa;    // fall of arctan(b sqrt(T)) per code density per code time
  double u_floor;  // code u at the floor temperature
  double t_floor;  // K
};

__device__ __forceinline__ double beta_cool_one(double u, double u_floor, double dt, double t_cool) {
  double decay = exp(-dt / t_cool);
  return u_floor + (u - u_floor) * decay;
}

__device__ __forceinline__ double brems_cool_one(double u, double rho, double dt, const BremsParams& c) {
  double t0 = c.tfac * u;
  if (t0 <= c.t_floor) return u;
  double th0 = atan(c.b * sqrt(t0));
  double th = th0 - c.kappa * rho * dt;
  double th_f = atan(c.b * sqrt(c.t_floor));
  if (th <= th_f) return c.u_floor;
  double ratio = tan(th) / tan(th0);
  return u * ratio * ratio;
}

// du/dt of the bremsstrahlung law (code units, <= 0).
__device__ __forceinline__ double brems_rate(double u, double rho, const BremsParams& c) {
  double t = c.tfac * u;
  return -2.0 * c.kappa / c.b * rho * sqrt(t) * (1.0 + c.b * c.b * t) / c.tfac;
}

}  // namespace nbk
