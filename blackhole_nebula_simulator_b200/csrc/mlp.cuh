// The learned cooling network: 3 inputs (log rho, log T, log dt, each scaled to [-1, 1] over the
// training hull) -> 64 -> 64 -> 64 (SiLU) -> 1 output, the fraction f = (u - u_new)/(u - u_floor)
// of the energy above the floor that one cooling step removes.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "cooling.cuh"

namespace nbk {

constexpr int MLP_IN = 3;
constexpr int MLP_H = 64;
// parameter offsets in the flat FP32 vector: W1 (64x3), b1, W2 (64x64), b2, W3 (64x64), b3,
// W4 (1x64), b4
constexpr int MLP_W1 = 0;
constexpr int MLP_B1 = MLP_W1 + MLP_H * MLP_IN;
constexpr int MLP_W2 = MLP_B1 + MLP_H;
constexpr int MLP_B2 = MLP_W2 + MLP_H * MLP_H;
constexpr int MLP_W3 = MLP_B2 + MLP_H;
constexpr int MLP_B3 = MLP_W3 + MLP_H * MLP_H;
constexpr int MLP_W4 = MLP_B3 + MLP_H;
constexpr int MLP_B4 = MLP_W4 + MLP_H;
constexpr int MLP_NPARAM = MLP_B4 + 1;  // 8641

// The training hull and the unit conversions of the inputs.
struct MlpHull {
  double rho_unit_cgs;  // g/cm^3 per code density
  double t_unit_s;      // s per code time
  double lrho_lo, lrho_hi;  // log10 rho [g/cm^3]
  double lt_lo, lt_hi;      // log10 T [K]
  double ldt_lo, ldt_hi;    // log10 dt [s]
  double check_tol;         // a-posteriori acceptance tolerance (fraction of u)
};

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
  float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// scaled inputs of one sample; false when it lies outside the hull
__device__ __forceinline__ bool mlp_inputs(double u, double rho, double dt, const BremsParams& bp,
                                           const MlpHull& hl, float x[3]) {
  double lr = log10(rho * hl.rho_unit_cgs);
  double lt = log10(bp.tfac * u);
  double ld = log10(dt * hl.t_unit_s);
  x[0] = (float)(2.0 * (lr - hl.lrho_lo) / (hl.lrho_hi - hl.lrho_lo) - 1.0);
  x[1] = (float)(2.0 * (lt - hl.lt_lo) / (hl.lt_hi - hl.lt_lo) - 1.0);
  x[2] = (float)(2.0 * (ld - hl.ldt_lo) / (hl.ldt_hi - hl.ldt_lo) - 1.0);
  return lr >= hl.lrho_lo && lr <= hl.lrho_hi && lt >= hl.lt_lo && lt <= hl.lt_hi &&
         ld >= hl.ldt_lo && ld <= hl.ldt_hi;
}

// the label: f of the exact integrator (0 at or below the floor)
__device__ __forceinline__ float mlp_label(double u, double rho, double dt, const BremsParams& bp) {
  double un = brems_cool_one(u, rho, dt, bp);
  double d = u - bp.u_floor;
  return d > 0 ? (float)((u - un) / d) : 0.0f;
}

}  // namespace nbk
