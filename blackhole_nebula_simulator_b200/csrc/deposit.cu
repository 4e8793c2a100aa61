// Particle -> grid deposition for the renderer (render/gasgrid.py:316-597 of the reference):
// each particle's fields (m, m T, m T^4, m v) go to the cells whose centres lie inside its
// support (q < 2), weighted by f(q) V_c and normalised; fewer than 8 such centres: trilinear
// weights in index space over the 8 nearest centres.  Weight beyond the grid goes to the
// `outside` total.  One thread per particle walks its candidate centres twice (sum of weights,
// then the atomic adds); the cell sums are FP64.  Compiled without fused multiply-add, so a
// particle's weights round like the reference's (the order of the atomic adds does not).
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "deposit.cuh"

namespace nbk {

constexpr int DEP_MIN_CELLS = 8;
constexpr int DEP_INNER_VIRTUAL = 64;  // virtual log shells below r_min (render/gasgrid.py:49)

__device__ __forceinline__ double py_mod(double a, double b) {  // Python's a % b, b > 0
  double r = fmod(a, b);
  if (r < 0.0) r += b;
  return r;
}
__device__ __forceinline__ int py_imod(int a, int b) { return ((a % b) + b) % b; }

__device__ __forceinline__ void particle_vals(int64_t p, const double* m, const double* t,
                                              const double* v, double* vals) {
  const double mp = m[p], tp = t[p];
  vals[0] = mp;
  vals[1] = mp * tp;
  vals[2] = mp * pow(tp, 4.0);
  vals[3] = mp * v[3 * p];
  vals[4] = mp * v[3 * p + 1];
  vals[5] = mp * v[3 * p + 2];
}

__device__ __forceinline__ void add_cell(double* acc, int64_t cell, double w, const double* vals) {
  double* c = acc + cell * DEP_FIELDS;
#pragma unroll
  for (int f = 0; f < DEP_FIELDS; ++f) atomicAdd(c + f, w * vals[f]);
}

// render/gasgrid.py:316-412 (_nb_log_kernel_pass): MODE 0 sums f V and counts the centres
// inside the support, MODE 1 adds the normalised weights and returns the mass beyond the grid
template <int MODE>
__device__ void log_pass(const LogGeom& g, double xp, double yp, double zp, double rr,
                         double th, double ph, double hp, int i_lo, int i_hi, int kid,
                         double inv, const double* vals, double* acc, double& wsum, int& n_in,
                         double& outside) {
  const double big = 2.0 * hp;
  const double ct0 = cos(th), st0 = sin(th);
  // q < 2 decided on d^2 against (2h)^2 with a relative margin of 1e-12 (sqrt(d^2) / h only
  // inside the margin); the weights take q = sqrt(d^2) (1 / h), within an ulp of the
  // reference's quotient
  const double big2 = big * big;
  const double in2 = big2 * (1.0 - 1e-12), out2 = big2 * (1.0 + 1e-12);
  const double ih = 1.0 / hp;
  for (int i = i_lo; i <= i_hi; ++i) {
    const double rc = g.r_min * exp((i + 0.5) * g.dlnr);
    const double cos_a = (rc * rc + rr * rr - big * big) / (2.0 * rc * rr);
    if (cos_a > 1.0) continue;
    int j0, j1;
    if (cos_a <= -1.0) {
      j0 = 0;
      j1 = g.nth - 1;
    } else {
      const double a = acos(cos_a);
      j0 = max(0, (int)floor((th - a) / g.dth) - 1);
      j1 = min(g.nth - 1, (int)floor((th + a) / g.dth) + 1);
    }
    const double r1 = g.r_min * exp(i * g.dlnr);
    const double r2 = r1 * exp(g.dlnr);
    const double vr = (r2 * r2 * r2 - r1 * r1 * r1) / 3.0;
    const bool ing = 0 <= i && i < g.nr;
    for (int j = j0; j <= j1; ++j) {
      const double ss = st0 * g.sth[j];
      bool full = true;
      int k0 = 0, k1 = g.nph - 1;
      if (ss > 1e-300 && cos_a > -1.0) {
        const double cd = (cos_a - ct0 * g.cth[j]) / ss;
        if (cd > 1.0 + 1e-12) continue;
        if (cd > -1.0) {
          const double dp = acos(fmin(cd, 1.0));
          k0 = (int)ceil((ph - dp) / g.dph - 0.5) - 1;
          k1 = (int)floor((ph + dp) / g.dph - 0.5) + 1;
          if (k1 - k0 + 1 < g.nph) full = false;
        }
      }
      if (full) {
        k0 = 0;
        k1 = g.nph - 1;
      }
      const double rst = rc * g.sth[j];
      const double dzc = rc * g.cth[j] - zp;
      const double vrt = vr * g.dcth[j] * g.dph;
      for (int kk = k0; kk <= k1; ++kk) {
        const int k = py_imod(kk, g.nph);
        const double dxc = rst * g.cph[k] - xp;
        const double dyc = rst * g.sph[k] - yp;
        const double dd = dxc * dxc + dyc * dyc + dzc * dzc;
        if (dd >= out2) continue;
        const double r = sqrt(dd);
        if (dd >= in2 && !(r / hp < 2.0)) continue;
        const double q = r * ih;
        {
          if (MODE == 0) {
            n_in += 1;
            wsum += kernel_f<double>(q, kid) * vrt;
          } else {
            const double w = kernel_f<double>(q, kid) * vrt * inv;
            if (ing)
              add_cell(acc, ((int64_t)i * g.nth + j) * g.nph + k, w, vals);
            else
              outside += w * vals[0];
          }
        }
      }
    }
  }
}

// render/gasgrid.py:415-531 (_nb_log_deposit_chunk)
__global__ void k_deposit_log(int64_t n, const double* __restrict__ x,
                              const double* __restrict__ h, const double* __restrict__ m,
                              const double* __restrict__ t, const double* __restrict__ v,
                              LogGeom g, int kid, double* __restrict__ acc, double* outside_sum,
                              unsigned long long* n_tri) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= n) return;
  double vals[DEP_FIELDS];
  particle_vals(p, m, t, v, vals);
  const double xp = x[3 * p], yp = x[3 * p + 1], zp = x[3 * p + 2];
  const double rr = sqrt(xp * xp + yp * yp + zp * zp);
  const double hp = h[p];
  const double big = 2.0 * hp;
  const double lnr0 = log(g.r_min);
  const int i_hi = (int)floor((log(rr + big) - lnr0) / g.dlnr);
  int i_lo = -DEP_INNER_VIRTUAL;
  if (!(big >= rr)) i_lo = max((int)floor((log(rr - big) - lnr0) / g.dlnr), -DEP_INNER_VIRTUAL);
  const double th = acos(fmin(1.0, fmax(-1.0, zp / rr)));
  const double ph = py_mod(atan2(yp, xp), 2.0 * 3.141592653589793);
  double wsum = 0.0, out = 0.0;
  int n_in = 0;
  log_pass<0>(g, xp, yp, zp, rr, th, ph, hp, i_lo, i_hi, kid, 0.0, vals, acc, wsum, n_in, out);
  if (n_in >= DEP_MIN_CELLS) {
    log_pass<1>(g, xp, yp, zp, rr, th, ph, hp, i_lo, i_hi, kid, 1.0 / wsum, vals, acc, wsum,
                n_in, out);
    if (out != 0.0) atomicAdd(outside_sum, out);
    return;
  }
  // trilinear fallback (render/gasgrid.py:217-237)
  atomicAdd(n_tri, 1ull);
  const double fr = log(rr / g.r_min) / g.dlnr - 0.5;
  const double fth = th / g.dth - 0.5;
  const double fph = ph / g.dph - 0.5;
  const int i0 = (int)floor(fr);
  int j0 = (int)floor(fth);
  const int k0 = (int)floor(fph);
  const double ti = fr - i0, tk = fph - k0;
  double tj = fth - j0;
  if (j0 < 0) {
    j0 = 0;
    tj = 0.0;
  }
  if (j0 > g.nth - 2) {
    j0 = g.nth - 2;
    tj = 1.0;
  }
  for (int di = 0; di < 2; ++di) {
    const double wi = di == 1 ? ti : 1.0 - ti;
    for (int dj = 0; dj < 2; ++dj) {
      const double wj = dj == 1 ? tj : 1.0 - tj;
      for (int dk = 0; dk < 2; ++dk) {
        const double wk = dk == 1 ? tk : 1.0 - tk;
        const double w = wi * wj * wk;
        const int i = i0 + di;
        if (0 <= i && i < g.nr)
          add_cell(acc, ((int64_t)i * g.nth + j0 + dj) * g.nph + py_imod(k0 + dk, g.nph), w, vals);
        else
          out += w * vals[0];
      }
    }
  }
  if (out != 0.0) atomicAdd(outside_sum, out);
}

// render/gasgrid.py:534-597 (_nb_box_deposit_chunk)
__global__ void k_deposit_box(int64_t n, const double* __restrict__ x,
                              const double* __restrict__ h, const double* __restrict__ m,
                              const double* __restrict__ t, const double* __restrict__ v,
                              double x0, double y0, double z0, double dx, int nb, int kid,
                              double* __restrict__ acc, double* outside_sum,
                              unsigned long long* n_tri) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= n) return;
  double vals[DEP_FIELDS];
  particle_vals(p, m, t, v, vals);
  const double xp = x[3 * p], yp = x[3 * p + 1], zp = x[3 * p + 2];
  const double hp = h[p];
  const double big = 2.0 * hp;
  const int a0 = (int)floor((xp - big - x0) / dx), a1 = (int)floor((xp + big - x0) / dx);
  const int b0 = (int)floor((yp - big - y0) / dx), b1 = (int)floor((yp + big - y0) / dx);
  const int c0 = (int)floor((zp - big - z0) / dx), c1 = (int)floor((zp + big - z0) / dx);
  // The candidate block holds every centre with q < 2.  Two shortcuts leave the result as the
  // full walk gives it: a row (a, b) only visits the chord of the support plus one cell each
  // side (the other centres fail q < 2), and a distance is compared as d^2 against (2h)^2
  // with a relative margin of 1e-12, taking sqrt(d^2) / h only inside the margin.
  const double big2 = big * big;
  const double in2 = big2 * (1.0 - 1e-12), out2 = big2 * (1.0 + 1e-12);
  auto inside = [&](double dd) {
    if (dd < in2) return true;
    if (dd >= out2) return false;
    return sqrt(dd) / hp < 2.0;
  };
  const double ih = 1.0 / hp;  // weights take q = sqrt(d^2) (1 / h), within an ulp of d / h
  auto chord = [&](double dxy2, int& lo, int& hi) {
    const double s = sqrt(fmax(out2 - dxy2, 0.0));
    lo = max(c0, (int)floor((zp - s - z0) / dx) - 1);
    hi = min(c1, (int)floor((zp + s - z0) / dx) + 1);
  };
  // a block wholly beyond the box puts all the particle's mass outside: only the count of
  // centres inside the support (kernel weights or trilinear fallback) is needed
  const bool beyond = a1 < 0 || a0 >= nb || b1 < 0 || b0 >= nb || c1 < 0 || c0 >= nb;
  double wsum = 0.0, out = 0.0;
  int n_in = 0;
  for (int a = a0; a <= a1; ++a) {
    const double dxc = x0 + (a + 0.5) * dx - xp;
    for (int b = b0; b <= b1; ++b) {
      const double dyc = y0 + (b + 0.5) * dx - yp;
      const double dxy2 = dxc * dxc + dyc * dyc;
      if (dxy2 >= out2) continue;
      int cl, ch;
      chord(dxy2, cl, ch);
      for (int c = cl; c <= ch; ++c) {
        const double dzc = z0 + (c + 0.5) * dx - zp;
        const double dd = dxc * dxc + dyc * dyc + dzc * dzc;
        if (inside(dd)) {
          n_in += 1;
          if (!beyond) wsum += kernel_f<double>(sqrt(dd) * ih, kid);
        }
      }
    }
  }
  if (n_in >= DEP_MIN_CELLS && beyond) {
    atomicAdd(outside_sum, vals[0]);
    return;
  }
  if (n_in >= DEP_MIN_CELLS) {
    const double inv = 1.0 / wsum;
    for (int a = a0; a <= a1; ++a) {
      const double dxc = x0 + (a + 0.5) * dx - xp;
      for (int b = b0; b <= b1; ++b) {
        const double dyc = y0 + (b + 0.5) * dx - yp;
        const double dxy2 = dxc * dxc + dyc * dyc;
        if (dxy2 >= out2) continue;
        int cl, ch;
        chord(dxy2, cl, ch);
        for (int c = cl; c <= ch; ++c) {
          const double dzc = z0 + (c + 0.5) * dx - zp;
          const double dd = dxc * dxc + dyc * dyc + dzc * dzc;
          if (inside(dd)) {
            const double w = kernel_f<double>(sqrt(dd) * ih, kid) * inv;
            if (0 <= a && a < nb && 0 <= b && b < nb && 0 <= c && c < nb)
              add_cell(acc, ((int64_t)a * nb + b) * nb + c, w, vals);
            else
              out += w * vals[0];
          }
        }
      }
    }
    if (out != 0.0) atomicAdd(outside_sum, out);
    return;
  }
  atomicAdd(n_tri, 1ull);
  const double fa = (xp - x0) / dx - 0.5, fb = (yp - y0) / dx - 0.5, fc = (zp - z0) / dx - 0.5;
  const int ia = (int)floor(fa), ib = (int)floor(fb), ic = (int)floor(fc);
  const double ta = fa - ia, tb = fb - ib, tc = fc - ic;
  for (int da = 0; da < 2; ++da) {
    const double wa = da == 1 ? ta : 1.0 - ta;
    for (int db = 0; db < 2; ++db) {
      const double wb = db == 1 ? tb : 1.0 - tb;
      for (int dc = 0; dc < 2; ++dc) {
        const double wc = dc == 1 ? tc : 1.0 - tc;
        const double w = wa * wb * wc;
        const int a = ia + da, b = ib + db, c = ic + dc;
        if (0 <= a && a < nb && 0 <= b && b < nb && 0 <= c && c < nb)
          add_cell(acc, ((int64_t)a * nb + b) * nb + c, w, vals);
        else
          out += w * vals[0];
      }
    }
  }
  if (out != 0.0) atomicAdd(outside_sum, out);
}

// render/gasgrid.py:293-313 (_finish): mass, rho = M / V, mass-weighted T, (sum m T^4 /
// sum m)^(1/4), mass-weighted v; empty cells 0.  vol[cell / per] is the cell's volume.
__global__ void k_grid_finish(int64_t ncell, const double* __restrict__ acc,
                              const double* __restrict__ vol, int64_t per, double* mass,
                              float* rho, float* t_mass, float* t_em, float* vel) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const double* a = acc + c * DEP_FIELDS;
  const double mc = a[0];
  const bool has = mc > 0.0;
  const double safe = has ? mc : 1.0;
  mass[c] = mc;
  rho[c] = (float)(mc / vol[c / per]);
  t_mass[c] = (float)(has ? a[1] / safe : 0.0);
  const double t4 = a[2] / safe;
  t_em[c] = (float)(has ? pow(t4 > 0.0 ? t4 : 0.0, 0.25) : 0.0);
#pragma unroll
  for (int d = 0; d < 3; ++d) vel[3 * c + d] = (float)(has ? a[3 + d] / safe : 0.0);
}

// render/gasgrid.py:757-788 (refine_sums): fine sums from the coarse sums' densities,
// trilinear in index space (theta and r clamped, phi periodic), times the fine volume; the
// fine mass is summed into msum for the rescaling
__device__ __forceinline__ void refine_axis(int i, int c, int nc, bool periodic, int& i0,
                                            int& i1, double& w) {
  double f = (i + 0.5) / c - 0.5;
  if (periodic) {
    const int b = (int)floor(f);
    i0 = py_imod(b, nc);
    i1 = py_imod(b + 1, nc);
    w = f - b;
    return;
  }
  f = fmin(fmax(f, 0.0), nc - 1.0);
  int b = 0;
  if (nc > 1) b = min((int)floor(f), nc - 2);
  i0 = b;
  i1 = min(b + 1, nc - 1);
  w = f - b;
}

__global__ void k_refine(const double* __restrict__ acc_c, const double* __restrict__ vc,
                         int nrc, int nthc, int nphc, const double* __restrict__ vf, int nr,
                         int nth, int nph, int cr, int ct, int cp, double* __restrict__ out,
                         double* msum) {
  const int64_t cell = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (cell >= (int64_t)nr * nth * nph) return;
  const int k = (int)(cell % nph);
  const int j = (int)((cell / nph) % nth);
  const int i = (int)(cell / ((int64_t)nph * nth));
  int ri[2], ti[2], pi[2];
  double rw, tw, pw;
  refine_axis(i, cr, nrc, false, ri[0], ri[1], rw);
  refine_axis(j, ct, nthc, false, ti[0], ti[1], tw);
  refine_axis(k, cp, nphc, true, pi[0], pi[1], pw);
  const double wr[2] = {1.0 - rw, rw}, wt[2] = {1.0 - tw, tw}, wp[2] = {1.0 - pw, pw};
  double s[DEP_FIELDS] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c) {
        const double w = wr[a] * wt[b] * wp[c];
        const int64_t cc = ((int64_t)ri[a] * nthc + ti[b]) * nphc + pi[c];
        const double vcc = vc[(int64_t)ri[a] * nthc + ti[b]];
#pragma unroll
        for (int f = 0; f < DEP_FIELDS; ++f) s[f] += w * (acc_c[cc * DEP_FIELDS + f] / vcc);
      }
  const double vfc = vf[(int64_t)i * nth + j];
#pragma unroll
  for (int f = 0; f < DEP_FIELDS; ++f) out[cell * DEP_FIELDS + f] = s[f] * vfc;
  atomicAdd(msum, s[0] * vfc);
}

__global__ void k_field_sum(int64_t ncell, const double* __restrict__ acc, double* sum) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c < ncell) atomicAdd(sum, acc[c * DEP_FIELDS]);
}

__global__ void k_refine_scale(int64_t nval, const double* __restrict__ sums, double* out) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= nval) return;
  const double fine = sums[0], coarse = sums[1];
  if (fine > 0.0) out[e] *= coarse / fine;
}

// ---------------------------------------------------------------- spatial order
// The particles are dealt to the deposition threads in the order of the cell holding their
// centre, so neighbouring threads add to neighbouring cells while those lines sit in L2 (in the
// caller's order each atomic add of a large grid travels to DRAM).  Keys: the grid's own linear
// cell index, with the out-of-grid cells clamped to one layer beyond each face.
__global__ void k_dep_keys_box(int64_t n, const double* __restrict__ x, double x0, double y0,
                               double z0, double dx, int nb, unsigned long long* keys,
                               int32_t* idx) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int e = nb + 2;
  const int a = min(max((int)floor((x[3 * p] - x0) / dx), -1), nb) + 1;
  const int b = min(max((int)floor((x[3 * p + 1] - y0) / dx), -1), nb) + 1;
  const int c = min(max((int)floor((x[3 * p + 2] - z0) / dx), -1), nb) + 1;
  keys[p] = ((unsigned long long)a * e + b) * e + c;
  idx[p] = (int32_t)p;
}

__global__ void k_dep_keys_log(int64_t n, const double* __restrict__ x, double r_min, double dlnr,
                               double dth, double dph, int nr, int nth, int nph,
                               unsigned long long* keys, int32_t* idx) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double xp = x[3 * p], yp = x[3 * p + 1], zp = x[3 * p + 2];
  const double rr = sqrt(xp * xp + yp * yp + zp * zp);
  const int i = min(max((int)floor(log(rr / r_min) / dlnr), -1), nr) + 1;
  const int j = min(max((int)floor(acos(fmin(1.0, fmax(-1.0, zp / rr))) / dth), 0), nth - 1);
  const int k = min(max((int)floor(py_mod(atan2(yp, xp), 2.0 * 3.141592653589793) / dph), 0), nph - 1);
  keys[p] = ((unsigned long long)i * nth + j) * nph + k;
  idx[p] = (int32_t)p;
}

__global__ void k_dep_gather(int64_t n, const int32_t* __restrict__ idx,
                             const double* __restrict__ x, const double* __restrict__ h,
                             const double* __restrict__ m, const double* __restrict__ t,
                             const double* __restrict__ v, double* __restrict__ out) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int64_t p = idx[q];
  double* xs = out;
  double* hs = out + 3 * n;
  double* ms = hs + n;
  double* ts = ms + n;
  double* vs = ts + n;
  for (int c = 0; c < 3; ++c) {
    xs[3 * q + c] = x[3 * p + c];
    vs[3 * q + c] = v[3 * p + c];
  }
  hs[q] = h[p];
  ms[q] = m[p];
  ts[q] = t[p];
}

void launch_deposit_keys(int64_t n, const double* x, int grid_kind, const LogGeom& g, double x0,
                         double y0, double z0, double dx, int nb, unsigned long long* keys,
                         int32_t* idx, cudaStream_t st) {
  if (n <= 0) return;
  if (grid_kind == 0)
    count_launch(), k_dep_keys_log<<<grid_for(n), NB_THREADS, 0, st>>>(
        n, x, g.r_min, g.dlnr, g.dth, g.dph, g.nr, g.nth, g.nph, keys, idx);
  else
    count_launch(), k_dep_keys_box<<<grid_for(n), NB_THREADS, 0, st>>>(n, x, x0, y0, z0, dx, nb,
                                                                        keys, idx);
}

void launch_deposit_gather(int64_t n, const int32_t* idx, const double* x, const double* h,
                           const double* m, const double* t, const double* v, double* out,
                           cudaStream_t st) {
  if (n > 0)
    count_launch(), k_dep_gather<<<grid_for(n), NB_THREADS, 0, st>>>(n, idx, x, h, m, t, v, out);
}

// ---------------------------------------------------------------- launchers
void launch_deposit_log(int64_t n, const double* x, const double* h, const double* m,
                        const double* t, const double* v, const LogGeom& g, int kid,
                        double* acc, double* outside, unsigned long long* n_tri,
                        cudaStream_t st) {
  if (n > 0)
    count_launch(), k_deposit_log<<<grid_for(n, 128), 128, 0, st>>>(n, x, h, m, t, v, g, kid,
                                                                      acc, outside, n_tri);
}

void launch_deposit_box(int64_t n, const double* x, const double* h, const double* m,
                        const double* t, const double* v, double x0, double y0, double z0,
                        double dx, int nb, int kid, double* acc, double* outside,
                        unsigned long long* n_tri, cudaStream_t st) {
  if (n > 0)
    count_launch(), k_deposit_box<<<grid_for(n, 128), 128, 0, st>>>(
        n, x, h, m, t, v, x0, y0, z0, dx, nb, kid, acc, outside, n_tri);
}

void launch_grid_finish(int64_t ncell, const double* acc, const double* vol, int64_t per,
                        double* mass, float* rho, float* t_mass, float* t_em, float* vel,
                        cudaStream_t st) {
  if (ncell > 0)
    count_launch(), k_grid_finish<<<grid_for(ncell), NB_THREADS, 0, st>>>(
        ncell, acc, vol, per, mass, rho, t_mass, t_em, vel);
}

void launch_refine_sums(const double* acc_c, const double* vol_c, int nrc, int nthc, int nphc,
                        const double* vol_f, int nr, int nth, int nph, int cr, int ct, int cp,
                        double* out, double* sums2, cudaStream_t st) {
  const int64_t nf = (int64_t)nr * nth * nph, nc = (int64_t)nrc * nthc * nphc;
  count_launch(), k_refine<<<grid_for(nf), NB_THREADS, 0, st>>>(
      acc_c, vol_c, nrc, nthc, nphc, vol_f, nr, nth, nph, cr, ct, cp, out, sums2);
  count_launch(), k_field_sum<<<grid_for(nc), NB_THREADS, 0, st>>>(nc, acc_c, sums2 + 1);
  count_launch(), k_refine_scale<<<grid_for(nf * DEP_FIELDS), NB_THREADS, 0, st>>>(
      nf * DEP_FIELDS, sums2, out);
}

}  // namespace nbk
