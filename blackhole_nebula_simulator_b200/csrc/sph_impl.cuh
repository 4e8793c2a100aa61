// SPH pair passes on neighbour lists (implementation, included by sph64.cu and sph32.cu): the h-rho Newton solve and the fused pressure + artificial
// viscosity (+ conductivity, + disc viscosity) force and du/dt pass.
//
// The density solve runs eight lanes per row with a shared-memory cache of the in-range entries
// (FP32) or one thread per row (FP64); the force pass eight lanes per row.  Both walk CSR lists.  They are templated on the list index type so the
// same code serves the caller-order int64 lists of the operator API and the engine's sorted int32
// lists, and on the arithmetic: FP64 (every pair term in double) or FP32 (positions as float
// offsets from cell centres, float pair terms, Kahan-compensated sums, the Newton update and all
// per-particle state in double).
#pragma once
#include "common.cuh"
#include "engine.cuh"
#include "sph.cuh"

namespace nbk {

// ---------------------------------------------------------------- position differences
// FP64: packed (x, y, z, w) doubles.  dx = x_j - x_i as the reference forms it.
struct Pos64 {
  const double4* p;
  static constexpr bool has_mass = false;
  struct Own {
    double4 a;
  };
  __device__ __forceinline__ void ready() {}
  __device__ __forceinline__ Own own(int64_t i) const { return Own{p[i]}; }
  __device__ __forceinline__ void diff(const Own& o, int64_t j, double& dx, double& dy,
                                       double& dz) const {
    const double4 b = p[j];
    dx = b.x - o.a.x;
    dy = b.y - o.a.y;
    dz = b.z - o.a.z;
  }
  __device__ __forceinline__ void diff(int64_t i, int64_t j, double& dx, double& dy,
                                       double& dz) const {
    diff(own(i), j, dx, dy, dz);
  }
  // the difference and particle j's smoothing length (from the hydro record)
  template <typename V4>
  __device__ __forceinline__ void diff_h(const Own& o, int64_t j, const V4* __restrict__ hydro,
                                         double& dx, double& dy, double& dz, double& hj) const {
    diff(o, j, dx, dy, dz);
    hj = (double)hydro[j].x;
  }
  template <typename V4>
  __device__ __forceinline__ void diff_h(int64_t i, int64_t j, const V4* __restrict__ hydro,
                                         double& dx, double& dy, double& dz, double& hj) const {
    diff_h(own(i), j, hydro, dx, dy, dz, hj);
  }
};

// FP32: per particle the cell of a uniform grid of edge `cell` (at most 1024 per axis) and the
// float offset from that cell's centre, packed as two float4: (offset x, y, z, mass) and (cell
// x, y, z as exact small floats, h: the smoothing length where the force pass needs it).  dx = (c_j - c_i) cell + (o_j - o_i): the cell difference
// is an exact float, and one fused multiply-add rounds the sum once, so the difference keeps full
// float precision at any distance from the origin.
struct Pos32 {
  const float4* p;
  float cell;
  const double* box6 = nullptr;  // grid corner and far corner; the edge is derived on the device
  static constexpr bool has_mass = true;
  struct Own {
    float4 a, c;
  };
  // edge of the grid cells: the largest side of the box over 1000, as the packing kernel uses
  __device__ __forceinline__ void ready() {
    if (box6) {
      double span = fmax(fmax(box6[3] - box6[0], box6[4] - box6[1]), box6[5] - box6[2]);
      cell = (float)fmax(span / 1000.0, 1e-30);
    }
  }
  __device__ __forceinline__ Own own(int64_t i) const { return Own{p[2 * i], p[2 * i + 1]}; }
  __device__ __forceinline__ float mass(int64_t j) const { return p[2 * j].w; }
  __device__ __forceinline__ void diff(const Own& o, int64_t j, float& dx, float& dy,
                                       float& dz) const {
    const float4 b = p[2 * j], cb = p[2 * j + 1];
    dx = fmaf(cb.x - o.c.x, cell, b.x - o.a.x);
    dy = fmaf(cb.y - o.c.y, cell, b.y - o.a.y);
    dz = fmaf(cb.z - o.c.z, cell, b.z - o.a.z);
  }
  __device__ __forceinline__ void diff(int64_t i, int64_t j, float& dx, float& dy,
                                       float& dz) const {
    diff(own(i), j, dx, dy, dz);
  }
  // the difference and particle j's smoothing length, from the same record
  template <typename V4>
  __device__ __forceinline__ void diff_h(const Own& o, int64_t j, const V4* __restrict__,
                                         float& dx, float& dy, float& dz, float& hj) const {
    const float4 b = p[2 * j], cb = p[2 * j + 1];
    dx = fmaf(cb.x - o.c.x, cell, b.x - o.a.x);
    dy = fmaf(cb.y - o.c.y, cell, b.y - o.a.y);
    dz = fmaf(cb.z - o.c.z, cell, b.z - o.a.z);
    hj = cb.w;
  }
  template <typename V4>
  __device__ __forceinline__ void diff_h(int64_t i, int64_t j, const V4* __restrict__ hydro,
                                         float& dx, float& dy, float& dz, float& hj) const {
    diff_h(own(i), j, hydro, dx, dy, dz, hj);
  }
};

__device__ __forceinline__ double sqdist(double dx, double dy, double dz) { return d2_exact(dx, dy, dz); }
__device__ __forceinline__ float sqdist(float dx, float dy, float dz) {
  return fmaf(dz, dz, fmaf(dy, dy, dx * dx));
}

template <typename R>
struct Acc;
template <>
struct Acc<double> {
  double s = 0.0;
  __device__ __forceinline__ void add(double v) { s += v; }
  __device__ __forceinline__ double get() const { return s; }
};
template <>
struct Acc<float> {
  Kahan k;
  __device__ __forceinline__ void add(float v) { k.add(v); }
  __device__ __forceinline__ double get() const { return (double)k.s; }
};

// ---------------------------------------------------------------- density
// Reference sim/sph.py:215-297 (_sums, _distances, _density_kernel): Newton-Raphson on
// f(h) = sum_j m_j W(r_ij, h) - m_i (eta/h)^3 inside a bisection bracket, tol * h0, at most 50
// iterations; the cap test near the search limit; Omega = 1 + h/(3 rho) sum m dW/dh (1 at h_max).
template <typename R, typename PosT, typename I>
__device__ void density_sums(const PosT& geo, int64_t i, const int64_t* off, const I* idx,
                             const double* mass, R r2max, R h, int kid, R cnorm, double& rs_out,
                             double& dws_out, int64_t& work) {
  Acc<R> rs, dws;
  R inv_h = R(1) / h;
  R ih2 = inv_h * inv_h;
  R ih3 = ih2 * inv_h;
  R ih4 = ih2 * ih2;
  for (int64_t e = off[i]; e < off[i + 1]; ++e) {
    int64_t j = (int64_t)idx[e];
    R dx, dy, dz;
    geo.diff(i, j, dx, dy, dz);
    R d2 = sqdist(dx, dy, dz);
    if (!(d2 < r2max)) continue;
    R q = sqrt(d2) * inv_h;
    if (q < R(2)) {
      work += 1;
      R fq = kernel_f<R>(q, kid);
      R m = (R)mass[j];
      rs.add(m * cnorm * ih3 * fq);
      dws.add(m * (-cnorm * ih4 * (R(3) * fq + q * kernel_df<R>(q, kid))));
    }
  }
  rs_out = rs.get();
  dws_out = dws.get();
}

// Sums over the cached in-range entries (r, m) of one row.
template <typename R>
__device__ __forceinline__ void cached_sums(const R* rr, const R* mm, int cnt, R h, int kid,
                                            R cnorm, double& rs_out, double& dws_out,
                                            int64_t& work) {
  Acc<R> rs, dws;
  R inv_h = R(1) / h;
  R ih2 = inv_h * inv_h;
  R ih3 = ih2 * inv_h;
  R ih4 = ih2 * ih2;
  for (int k = 0; k < cnt; ++k) {
    R q = rr[k] * inv_h;
    if (q < R(2)) {
      work += 1;
      R fq = kernel_f<R>(q, kid);
      R m = mm[k];
      rs.add(m * cnorm * ih3 * fq);
      dws.add(m * (-cnorm * ih4 * (R(3) * fq + q * kernel_df<R>(q, kid))));
    }
  }
  rs_out = rs.get();
  dws_out = dws.get();
}

// In-range entries a row may cache in its thread's local array (0: every sum walks the list; a
// per-thread cache in local memory measured slower than re-walking the curve-local list).
constexpr int DENSITY_CACHE = 0;

// One thread per row (the FP64 form: its shared-memory cache of (r, m) in double would hold
// occupancy too low for the row-group kernel below to pay off).

template <typename R, typename PosT, typename I>
__global__ void __launch_bounds__(NB_THREADS)
    k_density_thread(int64_t nrows, const int64_t* __restrict__ rows, PosT geo_in,
              const double* __restrict__ mass, const double* __restrict__ h_start,
              const double* __restrict__ h_search, const int64_t* __restrict__ off,
              const I* __restrict__ idx, DensityParams prm, const int32_t* __restrict__ out_map,
              double* __restrict__ h_out, double* __restrict__ rho, double* __restrict__ omega,
              int64_t* __restrict__ iters, int64_t* __restrict__ flags, int64_t* __restrict__ work) {
  PosT geo = geo_in;
  geo.ready();
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= nrows) return;
  int64_t i = rows ? rows[q] : q;
  int64_t o = out_map ? (int64_t)out_map[i] : q;
  double m_i = mass[i];
  double hs = fmin(h_search[i], prm.h_max);
  double r_max = 2.0 * hs;
  R r2max = (R)(r_max * r_max);
  const int kid = prm.kid;
  const R cn = (R)prm.cnorm;
  int64_t evals = 0;
  // distances and masses of the entries inside r_max (sim/sph.py:231-248): cached when
  // DENSITY_CACHE > 0, else recomputed from the list by every sum
  constexpr int CAP = DENSITY_CACHE > 0 ? DENSITY_CACHE : 1;
  R rr[CAP], mm[CAP];
  int cnt = 0;
  bool cached = DENSITY_CACHE > 0;
  if (DENSITY_CACHE > 0) {
    for (int64_t e = off[i]; e < off[i + 1]; ++e) {
      int64_t j = (int64_t)idx[e];
      R dx, dy, dz;
      geo.diff(i, j, dx, dy, dz);
      R d2 = sqdist(dx, dy, dz);
      if (!(d2 < r2max)) continue;
      if (cnt < DENSITY_CACHE) {
        rr[cnt] = sqrt(d2);
        mm[cnt] = (R)mass[j];
      } else {
        cached = false;
      }
      cnt += 1;
    }
  }
  auto sums = [&](R h, double& rs, double& dws) {
    if (cached)
      cached_sums<R>(rr, mm, cnt, h, kid, cn, rs, dws, evals);
    else
      density_sums<R>(geo, i, off, idx, mass, r2max, h, kid, cn, rs, dws, evals);
  };
  double lo = 0.0, hi = hs;
  double h = fmin(h_start[i], hi);
  double h0 = h;
  int flag = 3, it = 0;
  const double eta = prm.eta, e3 = eta * eta * eta;
  while (it < 50) {
    it += 1;
    double rs, dws;
    sums((R)h, rs, dws);
    double t = eta / h;
    double f = rs - m_i * (t * t * t);
    double h2 = h * h;
    double df = dws + 3.0 * m_i * e3 / (h2 * h2);
    if (f > 0)
      hi = h;
    else
      lo = h;
    double h_new = df > 0 ? h - f / df : 0.5 * (lo + hi);
    if (!(lo <= h_new && h_new <= hi)) h_new = 0.5 * (lo + hi);
    if (fabs(h_new - h) < prm.tol * h0) {
      h = h_new;
      flag = 0;
      break;
    }
    h = h_new;
  }
  if (h >= hs * (1 - 1e-3)) {
    double rs_lim, dummy;
    sums((R)hs, rs_lim, dummy);
    double t = eta / hs;
    if (rs_lim - m_i * (t * t * t) < 0) {
      h = hs;
      flag = hs >= prm.h_max ? 1 : 2;
    }
  }
  double rs, dws;
  sums((R)h, rs, dws);
  h_out[o] = h;
  rho[o] = rs;
  omega[o] = flag == 1 ? 1.0 : 1.0 + h / (3.0 * rs) * dws;
  if (iters) iters[o] = it;
  if (flags) flags[o] = flag;
  if (work) work[o] = evals;
}

// Sums over the 8 lanes of a row group (lanes 8g .. 8g+7 of a warp).  Every lane of the group ends
// with the same value (each butterfly step adds the same two operands on both lanes).  FP64: plain
// sums.  FP32: each lane's Kahan partial (s, -c) is combined pairwise with an exact two-sum, the
// rounding errors and the lanes' compensations carried in a second float.
__device__ __forceinline__ double group_total(double v) {
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double group_total(const Acc<double>& a) { return group_total(a.s); }
__device__ __forceinline__ double group_total(const Acc<float>& a) {
  float s = a.k.s, k = -a.k.c;
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) {
    float s2 = __shfl_xor_sync(0xffffffffu, s, o);
    float k2 = __shfl_xor_sync(0xffffffffu, k, o);
    float t = __fadd_rn(s, s2);
    float bp = __fsub_rn(t, s);
    float e = __fadd_rn(__fsub_rn(s, __fsub_rn(t, bp)), __fsub_rn(s2, bp));
    s = t;
    k = __fadd_rn(__fadd_rn(k, k2), e);
  }
  return (double)s + (double)k;
}

template <typename R>
struct DensityEntry;
#ifndef DENSITY_CAP
#define DENSITY_CAP 128
#endif
template <>
struct DensityEntry<float> {
  using T = float2;
  // entries inside r_in a row keeps in shared memory: 16 rows x 128 x 8 B = 16 KiB per block, so
  // 8 resident blocks (the register limit) leave most of the SM's L1 to the gathered records
  static constexpr int CAP = DENSITY_CAP;
  static constexpr int BLOCKS = 8;
};
template <>
struct DensityEntry<double> {
  using T = double2;
  static constexpr int CAP = 192;
  static constexpr int BLOCKS = 4;
};
constexpr int DENSITY_THREADS = 128;  // 16 rows per block
// rounds of 8 entries the list walk loads at once: 4 measured 3.55 ms per density launch on the
// 4M torus against 3.88 with 2 and 3.75 with 8
#ifndef DENSITY_UNROLL
#define DENSITY_UNROLL 4
#endif

// Eight lanes per row, four rows per warp.  The lanes of a row split its list (entry e to lane
// e mod 8, coalesced index loads) and store the distance and mass of every entry inside r_in =
// 2.1 h_start (the Newton iterates stay near the start h) in shared memory, in list order; each
// Newton iteration then sums the kernel terms over that cache and reduces across the eight lanes,
// so the lanes of a row take the same Newton steps.  A sum at an h whose support reaches past
// r_in adds the entries beyond it from the list (the same distances, recomputed); rows with more
// entries inside r_in than the cache holds re-walk their list in every sum.
template <typename R, typename PosT, typename I>
__global__ void __launch_bounds__(DENSITY_THREADS, DensityEntry<R>::BLOCKS)
    k_density(int64_t nrows, const int64_t* __restrict__ rows, PosT geo_in,
              const double* __restrict__ mass, const double* __restrict__ h_start,
              const double* __restrict__ h_search, const int64_t* __restrict__ off,
              const I* __restrict__ idx, DensityParams prm, const int32_t* __restrict__ out_map,
              double* __restrict__ h_out, double* __restrict__ rho, double* __restrict__ omega,
              int64_t* __restrict__ iters, int64_t* __restrict__ flags, int64_t* __restrict__ work) {
  PosT geo = geo_in;
  geo.ready();
  using E2 = typename DensityEntry<R>::T;
  constexpr int CAP = DensityEntry<R>::CAP;
  __shared__ E2 cache_s[DENSITY_THREADS / 8][CAP];
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, gl = lane & 7, g = lane >> 3;
  const int64_t q = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 4 + g;
  const bool live = q < nrows;
  if (!__any_sync(FULL, live)) return;  // warp-uniform
  E2* cache = cache_s[threadIdx.x >> 3];
  int64_t i = 0, o = 0, e0 = 0, e1 = 0;
  double m_i = 1.0, hs = 1.0;
  if (live) {
    i = rows ? rows[q] : q;
    o = out_map ? (int64_t)out_map[i] : q;
    m_i = mass[i];
    hs = fmin(h_search[i], prm.h_max);
    e0 = off[i];
    e1 = off[i + 1];
  }
  const typename PosT::Own me_rec = geo.own(i);  // the row's own record, loaded once
  auto mass_of = [&](int64_t j) -> R {
    if constexpr (PosT::has_mass)
      return (R)geo.mass(j);
    else
      return prm.massf ? (R)prm.massf[j] : (R)mass[j];
  };
  const double r_max = 2.0 * hs;
  const R r2max = (R)(r_max * r_max);
  const int kid = prm.kid;
  const R cn = (R)prm.cnorm;
  // the Newton iterates stay near the start h0 (the previous step's h): entries inside
  // r_in = 2.1 h0 are cached, and a sum at h adds the others only when r_in / h < 2 (else every
  // one of them has q >= 2, a zero term)
  const double h_first = live ? fmin(h_start[i], hs) : 1.0;
  const R r_in = (R)(2.1 * h_first);
  // distances and masses of the entries inside r_max (sim/sph.py:231-248), in list order
  const unsigned len = (unsigned)(e1 - e0);
  const unsigned maxlen = __reduce_max_sync(FULL, len);
  int cnt = 0;
  // DENSITY_UNROLL rounds of 8 entries per pass: their index, position and mass loads are issued
  // together (the walk is bound by the latency of those dependent gathers), then the rounds are
  // appended to the cache one after the other, so the cache holds the entries in list order
  constexpr int U = DENSITY_UNROLL;
  for (unsigned b = 0; b < maxlen; b += 8 * U) {
    int64_t jj[U];
    bool inr[U];
    R rr[U], mm[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const unsigned e = b + 8 * u + gl;
      jj[u] = e < len ? (int64_t)ld_stream(idx + e0 + e) : -1;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      inr[u] = false;
      rr[u] = R(0);
      mm[u] = R(0);
      if (jj[u] >= 0) {
        R dx, dy, dz;
        geo.diff(me_rec, jj[u], dx, dy, dz);
        R d2 = sqdist(dx, dy, dz);
        if (d2 < r2max) {
          inr[u] = true;
          rr[u] = sqrt(d2);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (inr[u]) mm[u] = mass_of(jj[u]);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const bool inner = inr[u] && rr[u] < r_in;
      const unsigned seg = (__ballot_sync(FULL, inner) >> (8 * g)) & 0xffu;
      const int pos = cnt + __popc(seg & ((1u << gl) - 1u));
      if (inner && pos < CAP) {  // overflow: the walk below instead
        E2 v;
        v.x = rr[u];
        v.y = mm[u];
        cache[pos] = v;
      }
      cnt += __popc(seg);
    }
  }
  __syncwarp();
  const bool cached = cnt <= CAP;
  int64_t evals = 0;
  // kernel sums at h of the rows whose `active` is set; every lane takes part in the reductions
  auto sums = [&](R h, bool active, double& rs_out, double& dws_out) {
    Acc<R> rs, dws;
    if (active) {
      R inv_h = R(1) / h;
      R ih2 = inv_h * inv_h;
      R ih3 = ih2 * inv_h;
      R ih4 = ih2 * ih2;
      auto term = [&](R rj, R mj) {
        R qq = rj * inv_h;
        if (qq < R(2)) {
          evals += 1;
          R fq = kernel_f<R>(qq, kid);
          rs.add(mj * cn * ih3 * fq);
          dws.add(mj * (-cn * ih4 * (R(3) * fq + qq * kernel_df<R>(qq, kid))));
        }
      };
      if (cached) {
        for (int t = gl; t < cnt; t += 8) {
          E2 v = cache[t];
          term(v.x, v.y);
        }
        if (!(r_in * inv_h >= R(2)))
          for (int64_t e = e0 + gl; e < e1; e += 8) {  // the entries beyond r_in
            int64_t j = (int64_t)idx[e];
            R dx, dy, dz;
            geo.diff(me_rec, j, dx, dy, dz);
            R d2 = sqdist(dx, dy, dz);
            if (!(d2 < r2max)) continue;
            const R rj = sqrt(d2);
            if (rj < r_in) continue;
            term(rj, mass_of(j));
          }
      } else {
        for (int64_t e = e0 + gl; e < e1; e += 8) {
          int64_t j = (int64_t)idx[e];
          R dx, dy, dz;
          geo.diff(me_rec, j, dx, dy, dz);
          R d2 = sqdist(dx, dy, dz);
          if (!(d2 < r2max)) continue;
          term(sqrt(d2), mass_of(j));
        }
      }
    }
    rs_out = group_total(rs);
    dws_out = group_total(dws);
  };
  double lo = 0.0, hi = hs;
  double h = live ? fmin(h_start[i], hi) : 1.0;
  double h0 = h;
  int flag = 3, it = 0;
  bool done = !live;
  const double eta = prm.eta, e3 = eta * eta * eta;
  while (__any_sync(FULL, !done)) {
    double rs, dws;
    sums((R)h, !done, rs, dws);
    if (!done) {
      it += 1;
      double t = eta / h;
      double f = rs - m_i * (t * t * t);
      double h2 = h * h;
      double df = dws + 3.0 * m_i * e3 / (h2 * h2);
      if (f > 0)
        hi = h;
      else
        lo = h;
      double h_new = df > 0 ? h - f / df : 0.5 * (lo + hi);
      if (!(lo <= h_new && h_new <= hi)) h_new = 0.5 * (lo + hi);
      if (fabs(h_new - h) < prm.tol * h0) {
        flag = 0;
        done = true;
      } else if (it >= 50) {
        done = true;
      }
      h = h_new;
    }
  }
  const bool cap_test = live && h >= hs * (1 - 1e-3);
  if (__any_sync(FULL, cap_test)) {
    double rs_lim, dummy;
    sums((R)hs, cap_test, rs_lim, dummy);
    double t = eta / hs;
    if (cap_test && rs_lim - m_i * (t * t * t) < 0) {
      h = hs;
      flag = hs >= prm.h_max ? 1 : 2;
    }
  }
  double rs, dws;
  sums((R)h, live, rs, dws);
#pragma unroll
  for (int of = 4; of > 0; of >>= 1) evals += __shfl_xor_sync(FULL, evals, of);
  if (live && gl == 0) {
    h_out[o] = h;
    rho[o] = rs;
    omega[o] = flag == 1 ? 1.0 : 1.0 + h / (3.0 * rs) * dws;
    if (iters) iters[o] = it;
    if (flags) flags[o] = flag;
    if (work) work[o] = evals;
  }
}

// ---------------------------------------------------------------- forces
// Reference sim/sph.py:519-652 (_forces_kernel, no reconstruction) and sim/sph.py:1084-1117
// (_disc_kernel).  r_ab = x_a - x_b; F(h) = dW/dr; pair terms antisymmetric.
template <typename R>
__device__ __forceinline__ R dwdr(R r, R h, int kid, R cnorm) {
  R h2 = h * h;
  return cnorm / (h2 * h2) * kernel_df<R>(r / h, kid);
}

constexpr int FORCE_QUEUE = 64;  // interacting entries a row queues before its lanes drain them
#ifndef FORCE_UNROLL
#define FORCE_UNROLL 4
#endif
// rounds of eight entries the walk launch (MODE 1) issues at once, and its resident blocks
#ifndef WALK_UNROLL
#define WALK_UNROLL 4
#endif
#ifndef WALK_BLOCKS
#define WALK_BLOCKS 6
#endif
#ifndef WALK_OWN
#define WALK_OWN 0  // 1: the walk launch keeps the row's own record in registers
#endif
// resident blocks per SM of the FP32 force pass (registers: 65536 / (256 * 4) = 64, a few spilled;
// measured on the 4M torus 4.26 ms per launch against 4.59 with 3 blocks and 80 registers and
// 5.63 with 2); the FP64 form keeps 2, its doubles would spill; the reconstruction forms, with
// two 3x3 gradients per pair, 2 and 1
#ifndef FORCE_BLOCKS_PER_SM_FP32
#define FORCE_BLOCKS_PER_SM_FP32 4
#endif

// Fused pressure + artificial viscosity (+ conductivity) + P dV (+ disc viscosity) pass.  Eight
// lanes per row (lanes 8g .. 8g+7 of a warp), each taking every eighth list entry; the pair terms
// are summed per lane and then over the row's lanes.
// MODE 0: the walk queues the interacting entries and drains them into the pair terms as it
// goes.  The same pass can run as two launches: MODE 1 only walks, writing every row's
// interacting entries (self included, list order) to prm.tidx / prm.tcnt, with few registers
// and so many resident warps to hide the walk's dependent loads; MODE 2 then reads those
// entries, every lane busy on pair terms, with no walk state alive beside the accumulators.
template <int MODE, typename R, bool RECON>
struct ForceBlocks {
  static constexpr int value = MODE == 1 ? WALK_BLOCKS
                               : sizeof(R) == 4 ? (RECON ? 2 : FORCE_BLOCKS_PER_SM_FP32)
                                                : (RECON ? 1 : 2);
};

template <typename R, typename PosT, typename I, typename V4, bool RECON, int MODE = 0>
__global__ void __launch_bounds__(NB_THREADS, (ForceBlocks<MODE, R, RECON>::value))
    k_forces_g(int64_t nrows, const int64_t* __restrict__ rows, PosT geo_in,
             const V4* __restrict__ vm,    // (vx, vy, vz, mass)
             const V4* __restrict__ hydro, // (h, rho, omega, P)
             const V4* __restrict__ aux,   // (u, c_s, alpha, unused)
             const int64_t* __restrict__ off, const I* __restrict__ idx, ForceParams prm,
             const int32_t* __restrict__ out_map, ForceOut out) {
  PosT geo = geo_in;
  geo.ready();
  const unsigned FULL = 0xffffffffu;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t q = t >> 3;
  const int gl = (int)(t & 7);
  const bool live = q < nrows;
  if (!__any_sync(FULL, live)) return;  // warp-uniform
  int64_t a = 0, o = 0;
  if (live) {
    a = rows ? rows[q] : q;
    o = out_map ? (int64_t)out_map[a] : q;
  }
  const V4 va = vm[a], ha = hydro[a], xa = aux[a];
  const R h_a = (R)ha.x, rho_a = (R)ha.y, om_a = (R)ha.z, P_a = (R)ha.w;
  const R inv_or_a = R(1) / (om_a * rho_a);
  const R inv_orr_a = R(1) / (om_a * rho_a * rho_a);
  const R cs_a = (R)xa.y, al_a = (R)xa.z, u_a = (R)xa.x;
  const R beta = (R)prm.beta, alpha_u = (R)prm.alpha_u, aav = (R)prm.disc_alpha_av;
  const R cn = (R)prm.cnorm;
  const int kid = prm.kid;
  Acc<R> ax, ay, az, work, heat, vheat, cheat, dax, day, daz, dheat;
  R vmax = prm.use_visc ? cs_a : R(0);
  int64_t npairs = 0;
  // the row's list in rounds of eight entries: lanes test their entry, the interacting ones are
  // queued in shared memory in list order, and full queues are drained with all eight lanes
  // busy on pair terms
  __shared__ int32_t queue_s[NB_THREADS / 8][FORCE_QUEUE + 8 * FORCE_UNROLL];
  int32_t* pq = queue_s[threadIdx.x >> 3];
  const int g = (threadIdx.x & 31) >> 3;
  const int64_t e_beg = live ? off[a] : 0, e_end = live ? off[a + 1] : 0;
  const unsigned len = (unsigned)(e_end - e_beg);
  const unsigned maxlen = __reduce_max_sync(FULL, len);
  int pc = 0;
  // velocity reconstruction (sim/sph.py:568-609; physics/viscosity.py:116-158): the jump that
  // drives q is the velocity difference extrapolated to the pair midpoint with each side's
  // gradient, limited by the van Leer limiter of their projections and by the closeness factor;
  // the shock heating keeps the actual v_ab . r_hat
  R Ga[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) {
    if constexpr (!RECON)
      Ga[e] = R(0);
    else if constexpr (sizeof(R) == 4)
      Ga[e] = prm.gv32[9 * a + e];
    else
      Ga[e] = (R)prm.gv64[9 * a + e];
  }
  const R eta_crit = (R)prm.eta_crit, eta_fold = (R)prm.eta_fold;
  auto recon_visc = [&](int64_t b, R dx0, R dx1, R dx2, R r, R rx, R ry, R rz, R h_b, R vdotr,
                        const V4& vb, const V4& xb, R rho_b, R m_b, R fa, R& num_a, R& num_b) {
    R Gb[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      if constexpr (sizeof(R) == 4)
        Gb[e] = prm.gv32[9 * b + e];
      else
        Gb[e] = (R)prm.gv64[9 * b + e];
    }
    const R ga0 = Ga[0] * dx0 + Ga[1] * dx1 + Ga[2] * dx2;
    const R ga1 = Ga[3] * dx0 + Ga[4] * dx1 + Ga[5] * dx2;
    const R ga2 = Ga[6] * dx0 + Ga[7] * dx1 + Ga[8] * dx2;
    const R gb0 = Gb[0] * dx0 + Gb[1] * dx1 + Gb[2] * dx2;
    const R gb1 = Gb[3] * dx0 + Gb[4] * dx1 + Gb[5] * dx2;
    const R gb2 = Gb[6] * dx0 + Gb[7] * dx1 + Gb[8] * dx2;
    const R pa = dx0 * ga0 + dx1 * ga1 + dx2 * ga2;
    const R pb = dx0 * gb0 + dx1 * gb1 + dx2 * gb2;
    R phi = R(0);
    if (pb != R(0)) {
      const R ratio = pa / pb;
      if (ratio > R(0)) {
        const R t = R(4) * ratio / ((R(1) + ratio) * (R(1) + ratio));
        phi = t < R(1) ? t : R(1);
      }
    }
    if (prm.closeness) {
      const R e_a = r / h_a, e_b = r / h_b;
      const R eta_ab = e_b < e_a ? e_b : e_a;
      if (eta_ab < eta_crit) {
        const R t = (eta_ab - eta_crit) / eta_fold;
        phi *= exp(-t * t);
      }
    }
    const R hp = R(0.5) * phi;
    R vdr = (((R)va.x - hp * ga0) - ((R)vb.x + hp * gb0)) * rx +
            (((R)va.y - hp * ga1) - ((R)vb.y + hp * gb1)) * ry +
            (((R)va.z - hp * ga2) - ((R)vb.z + hp * gb2)) * rz;
    bool on = vdr < R(0) && vdotr < R(0);
    if (prm.gate == 1)
      on = vdr < R(0);
    else if (prm.gate == 2 && vdotr > vdr)
      vdr = vdotr;
    const R vsig_a = al_a * cs_a + beta * fabs(vdr);
    const R vsig_b = (R)xb.z * (R)xb.y + beta * fabs(vdr);
    const R vsig_cfl = al_a * cs_a + beta * fabs(vdotr);
    if (vsig_cfl > vmax) vmax = vsig_cfl;
    if (on) {
      num_a += R(-0.5) * rho_a * vsig_a * vdr;
      num_b += R(-0.5) * rho_b * vsig_b * vdr;
      R dh = m_b * vsig_a * R(0.5) * vdr * vdotr * fa * inv_or_a;
      heat.add(-dh);
      vheat.add(-dh);
    }
  };
  auto pair = [&](int64_t b) {
    R ddx, ddy, ddz;
    geo.diff(a, b, ddx, ddy, ddz);  // x_b - x_a
    const V4 hb4 = hydro[b];
    const R h_b = (R)hb4.x;
    R d2 = sqdist(ddx, ddy, ddz);
    npairs += 1;
    const V4 vb = vm[b];
    const R rho_b = (R)hb4.y, om_b = (R)hb4.z, P_b = (R)hb4.w;
    const R m_b = (R)vb.w;
    R r = sqrt(d2);
    R rx = -ddx / r, ry = -ddy / r, rz = -ddz / r;  // r_hat of x_a - x_b
    R fa = dwdr<R>(r, h_a, kid, cn);
    R fb = dwdr<R>(r, h_b, kid, cn);
    // velocity differences are formed in double before rounding, so a large common (orbital)
    // velocity costs the FP32 path no precision
    const R dvx = (R)(va.x - vb.x), dvy = (R)(va.y - vb.y), dvz = (R)(va.z - vb.z);
    R vdotr = dvx * rx + dvy * ry + dvz * rz;
    R num_a = P_a, num_b = P_b;
    R inv_orr_b = R(1) / (om_b * rho_b * rho_b);
    if (prm.use_sph) {
      if (prm.use_visc) {
        const V4 xb = aux[b];
        if constexpr (RECON) {
          recon_visc(b, -ddx, -ddy, -ddz, r, rx, ry, rz, h_b, vdotr, vb, xb, rho_b, m_b, fa,
                     num_a, num_b);
        } else {
          R vsig_a = al_a * cs_a + beta * fabs(vdotr);
          R vsig_b = (R)xb.z * (R)xb.y + beta * fabs(vdotr);
          if (vsig_a > vmax) vmax = vsig_a;
          if (vdotr < R(0)) {
            num_a += R(-0.5) * rho_a * vsig_a * vdotr;
            num_b += R(-0.5) * rho_b * vsig_b * vdotr;
            R dh = m_b * vsig_a * R(0.5) * vdotr * vdotr * fa * inv_or_a;
            heat.add(-dh);
            vheat.add(-dh);
          }
        }
        if (prm.use_cond) {
          R vu;
          if (prm.cond_signal == 0)
            vu = sqrt(fabs(P_a - P_b) / (R(0.5) * (rho_a + rho_b)));
          else
            vu = fabs(vdotr);
          R dc = m_b * alpha_u * vu * (R)(xa.x - xb.x) * R(0.5) *
                 (fa * inv_or_a + fb / (om_b * rho_b));
          heat.add(dc);
          cheat.add(dc);
        }
      }
      R f = m_b * (num_a * inv_orr_a * fa + num_b * inv_orr_b * fb);
      ax.add(-f * rx);
      ay.add(-f * ry);
      az.add(-f * rz);
      work.add(m_b * vdotr * fa);
    }
    if (prm.use_disc) {
      // the reference's disc kernel forms its terms in its own order (sim/sph.py:1097-1114)
      const V4 xb = aux[b];
      R ex = -ddx, ey = -ddy, ez = -ddz;  // x_a - x_b
      R vdr = dvx * ex / r;
      vdr = vdr + dvy * ey / r;
      vdr = vdr + dvz * ez / r;
      R qa = -rho_a * h_a / (R(2) * r) * aav * cs_a * vdr * (R(1) / (om_a * rho_a * rho_a));
      R qb = -rho_b * h_b / (R(2) * r) * aav * (R)xb.y * vdr / (om_b * rho_b * rho_b);
      R f = m_b * (qa * fa + qb * fb);
      dax.add(-(f * ex / r));
      day.add(-(f * ey / r));
      daz.add(-(f * ez / r));
      dheat.add(m_b * qa * vdr * fa);
    }
    };
  // FP32 form: the same terms with one reciprocal square root per pair and reciprocals of the
  // per-particle denominators instead of divisions (rounding differs from the FP64 form by a few
  // float ulps, far inside the FP32 tolerances)
  const R ih_a = R(1) / h_a;
  const R cn4_a = cn * (ih_a * ih_a) * (ih_a * ih_a);
  auto pair_fast = [&](int64_t b) {
    R ddx, ddy, ddz;
    geo.diff(a, b, ddx, ddy, ddz);  // x_b - x_a
    const V4 hb4 = hydro[b];
    const R h_b = (R)hb4.x;
    const R d2 = sqdist(ddx, ddy, ddz);
    npairs += 1;
    const V4 vb = vm[b];
    const R rho_b = (R)hb4.y, om_b = (R)hb4.z, P_b = (R)hb4.w;
    const R m_b = (R)vb.w;
    const R inv_r = rsqrtf(d2);
    const R r = d2 * inv_r;
    const R rx = -ddx * inv_r, ry = -ddy * inv_r, rz = -ddz * inv_r;  // r_hat of x_a - x_b
    const R ih_b = __frcp_rn(h_b);
    const R fa = cn4_a * kernel_df<R>(r * ih_a, kid);
    const R fb = cn * (ih_b * ih_b) * (ih_b * ih_b) * kernel_df<R>(r * ih_b, kid);
    const R dvx = (R)(va.x - vb.x), dvy = (R)(va.y - vb.y), dvz = (R)(va.z - vb.z);
    const R vdotr = dvx * rx + dvy * ry + dvz * rz;
    R num_a = P_a, num_b = P_b;
    const R inv_orr_b = __frcp_rn(om_b * rho_b * rho_b);
    if (prm.use_sph) {
      if (prm.use_visc) {
        const V4 xb = aux[b];
        if constexpr (RECON) {
          recon_visc(b, -ddx, -ddy, -ddz, r, rx, ry, rz, h_b, vdotr, vb, xb, rho_b, m_b, fa,
                     num_a, num_b);
        } else {
          R vsig_a = al_a * cs_a + beta * fabs(vdotr);
          R vsig_b = (R)xb.z * (R)xb.y + beta * fabs(vdotr);
          if (vsig_a > vmax) vmax = vsig_a;
          if (vdotr < R(0)) {
            num_a += R(-0.5) * rho_a * vsig_a * vdotr;
            num_b += R(-0.5) * rho_b * vsig_b * vdotr;
            R dh = m_b * vsig_a * R(0.5) * vdotr * vdotr * fa * inv_or_a;
            heat.add(-dh);
            vheat.add(-dh);
          }
        }
        if (prm.use_cond) {
          R vu;
          if (prm.cond_signal == 0)
            vu = sqrt(fabs(P_a - P_b) * __frcp_rn(R(0.5) * (rho_a + rho_b)));
          else
            vu = fabs(vdotr);
          R dc = m_b * alpha_u * vu * (R)(xa.x - xb.x) * R(0.5) *
                 (fa * inv_or_a + fb * inv_orr_b * rho_b);
          heat.add(dc);
          cheat.add(dc);
        }
      }
      R f = m_b * (num_a * inv_orr_a * fa + num_b * inv_orr_b * fb);
      ax.add(-f * rx);
      ay.add(-f * ry);
      az.add(-f * rz);
      work.add(m_b * vdotr * fa);
    }
    if (prm.use_disc) {
      const V4 xb = aux[b];
      const R vdr = vdotr;  // v_ab . (x_a - x_b) / r
      R qa = -rho_a * h_a * R(0.5) * inv_r * aav * cs_a * vdr * inv_orr_a;
      R qb = -rho_b * h_b * R(0.5) * inv_r * aav * (R)xb.y * vdr * inv_orr_b;
      R f = m_b * (qa * fa + qb * fb);
      dax.add(-(f * rx));
      day.add(-(f * ry));
      daz.add(-(f * rz));
      dheat.add(m_b * qa * vdr * fa);
    }
  };
  auto drain = [&]() {
    for (int k2 = gl; k2 < pc; k2 += 8) {
      if constexpr (sizeof(R) == 4)
        pair_fast((int64_t)pq[k2]);
      else
        pair((int64_t)pq[k2]);
    }
    __syncwarp();
    pc = 0;
  };
  // with prm.tidx the row's interacting entries (self included), in list order, are also
  // written out for the level limiter: exactly the reference's FP64 test, which the FP32 form
  // takes from prm.pos64 where its float test falls within 1e-5 of the boundary
  int m_tot = 0;
  if constexpr (MODE == 2) {
    // the interacting entries the walk launch wrote (self included: skipped here)
    const int cnt = live ? prm.tcnt[q] : 0;
    for (int k2 = gl; k2 < cnt; k2 += 8) {
      const int64_t b = (int64_t)ld_stream(prm.tidx + e_beg + k2);
      if (b == a) continue;
      if constexpr (sizeof(R) == 4)
        pair_fast(b);
      else
        pair(b);
    }
  }
  // FORCE_UNROLL rounds of eight entries at a time: their index and position loads are issued
  // together, then the rounds are queued one after the other in list order
  constexpr int FU = MODE == 1 ? WALK_UNROLL : FORCE_UNROLL;
  const typename PosT::Own me_walk = geo.own(a);
  for (unsigned base = 0; MODE != 2 && base < maxlen; base += 8 * FU) {
    int64_t bb[FU];
    bool take[FU], tight[FU];
#pragma unroll
    for (int u = 0; u < FU; ++u) {
      const unsigned e = base + 8 * u + gl;
      bb[u] = e < len ? (int64_t)ld_stream(idx + e_beg + e) : -1;
    }
#pragma unroll
    for (int u = 0; u < FU; ++u) {
      const int64_t b = bb[u];
      take[u] = false;
      tight[u] = false;
      if (b >= 0) {
        if (b != a) {
          bool tk = true;
          if (prm.tighten) {
            R ddx, ddy, ddz, h_b;
            if constexpr (MODE == 1 && WALK_OWN)
              geo.diff_h(me_walk, b, hydro, ddx, ddy, ddz, h_b);
            else
              geo.diff_h(a, b, hydro, ddx, ddy, ddz, h_b);
            R rr = R(2) * (h_a > h_b ? h_a : h_b);
            const R d2 = sqdist(ddx, ddy, ddz), r2 = rr * rr;
            tk = d2 < r2;
            if constexpr (sizeof(R) == 4) {
              if (prm.pos64 && d2 > r2 * R(1.0 - 1e-5) && d2 < r2 * R(1.0 + 1e-5)) {
                const double4 pa = prm.pos64[a], pb = prm.pos64[b];
                const double e2 = d2_exact(pb.x - pa.x, pb.y - pa.y, pb.z - pa.z);
                const double er = 2.0 * fmax(pa.w, pb.w);
                tk = e2 < er * er;
              }
            }
          }
          take[u] = tk;
          tight[u] = tk;
        } else {
          tight[u] = true;  // self: listed for the limiter, not a pair
        }
      }
    }
#pragma unroll
    for (int u = 0; u < FU; ++u) {
      if constexpr (MODE == 0) {
        unsigned seg = (__ballot_sync(FULL, take[u]) >> (8 * g)) & 0xffu;
        if (take[u]) pq[pc + __popc(seg & ((1u << gl) - 1u))] = (int32_t)bb[u];
        pc += __popc(seg);
      }
      if (prm.tidx) {
        const unsigned tseg = (__ballot_sync(FULL, tight[u]) >> (8 * g)) & 0xffu;
        if (tight[u])
          prm.tidx[e_beg + m_tot + __popc(tseg & ((1u << gl) - 1u))] = (int32_t)bb[u];
        m_tot += __popc(tseg);
      }
    }
    if (MODE == 0 && __any_sync(FULL, pc > FORCE_QUEUE - 8)) drain();
  }
  if constexpr (MODE == 0) drain();
  if (MODE != 2 && prm.tcnt && live && gl == 0) prm.tcnt[q] = m_tot;
  if constexpr (MODE == 1) return;  // the walk launch writes only the entries and counts
  // sums over the row's eight lanes (uniform flags: every lane takes part in every reduction)
  double s_ax = 0, s_ay = 0, s_az = 0, s_work = 0, s_heat = 0, s_vheat = 0, s_cheat = 0;
  double s_dax = 0, s_day = 0, s_daz = 0, s_dheat = 0;
  if (prm.use_sph) {
    s_ax = group_total(ax);
    s_ay = group_total(ay);
    s_az = group_total(az);
    s_work = group_total(work);
    s_heat = group_total(heat);
    s_vheat = group_total(vheat);
    s_cheat = group_total(cheat);
  }
  if (prm.use_disc) {
    s_dax = group_total(dax);
    s_day = group_total(day);
    s_daz = group_total(daz);
    s_dheat = group_total(dheat);
  }
#pragma unroll
  for (int of = 4; of > 0; of >>= 1) {
    R vo = __shfl_xor_sync(FULL, vmax, of);
    vmax = vo > vmax ? vo : vmax;
    npairs += __shfl_xor_sync(FULL, npairs, of);
  }
  if (!live || gl != 0) return;
  if (prm.use_sph) {
    double du = (double)P_a * (double)inv_or_a / (double)rho_a * s_work + s_heat;
    if (out.acc) {
      out.acc[3 * o + 0] = s_ax;
      out.acc[3 * o + 1] = s_ay;
      out.acc[3 * o + 2] = s_az;
    }
    if (out.dudt) out.dudt[o] = du;
    if (out.vsig) out.vsig[o] = (double)vmax;
    if (out.vheat) out.vheat[o] = s_vheat;
    if (out.cheat) out.cheat[o] = s_cheat;
  }
  if (prm.use_disc) {
    if (out.dacc) {
      out.dacc[3 * o + 0] = s_dax;
      out.dacc[3 * o + 1] = s_day;
      out.dacc[3 * o + 2] = s_daz;
    }
    if (out.ddudt) out.ddudt[o] = s_dheat;
  }
  if (out.pairs) out.pairs[o] = npairs;
}

// ---------------------------------------------------------------- corrected gradients
// Reference sim/sph.py:693-902 (_near_singular, _velocity_gradient_kernel, _gradients_kernel):
//     R_lj = sum_b m_b (x_b - x_a)^l dW_ab(h_a)/dx_a^j,  G_kj = sum_b m_b (v_b - v_a)^k dW/dx_a^j,
//     dv/dx = G R^-1 (the same with accelerations for d(div v)/dt),
// with dW_ab(h_a)/dx_a = (x_a - x_b) F(r, h_a) / r.  Fewer than 4 list entries (self excluded),
// tr R <= 0 or |det R| < 1e-6 (tr R / 3)^3: G / (tr R / 3) instead (0 when tr R <= 0).  R^-1 is
// the adjugate over the determinant.  Eight lanes per row, FP64 only (the FP32 form converts).
constexpr double SINGULAR_TOL = 1e-6;

__device__ __forceinline__ double det3(const double* m) {
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
         m[2] * (m[3] * m[7] - m[4] * m[6]);
}

// g <- g R^-1 (or the fallback) for the gradient sums g (3x3 row-major)
template <int NG>
__device__ __forceinline__ void corrected_gradients(const double* rm, int64_t cnt, double (*g)[9]) {
  const double scale = (rm[0] + rm[4] + rm[8]) / 3.0;
  const double det = det3(rm);
  const bool singular =
      cnt < 4 || !(scale > 0.0) || !(fabs(det) >= SINGULAR_TOL * scale * scale * scale);
  if (singular) {
    const double inv_s = scale > 0.0 ? 1.0 / scale : 0.0;
#pragma unroll
    for (int k = 0; k < NG; ++k)
#pragma unroll
      for (int e = 0; e < 9; ++e) g[k][e] = g[k][e] * inv_s;
    return;
  }
  double ri[9];
  ri[0] = (rm[4] * rm[8] - rm[5] * rm[7]) / det;
  ri[1] = (rm[2] * rm[7] - rm[1] * rm[8]) / det;
  ri[2] = (rm[1] * rm[5] - rm[2] * rm[4]) / det;
  ri[3] = (rm[5] * rm[6] - rm[3] * rm[8]) / det;
  ri[4] = (rm[0] * rm[8] - rm[2] * rm[6]) / det;
  ri[5] = (rm[2] * rm[3] - rm[0] * rm[5]) / det;
  ri[6] = (rm[3] * rm[7] - rm[4] * rm[6]) / det;
  ri[7] = (rm[1] * rm[6] - rm[0] * rm[7]) / det;
  ri[8] = (rm[0] * rm[4] - rm[1] * rm[3]) / det;
#pragma unroll
  for (int k = 0; k < NG; ++k) {
    double o[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
        o[3 * i + j] = g[k][3 * i + 0] * ri[j] + g[k][3 * i + 1] * ri[3 + j] +
                       g[k][3 * i + 2] * ri[6 + j];
#pragma unroll
    for (int e = 0; e < 9; ++e) g[k][e] = o[e];
  }
}

// physics/viscosity.py:83-113: xi (Balsara), alpha_loc, decay time, then the jump to alpha_loc
// or the backward-Euler decay toward it, for the particle at output index o
__device__ __forceinline__ void switch_update(const GradOut& out, int64_t o, double div,
                                              double curl, double ddiv) {
  // physics/viscosity.py:83-113: xi (Balsara), alpha_loc, decay time, the jump or the decay
  const double d2 = div * div, cc2 = curl * curl;
  const double xi = d2 + cc2 > 0.0 ? d2 / (d2 + cc2) : 0.0;
  const double mdd = -ddiv < 0.0 ? 0.0 : -ddiv;  // max(-d(div v)/dt, 0); NaN stays NaN
  const double h = out.h[o], cs = out.cs[o];
  const double al = 10.0 * h * h * (xi * mdd) / (cs * cs);
  const double a_loc = al > 1.0 ? 1.0 : al;  // min(alpha_loc, alpha_max = 1)
  const double dt =
      out.n_beg ? 2.0 * (0.5 * (double)(out.n_end[o] - out.n_beg[o]) * out.tick) : out.dt;
  const double tau = h / (0.1 * cs);
  const double alpha = out.alpha[o];
  const double decayed = (alpha + a_loc * dt / tau) / (1.0 + dt / tau);
  out.alpha[o] = a_loc > alpha ? a_loc : decayed;
}

template <typename I, bool ACC>
__global__ void __launch_bounds__(NB_THREADS)
    k_gradients(int64_t nrows, const int64_t* __restrict__ rows, Pos64 geo,
                const double4* __restrict__ vm,     // (vx, vy, vz, mass)
                const double4* __restrict__ hydro,  // (h, ...)
                const double4* __restrict__ acc,    // (ax, ay, az, -), with ACC
                const int64_t* __restrict__ off, const I* __restrict__ idx, GradParams prm,
                const int32_t* __restrict__ out_map, GradOut out) {
  const unsigned FULL = 0xffffffffu;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t q = t >> 3;
  const int gl = (int)(t & 7);
  bool live = q < nrows;
  int64_t a = 0, o = 0;
  if (live) {
    a = rows ? rows[q] : q;
    o = out_map ? (int64_t)out_map[a] : q;
    if (!rows && prm.mask && !prm.mask[o]) live = false;
  }
  if (!__any_sync(FULL, live)) return;  // warp-uniform
  const double4 va = vm[a];
  const double h_a = hydro[a].x;
  double4 aa = make_double4(0.0, 0.0, 0.0, 0.0);
  if (ACC) aa = acc[a];
  double rm[9], g[ACC ? 2 : 1][9];
#pragma unroll
  for (int e = 0; e < 9; ++e) {
    rm[e] = 0.0;
    g[0][e] = 0.0;
    if (ACC) g[ACC ? 1 : 0][e] = 0.0;
  }
  int cnt = 0;
  // eight lanes per row, each taking every eighth list entry; the sums are then added over
  // the row's lanes
  const int64_t e0 = live ? off[a] : 0, e1 = live ? off[a + 1] : 0;
  for (int64_t k = e0 + gl; k < e1; k += 8) {
    const int64_t b = (int64_t)ld_stream(idx + k);
    if (b == a) continue;
    double ddx, ddy, ddz;
    geo.diff(a, b, ddx, ddy, ddz);  // x_b - x_a
    if (prm.tighten) {
      const double h_b = hydro[b].x;
      const double rr = 2.0 * (h_a > h_b ? h_a : h_b);
      if (!(sqdist(ddx, ddy, ddz) < rr * rr)) continue;
    }
    cnt += 1;
    const double dx[3] = {-ddx, -ddy, -ddz};  // x_a - x_b
    const double r = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
    const double f = dwdr<double>(r, h_a, prm.kid, prm.cnorm) / r;
    const double4 vb = vm[b];
    const double dv[3] = {vb.x - va.x, vb.y - va.y, vb.z - va.z};
    double da[3] = {0.0, 0.0, 0.0};
    if (ACC) {
      const double4 ab = acc[b];
      da[0] = ab.x - aa.x;
      da[1] = ab.y - aa.y;
      da[2] = ab.z - aa.z;
    }
    const double mf = vb.w * f;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const double gj = mf * dx[j];
        rm[3 * i + j] -= dx[i] * gj;
        g[0][3 * i + j] += dv[i] * gj;
        if (ACC) g[ACC ? 1 : 0][3 * i + j] += da[i] * gj;
      }
  }
#pragma unroll
  for (int of = 4; of > 0; of >>= 1) {
    cnt += __shfl_xor_sync(FULL, cnt, of);
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      rm[e] += __shfl_xor_sync(FULL, rm[e], of);
      g[0][e] += __shfl_xor_sync(FULL, g[0][e], of);
      if (ACC) g[ACC ? 1 : 0][e] += __shfl_xor_sync(FULL, g[ACC ? 1 : 0][e], of);
    }
  }
  if (!live || gl != 0) return;
  corrected_gradients<ACC ? 2 : 1>(rm, cnt, g);
  const double* dv = g[0];
  if (out.gv) {
#pragma unroll
    for (int e = 0; e < 9; ++e) out.gv[9 * a + e] = dv[e];
  }
  if (!ACC) return;
  const double* dacc = g[ACC ? 1 : 0];
  const double div = dv[0] + dv[4] + dv[8];
  const double c0 = dv[7] - dv[5], c1 = dv[2] - dv[6], c2 = dv[3] - dv[1];
  const double curl = sqrt(c0 * c0 + c1 * c1 + c2 * c2);
  double sdd = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) sdd += dv[3 * i + j] * dv[3 * j + i];
  const double ddiv = dacc[0] + dacc[4] + dacc[8] - sdd;
  if (out.div) out.div[o] = div;
  if (out.curl) out.curl[o] = curl;
  if (out.ddiv) out.ddiv[o] = ddiv;
  if (out.alpha) switch_update(out, o, div, curl, ddiv);
}

// The switch and the reconstruction's gradients of a step in one walk of the cached lists
// (sorted order).  A list entry adds to R, G (and the acceleration sum) only where
// F(r, h_a) != 0, i.e. r / h_a < 2, and such an entry always passes the tightening test
// (r < 2 h_a <= 2 max(h_a, h_b)); the other entries add exact zeros.  So the sums over a row's
// tightened list (the switch, and the reconstruction of shared steps) and over its untightened
// list (the reconstruction of block steps) are the same sums over the same nonzero terms in
// the same order, and only the entry counts of the singular-matrix test differ: both are kept.
//   live: particles whose gradient the reconstruction needs (mask, caller order; null = all),
//         or none without it; rows: the switch's rows (sorted mask; null = no switch)
template <typename I, bool SW>
__global__ void __launch_bounds__(NB_THREADS)
    k_shock_grad(int64_t n, Pos64 geo, const double4* __restrict__ vm,
                 const double4* __restrict__ hydro, const double4* __restrict__ acc,
                 const int64_t* __restrict__ off, const I* __restrict__ idx, int kid,
                 double cnorm, int recon, int recon_full, const uint8_t* __restrict__ live_mask,
                 const uint8_t* __restrict__ row_sorted, const int32_t* __restrict__ perm,
                 GradOut out) {
  const unsigned FULL = 0xffffffffu;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t a = t >> 3;
  const int gl = (int)(t & 7);
  bool need_g = false, is_row = false;
  int64_t o = 0;
  if (a < n) {
    o = perm[a];
    need_g = recon && (!live_mask || live_mask[o]);
    is_row = SW && row_sorted[a];
  }
  const bool live = need_g || is_row;
  if (!__any_sync(FULL, live)) return;  // warp-uniform
  const double4 va = vm[live ? a : 0];
  const double h_a = hydro[live ? a : 0].x;
  double4 aa = make_double4(0.0, 0.0, 0.0, 0.0);
  if (SW && is_row) aa = acc[a];
  double rm[9], gv[9], ga[SW ? 9 : 1];
#pragma unroll
  for (int e = 0; e < 9; ++e) {
    rm[e] = 0.0;
    gv[e] = 0.0;
    if (SW) ga[SW ? e : 0] = 0.0;
  }
  int cnt_f = 0, cnt_t = 0;
  const int64_t e0 = live ? off[a] : 0, e1 = live ? off[a + 1] : 0;
  for (int64_t k = e0 + gl; k < e1; k += 8) {
    const int64_t b = (int64_t)ld_stream(idx + k);
    if (b == a) continue;
    cnt_f += 1;
    double ddx, ddy, ddz;
    geo.diff(a, b, ddx, ddy, ddz);  // x_b - x_a
    const double d2 = sqdist(ddx, ddy, ddz);
    const double h_b = hydro[b].x;
    const double rr = 2.0 * (h_a > h_b ? h_a : h_b);
    if (d2 < rr * rr) cnt_t += 1;
    const double dx[3] = {-ddx, -ddy, -ddz};  // x_a - x_b
    const double r = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
    if (!(r / h_a < 2.0)) continue;  // F(r, h_a) = 0: every term below is an exact zero
    const double f = dwdr<double>(r, h_a, kid, cnorm) / r;
    const double4 vb = vm[b];
    const double dv[3] = {vb.x - va.x, vb.y - va.y, vb.z - va.z};
    double da[3] = {0.0, 0.0, 0.0};
    if (SW && is_row) {
      const double4 ab = acc[b];
      da[0] = ab.x - aa.x;
      da[1] = ab.y - aa.y;
      da[2] = ab.z - aa.z;
    }
    const double mf = vb.w * f;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const double gj = mf * dx[j];
        rm[3 * i + j] -= dx[i] * gj;
        gv[3 * i + j] += dv[i] * gj;
        if (SW) ga[SW ? 3 * i + j : 0] += da[i] * gj;
      }
  }
#pragma unroll
  for (int of = 4; of > 0; of >>= 1) {
    cnt_f += __shfl_xor_sync(FULL, cnt_f, of);
    cnt_t += __shfl_xor_sync(FULL, cnt_t, of);
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      rm[e] += __shfl_xor_sync(FULL, rm[e], of);
      gv[e] += __shfl_xor_sync(FULL, gv[e], of);
      if (SW) ga[SW ? e : 0] += __shfl_xor_sync(FULL, ga[SW ? e : 0], of);
    }
  }
  if (!live || gl != 0) return;
  if (need_g) {
    double g1[1][9];
#pragma unroll
    for (int e = 0; e < 9; ++e) g1[0][e] = gv[e];
    corrected_gradients<1>(rm, recon_full ? cnt_f : cnt_t, g1);
#pragma unroll
    for (int e = 0; e < 9; ++e) out.gv[9 * a + e] = g1[0][e];
  }
  if (SW && is_row) {
    double g2[2][9];
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      g2[0][e] = gv[e];
      g2[1][e] = ga[SW ? e : 0];
    }
    corrected_gradients<2>(rm, cnt_t, g2);
    const double* dvm = g2[0];
    const double* dam = g2[1];
    const double div = dvm[0] + dvm[4] + dvm[8];
    const double c0 = dvm[7] - dvm[5], c1 = dvm[2] - dvm[6], c2 = dvm[3] - dvm[1];
    const double curl = sqrt(c0 * c0 + c1 * c1 + c2 * c2);
    double sdd = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) sdd += dvm[3 * i + j] * dvm[3 * j + i];
    const double ddiv = dam[0] + dam[4] + dam[8] - sdd;
    switch_update(out, o, div, curl, ddiv);
  }
}

}  // namespace nbk
