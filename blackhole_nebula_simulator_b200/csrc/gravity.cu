// The hole's gravity in FP64: the Tejeda-Rosswog generalized-Newtonian Hamiltonian
//     H = 1/2 A |p|^2 + 1/2 C (p.x)^2 - 1/r,   A = (r-2)/r,  C = -2 (r-2)/r^4,
// integrated per particle by the implicit generalized leapfrog (reference sim/integrator.py:
// 29-198; physics/gravity.py:61-121), and the per-particle pieces of the energy and angular
// momentum ledger (sim/coupled.py:261-270), reduced pairwise in a fixed order.
#include "common.cuh"
#include "gravity.cuh"

namespace nbk {

__global__ void k_glf_many(int64_t n, const double* __restrict__ x, const double* __restrict__ p,
                           const double* __restrict__ dt, double dt_scalar,
                           double* __restrict__ xo, double* __restrict__ po,
                           int64_t* __restrict__ iters) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double xi[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
  double pi[3] = {p[3 * i], p[3 * i + 1], p[3 * i + 2]};
  double a[3], b[3];
  int it = glf_one(xi, pi, dt ? dt[i] : dt_scalar, a, b);
  for (int k = 0; k < 3; ++k) {
    xo[3 * i + k] = a[k];
    po[3 * i + k] = b[k];
  }
  if (iters) iters[i] = it;
}

__global__ void k_v_from_p(int64_t n, const double* __restrict__ x, const double* __restrict__ p,
                           double* __restrict__ v) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double xi[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
  double pi[3] = {p[3 * i], p[3 * i + 1], p[3 * i + 2]};
  double w[3];
  gn_dh_dp(xi, pi, w);
  for (int k = 0; k < 3; ++k) v[3 * i + k] = w[k];
}

// p = f v + g rdot x/r, f = r/(r-2), g = 2r/(r-2)^2, rdot = x.v/r (physics/gravity.py:66-77).
__global__ void k_p_from_v(int64_t n, const double* __restrict__ x, const double* __restrict__ v,
                           double* __restrict__ p) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double xi[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
  double vi[3] = {v[3 * i], v[3 * i + 1], v[3 * i + 2]};
  double r = sqrt(xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2]);
  double f = r / (r - 2.0);
  double g = 2.0 * r / ((r - 2.0) * (r - 2.0));
  double rdot = (xi[0] * vi[0] + xi[1] * vi[1] + xi[2] * vi[2]) / r;
  for (int k = 0; k < 3; ++k) p[3 * i + k] = f * vi[k] + g * rdot * xi[k] / r;
}

// Ledger terms per particle: m (H + u), m |H|, m (x cross p), m p.  Block sums in a fixed tree
// order, then one block adds the block sums in index order: the same bits on every run.
constexpr int LEDGER_TERMS = 9;

__global__ void k_ledger_partial(int64_t n, const double* __restrict__ x,
                                 const double* __restrict__ p, const double* __restrict__ u,
                                 const double* __restrict__ m, double* __restrict__ part) {
  __shared__ double s[LEDGER_TERMS][NB_THREADS];
  double acc[LEDGER_TERMS];
  for (int t = 0; t < LEDGER_TERMS; ++t) acc[t] = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double xi[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
    double pi[3] = {p[3 * i], p[3 * i + 1], p[3 * i + 2]};
    double r = sqrt(xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2]);
    double a = (r - 2.0) / r, c = -2.0 * (r - 2.0) / (r * r * r * r);
    double px = pi[0] * xi[0] + pi[1] * xi[1] + pi[2] * xi[2];
    double H = 0.5 * a * (pi[0] * pi[0] + pi[1] * pi[1] + pi[2] * pi[2]) + 0.5 * c * px * px - 1.0 / r;
    double mi = m[i];
    acc[0] += mi * (H + u[i]);
    acc[1] += mi * fabs(H);
    acc[2] += mi * (xi[1] * pi[2] - xi[2] * pi[1]);
    acc[3] += mi * (xi[2] * pi[0] - xi[0] * pi[2]);
    acc[4] += mi * (xi[0] * pi[1] - xi[1] * pi[0]);
    acc[5] += mi * pi[0];
    acc[6] += mi * pi[1];
    acc[7] += mi * pi[2];
    acc[8] += mi;
  }
  for (int t = 0; t < LEDGER_TERMS; ++t) s[t][threadIdx.x] = acc[t];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int t = 0; t < LEDGER_TERMS; ++t) s[t][threadIdx.x] += s[t][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int t = 0; t < LEDGER_TERMS; ++t) part[LEDGER_TERMS * blockIdx.x + t] = s[t][0];
}

__global__ void k_sum_partials(int nb, int terms, const double* __restrict__ part,
                               double* __restrict__ out) {
  int t = threadIdx.x;
  if (t >= terms) return;
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s += part[terms * b + t];
  out[t] = s;
}

// Orbit level (sim/integrator.py:201-210): smallest k with dt_max / 2^k <= eta r^1.5 (K_MAX + 1
// when none), halving dt_max like the reference so the same k comes out.
__device__ __forceinline__ int orbit_level(double r, double eta, double dt_max) {
  double target = eta * pow(r, 1.5);
  double dt = dt_max;
  int k = 0;
  while (dt > target && k <= 40) {
    dt *= 0.5;
    k += 1;
  }
  return k;
}

// One orbit per thread on the integer tick timeline (tick = dt_max / 2^40) until tick n_end,
// recording every step (sim/integrator.py:220-253).  eta > 0: quantized adaptive steps; else
// fixed dt_max.  nrec[o] = records, or a negative failure code (-1/-2/-3 GLF, -4 level, -5 full).
__global__ void k_integrate_orbit(int norb, const double* __restrict__ state0, double dt_max,
                                  double eta, int64_t n_end, int64_t max_records,
                                  double* __restrict__ t_out, double* __restrict__ s_out,
                                  int64_t* __restrict__ it_out, int64_t* __restrict__ nrec) {
  int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= norb) return;
  const double tick = dt_max / 1099511627776.0;  // 2^40
  double x[3] = {state0[6 * o], state0[6 * o + 1], state0[6 * o + 2]};
  double p[3] = {state0[6 * o + 3], state0[6 * o + 4], state0[6 * o + 5]};
  double* T = t_out + (int64_t)o * max_records;
  double* S = s_out + (int64_t)o * max_records * 6;
  int64_t* I = it_out + (int64_t)o * max_records;
  int64_t n = 0, m = 0;
  T[0] = 0.0;
  for (int c = 0; c < 3; ++c) {
    S[c] = x[c];
    S[3 + c] = p[c];
  }
  I[0] = 0;
  while (n < n_end) {
    if (m + 1 >= max_records) {
      nrec[o] = -5;
      return;
    }
    int k = 0;
    if (eta > 0.0) k = orbit_level(sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]), eta, dt_max);
    while (k <= 40 && ((int64_t)1 << (40 - k)) > n_end - n) k += 1;  // never past the end
    if (k > 40) {
      nrec[o] = -4;
      return;
    }
    int64_t steps = (int64_t)1 << (40 - k);
    double xo[3], po[3];
    int it = glf_one(x, p, dt_max / (double)((int64_t)1 << k), xo, po);
    if (it < 0) {
      nrec[o] = it;
      return;
    }
    for (int c = 0; c < 3; ++c) {
      x[c] = xo[c];
      p[c] = po[c];
    }
    n += steps;
    m += 1;
    T[m] = (double)n * tick;
    for (int c = 0; c < 3; ++c) {
      S[6 * m + c] = x[c];
      S[6 * m + 3 + c] = p[c];
    }
    I[m] = it;
  }
  nrec[o] = m + 1;
}

void launch_integrate_orbit(int norb, const double* state0, double dt_max, double eta,
                            int64_t n_end, int64_t max_records, double* t_out, double* s_out,
                            int64_t* it_out, int64_t* nrec, cudaStream_t st) {
  if (norb > 0)
    count_launch(), k_integrate_orbit<<<(norb + 63) / 64, 64, 0, st>>>(norb, state0, dt_max, eta, n_end,
                                                                     max_records, t_out, s_out,
                                                                     it_out, nrec);
}

void launch_glf(int64_t n, const double* x, const double* p, const double* dt, double dt_scalar,
                double* xo, double* po, int64_t* iters, cudaStream_t st) {
  if (n > 0)
    count_launch(), k_glf_many<<<grid_for(n, 128), 128, 0, st>>>(n, x, p, dt, dt_scalar, xo, po, iters);
}

void launch_v_from_p(int64_t n, const double* x, const double* p, double* v, cudaStream_t st) {
  if (n > 0) count_launch(), k_v_from_p<<<grid_for(n), NB_THREADS, 0, st>>>(n, x, p, v);
}

void launch_p_from_v(int64_t n, const double* x, const double* v, double* p, cudaStream_t st) {
  if (n > 0) count_launch(), k_p_from_v<<<grid_for(n), NB_THREADS, 0, st>>>(n, x, v, p);
}

int ledger_blocks(int64_t n) { return (int)std::min<int64_t>(grid_for(n), 592); }

void launch_ledger(int64_t n, const double* x, const double* p, const double* u, const double* m,
                   double* part, double* out, cudaStream_t st) {
  int nb = ledger_blocks(n);
  count_launch(), k_ledger_partial<<<nb, NB_THREADS, 0, st>>>(n, x, p, u, m, part);
  count_launch(), k_sum_partials<<<1, 32, 0, st>>>(nb, LEDGER_TERMS, part, out);
}

}  // namespace nbk
