// The reference's step drivers on device state: the hydro evaluation of active rows and their
// neighbours (sim/blocks.py:217-315; sim/coupled.py:145-195), the shared kick-flow-kick step
// (sim/coupled.py:198-258), and the block-timestep system step with levels, limiter, wake-up and
// opening kicks on the int64 tick timeline (sim/blocks.py:318-563, sim/timesteps.py:21-59).
//
// Compiled without fused multiply-add: every kick, drift and cooling update rounds like the
// reference's NumPy expressions.
#include <cub/cub.cuh>

#include "common.cuh"
#include "cooling.cuh"
#include "engine.cuh"
#include "gravity.cuh"
#include "steps.cuh"

namespace nbk {

__device__ __forceinline__ int64_t ticks_of(int64_t level) { return (int64_t)1 << (K_MAX - level); }

__device__ __forceinline__ double norm3(const double* v) {
  return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
}

__global__ void k_fill_u8(int64_t n, uint8_t v, uint8_t* __restrict__ m) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) m[i] = v;
}

__global__ void k_any_nonpositive(int64_t n, const double* __restrict__ u, int* err) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n && !(u[i] > 0.0)) set_error(err, ERR_NONPOSITIVE_U);
}

__global__ void k_set_rows(int64_t nrows, const int64_t* __restrict__ rows, double v,
                           double* __restrict__ a) {
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q < nrows) a[rows[q]] = v;
}

__global__ void k_iota(int64_t n, int64_t* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = i;
}

// Heat budget of the block steps (sim/blocks.py:434-440): a kick u += dt du/dt of particle i split
// into its viscous, conductive, disc-viscous and P dV parts.  hv null: no budget kept.
struct HeatBook {
  const double* vh = nullptr;  // parts of du/dt at the last force evaluation
  const double* ch = nullptr;
  const double* dh = nullptr;
  double* hv = nullptr;  // accumulated parts
  double* hc = nullptr;
  double* hd = nullptr;
  double* hp = nullptr;
};

static HeatBook heat_of(const nb_state* s) {
  HeatBook b;
  if (!s->heat_visc) return b;
  b.vh = s->visc_heating;
  b.ch = s->cond_heating;
  b.dh = s->disk_heating;
  b.hv = s->heat_visc;
  b.hc = s->heat_cond;
  b.hd = s->heat_disk;
  b.hp = s->heat_pdv;
  return b;
}

__device__ __forceinline__ void book_heat(const HeatBook& b, int64_t i, double dt, double dudt) {
  if (!b.hv) return;
  const double v = b.vh ? b.vh[i] : 0.0;
  const double c = b.ch ? b.ch[i] : 0.0;
  const double d = b.dh ? b.dh[i] : 0.0;
  b.hv[i] += dt * v;
  b.hc[i] += dt * c;
  b.hd[i] += dt * d;
  b.hp[i] += dt * (dudt - v - c - d);
}

static BremsParams brems_of(const nb_params* prm) {
  BremsParams b;
  b.tfac = prm->brems_tfac;
  b.b = prm->brems_b;
  b.kappa = prm->brems_kappa;
  b.u_floor = prm->u_floor;
  b.t_floor = prm->brems_t_floor;
  return b;
}

// ---------------------------------------------------------------- hydro of the active rows
// sim/blocks.py:217-239 (_density_touched) and 242-315 (_hydro_rows): density for the rows and
// every neighbour in the cached lists, widened until every interacting neighbour is fresh; then
// the fused EOS + force pass for the rows.
int hydro_rows(Engine& E, nb_state* s, const nb_params* prm, int64_t nrows, const int64_t* rows,
               const double* vel, const double* u, cudaStream_t st, const ShockStep& sk) {
  Workspace& W = E.ws;
  int64_t n = s->n;
  NB_TRY(W.ensure(E, n));
  count_launch(), k_any_nonpositive<<<grid_for(n), NB_THREADS, 0, st>>>(n, u, E.d_err);
  W.pend_err = true;  // read with the touched set's count, before any state is written
  // todo = every particle without a cache, else rows and their cached-list neighbours
  // (full_marks: the todo set holds every particle or every list entry of the rows on the lists
  // that are cached now)
  bool full_marks = true;
  if (!W.cache.valid || W.cache.n != n || E.lists.n != n) {
    count_launch(), k_fill_u8<<<grid_for(n), NB_THREADS, 0, st>>>(n, 1, W.m_need);
  } else {
    NB_CUDA(cudaMemsetAsync(W.m_need, 0, n, st));
    E.prof.begin(st);
    NB_TRY(mark_rows(E, nrows, rows, 0, s->x, s->h, W.m_need, st));
    E.prof.end(PROF_MARKS, st, (double)nrows, 0.0);
  }
  NB_CUDA(cudaMemsetAsync(W.m_done, 0, n, st));
  const int64_t builds_in = s->builds;
  bool settled = false;
  for (int it = 0; it < 8; ++it) {
    int64_t ntodo = 0;
    // on cached lists, the first reuse test runs on the todo mask before its count is read, and
    // its outcome comes back with the count (W.d_i64[1])
    int first_fail = -1;
    const bool pre = it == 0 && W.cache.valid && W.cache.n == n && E.lists.n == n && n > 0;
    if (pre) {
      NB_CUDA(cudaMemsetAsync(W.d_i64 + 1, 0, sizeof(int64_t), st));
      NB_TRY(reuse_first_test(E, n, s->x, s->h, W.m_need, reinterpret_cast<int*>(W.d_i64 + 1), st));
      int64_t fail64 = 0;
      NB_TRY(select_mask(E, n, W.m_need, W.rows2, &ntodo, st, &fail64));
      first_fail = fail64 != 0;
    } else {
      NB_TRY(select_mask(E, n, W.m_need, W.rows2, &ntodo, st));
    }
    if (ntodo == 0) {
      settled = true;
      break;
    }
    const int64_t builds0 = s->builds;
    NB_TRY(compute_density(E, n, s->x, s->mass, s->h, s->rho, s->omega, ntodo, W.rows2, prm,
                           &s->builds, &s->reuses, st, pre ? W.m_need : nullptr, first_fail));
    mask_or(n, W.m_need, W.m_done, st);
    // Reused lists are complete for every pair within 2 max(h_i, h_j) at the new h (the reuse
    // test proves it for the search limits the solve was capped at), so the interacting
    // neighbours of the rows are list entries of the rows, all of them done already: the
    // marking pass below would find nothing new.
    if (full_marks && s->builds == builds0) {
      settled = true;
      break;
    }
    full_marks = false;
    // interacting neighbours of the rows at the current h
    NB_CUDA(cudaMemsetAsync(W.m_tmp, 0, n, st));
    E.prof.begin(st);
    NB_TRY(mark_rows(E, nrows, rows, 1, s->x, s->h, W.m_tmp, st));
    E.prof.end(PROF_MARKS, st, (double)nrows, 0.0);
    mask_and_not(n, W.m_tmp, W.m_done, W.m_need, st);
  }
  if (!settled) {
    int64_t ntodo = 0;
    NB_TRY(select_mask(E, n, W.m_need, W.rows2, &ntodo, st));
    if (ntodo != 0) {
      std::snprintf(E.last_error, sizeof(E.last_error),
                    "neighbour set of the active particles did not settle");
      return NB_ERR_TOUCHED;
    }
  }
  if (prm->viscosity && !prm->visc_switch)
    count_launch(), k_set_rows<<<grid_for(nrows), NB_THREADS, 0, st>>>(nrows, rows, prm->alpha_const, s->alpha);
  ShockStep sk2 = sk;
  sk2.touched_covers_lists = s->builds == builds_in;  // no rebuild since the first marking
  return engine_forces(E, s, vel, u, nrows, rows, prm, W.m_done, sk2, st);
}

// ---------------------------------------------------------------- shared step
__global__ void k_kick_half(int64_t n, const double* __restrict__ p, const double* __restrict__ a,
                            const double* __restrict__ u, const double* __restrict__ dudt,
                            double half, double* __restrict__ p_out, double* __restrict__ u_out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int c = 0; c < 3; ++c) p_out[3 * i + c] = p[3 * i + c] + half * a[3 * i + c];
  u_out[i] = u[i] + half * dudt[i];
}

// cooling over dt at mid-step (sim/coupled.py:244-251): u_half <- cooled, dm = m (u_half - u_new)
__global__ void k_cool_shared(int64_t n, int law, const double* __restrict__ x0,
                              const double* __restrict__ x1, const double* __restrict__ rho,
                              const double* __restrict__ m, double dt, double beta,
                              double u_floor, BremsParams bp, double* __restrict__ u_half,
                              double* __restrict__ dm) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double uh = u_half[i], un;
  if (law == 1) {
    double r_mid = 0.5 * (norm3(x0 + 3 * i) + norm3(x1 + 3 * i));
    double t_cool = beta / pow(r_mid, -1.5);
    un = beta_cool_one(uh, u_floor, dt, t_cool);
  } else {
    un = brems_cool_one(uh, rho[i], dt, bp);
  }
  dm[i] = m[i] * (uh - un);
  u_half[i] = un;
}

__global__ void k_pred_shared(int64_t n, const double* __restrict__ p_flow,
                              const double* __restrict__ a, const double* __restrict__ u_half,
                              const double* __restrict__ dudt, double half,
                              double* __restrict__ p_pred, double* __restrict__ u_pred) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int c = 0; c < 3; ++c) p_pred[3 * i + c] = p_flow[3 * i + c] + half * a[3 * i + c];
  u_pred[i] = u_half[i] + half * dudt[i];
}


static int glf_status(Engine& E, int64_t n, const int64_t* iters, cudaStream_t st) {
  size_t tmp = E.cub_bytes;
  NB_CUDA(cub::DeviceReduce::Min(E.cub_tmp, tmp, iters, E.ws.d_i64, (int)n, st));
  NB_CUDA(cudaMemcpyAsync(E.ws.h_i64, E.ws.d_i64, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  NB_CUDA(host_sync(st));
  int64_t worst = E.ws.h_i64[0];
  if (worst >= 0) return 0;
  const char* msg = worst == -1   ? "stage 1 (p_half) did not converge in 10 iterations: time step too large"
                    : worst == -2 ? "stage 2 (x1) did not converge in 10 iterations: time step too large"
                                  : "particle inside r = 2.5";
  std::snprintf(E.last_error, sizeof(E.last_error), "%s", msg);
  return worst == -1 ? NB_ERR_GLF_P_HALF : worst == -2 ? NB_ERR_GLF_X1 : NB_ERR_GLF_RADIUS;
}

static int sum_doubles(Engine& E, int64_t n, const double* a, double* out, cudaStream_t st) {
  if (n <= 0) {
    *out = 0.0;
    return 0;
  }
  size_t tmp = E.cub_bytes;
  NB_CUDA(cub::DeviceReduce::Sum(E.cub_tmp, tmp, a, E.ws.d_tmp, (int)n, st));
  NB_CUDA(cudaMemcpyAsync(E.ws.h_dbl, E.ws.d_tmp, sizeof(double), cudaMemcpyDeviceToHost, st));
  NB_CUDA(host_sync(st));
  *out = E.ws.h_dbl[0];
  return 0;
}

int coupled_initialise(Engine& E, nb_state* s, const nb_params* prm, cudaStream_t st) {
  Workspace& W = E.ws;
  int64_t n = s->n;
  NB_TRY(W.ensure(E, n));
  W.cache.valid = false;
  count_launch(), k_iota<<<grid_for(n), NB_THREADS, 0, st>>>(n, W.rows);
  W.rows_ver += 1;
  launch_v_from_p(n, s->x, s->p, W.v_eval, st);
  NB_TRY(hydro_rows(E, s, prm, n, W.rows, W.v_eval, s->u, st));
  return pending_flush(E, st);
}

int coupled_step(Engine& E, nb_state* s, const nb_params* prm, double dt, cudaStream_t st) {
  Workspace& W = E.ws;
  int64_t n = s->n;
  NB_TRY(W.ensure(E, n));
  double half = 0.5 * dt;
  // p_half, u_half; gravity flow over dt
  double* u_half = W.d_uh;
  count_launch(), k_kick_half<<<grid_for(n), NB_THREADS, 0, st>>>(n, s->p, s->a_hydro, s->u, s->dudt, half,
                                                  W.v_tmp, u_half);
  E.prof.begin(st);
  launch_glf(n, s->x, W.v_tmp, nullptr, dt, W.v_pred, W.v_flow, W.iters, st);
  E.prof.end(PROF_FLOW, st, (double)n, 0.0);
  NB_TRY(glf_status(E, n, W.iters, st));
  if (prm->cooling == 1 || prm->cooling == 2) {
    count_launch(), k_cool_shared<<<grid_for(n), NB_THREADS, 0, st>>>(n, prm->cooling, s->x, W.v_pred, s->rho,
                                                      s->mass, dt, prm->cooling_beta,
                                                      prm->u_floor, brems_of(prm), u_half, W.d_dm);
    double de = 0;
    NB_TRY(sum_doubles(E, n, W.d_dm, &de, st));
    s->e_radiated += de;
  }
  // predicted state: x1, p_flow, u_half + dt/2 dudt; predictor momentum for velocities
  NB_CUDA(cudaMemcpyAsync(s->x, W.v_pred, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, st));
  count_launch(), k_pred_shared<<<grid_for(n), NB_THREADS, 0, st>>>(n, W.v_flow, s->a_hydro, u_half, s->dudt,
                                                    half, W.v_tmp, s->u);
  launch_v_from_p(n, s->x, W.v_tmp, W.v_eval, st);
  count_launch(), k_iota<<<grid_for(n), NB_THREADS, 0, st>>>(n, W.rows);
  W.rows_ver += 1;
  ShockStep sk;
  sk.switch_on = 1;
  sk.dt = dt;
  NB_TRY(hydro_rows(E, s, prm, n, W.rows, W.v_eval, s->u, st, sk));
  // closing kick with the new forces
  count_launch(), k_pred_shared<<<grid_for(n), NB_THREADS, 0, st>>>(n, W.v_flow, s->a_hydro, u_half, s->dudt,
                                                    half, s->p, s->u);
  s->particle_steps += n;
  s->last_active = n;
  NB_CUDA(cudaGetLastError());
  return pending_flush(E, st);
}

// sim/coupled.py:213-226: min over particles of C_cour h / v_sig, C_force sqrt(h / |a|),
// viscous 0.25 h^2 / nu and eta_orb r^(3/2).
// Bremsstrahlung time-step limit (this project's criterion; the reference's beta-cooling is
// exact at any step): C_cool u / |du/dt| for gas above the floor temperature, else inf.
constexpr double C_COOL = 0.25;
__device__ __forceinline__ double cooling_dt(int law, double u, double rho, const BremsParams& bp) {
  if ((law != 2 && law != 3) || !(bp.tfac * u > bp.t_floor)) return INFINITY;
  double rate = fabs(brems_rate(u, rho, bp));
  return rate > 0 ? C_COOL * u / rate : INFINITY;
}

__global__ void k_stable_dt(int64_t n, const double* __restrict__ h, const double* __restrict__ vsig,
                            const double* __restrict__ a, const double* __restrict__ nu,
                            const double* __restrict__ x, double courant, double c_force,
                            double eta_orb, int law, const double* __restrict__ u,
                            const double* __restrict__ rho, BremsParams bp,
                            double* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double dt = courant * (h[i] / vsig[i]);
  double amag = norm3(a + 3 * i);
  if (amag > 0) dt = fmin(dt, c_force * sqrt(h[i] / amag));
  if (nu && nu[i] > 0) dt = fmin(dt, 0.25 * h[i] * h[i] / nu[i]);
  double r = norm3(x + 3 * i);
  dt = fmin(dt, eta_orb * pow(r, 1.5));
  out[i] = fmin(dt, cooling_dt(law, u[i], rho[i], bp));
}

int coupled_stable_dt(Engine& E, nb_state* s, const nb_params* prm, double* dt, cudaStream_t st) {
  Workspace& W = E.ws;
  int64_t n = s->n;
  NB_TRY(W.ensure(E, n));
  count_launch(), k_stable_dt<<<grid_for(n), NB_THREADS, 0, st>>>(n, s->h, s->vsig_max, s->a_hydro,
                                                  prm->disc_alpha_av > 0 ? s->nu : nullptr, s->x,
                                                  prm->courant, prm->c_force, prm->eta_orb,
                                                  prm->cooling, s->u, s->rho, brems_of(prm), W.d_b);
  size_t tmp = E.cub_bytes;
  NB_CUDA(cub::DeviceReduce::Min(E.cub_tmp, tmp, W.d_b, W.d_tmp, (int)n, st));
  NB_CUDA(cudaMemcpyAsync(W.h_dbl, W.d_tmp, sizeof(double), cudaMemcpyDeviceToHost, st));
  NB_CUDA(host_sync(st));
  *dt = W.h_dbl[0];
  return 0;
}

// ---------------------------------------------------------------- block steps
// gravity flow of every particle to tick n_next from its step start, the predictor momentum,
// and the active flags (sim/blocks.py:506-517)
__global__ void k_block_flow(int64_t n, const int64_t* __restrict__ n_next_p, double tick,
                             const double* __restrict__ x_beg, const double* __restrict__ p_half,
                             const int64_t* __restrict__ n_beg, const int64_t* __restrict__ n_end,
                             const double* __restrict__ a, double* __restrict__ x,
                             double* __restrict__ p_flow, double* __restrict__ p_pred,
                             double* __restrict__ v_eval, int64_t* __restrict__ iters,
                             uint8_t* __restrict__ active) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t n_next = *n_next_p;
  double s = (double)(n_next - n_beg[i]) * tick;
  double half_len = 0.5 * (double)(n_end[i] - n_beg[i]) * tick;
  double xb[3] = {x_beg[3 * i], x_beg[3 * i + 1], x_beg[3 * i + 2]};
  double pb[3] = {p_half[3 * i], p_half[3 * i + 1], p_half[3 * i + 2]};
  double xo[3], po[3], pp[3];
  iters[i] = glf_one(xb, pb, s, xo, po);
  double lag = s - half_len;
  for (int c = 0; c < 3; ++c) {
    pp[c] = po[c] + lag * a[3 * i + c];
    x[3 * i + c] = xo[c];
    p_flow[3 * i + c] = po[c];
    p_pred[3 * i + c] = pp[c];
  }
  if (v_eval) {  // the velocity of the predicted momentum at the new position (k_v_from_p's)
    double w[3];
    gn_dh_dp(xo, pp, w);
    for (int c = 0; c < 3; ++c) v_eval[3 * i + c] = w[c];
  }
  active[i] = n_end[i] == n_next;
}

// cooling at mid-step of every particle over its elapsed time s (exact laws), radiated energy of
// the active rows, and the predicted u (sim/blocks.py:518-538)
__global__ void k_block_cool(int64_t n, int law, int64_t n_next, double tick,
                             const int64_t* __restrict__ n_beg, const int64_t* __restrict__ n_end,
                             const double* __restrict__ x_beg, const double* __restrict__ x,
                             const double* __restrict__ rho, const double* __restrict__ m,
                             const double* __restrict__ dudt, double beta, double u_floor,
                             BremsParams bp, const double* __restrict__ uc_in,
                             double* __restrict__ u_half, double* __restrict__ u,
                             double* __restrict__ lum, double* __restrict__ dm,
                             double* __restrict__ heat_cool) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = (double)(n_next - n_beg[i]) * tick;
  double half_len = 0.5 * (double)(n_end[i] - n_beg[i]) * tick;
  double uh = u_half[i];
  bool act = n_end[i] == n_next;
  double uc = uh;
  if (law == 1) {
    double r_mid = 0.5 * (norm3(x_beg + 3 * i) + norm3(x + 3 * i));
    double t_cool = beta / pow(r_mid, -1.5);
    uc = beta_cool_one(uh, u_floor, s, t_cool);
  } else if (law == 2) {
    uc = brems_cool_one(uh, rho[i], s, bp);
  } else if (law == 3) {
    // the network's result closes the step; the provisional prediction of a particle in mid-step
    // takes the exact integrator (cheaper than the network, and replaced when the step closes)
    uc = act ? uc_in[i] : brems_cool_one(uh, rho[i], s, bp);
  }
  if (law != 0) {
    double d = act ? m[i] * (uh - uc) : 0.0;
    dm[i] = d;
    if (act) {
      lum[i] = d / (2.0 * half_len);
      if (heat_cool) heat_cool[i] += uh - uc;
      u_half[i] = uc;
    }
  }
  u[i] = uc + (s - half_len) * dudt[i];
}

// inputs of the network for the rows: u_half, rho and the elapsed time of each row's step
__global__ void k_gather_cool_rows(int64_t nrows, const int64_t* __restrict__ rows, int64_t n_next,
                                   double tick, const int64_t* __restrict__ n_beg,
                                   const double* __restrict__ u_half, const double* __restrict__ rho,
                                   double* __restrict__ ug, double* __restrict__ rg,
                                   double* __restrict__ sg) {
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= nrows) return;
  int64_t i = rows[q];
  ug[q] = u_half[i];
  rg[q] = rho[i];
  sg[q] = (double)(n_next - n_beg[i]) * tick;
}

__global__ void k_scatter_rows_d(int64_t nrows, const int64_t* __restrict__ rows,
                                 const double* __restrict__ v, double* __restrict__ out) {
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q < nrows) out[rows[q]] = v[q];
}

// closing kicks of the rows (sim/blocks.py:544-547)
__global__ void k_block_close(int64_t nrows, const int64_t* __restrict__ rows, double tick,
                              const int64_t* __restrict__ n_beg, const int64_t* __restrict__ n_end,
                              const double* __restrict__ p_flow, const double* __restrict__ a,
                              const double* __restrict__ u_half, const double* __restrict__ dudt,
                              double* __restrict__ p_pred, double* __restrict__ u, HeatBook hb) {
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= nrows) return;
  int64_t i = rows[q];
  double half_len = 0.5 * (double)(n_end[i] - n_beg[i]) * tick;
  for (int c = 0; c < 3; ++c) p_pred[3 * i + c] = p_flow[3 * i + c] + half_len * a[3 * i + c];
  u[i] = u_half[i] + half_len * dudt[i];
  book_heat(hb, i, half_len, dudt[i]);
}

// wanted level of the rows: orbit, Courant, force and viscous criteria (sim/blocks.py:318-334),
// level_for_dt (sim/timesteps.py:26-39), forced offset, allowed_level (sim/timesteps.py:47-59)
__global__ void k_wanted_levels(int64_t nrows, const int64_t* __restrict__ rows, int64_t tick_n,
                                double dt_max, const double* __restrict__ h,
                                const double* __restrict__ vsig, const double* __restrict__ a,
                                const double* __restrict__ nu, const double* __restrict__ x,
                                double courant, double c_force, double eta_orb, int law,
                                const double* __restrict__ u, const double* __restrict__ rho,
                                BremsParams bp, const int64_t* __restrict__ offset,
                                int64_t* __restrict__ level, int* err) {
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= nrows) return;
  int64_t i = rows[q];
  double hi = h[i];
  double dt = courant * hi / vsig[i];
  double amag = norm3(a + 3 * i);
  if (amag > 0) dt = fmin(dt, c_force * sqrt(hi / amag));
  if (nu && nu[i] > 0) dt = fmin(dt, 0.25 * (hi * hi) / nu[i]);
  dt = fmin(dt, eta_orb * pow(norm3(x + 3 * i), 1.5));
  dt = fmin(dt, cooling_dt(law, u[i], rho[i], bp));
  if (!(dt > 0)) {
    set_error(err, ERR_DT);
    return;
  }
  double kd = ceil(log2(dt_max / dt) - 1e-12);
  int64_t k = (int64_t)kd;
  if (k < 0) k = 0;
  if (k <= 62 && dt_max / exp2((double)k) > dt) k += 1;
  if (k > K_MAX) {
    set_error(err, ERR_LEVEL);
    return;
  }
  k += offset ? offset[i] : 0;
  int64_t cur = level[i];
  int64_t nw = k >= cur ? k : cur;
  if (k < cur) {
    for (int64_t kk = k; kk < cur; ++kk) {
      if (kk >= 0 && kk <= K_MAX && tick_n % ticks_of(kk) == 0) {
        nw = kk;
        break;
      }
    }
  }
  level[i] = nw;
}

// The interacting entries (r < 2 max(h_i, h_j), the reference's FP64 test) of the rows, written
// into the rows' own stretches of the list storage (tidx[off[k] ..], tcnt[q] of them), so the
// limiter sweeps and the wake-up walk short lists without distance tests.  Eight lanes per row;
// a group ballot keeps the entries in list order.
__global__ void k_tight_rows(int64_t nrows, const int64_t* __restrict__ rows_s,
                             const int64_t* __restrict__ off, const int32_t* __restrict__ idx,
                             const double4* __restrict__ pk, int32_t* __restrict__ tidx,
                             int32_t* __restrict__ tcnt) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t q = t >> 3;
  const int gl = (int)(t & 7), g = (int)((threadIdx.x & 31) >> 3);
  const bool live = q < nrows;
  if (!__any_sync(0xffffffffu, live)) return;  // warp-uniform
  int64_t k = live ? rows_s[q] : 0;
  const int64_t e0 = live ? off[k] : 0, e1 = live ? off[k + 1] : 0;
  const unsigned len = (unsigned)(e1 - e0);
  const unsigned maxlen = __reduce_max_sync(0xffffffffu, len);
  double4 me = live ? pk[k] : make_double4(0, 0, 0, 0);
  int m = 0;
  for (unsigned b = 0; b < maxlen; b += 8) {
    bool take = false;
    int32_t js = 0;
    if (b + gl < len) {
      js = ld_stream(idx + e0 + b + gl);
      double4 o = pk[js];
      double d2 = d2_exact(o.x - me.x, o.y - me.y, o.z - me.z);
      double rr = 2.0 * fmax(me.w, o.w);
      take = d2 < rr * rr;
    }
    unsigned seg = (__ballot_sync(0xffffffffu, take) >> (8 * g)) & 0xffu;
    if (take) tidx[e0 + m + __popc(seg & ((1u << gl) - 1u))] = js;
    m += __popc(seg);
  }
  if (live && gl == 0) tcnt[q] = m;
}

// one sweep of the level limiter (sim/blocks.py:337-353) over the rows' interacting entries, on
// curve-ordered rows and a sorted copy of the levels (eight lanes per row); the least fixed point
// above the start is unique, so in-place sweeps reach the reference's levels
__global__ void k_limit_sweep_t(int64_t nrows, const int64_t* __restrict__ rows_s,
                                const int64_t* __restrict__ off, const int32_t* __restrict__ tidx,
                                const int32_t* __restrict__ tcnt, int max_gap,
                                int32_t* level_s, int* changed) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t q = t >> 3;
  const int gl = (int)(t & 7);
  const bool live = q < nrows;
  int64_t k = 0;
  int need = INT_MIN;
  if (live) {
    k = rows_s[q];
    need = ((volatile int32_t*)level_s)[k];
    const int32_t* tl = tidx + off[k];
    for (int c = gl; c < tcnt[q]; c += 8) {
      int lj = ((volatile int32_t*)level_s)[tl[c]];
      if (lj - max_gap > need) need = lj - max_gap;
    }
  }
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) {
    int other = __shfl_xor_sync(0xffffffffu, need, o);
    need = other > need ? other : need;
  }
  if (live && gl == 0 && need > ((volatile int32_t*)level_s)[k]) {
    atomicMax(&level_s[k], need);
    *changed = 1;
  }
}

// _wake_targets (sim/blocks.py:356-364): need[j] = max over active i of level_i - max_gap, over
// the rows' interacting entries into a sorted need array (eight lanes per row).  k_cut_steps acts
// on j only where need[j] > level[j], so a contribution that is not above j's own level cannot
// change what it does and is skipped (a load instead of an atomic): need[j] stays below or at
// level[j] exactly where it did, and keeps its maximum where it is above.
__global__ void k_wake_need_t(int64_t nrows, const int64_t* __restrict__ rows_s,
                              const int64_t* __restrict__ off, const int32_t* __restrict__ tidx,
                              const int32_t* __restrict__ tcnt, const int32_t* __restrict__ level_s,
                              int max_gap, int32_t* __restrict__ need_s) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t q = t >> 3;
  const int gl = (int)(t & 7);
  if (q >= nrows) return;
  int64_t k = rows_s[q];
  const int v = level_s[k] - max_gap;
  const int32_t* tl = tidx + off[k];
  for (int c = gl; c < tcnt[q]; c += 8) {
    const int32_t j = tl[c];
    if (v > level_s[j]) atomicMax(&need_s[j], v);
  }
}

// levels (at most K_MAX) in sorted order as 32-bit integers, for the sweeps' gathers
__global__ void k_gather_level32(int64_t n, const int32_t* __restrict__ perm,
                                 const int64_t* __restrict__ a, int32_t* __restrict__ out) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < n) out[k] = (int32_t)a[perm[k]];
}

__global__ void k_fill_i32(int64_t n, int32_t v, int32_t* __restrict__ a) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

__global__ void k_scatter_rows_level32(int64_t nrows, const int64_t* __restrict__ rows_s,
                                       const int32_t* __restrict__ perm,
                                       const int32_t* __restrict__ a_s, int64_t* __restrict__ a) {
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= nrows) return;
  int64_t k = rows_s[q];
  a[perm[k]] = a_s[k];
}

__global__ void k_scatter_level32(int64_t n, const int32_t* __restrict__ perm,
                                  const int32_t* __restrict__ a_s, int64_t* __restrict__ a) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < n) a[perm[k]] = a_s[k];
}

// _land (sim/blocks.py:383-393) and the K_MAX check of _choose_levels
__global__ void k_land(int64_t nrows, const int64_t* __restrict__ rows, int64_t tick_n,
                       int64_t n_stop, int64_t* __restrict__ level, int* err) {
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= nrows) return;
  int64_t i = rows[q];
  int64_t k = level[i];
  if (tick_n < n_stop) {
    for (int guard = 0; guard < 64; ++guard) {
      int64_t kk = k < K_MAX ? k : K_MAX;
      if (!(tick_n + ticks_of(kk) > n_stop)) break;
      k += 1;
    }
  }
  if (k > K_MAX) set_error(err, ERR_LEVEL);
  level[i] = k;
}

// _cut_steps / _cut_to (sim/blocks.py:404-431): shorten running steps longer than `need` allows
__global__ void k_cut_steps(int64_t n, int64_t tick_n, double tick, const int64_t* __restrict__ need,
                            const double* __restrict__ a, const double* __restrict__ dudt,
                            int64_t* __restrict__ level, int64_t* __restrict__ n_end,
                            double* __restrict__ p_half, double* __restrict__ u_half,
                            unsigned long long* __restrict__ woken, const int* __restrict__ err,
                            HeatBook hb) {
  int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= n || *err) return;  // a failed landing leaves the state as it was
  int64_t nd = need[j];
  if (!(n_end[j] > tick_n && nd > level[j])) return;
  int64_t t_new = ticks_of(nd);
  int64_t end_new = (tick_n / t_new + 1) * t_new;
  level[j] = nd;
  if (end_new < n_end[j]) {
    double d_len = (double)(end_new - n_end[j]) * tick;
    for (int c = 0; c < 3; ++c) p_half[3 * j + c] += 0.5 * d_len * a[3 * j + c];
    u_half[j] += 0.5 * d_len * dudt[j];
    book_heat(hb, j, 0.5 * d_len, dudt[j]);
    n_end[j] = end_new;
    atomicAdd(woken, 1ull);
  }
}

// _open (sim/blocks.py:443-452)
__global__ void k_open(int64_t nrows, const int64_t* __restrict__ rows, int64_t tick_n, double tick,
                       const int64_t* __restrict__ level, const double* __restrict__ x,
                       const double* __restrict__ p, const double* __restrict__ u,
                       const double* __restrict__ a, const double* __restrict__ dudt,
                       int64_t* __restrict__ n_beg, int64_t* __restrict__ n_end,
                       double* __restrict__ x_beg, double* __restrict__ p_half,
                       double* __restrict__ u_half, const int* __restrict__ err, HeatBook hb) {
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= nrows || *err) return;  // a failed landing leaves the state as it was
  int64_t i = rows[q];
  int64_t t = ticks_of(level[i]);
  double length = (double)t * tick;
  n_beg[i] = tick_n;
  n_end[i] = tick_n + t;
  for (int c = 0; c < 3; ++c) {
    x_beg[3 * i + c] = x[3 * i + c];
    p_half[3 * i + c] = p[3 * i + c] + 0.5 * length * a[3 * i + c];
  }
  u_half[i] = u[i] + 0.5 * length * dudt[i];
  book_heat(hb, i, 0.5 * length, dudt[i]);
}

__global__ void k_fill_i64(int64_t n, int64_t v, int64_t* __restrict__ a) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

// sim/blocks.py:367-380 (_choose_levels) followed by _open for the rows
static int choose_levels_and_open(Engine& E, nb_state* s, const nb_params* prm, int64_t nrows,
                                  const int64_t* rows, cudaStream_t st) {
  Workspace& W = E.ws;
  Lists& L = E.lists;
  int64_t n = s->n;
  // sorted levels and wake-up needs as 32-bit integers in the int64 scratch arrays
  int32_t* lvl_s = reinterpret_cast<int32_t*>(W.i_lvl);
  int32_t* need_s = reinterpret_cast<int32_t*>(W.i_tmp2);
  if (nrows == 0) return 0;
  count_launch(), k_wanted_levels<<<grid_for(nrows), NB_THREADS, 0, st>>>(
      nrows, rows, s->tick_n, prm->dt_max, s->h, s->vsig_max, s->a_hydro,
      prm->disc_alpha_av > 0 ? s->nu : nullptr, s->x, prm->courant, prm->c_force, prm->eta_orb,
      prm->cooling, s->u, s->rho, brems_of(prm), s->level_offset, s->level, E.d_err);
  W.pend_err = true;  // read with the first limiter sweep's flag (or by the landing check)
  int64_t ns = 0;
  if (prm->limiter) {
    // the rows' interacting entries, once for every sweep and the wake-up walk (already written
    // by the force pass of these rows on these lists, when it ran just before); the sorted
    // (x, h) are needed only to find them here
    const bool have_tight = rows == W.rows && W.tight_ver == W.rows_ver &&
                            W.tight_gen == L.gen && W.tight_n == nrows;
    // curve-ordered rows, and a sorted copy of the levels
    if (have_tight)
      NB_TRY(sorted_rows(E, nrows, rows, &ns, st));
    else
      NB_TRY(sorted_rows_and_pack(E, nrows, rows, s->x, s->h, &ns, st));
    count_launch(), k_gather_level32<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, s->level, lvl_s);
    if (!have_tight) {
      NB_TRY(E.ensure_tight(L.total));
      count_launch(), k_tight_rows<<<grid_for(ns * 8), NB_THREADS, 0, st>>>(ns, W.rows_s, L.off, L.idx, W.pk0,
                                                                         E.tidx, W.i32a);
    }
    // small active sets: sweeps in batches of 4 between host reads (a sweep costs microseconds,
    // a round trip more), each with its own change flag; a sweep that changes nothing leaves a
    // fixed point, which later sweeps keep, so the batch's last flag says whether the levels
    // have settled.  Large sets: one sweep per read (a sweep costs more than the round trip).
    const int batch = ns < 65536 ? 4 : 1;
    bool settled = false;
    for (int sweep = 0; sweep < 4096; sweep += batch) {
      NB_CUDA(cudaMemsetAsync(W.d_int, 0, sizeof(int) * batch, st));
      for (int b = 0; b < batch; ++b)
        count_launch(), k_limit_sweep_t<<<grid_for(ns * 8), NB_THREADS, 0, st>>>(
            ns, W.rows_s, L.off, E.tidx, W.i32a, (int)prm->max_gap, lvl_s, W.d_int + b);
      NB_CUDA(cudaMemcpyAsync(W.h_int, W.d_int + batch - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
      NB_TRY(pending_enqueue(E, st));
      NB_CUDA(host_sync(st));
      NB_TRY(pending_finish(E, st));
      if (W.h_int[0] == 0) {
        settled = true;
        break;
      }
    }
    if (!settled) return set_host_error(E, "level limiter did not settle");
    count_launch(), k_scatter_rows_level32<<<grid_for(ns), NB_THREADS, 0, st>>>(ns, W.rows_s, L.perm, lvl_s, s->level);
  }
  count_launch(), k_land<<<grid_for(nrows), NB_THREADS, 0, st>>>(nrows, rows, s->tick_n, s->n_stop, s->level, E.d_err);
  W.pend_err = true;  // read with the wake-up count (the kernels below skip their writes on it)
  if (prm->limiter) {
    // levels after _land, sorted; need in sorted order, then back to the caller's order
    count_launch(), k_gather_level32<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, s->level, lvl_s);
    count_launch(), k_fill_i32<<<grid_for(n), NB_THREADS, 0, st>>>(n, -1, need_s);
    count_launch(), k_wake_need_t<<<grid_for(ns * 8), NB_THREADS, 0, st>>>(ns, W.rows_s, L.off, E.tidx, W.i32a,
                                                                     lvl_s, (int)prm->max_gap, need_s);
    count_launch(), k_scatter_level32<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, need_s, W.need);
    // the wake-up count is read with the step's last checks (no round trip of its own)
    if (W.pend_woken) NB_TRY(pending_flush(E, st));
    NB_CUDA(cudaMemsetAsync(W.d_scal_i + 2, 0, sizeof(int64_t), st));
    count_launch(), k_cut_steps<<<grid_for(n), NB_THREADS, 0, st>>>(n, s->tick_n, s->tick, W.need, s->a_hydro,
                                                    s->dudt, s->level, s->n_end, s->p_half,
                                                    s->u_half, (unsigned long long*)(W.d_scal_i + 2), E.d_err,
                                                    heat_of(s));
    W.pend_woken = &s->woken;
  }
  count_launch(), k_open<<<grid_for(nrows), NB_THREADS, 0, st>>>(nrows, rows, s->tick_n, s->tick, s->level, s->x,
                                                 s->p, s->u, s->a_hydro, s->dudt, s->n_beg,
                                                 s->n_end, s->x_beg, s->p_half, s->u_half, E.d_err,
                                                 heat_of(s));
  NB_CUDA(cudaGetLastError());
  return 0;
}

// sim/blocks.py:455-499 (initialise): the caller has filled x, p (from v), u, mass, h, alpha and
// zeroed the rest; every particle is evaluated, gets its level and opens its first step.
int block_initialise(Engine& E, nb_state* s, const nb_params* prm, cudaStream_t st) {
  Workspace& W = E.ws;
  int64_t n = s->n;
  NB_TRY(W.ensure(E, n));
  W.cache.valid = false;
  count_launch(), k_iota<<<grid_for(n), NB_THREADS, 0, st>>>(n, W.rows);
  W.rows_ver += 1;
  launch_v_from_p(n, s->x, s->p, W.v_eval, st);
  ShockStep sk;
  sk.recon_full = 1;
  sk.want_tight = 1;
  NB_TRY(hydro_rows(E, s, prm, n, W.rows, W.v_eval, s->u, st, sk));
  count_launch(), k_fill_i64<<<grid_for(n), NB_THREADS, 0, st>>>(n, 0, s->level);
  NB_TRY(choose_levels_and_open(E, s, prm, n, W.rows, st));
  return pending_flush(E, st);
}

// sim/blocks.py:502-563 (advance): one system step to the earliest step end.  rows_out (optional,
// device, n) receives the active rows; their number is s->last_active.
int block_advance(Engine& E, nb_state* s, const nb_params* prm, int64_t* rows_out,
                  cudaStream_t st, double* v_eval_out, double* u_eval_out) {
  Workspace& W = E.ws;
  int64_t n = s->n;
  NB_TRY(W.ensure(E, n));
  size_t tmp = E.cub_bytes;
  // the earliest step end stays on the device for the flow and the active flags; the host reads
  // it with the active count
  NB_CUDA(cub::DeviceReduce::Min(E.cub_tmp, tmp, s->n_end, W.d_i64 + 1, (int)n, st));
  // flow of every particle from its step start; predictor momenta; active flags
  E.prof.begin(st);
  count_launch(), k_block_flow<<<grid_for(n, 128), 128, 0, st>>>(n, W.d_i64 + 1, s->tick, s->x_beg, s->p_half, s->n_beg,
                                                 s->n_end, s->a_hydro, s->x, W.v_flow, W.v_pred,
                                                 W.v_eval, W.iters, W.m_rows);
  E.prof.end(PROF_FLOW, st, (double)n, 0.0);
  {
    // the flow's worst iteration code, read with the active count just below
    size_t tmp2 = E.cub_bytes;
    NB_CUDA(cub::DeviceReduce::Min(E.cub_tmp, tmp2, W.iters, W.d_scal_i, (int)n, st));
    W.pend_glf = true;
  }
  int64_t nrows = 0, n_next = 0;
  NB_TRY(select_mask(E, n, W.m_rows, W.rows, &nrows, st, &n_next));
  W.rows_ver += 1;
  E.prof.begin(st);
  if (prm->cooling == 3 && nrows > 0) {
    // the network's cooled u_half of the particles whose steps close (exact fallback inside)
    count_launch(), k_gather_cool_rows<<<grid_for(nrows), NB_THREADS, 0, st>>>(
        nrows, W.rows, n_next, s->tick, s->n_beg, s->u_half, s->rho, W.d_a, W.d_b, W.d_hg);
    NB_TRY(mlp_cool(E, nrows, W.d_a, W.d_b, W.d_hg, 0.0, &prm->mlp, W.d_tmp, nullptr, st));
    count_launch(), k_scatter_rows_d<<<grid_for(nrows), NB_THREADS, 0, st>>>(nrows, W.rows, W.d_tmp, W.d_c);
  }
  count_launch(), k_block_cool<<<grid_for(n), NB_THREADS, 0, st>>>(
      n, prm->cooling, n_next, s->tick, s->n_beg, s->n_end, s->x_beg, s->x, s->rho, s->mass,
      s->dudt, prm->cooling_beta, prm->u_floor, brems_of(prm), W.d_c, s->u_half, s->u,
      s->luminosity, W.d_dm, s->heat_visc ? s->heat_cool : nullptr);
  E.prof.end(PROF_COOL, st, (double)nrows, 0.0);
  if (prm->cooling != 0) {
    // radiated energy of the closing steps, added to the ledger at the next read
    size_t tmp2 = E.cub_bytes;
    NB_CUDA(cub::DeviceReduce::Sum(E.cub_tmp, tmp2, W.d_dm, W.d_scal, (int)n, st));
    W.pend_erad = &s->e_radiated;
  }
  s->tick_n = n_next;  // W.v_eval: written by the flow kernel
  ShockStep sk;
  sk.switch_on = 1;
  sk.n_beg = s->n_beg;
  sk.n_end = s->n_end;
  sk.tick = s->tick;
  sk.recon_full = 1;
  sk.want_tight = 1;
  NB_TRY(hydro_rows(E, s, prm, nrows, W.rows, W.v_eval, s->u, st, sk));
  // the evaluation's velocities and (predicted) energies, for a removal that recomputes forces
  const bool split = v_eval_out != nullptr;
  if (split) {
    NB_CUDA(cudaMemcpyAsync(v_eval_out, W.v_eval, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, st));
    NB_CUDA(cudaMemcpyAsync(u_eval_out, s->u, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  }
  count_launch(), k_block_close<<<grid_for(nrows), NB_THREADS, 0, st>>>(nrows, W.rows, s->tick, s->n_beg, s->n_end,
                                                       W.v_flow, s->a_hydro, s->u_half, s->dudt,
                                                       W.v_pred, s->u, heat_of(s));
  NB_CUDA(cudaMemcpyAsync(s->p, W.v_pred, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, st));
  if (!split) {
    E.prof.begin(st);
    NB_TRY(choose_levels_and_open(E, s, prm, nrows, W.rows, st));
    E.prof.end(PROF_LEVELS, st, (double)nrows, 0.0);
  }
  NB_TRY(pending_flush(E, st));
  if (rows_out && nrows > 0)
    NB_CUDA(cudaMemcpyAsync(rows_out, W.rows, sizeof(int64_t) * nrows, cudaMemcpyDeviceToDevice, st));
  s->last_active = nrows;
  s->particle_steps += nrows;
  return 0;
}

// The second half of a split system step (removal with removal_sync, sim/blocks.py:541-549):
// rows (caller order, already renumbered by the caller's removal) get their forces again at the
// evaluation's velocities and energies (the switch not advanced), or not when redo == 0; then
// their levels are chosen and their next steps opened.
int block_finish(Engine& E, nb_state* s, const nb_params* prm, int64_t nrows, const int64_t* rows,
                 int redo, const double* v_eval, const double* u_eval, cudaStream_t st) {
  Workspace& W = E.ws;
  const int64_t n = s->n;
  NB_TRY(W.ensure(E, n));
  if (nrows > 0)
    NB_CUDA(cudaMemcpyAsync(W.rows, rows, sizeof(int64_t) * nrows, cudaMemcpyDeviceToDevice, st));
  W.rows_ver += 1;
  if (redo && nrows > 0) {
    ShockStep sk;
    sk.recon_full = 1;
  sk.want_tight = 1;
    NB_TRY(hydro_rows(E, s, prm, nrows, W.rows, v_eval, u_eval, st, sk));
  }
  E.prof.begin(st);
  NB_TRY(choose_levels_and_open(E, s, prm, nrows, W.rows, st));
  E.prof.end(PROF_LEVELS, st, (double)nrows, 0.0);
  return pending_flush(E, st);
}

// sim/blocks.py:593-627 (_wake_for_removal, its list walk and _cut_to): for every pair (a, b) of
// a row's cached list, a doomed particle's neighbour must end its step by the doomed one's end
// (its level label raised to the doomed one's), in both directions; running steps that end later
// are cut, the opening kick corrected to the new length (Durier Eq. C5).
__global__ void k_doomed_walk(int64_t nrows, const int64_t* __restrict__ rows_s,
                              const int64_t* __restrict__ off, const int32_t* __restrict__ idx,
                              const int32_t* __restrict__ perm, const uint8_t* __restrict__ doomed,
                              const int64_t* __restrict__ n_end, const int64_t* __restrict__ level,
                              unsigned long long* end, long long* label) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= nrows) return;
  const int64_t as = rows_s[q];
  const int64_t a = perm[as];
  const bool da = doomed[a];
  for (int64_t k = off[as]; k < off[as + 1]; ++k) {
    const int64_t bs = idx[k];
    if (bs == as) continue;
    const int64_t b = perm[bs];
    if (da) {
      atomicMin(end + b, (unsigned long long)n_end[a]);
      atomicMax(label + b, (long long)level[a]);
    }
    if (doomed[b]) {
      atomicMin(end + a, (unsigned long long)n_end[b]);
      atomicMax(label + a, (long long)level[b]);
    }
  }
}

__global__ void k_cut_doomed(int64_t n, int64_t tick_n, double tick,
                             const unsigned long long* __restrict__ end,
                             const long long* __restrict__ label, int64_t* __restrict__ n_end,
                             int64_t* __restrict__ level, double* __restrict__ p_half,
                             double* __restrict__ u_half, const double* __restrict__ a,
                             const double* __restrict__ dudt, unsigned long long* woken,
                             HeatBook hb) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t e = (int64_t)end[i];
  if (!(e < n_end[i] && n_end[i] > tick_n)) return;
  level[i] = (int64_t)label[i];
  const double d_len = (double)(e - n_end[i]) * tick;
  for (int c = 0; c < 3; ++c) p_half[3 * i + c] += 0.5 * d_len * a[3 * i + c];
  u_half[i] += 0.5 * d_len * dudt[i];
  book_heat(hb, i, 0.5 * d_len, dudt[i]);
  n_end[i] = e;
  atomicAdd(woken, 1ull);
}

__global__ void k_fill_u64(int64_t n, unsigned long long v, unsigned long long* out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = v;
}

__global__ void k_copy_level(int64_t n, const int64_t* __restrict__ level, long long* out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = (long long)level[i];
}

int block_wake_doomed(Engine& E, nb_state* s, int64_t nrows, const int64_t* rows,
                      const uint8_t* doomed, cudaStream_t st) {
  Workspace& W = E.ws;
  const int64_t n = s->n;
  NB_TRY(W.ensure(E, n));
  if (nrows == 0) return 0;
  if (E.lists.n != n) {
    std::snprintf(E.last_error, sizeof(E.last_error), "no cached lists for the current particles");
    return NB_ERR_INPUT;
  }
  Lists& L = E.lists;
  NB_CUDA(cudaMemcpyAsync(W.rows, rows, sizeof(int64_t) * nrows, cudaMemcpyDeviceToDevice, st));
  W.rows_ver += 1;
  int64_t ns = 0;
  NB_TRY(sorted_rows_and_pack(E, nrows, W.rows, s->x, s->h, &ns, st));
  unsigned long long* end = reinterpret_cast<unsigned long long*>(W.i_tmp);
  long long* label = reinterpret_cast<long long*>(W.i_tmp2);
  count_launch(), k_fill_u64<<<grid_for(n), NB_THREADS, 0, st>>>(n, 0x7fffffffffffffffull, end);
  count_launch(), k_copy_level<<<grid_for(n), NB_THREADS, 0, st>>>(n, s->level, label);
  count_launch(), k_doomed_walk<<<grid_for(ns), NB_THREADS, 0, st>>>(
      ns, W.rows_s, L.off, L.idx, L.perm, doomed, s->n_end, s->level, end, label);
  NB_CUDA(cudaMemsetAsync(W.d_i64, 0, sizeof(int64_t), st));
  count_launch(), k_cut_doomed<<<grid_for(n), NB_THREADS, 0, st>>>(
      n, s->tick_n, s->tick, end, label, s->n_end, s->level, s->p_half, s->u_half, s->a_hydro,
      s->dudt, reinterpret_cast<unsigned long long*>(W.d_i64), heat_of(s));
  NB_CUDA(cudaMemcpyAsync(W.h_i64, W.d_i64, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  NB_CUDA(host_sync(st));
  s->woken += W.h_i64[0];
  return check_device_error(E, st);
}

// run()'s prologue (sim/blocks.py:727-734): re-open the steps opened at this tick that would end
// past n_stop so they land on it
__global__ void k_fresh(int64_t n, int64_t tick_n, int64_t n_stop, const int64_t* __restrict__ n_beg,
                        const int64_t* __restrict__ n_end, uint8_t* __restrict__ m) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) m[i] = n_beg[i] == tick_n && n_end[i] > n_stop;
}

__global__ void k_open_only(int64_t nrows, const int64_t* __restrict__ rows, int64_t tick_n,
                            double tick, const int64_t* __restrict__ level,
                            const double* __restrict__ x, const double* __restrict__ p,
                            const double* __restrict__ u, const double* __restrict__ a,
                            const double* __restrict__ dudt, int64_t* __restrict__ n_beg,
                            int64_t* __restrict__ n_end, double* __restrict__ x_beg,
                            double* __restrict__ p_half, double* __restrict__ u_half,
                            HeatBook hb) {
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= nrows) return;
  int64_t i = rows[q];
  int64_t t = ticks_of(level[i]);
  double length = (double)t * tick;
  n_beg[i] = tick_n;
  n_end[i] = tick_n + t;
  for (int c = 0; c < 3; ++c) {
    x_beg[3 * i + c] = x[3 * i + c];
    p_half[3 * i + c] = p[3 * i + c] + 0.5 * length * a[3 * i + c];
  }
  u_half[i] = u[i] + 0.5 * length * dudt[i];
  // run() re-opens through _open, which books the opening kick again (sim/blocks.py:733, 451)
  book_heat(hb, i, 0.5 * length, dudt[i]);
}

int block_land(Engine& E, nb_state* s, const nb_params* prm, cudaStream_t st) {
  (void)prm;
  Workspace& W = E.ws;
  int64_t n = s->n;
  NB_TRY(W.ensure(E, n));
  count_launch(), k_fresh<<<grid_for(n), NB_THREADS, 0, st>>>(n, s->tick_n, s->n_stop, s->n_beg, s->n_end, W.m_tmp);
  int64_t nf = 0;
  NB_TRY(select_mask(E, n, W.m_tmp, W.rows2, &nf, st));
  if (nf == 0) return 0;
  count_launch(), k_land<<<grid_for(nf), NB_THREADS, 0, st>>>(nf, W.rows2, s->tick_n, s->n_stop, s->level, E.d_err);
  NB_TRY(check_device_error(E, st));
  count_launch(), k_open_only<<<grid_for(nf), NB_THREADS, 0, st>>>(nf, W.rows2, s->tick_n, s->tick, s->level, s->x,
                                                   s->p, s->u, s->a_hydro, s->dudt, s->n_beg,
                                                   s->n_end, s->x_beg, s->p_half, s->u_half,
                                                   heat_of(s));
  NB_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace nbk
