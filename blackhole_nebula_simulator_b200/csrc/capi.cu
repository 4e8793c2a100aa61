// extern "C" entry points of libnebula_b200.so (declared in include/nebula_b200.h).
#include <cub/cub.cuh>

#include <new>

#include "../../include/nebula_b200.h"
#include "common.cuh"
#include "cooling.cuh"
#include "deposit.cuh"
#include "engine.cuh"
#include "eos.cuh"
#include "gravity.cuh"
#include "sph.cuh"
#include "steps.cuh"

namespace nbk {
unsigned long long g_launch_count = 0;
unsigned long long g_sync_count = 0;
}

using nbk::Engine;

namespace {

cudaStream_t S(void* stream) { return (cudaStream_t)stream; }

int begin(nb_ctx* ctx) {
  if (!ctx) return NB_ERR_INPUT;
  Engine& E = ctx->E;
  E.last_error[0] = 0;
  // checks left pending by a call that failed part-way belong to that call
  E.ws.pend_err = E.ws.pend_glf = false;
  E.ws.pend_erad = nullptr;
  E.ws.pend_woken = nullptr;
  NB_CUDA(cudaSetDevice(E.device));
  return 0;
}

__global__ void k_eos_op(int64_t n, const double* __restrict__ rho, const double* __restrict__ u,
                         nbk::EosParams ep, double* __restrict__ P, double* __restrict__ cs,
                         double* __restrict__ T, double* __restrict__ beta, int* err) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double ui = u[i];
  if (!(ui > 0.0)) {
    nbk::set_error(err, nbk::ERR_NONPOSITIVE_U);
    return;
  }
  double p, c, t, b;
  nbk::eos_point(ep, rho[i], ui, p, c, t, b, err);
  P[i] = p;
  cs[i] = c;
  if (T) T[i] = t;
  if (beta) beta[i] = b;
}

__global__ void k_beta(int64_t n, const double* __restrict__ u, const double* __restrict__ uf,
                       const double* __restrict__ dt, const double* __restrict__ tc,
                       double* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = nbk::beta_cool_one(u[i], uf[i], dt[i], tc[i]);
}

__global__ void k_brems(int64_t n, const double* __restrict__ u, const double* __restrict__ rho,
                        const double* __restrict__ dt, double dt_scalar, nbk::BremsParams bp,
                        double* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = nbk::brems_cool_one(u[i], rho[i], dt ? dt[i] : dt_scalar, bp);
}

// sim/neighbours.py:284-323 on caller lists
__global__ void k_tighten(int64_t nrows, const int64_t* __restrict__ rows, const double* __restrict__ pos,
                          const double* __restrict__ h, const int64_t* __restrict__ off,
                          const int64_t* __restrict__ idx, int64_t* __restrict__ counts,
                          const int64_t* __restrict__ out_off, int64_t* __restrict__ out_idx) {
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= nrows) return;
  int64_t i = rows ? rows[q] : q;
  int64_t m = 0;
  for (int64_t e = off[i]; e < off[i + 1]; ++e) {
    int64_t j = idx[e];
    double d2 = nbk::d2_exact(pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                              pos[3 * j + 2] - pos[3 * i + 2]);
    double rr = 2.0 * fmax(h[i], h[j]);
    if (d2 < rr * rr) {
      if (out_off) out_idx[out_off[i] + m] = j;
      m += 1;
    }
  }
  if (!out_off) counts[i] = m;
}

double cnorm_of(int kid) { return kid == 0 ? 1.0 / M_PI : 495.0 / (256.0 * M_PI); }

nbk::BremsParams brems_params(const nb_params* prm) {
  nbk::BremsParams b;
  b.tfac = prm->brems_tfac;
  b.b = prm->brems_b;
  b.kappa = prm->brems_kappa;
  b.u_floor = prm->u_floor;
  b.t_floor = prm->brems_t_floor;
  return b;
}

int check_params(Engine& E, const nb_params* prm) {
  if (!prm) return nbk::set_host_error(E, "params missing"), NB_ERR_INPUT;
  if (prm->kernel_id != 0 && prm->kernel_id != 1) {
    nbk::set_host_error(E, "kernel_id must be 0 (cubic) or 1 (wendland_c4)");
    return NB_ERR_INPUT;
  }
  if (prm->precision != 0 && prm->precision != 1) {
    nbk::set_host_error(E, "precision must be 0 (fp64) or 1 (fp32)");
    return NB_ERR_INPUT;
  }
  return 0;
}

}  // namespace

extern "C" {

int nb_version(void) { return 1; }
int64_t nb_state_size(void) { return (int64_t)sizeof(nb_state); }
int64_t nb_params_size(void) { return (int64_t)sizeof(nb_params); }

int64_t nb_launch_count(void) { return (int64_t)__atomic_load_n(&nbk::g_launch_count, __ATOMIC_RELAXED); }
int64_t nb_sync_count(void) { return (int64_t)__atomic_load_n(&nbk::g_sync_count, __ATOMIC_RELAXED); }

nb_ctx* nb_create(int device) {
  nb_ctx* c = new (std::nothrow) nb_ctx();
  if (!c) return nullptr;
  c->E.device = device;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete c;
    return nullptr;
  }
  if (c->E.ensure_n(1) != 0) {
    c->E.release();
    delete c;
    return nullptr;
  }
  return c;
}

void nb_destroy(nb_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->E.device);
  cudaDeviceSynchronize();
  ctx->E.release();
  delete ctx;
}

const char* nb_last_error(nb_ctx* ctx) { return ctx ? ctx->E.last_error : "no context"; }

int nb_reset_cache(nb_ctx* ctx) {
  NB_TRY(begin(ctx));
  ctx->E.ws.cache.valid = false;
  return 0;
}

int nb_find_neighbours(nb_ctx* ctx, int64_t n, const double* pos, const double* h,
                       int64_t* offset, int64_t* total, void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  if (n < 0 || n > 2000000000) return nbk::set_host_error(E, "n out of range"), NB_ERR_INPUT;
  NB_TRY(nbk::build_lists(E, n, pos, h, S(stream)));
  *total = E.lists.total;
  if (n == 0) {
    NB_CUDA(cudaMemsetAsync(offset, 0, sizeof(int64_t), S(stream)));
    return 0;
  }
  return nbk::export_lists_offsets(E, offset, S(stream));
}

int nb_neighbours_export(nb_ctx* ctx, int64_t* offset, int64_t* index, void* stream) {
  NB_TRY(begin(ctx));
  return nbk::export_lists(ctx->E, offset, index, S(stream));
}

int nb_cell_geometry(nb_ctx* ctx, int64_t n, const double* pos, const double* h, double* lo,
                     double* inv_cell, int64_t* ncell, void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  if (n <= 0 || n > 2000000000) return nbk::set_host_error(E, "n out of range"), NB_ERR_INPUT;
  int r = nbk::cell_geometry(E, n, pos, h, lo, inv_cell, ncell, S(stream));
  return r == -1 ? NB_ERR_INPUT : r;
}

int nb_build_cells(nb_ctx* ctx, int64_t n, const double* pos, const double* lo,
                   const double* inv_cell, const int64_t* ncell, int64_t* start, int64_t* order,
                   void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  if (n < 0 || n > 2000000000) return nbk::set_host_error(E, "n out of range"), NB_ERR_INPUT;
  int r = nbk::build_cells(E, n, pos, lo, inv_cell, ncell, start, order, S(stream));
  return r == -1 ? NB_ERR_INPUT : r;
}

int nb_tighten(nb_ctx* ctx, int64_t n, const double* pos, const double* h, const int64_t* offset,
               const int64_t* index, int64_t nrows, const int64_t* rows, int64_t* counts,
               const int64_t* out_off, int64_t* out_idx, void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  if (!out_off) NB_CUDA(cudaMemsetAsync(counts, 0, sizeof(int64_t) * n, S(stream)));
  if (nrows > 0)
    nbk::count_launch(), k_tighten<<<nbk::grid_for(nrows), NB_THREADS, 0, S(stream)>>>(nrows, rows, pos, h, offset,
                                                                  index, counts, out_off, out_idx);
  NB_CUDA(cudaGetLastError());
  return nbk::check_device_error(E, S(stream));
}

int nb_density(nb_ctx* ctx, int64_t n, const double* pos, const double* mass,
               const double* h_start, const double* h_search, const int64_t* offset,
               const int64_t* index, int64_t nrows, const int64_t* rows, int kernel_id,
               double eta, double tol, double h_max, double* h_out, double* rho, double* omega,
               int64_t* iters, int64_t* flags, void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  if (kernel_id != 0 && kernel_id != 1) return nbk::set_host_error(E, "bad kernel_id"), NB_ERR_INPUT;
  NB_TRY(E.ws.ensure(E, n));
  nbk::pack_pos(n, pos, nullptr, E.ws.pk0, S(stream));
  nbk::DensityParams dp{kernel_id, cnorm_of(kernel_id), eta, tol, h_max};
  nbk::launch_density64<int64_t>(rows ? nrows : n, rows, E.ws.pk0, mass, h_start, h_search,
                                 offset, index, dp, nullptr, h_out, rho, omega, iters, flags,
                                 nullptr, S(stream));
  NB_CUDA(cudaGetLastError());
  return nbk::check_device_error(E, S(stream));
}

static int forces_impl(nb_ctx* ctx, int64_t n, const double* pos, const double* vel,
                       const double* mass, const double* h, const double* rho,
                       const double* omega, const double* pressure, const double* u,
                       const double* c_s, const double* alpha, const double* grad_v,
                       const int64_t* offset, const int64_t* index, int64_t nrows,
                       const int64_t* rows, int kernel_id, double beta, double alpha_u,
                       int cond_signal, int closeness, double eta_crit, double eta_fold,
                       int gate, double* acc, double* dudt, double* vsig_max, double* vheat,
                       double* cheat, void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  if (kernel_id != 0 && kernel_id != 1) return nbk::set_host_error(E, "bad kernel_id"), NB_ERR_INPUT;
  NB_TRY(E.ws.ensure(E, n));
  nbk::Workspace& W = E.ws;
  cudaStream_t st = S(stream);
  nbk::pack_pos(n, pos, nullptr, W.pk0, st);
  nbk::pack_vm(n, vel, mass, W.pk1, st);
  nbk::pack4(n, h, rho, omega, pressure, W.pk2, st);
  nbk::pack4(n, u, c_s, alpha, nullptr, W.pk3, st);
  nbk::ForceParams fp{};
  fp.kid = kernel_id;
  fp.cnorm = cnorm_of(kernel_id);
  fp.use_sph = 1;
  fp.use_visc = alpha != nullptr && c_s != nullptr;
  fp.use_cond = fp.use_visc && u != nullptr;
  fp.cond_signal = cond_signal;
  fp.beta = beta;
  fp.alpha_u = alpha_u;
  fp.use_disc = 0;
  fp.tighten = 0;
  if (grad_v && fp.use_visc) {
    if (gate < 0 || gate > 2) return nbk::set_host_error(E, "bad reconstruction gate"), NB_ERR_INPUT;
    fp.use_recon = 1;
    fp.closeness = closeness;
    fp.eta_crit = eta_crit;
    fp.eta_fold = eta_fold;
    fp.gate = gate;
    fp.gv64 = grad_v;
  }
  nbk::ForceOut fo;
  fo.acc = acc;
  fo.dudt = dudt;
  fo.vsig = vsig_max;
  fo.vheat = vheat;
  fo.cheat = cheat;
  nbk::launch_forces64<int64_t>(rows ? nrows : n, rows, W.pk0, W.pk1, W.pk2, W.pk3, offset, index,
                                fp, nullptr, fo, st);
  NB_CUDA(cudaGetLastError());
  return nbk::check_device_error(E, st);
}

int nb_forces(nb_ctx* ctx, int64_t n, const double* pos, const double* vel, const double* mass,
              const double* h, const double* rho, const double* omega, const double* pressure,
              const double* u, const double* c_s, const double* alpha, const int64_t* offset,
              const int64_t* index, int64_t nrows, const int64_t* rows, int kernel_id,
              double beta, double alpha_u, int cond_signal, double* acc, double* dudt,
              double* vsig_max, double* vheat, double* cheat, void* stream) {
  return forces_impl(ctx, n, pos, vel, mass, h, rho, omega, pressure, u, c_s, alpha, nullptr,
                     offset, index, nrows, rows, kernel_id, beta, alpha_u, cond_signal, 1, 0.0,
                     0.2, 2, acc, dudt, vsig_max, vheat, cheat, stream);
}

int nb_forces_recon(nb_ctx* ctx, int64_t n, const double* pos, const double* vel,
                    const double* mass, const double* h, const double* rho, const double* omega,
                    const double* pressure, const double* u, const double* c_s,
                    const double* alpha, const double* grad_v, const int64_t* offset,
                    const int64_t* index, int64_t nrows, const int64_t* rows, int kernel_id,
                    double beta, double alpha_u, int cond_signal, int closeness, double eta_crit,
                    double eta_fold, int gate, double* acc, double* dudt, double* vsig_max,
                    double* vheat, double* cheat, void* stream) {
  if (!grad_v) {
    NB_TRY(begin(ctx));
    return nbk::set_host_error(ctx->E, "grad_v missing"), NB_ERR_INPUT;
  }
  return forces_impl(ctx, n, pos, vel, mass, h, rho, omega, pressure, u, c_s, alpha, grad_v,
                     offset, index, nrows, rows, kernel_id, beta, alpha_u, cond_signal,
                     closeness, eta_crit, eta_fold, gate, acc, dudt, vsig_max, vheat, cheat,
                     stream);
}

int nb_gradients(nb_ctx* ctx, int64_t n, const double* pos, const double* vel,
                 const double* acc, const double* mass, const double* h, const int64_t* offset,
                 const int64_t* index, int64_t nrows, const int64_t* rows, int kernel_id,
                 double* div_v, double* curl_v, double* ddivv_dt, void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  if (kernel_id != 0 && kernel_id != 1) return nbk::set_host_error(E, "bad kernel_id"), NB_ERR_INPUT;
  if (!acc) return nbk::set_host_error(E, "accelerations missing"), NB_ERR_INPUT;
  NB_TRY(E.ws.ensure(E, std::max<int64_t>(n, 1)));
  nbk::Workspace& W = E.ws;
  cudaStream_t st = S(stream);
  nbk::pack_pos(n, pos, nullptr, W.pk0, st);
  nbk::pack_vm(n, vel, mass, W.pk1, st);
  nbk::pack4(n, h, nullptr, nullptr, nullptr, W.pk2, st);
  nbk::pack_pos(n, acc, nullptr, W.pk3, st);
  nbk::GradParams gp{kernel_id, cnorm_of(kernel_id), 0};
  nbk::GradOut go;
  go.div = div_v;
  go.curl = curl_v;
  go.ddiv = ddivv_dt;
  nbk::launch_gradients<int64_t>(rows ? nrows : n, rows, W.pk0, W.pk1, W.pk2, W.pk3, offset,
                                 index, gp, nullptr, go, st);
  NB_CUDA(cudaGetLastError());
  return nbk::check_device_error(E, st);
}

int nb_velocity_gradients(nb_ctx* ctx, int64_t n, const double* pos, const double* vel,
                          const double* mass, const double* h, const int64_t* offset,
                          const int64_t* index, int64_t nrows, const int64_t* rows,
                          int kernel_id, double* out, void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  if (kernel_id != 0 && kernel_id != 1) return nbk::set_host_error(E, "bad kernel_id"), NB_ERR_INPUT;
  NB_TRY(E.ws.ensure(E, std::max<int64_t>(n, 1)));
  nbk::Workspace& W = E.ws;
  cudaStream_t st = S(stream);
  nbk::pack_pos(n, pos, nullptr, W.pk0, st);
  nbk::pack_vm(n, vel, mass, W.pk1, st);
  nbk::pack4(n, h, nullptr, nullptr, nullptr, W.pk2, st);
  nbk::GradParams gp{kernel_id, cnorm_of(kernel_id), 0};
  nbk::GradOut go;
  go.gv = out;
  nbk::launch_gradients<int64_t>(rows ? nrows : n, rows, W.pk0, W.pk1, W.pk2, nullptr, offset,
                                 index, gp, nullptr, go, st);
  NB_CUDA(cudaGetLastError());
  return nbk::check_device_error(E, st);
}

int nb_disc_forces(nb_ctx* ctx, int64_t n, const double* pos, const double* vel,
                   const double* mass, const double* h, const double* rho, const double* omega,
                   const double* c_s, double alpha_av, const int64_t* offset, const int64_t* index,
                   int64_t nrows, const int64_t* rows, int kernel_id, double* acc, double* dudt,
                   void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  if (kernel_id != 0 && kernel_id != 1) return nbk::set_host_error(E, "bad kernel_id"), NB_ERR_INPUT;
  NB_TRY(E.ws.ensure(E, n));
  nbk::Workspace& W = E.ws;
  cudaStream_t st = S(stream);
  nbk::pack_pos(n, pos, nullptr, W.pk0, st);
  nbk::pack_vm(n, vel, mass, W.pk1, st);
  nbk::pack4(n, h, rho, omega, nullptr, W.pk2, st);
  nbk::pack4(n, nullptr, c_s, nullptr, nullptr, W.pk3, st);
  nbk::ForceParams fp{};
  fp.kid = kernel_id;
  fp.cnorm = cnorm_of(kernel_id);
  fp.use_sph = 0;
  fp.use_disc = 1;
  fp.disc_alpha_av = alpha_av;
  fp.tighten = 0;
  nbk::ForceOut fo;
  fo.dacc = acc;
  fo.ddudt = dudt;
  nbk::launch_forces64<int64_t>(rows ? nrows : n, rows, W.pk0, W.pk1, W.pk2, W.pk3, offset, index,
                                fp, nullptr, fo, st);
  NB_CUDA(cudaGetLastError());
  return nbk::check_device_error(E, st);
}

int nb_glf_step_many(nb_ctx* ctx, int64_t n, const double* x, const double* p, const double* dt,
                     double dt_scalar, double* x1, double* p1, int64_t* iters, void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  NB_TRY(E.ws.ensure(E, n));
  cudaStream_t st = S(stream);
  int64_t* it = iters ? iters : E.ws.iters;
  nbk::launch_glf(n, x, p, dt, dt_scalar, x1, p1, it, st);
  NB_CUDA(cudaGetLastError());
  if (n == 0) return 0;
  size_t tmp = E.cub_bytes;
  NB_CUDA(cub::DeviceReduce::Min(E.cub_tmp, tmp, it, E.ws.d_i64, (int)n, st));
  NB_CUDA(cudaMemcpyAsync(E.ws.h_i64, E.ws.d_i64, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  NB_CUDA(nbk::host_sync(st));
  int64_t w = E.ws.h_i64[0];
  if (w >= 0) return 0;
  nbk::set_host_error(E, w == -1   ? "stage 1 (p_half) did not converge in 10 iterations: time step too large"
                         : w == -2 ? "stage 2 (x1) did not converge in 10 iterations: time step too large"
                                   : "particle inside r = 2.5");
  return w == -1 ? NB_ERR_GLF_P_HALF : w == -2 ? NB_ERR_GLF_X1 : NB_ERR_GLF_RADIUS;
}

int nb_integrate_orbit(nb_ctx* ctx, int norb, const double* state0, double dt_max, double eta,
                       int64_t n_end, int64_t max_records, double* t_out, double* s_out,
                       int64_t* it_out, int64_t* nrec, void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  nbk::launch_integrate_orbit(norb, state0, dt_max, eta, n_end, max_records, t_out, s_out, it_out,
                              nrec, S(stream));
  NB_CUDA(cudaGetLastError());
  NB_CUDA(nbk::host_sync(S(stream)));
  return 0;
}

int nb_gn_v_from_p(nb_ctx* ctx, int64_t n, const double* x, const double* p, double* v, void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  nbk::launch_v_from_p(n, x, p, v, S(stream));
  NB_CUDA(cudaGetLastError());
  return 0;
}

int nb_gn_p_from_v(nb_ctx* ctx, int64_t n, const double* x, const double* v, double* p, void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  nbk::launch_p_from_v(n, x, v, p, S(stream));
  NB_CUDA(cudaGetLastError());
  return 0;
}

int nb_beta_cool(nb_ctx* ctx, int64_t n, const double* u, const double* u_floor, const double* dt,
                 const double* t_cool, double* out, void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  if (n > 0) nbk::count_launch(), k_beta<<<nbk::grid_for(n), NB_THREADS, 0, S(stream)>>>(n, u, u_floor, dt, t_cool, out);
  NB_CUDA(cudaGetLastError());
  return 0;
}

int nb_brems_cool(nb_ctx* ctx, int64_t n, const double* u, const double* rho, const double* dt,
                  double dt_scalar, const nb_params* prm, double* out, void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  if (!prm) return nbk::set_host_error(E, "params missing"), NB_ERR_INPUT;
  if (n > 0)
    nbk::count_launch(), k_brems<<<nbk::grid_for(n), NB_THREADS, 0, S(stream)>>>(n, u, rho, dt, dt_scalar,
                                                            brems_params(prm), out);
  NB_CUDA(cudaGetLastError());
  return 0;
}

int nb_eos(nb_ctx* ctx, int64_t n, const double* rho, const double* u, const nb_params* prm,
           double* P, double* c_s, double* T, double* beta, void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  if (!prm) return nbk::set_host_error(E, "params missing"), NB_ERR_INPUT;
  if (prm->eos < 0 || prm->eos > 2) return nbk::set_host_error(E, "unknown equation of state"), NB_ERR_INPUT;
  NB_TRY(E.ensure_n(std::max<int64_t>(n, 1)));
  if (n > 0)
    nbk::count_launch(), k_eos_op<<<nbk::grid_for(n), NB_THREADS, 0, S(stream)>>>(
        n, rho, u, nbk::eos_of(prm), P, c_s, T, beta, E.d_err);
  NB_CUDA(cudaGetLastError());
  return nbk::check_device_error(E, S(stream));
}

// ---------------------------------------------------------------- grid deposition
// Large inputs are deposited in the spatial order of their centres' cells (sorted keys, gathered
// copies of the particle data): neighbouring threads then add to neighbouring cells.
constexpr int64_t DEPOSIT_SORT_MIN = 1 << 16;

static int deposit_order(Engine& E, int64_t n, int kind, const nbk::LogGeom& g, double x0,
                         double y0, double z0, double dx, int nb, const double*& x,
                         const double*& h, const double*& m, const double*& t, const double*& v,
                         cudaStream_t st) {
  if (n < DEPOSIT_SORT_MIN) return 0;
  NB_TRY(E.ensure_deposit(n));
  nbk::launch_deposit_keys(n, x, kind, g, x0, y0, z0, dx, nb, E.dep_k0, E.dep_i0, st);
  const unsigned long long max_key =
      kind == 0 ? (unsigned long long)(g.nr + 2) * g.nth * g.nph
                : (unsigned long long)(nb + 2) * (nb + 2) * (nb + 2);
  int bits = 1;
  while (bits < 64 && (1ull << bits) <= max_key) ++bits;
  cub::DoubleBuffer<unsigned long long> kb(E.dep_k0, E.dep_k1);
  cub::DoubleBuffer<int32_t> vb(E.dep_i0, E.dep_i1);
  size_t tmp = E.cub_bytes;
  NB_CUDA(cub::DeviceRadixSort::SortPairs(E.cub_tmp, tmp, kb, vb, (int)n, 0, bits, st));
  nbk::launch_deposit_gather(n, vb.Current(), x, h, m, t, v, E.dep_buf, st);
  x = E.dep_buf;
  h = E.dep_buf + 3 * n;
  m = h + n;
  t = m + n;
  v = t + n;
  return 0;
}

static int deposit_finish_host(nbk::Engine& E, double* outside, int64_t* n_trilinear,
                               cudaStream_t st) {
  NB_CUDA(cudaGetLastError());
  NB_CUDA(cudaMemcpyAsync(outside, E.ws.d_scal, sizeof(double), cudaMemcpyDeviceToHost, st));
  NB_CUDA(cudaMemcpyAsync(n_trilinear, E.ws.d_i64, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  NB_CUDA(nbk::host_sync(st));
  return 0;
}

int nb_deposit_log(nb_ctx* ctx, int64_t n, const double* x, const double* h, const double* m,
                   const double* t, const double* v, double r_min, double dlnr, double dth,
                   double dph, int nr, int nth, int nph, int kernel_id, const double* sth,
                   const double* cth, const double* dcth, const double* cph, const double* sph,
                   double* acc, double* outside, int64_t* n_trilinear, void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  if (kernel_id != 0 && kernel_id != 1) return nbk::set_host_error(E, "bad kernel_id"), NB_ERR_INPUT;
  if (nr < 1 || nth < 2 || nph < 1 || !(r_min > 0.0) || !(dlnr > 0.0))
    return nbk::set_host_error(E, "bad log-spherical grid"), NB_ERR_INPUT;
  if (!outside || !n_trilinear) return nbk::set_host_error(E, "outputs missing"), NB_ERR_INPUT;
  cudaStream_t st = S(stream);
  NB_TRY(E.ws.ensure(E, std::max<int64_t>(E.ws.cap, 1024)));
  const int64_t ncell = (int64_t)nr * nth * nph;
  NB_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * nbk::DEP_FIELDS * ncell, st));
  NB_CUDA(cudaMemsetAsync(E.ws.d_scal, 0, sizeof(double), st));
  NB_CUDA(cudaMemsetAsync(E.ws.d_i64, 0, sizeof(int64_t), st));
  nbk::LogGeom g{r_min, dlnr, dth, dph, nr, nth, nph, sth, cth, dcth, cph, sph};
  NB_TRY(deposit_order(E, n, 0, g, 0.0, 0.0, 0.0, 0.0, 0, x, h, m, t, v, st));
  nbk::launch_deposit_log(n, x, h, m, t, v, g, kernel_id, acc, E.ws.d_scal,
                          (unsigned long long*)E.ws.d_i64, st);
  return deposit_finish_host(E, outside, n_trilinear, st);
}

int nb_deposit_box(nb_ctx* ctx, int64_t n, const double* x, const double* h, const double* m,
                   const double* t, const double* v, double x0, double y0, double z0, double dx,
                   int nb, int kernel_id, double* acc, double* outside, int64_t* n_trilinear,
                   void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  if (kernel_id != 0 && kernel_id != 1) return nbk::set_host_error(E, "bad kernel_id"), NB_ERR_INPUT;
  if (nb < 1 || !(dx > 0.0)) return nbk::set_host_error(E, "bad box"), NB_ERR_INPUT;
  if (!outside || !n_trilinear) return nbk::set_host_error(E, "outputs missing"), NB_ERR_INPUT;
  cudaStream_t st = S(stream);
  NB_TRY(E.ws.ensure(E, std::max<int64_t>(E.ws.cap, 1024)));
  const int64_t ncell = (int64_t)nb * nb * nb;
  NB_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * nbk::DEP_FIELDS * ncell, st));
  NB_CUDA(cudaMemsetAsync(E.ws.d_scal, 0, sizeof(double), st));
  NB_CUDA(cudaMemsetAsync(E.ws.d_i64, 0, sizeof(int64_t), st));
  const nbk::LogGeom none{};
  NB_TRY(deposit_order(E, n, 1, none, x0, y0, z0, dx, nb, x, h, m, t, v, st));
  nbk::launch_deposit_box(n, x, h, m, t, v, x0, y0, z0, dx, nb, kernel_id, acc, E.ws.d_scal,
                          (unsigned long long*)E.ws.d_i64, st);
  return deposit_finish_host(E, outside, n_trilinear, st);
}

int nb_grid_finish(nb_ctx* ctx, int64_t ncell, const double* acc, const double* vol,
                   int64_t cells_per_volume, double* mass, float* rho, float* t_mass,
                   float* t_em, float* vel, void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  if (cells_per_volume < 1) return nbk::set_host_error(E, "bad volume layout"), NB_ERR_INPUT;
  nbk::launch_grid_finish(ncell, acc, vol, cells_per_volume, mass, rho, t_mass, t_em, vel,
                          S(stream));
  NB_CUDA(cudaGetLastError());
  return 0;
}

int nb_refine_sums(nb_ctx* ctx, const double* acc_c, const double* vol_c, int nrc, int nthc,
                   int nphc, const double* vol_f, int nr, int nth, int nph, int cr, int ct,
                   int cp, double* out, void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  if (cr < 1 || ct < 1 || cp < 1 || nrc < 1 || nthc < 1 || nphc < 1 || nrc * cr != nr ||
      nthc * ct != nth || nphc * cp != nph)
    return nbk::set_host_error(E, "coarse grid does not divide the fine grid"), NB_ERR_INPUT;
  cudaStream_t st = S(stream);
  NB_TRY(E.ws.ensure(E, std::max<int64_t>(E.ws.cap, 1024)));
  NB_CUDA(cudaMemsetAsync(E.ws.d_scal, 0, 2 * sizeof(double), st));
  nbk::launch_refine_sums(acc_c, vol_c, nrc, nthc, nphc, vol_f, nr, nth, nph, cr, ct, cp, out,
                          E.ws.d_scal, st);
  NB_CUDA(cudaGetLastError());
  return 0;
}

int nb_ledger(nb_ctx* ctx, int64_t n, const double* x, const double* p, const double* u,
              const double* mass, double* out, void* stream) {
  NB_TRY(begin(ctx));
  Engine& E = ctx->E;
  cudaStream_t st = S(stream);
  NB_TRY(E.ws.ensure(E, std::max<int64_t>(n, 1)));
  nbk::launch_ledger(n, x, p, u, mass, E.red, E.ws.d_tmp, st);
  NB_CUDA(cudaMemcpyAsync(E.ws.h_dbl, E.ws.d_tmp, sizeof(double) * 9, cudaMemcpyDeviceToHost, st));
  NB_CUDA(nbk::host_sync(st));
  for (int t = 0; t < 9; ++t) out[t] = E.ws.h_dbl[t];
  return 0;
}

int nb_coupled_initialise(nb_ctx* ctx, nb_state* st, const nb_params* prm, void* stream) {
  NB_TRY(begin(ctx));
  NB_TRY(check_params(ctx->E, prm));
  return nbk::coupled_initialise(ctx->E, st, prm, S(stream));
}

int nb_coupled_step(nb_ctx* ctx, nb_state* st, const nb_params* prm, double dt, void* stream) {
  NB_TRY(begin(ctx));
  NB_TRY(check_params(ctx->E, prm));
  return nbk::coupled_step(ctx->E, st, prm, dt, S(stream));
}

int nb_coupled_stable_dt(nb_ctx* ctx, nb_state* st, const nb_params* prm, double* dt_out,
                         void* stream) {
  NB_TRY(begin(ctx));
  NB_TRY(check_params(ctx->E, prm));
  return nbk::coupled_stable_dt(ctx->E, st, prm, dt_out, S(stream));
}

int nb_block_initialise(nb_ctx* ctx, nb_state* st, const nb_params* prm, void* stream) {
  NB_TRY(begin(ctx));
  NB_TRY(check_params(ctx->E, prm));
  return nbk::block_initialise(ctx->E, st, prm, S(stream));
}

int nb_block_advance(nb_ctx* ctx, nb_state* st, const nb_params* prm, int64_t* rows_out,
                     void* stream) {
  NB_TRY(begin(ctx));
  NB_TRY(check_params(ctx->E, prm));
  return nbk::block_advance(ctx->E, st, prm, rows_out, S(stream));
}

int nb_block_advance_split(nb_ctx* ctx, nb_state* st, const nb_params* prm, int64_t* rows_out,
                           double* v_eval_out, double* u_eval_out, void* stream) {
  NB_TRY(begin(ctx));
  NB_TRY(check_params(ctx->E, prm));
  if (!v_eval_out || !u_eval_out)
    return nbk::set_host_error(ctx->E, "evaluation buffers missing"), NB_ERR_INPUT;
  return nbk::block_advance(ctx->E, st, prm, rows_out, S(stream), v_eval_out, u_eval_out);
}

int nb_block_finish(nb_ctx* ctx, nb_state* st, const nb_params* prm, int64_t nrows,
                    const int64_t* rows, int redo, const double* v_eval, const double* u_eval,
                    void* stream) {
  NB_TRY(begin(ctx));
  NB_TRY(check_params(ctx->E, prm));
  if (redo && (!v_eval || !u_eval))
    return nbk::set_host_error(ctx->E, "evaluation buffers missing"), NB_ERR_INPUT;
  return nbk::block_finish(ctx->E, st, prm, nrows, rows, redo, v_eval, u_eval, S(stream));
}

int nb_block_wake_doomed(nb_ctx* ctx, nb_state* st, int64_t nrows, const int64_t* rows,
                         const uint8_t* doomed, void* stream) {
  NB_TRY(begin(ctx));
  return nbk::block_wake_doomed(ctx->E, st, nrows, rows, doomed, S(stream));
}

int nb_block_land(nb_ctx* ctx, nb_state* st, const nb_params* prm, void* stream) {
  NB_TRY(begin(ctx));
  NB_TRY(check_params(ctx->E, prm));
  return nbk::block_land(ctx->E, st, prm, S(stream));
}

int nb_profile(nb_ctx* ctx, int on) {
  NB_TRY(begin(ctx));
  nbk::Prof& P = ctx->E.prof;
  nbk::Engine& E = ctx->E;
  P.flush();
  P.on = on != 0;
  P.open = false;
  for (int c = 0; c < nbk::PROF_NCAT; ++c) {
    P.ms[c] = 0;
    P.launches[c] = 0;
    P.units[c] = 0;
    P.pairs[c] = 0;
  }
  if (P.on) {
    if (P.ensure() != 0) return nbk::set_host_error(E, "profile events could not be created");
    NB_CUDA(cudaMemset(P.d_pairs, 0, sizeof(unsigned long long) * nbk::PROF_NCAT));
  }
  return 0;
}

int nb_profile_read(nb_ctx* ctx, double* out) {
  NB_TRY(begin(ctx));
  nbk::Prof& P = ctx->E.prof;
  nbk::Engine& E = ctx->E;
  P.flush();
  unsigned long long dev[nbk::PROF_NCAT] = {0};
  if (P.d_pairs) NB_CUDA(cudaMemcpy(dev, P.d_pairs, sizeof(dev), cudaMemcpyDeviceToHost));
  for (int c = 0; c < nbk::PROF_NCAT; ++c) {
    out[4 * c + 3] = P.pairs[c] + (double)dev[c];
    out[4 * c + 0] = P.ms[c];
    out[4 * c + 1] = (double)P.launches[c];
    out[4 * c + 2] = P.units[c];
  }
  return 0;
}

}  // extern "C"
