/*
 * nebula_b200.h — C ABI of libnebula_b200.so, the sm_100a SPH step of Blackhole-Nebula-Simulator.
 *
 * Every array argument is a DEVICE pointer (e.g. torch.Tensor.data_ptr() of a CUDA tensor) in
 * the caller's particle order, C-contiguous: positions, velocities and momenta are (n, 3)
 * float64, per-particle scalars (n,) float64, neighbour lists CSR int64 (offset n+1, index
 * total).  "rows" selects particles (int64 indices) whose results are written in rows order,
 * exactly like the reference's ``rows`` argument.  `stream` is a cudaStream_t (NULL: the legacy
 * default stream).  Nothing calls exit() or traps on the device.
 *
 * Return value: 0 = success; NB_ERR_* > 0 = a domain error that maps to one of the reference's
 * exceptions (message in nb_last_error); < 0 = a CUDA or host error (message in nb_last_error).
 */
#ifndef NEBULA_B200_H
#define NEBULA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* domain errors (reference exception in brackets) */
#define NB_ERR_GLF_P_HALF 11      /* [GLFConvergenceError] stage 1 did not converge */
#define NB_ERR_GLF_X1 12          /* [GLFConvergenceError] stage 2 did not converge */
#define NB_ERR_GLF_RADIUS 13      /* [GLFConvergenceError] particle inside r = 2.5 */
#define NB_ERR_SEARCH 20          /* [RuntimeError] smoothing lengths kept outgrowing the search */
#define NB_ERR_TOUCHED 21         /* [RuntimeError] neighbour set of the active particles did not settle */
#define NB_ERR_NONPOSITIVE_U 22   /* [FloatingPointError] non-positive internal energy */
#define NB_ERR_LEVEL 23           /* [ValueError] a level beyond K_MAX */
#define NB_ERR_DT 24              /* [ValueError] time steps must be positive */
#define NB_ERR_UNSUPPORTED 25     /* [NotImplementedError] option outside the CUDA path */
#define NB_ERR_INPUT 26           /* [ValueError] bad argument */
#define NB_ERR_EOS_RANGE 27       /* [ValueError] u outside the gas + radiation EOS bracket [1, 1e13] K */
#define NB_ERR_EOS 28             /* [RuntimeError] gas + radiation temperature did not converge */

#if defined(__GNUC__)
#define NB_API __attribute__((visibility("default")))
#else
#define NB_API
#endif

typedef struct nb_ctx nb_ctx;

/* The learned cooling step (no reference counterpart): the bremsstrahlung law, the unit
 * conversions of the network's inputs and its training hull (log10 rho [g/cm^3], log10 T [K],
 * log10 dt [s]), the tolerance of the a-posteriori check (a fraction of u) and the stride of
 * the exact-integrator comparison ("judge", 0: off). */
typedef struct nb_mlp_params {
  double tfac, b, kappa, u_floor, t_floor;
  double rho_unit_cgs, t_unit_s;
  double lrho_lo, lrho_hi, lt_lo, lt_hi, ldt_lo, ldt_hi;
  double check_tol;
  int judge;
} nb_mlp_params;

/* Physics and numerics of one run: the fields of the reference's HydroConfig, CoupledConfig and
 * BlockConfig that the CUDA path implements (sim/hydro.py:53-98, sim/coupled.py:62-75,
 * sim/blocks.py:83-100). */
typedef struct nb_params {
  int kernel_id;          /* 0 cubic spline, 1 Wendland C4 */
  double cnorm, eta, tol, h_max, skin;
  double gamma;
  int viscosity, conductivity, cond_signal;
  double alpha_const, beta, alpha_u;
  double disc_alpha_av;   /* > 0: disc viscosity (Option B) */
  double courant, c_force, eta_orb;
  int precision;          /* 0: FP64 pair arithmetic, 1: FP32 (cell offsets, Kahan sums) */
  int cooling;            /* 0 none, 1 beta-cooling, 2 bremsstrahlung (exact), 3 brems via MLP */
  double cooling_beta;    /* beta of beta-cooling */
  double u_floor;         /* code u at the floor temperature */
  double brems_tfac, brems_b, brems_kappa, brems_t_floor;
  double dt_max;          /* block steps: level-0 step */
  int limiter, max_gap;
  nb_mlp_params mlp;      /* cooling 3: the network (weights set by nb_mlp_train / nb_mlp_weights) */
  int eos;                /* 0 ideal gas (gamma), 1 gas + radiation, 2 radiation limit (P = rho u / 3) */
  double eos_rho_si;      /* gas + radiation: kg/m^3 per code density (the run's GasUnits) */
  double eos_u_si;        /* J/kg per code specific energy (c^2) */
  double eos_a1;          /* 3 k / (2 mu m_p) [J/(kg K)] */
  double eos_a_rad;       /* radiation constant [J m^-3 K^-4] */
  int visc_switch;        /* Cullen-Dehnen switch: alpha of the rows advanced at each step */
  int recon;              /* velocity reconstruction in the viscosity */
  int recon_closeness;    /* its closeness factor (Frontiere et al. 2017 Eq. 51) */
  int recon_gate;         /* 0 both jumps approaching, 1 reconstructed jump only, 2 min-mod */
  double recon_eta_crit;  /* 1 / hfact */
  double recon_eta_fold;
} nb_params;

/* Device state of a run (the fields of the reference's GasState / BlockState that the step
 * reads or writes).  Block-step fields may be NULL for the shared step. */
typedef struct nb_state {
  int64_t n;
  double *x, *p, *u, *mass, *h, *alpha, *a_hydro, *dudt, *rho, *omega, *c_s, *vsig_max, *nu;
  double *visc_heating;
  int64_t *level, *n_beg, *n_end, *level_offset;
  double *x_beg, *p_half, *u_half, *luminosity;
  int64_t tick_n, n_stop;
  double t0, tick;
  double e_radiated;
  int64_t particle_steps, woken, last_active, pairs;
  int64_t builds, reuses;
  /* block steps: the parts of du/dt at each particle's last force evaluation (viscous heating is
   * visc_heating above) and the heat budget since the start, what each part of du/dt and the
   * cooling added to u (sim/blocks.py:142-154, 434-440).  heat_visc NULL: no budget kept;
   * cond_heating / disk_heating may be NULL without conductivity / disc viscosity. */
  double *cond_heating, *disk_heating;
  double *heat_visc, *heat_cond, *heat_disk, *heat_pdv, *heat_cool;
} nb_state;

/* ---------------------------------------------------------------- context */
NB_API nb_ctx* nb_create(int device);
NB_API void nb_destroy(nb_ctx* ctx);
NB_API const char* nb_last_error(nb_ctx* ctx);
NB_API int nb_version(void);
/* sizeof(nb_state) and sizeof(nb_params) of this build (bindings check their mirrors). */
NB_API int64_t nb_state_size(void);
NB_API int64_t nb_params_size(void);
/* Number of this library's own kernels launched so far by this process (all contexts). */
NB_API int64_t nb_launch_count(void);
/* Number of host waits on a stream this library has made so far (all contexts). */
NB_API int64_t nb_sync_count(void);

/* ---------------------------------------------------------------- operators
 * One-for-one replacements of the reference's inner functions (sim/neighbours.py, sim/sph.py,
 * sim/integrator.py, sim/fastphys.py, physics/cooling.py). */

/* find_neighbours_numba (sim/neighbours.py:240-281): builds the symmetric lists
 * {j : r_ij < 2 max(h_i, h_j)} (no periodic box) and writes offset (n+1) and *total (host).
 * nb_neighbours_export then writes index (total) with every row sorted ascending. */
NB_API int nb_find_neighbours(nb_ctx* ctx, int64_t n, const double* pos, const double* h, int64_t* offset,
                       int64_t* total, void* stream);
NB_API int nb_neighbours_export(nb_ctx* ctx, int64_t* offset, int64_t* index, void* stream);

/* The reference's cell grid.  nb_cell_geometry: find_neighbours_numba's grid geometry without
 * a periodic box (sim/neighbours.py:250-265): lo (3) = the smallest coordinates, cell = max(
 * median(h), max(span) / 160, 1e-300), ncell (3) = floor(span / cell) + 1, inv_cell (3) = 1 /
 * cell, written to host memory (the call synchronises its stream).  nb_build_cells: _build_grid
 * (sim/neighbours.py:106-126): cell (cx * ny + cy) * nz + cz of each particle with
 * k = floor((x - lo) * inv_cell) clamped to [0, ncell - 1], rounded as the reference's, and the
 * stable counting sort: start (ncx * ncy * ncz + 1) and order (n, ascending index within a
 * cell); lo, inv_cell and ncell are host arrays. */
NB_API int nb_cell_geometry(nb_ctx* ctx, int64_t n, const double* pos, const double* h,
                            double* lo, double* inv_cell, int64_t* ncell, void* stream);
NB_API int nb_build_cells(nb_ctx* ctx, int64_t n, const double* pos, const double* lo,
                          const double* inv_cell, const int64_t* ncell, int64_t* start,
                          int64_t* order, void* stream);

/* tighten (sim/neighbours.py:284-323), two calls: out_off == NULL writes counts (n) of the kept
 * entries per row; then with out_off (n+1, the caller's prefix sum) writes out_idx. */
NB_API int nb_tighten(nb_ctx* ctx, int64_t n, const double* pos, const double* h, const int64_t* offset,
               const int64_t* index, int64_t nrows, const int64_t* rows, int64_t* counts,
               const int64_t* out_off, int64_t* out_idx, void* stream);

/* density_numba (sim/sph.py:300-326): results (nrows) in rows order (rows NULL: all n). */
NB_API int nb_density(nb_ctx* ctx, int64_t n, const double* pos, const double* mass,
               const double* h_start, const double* h_search, const int64_t* offset,
               const int64_t* index, int64_t nrows, const int64_t* rows, int kernel_id,
               double eta, double tol, double h_max, double* h_out, double* rho, double* omega,
               int64_t* iters, int64_t* flags, void* stream);

/* forces_numba without reconstruction (sim/sph.py:655-690).  u NULL: no conductivity; alpha or
 * c_s NULL: no viscosity.  vheat / cheat may be NULL. */
NB_API int nb_forces(nb_ctx* ctx, int64_t n, const double* pos, const double* vel, const double* mass,
              const double* h, const double* rho, const double* omega, const double* pressure,
              const double* u, const double* c_s, const double* alpha, const int64_t* offset,
              const int64_t* index, int64_t nrows, const int64_t* rows, int kernel_id,
              double beta, double alpha_u, int cond_signal, double* acc, double* dudt,
              double* vsig_max, double* vheat, double* cheat, void* stream);

/* forces_numba with velocity reconstruction (sim/sph.py:655-690 with shock.reconstruction,
 * the branch at sim/sph.py:568-609): nb_forces plus grad_v (n, 3, 3) of every particle, the
 * closeness factor switch, eta_crit, eta_fold and the gate (ShockCapturing.recon_gate). */
NB_API int nb_forces_recon(nb_ctx* ctx, int64_t n, const double* pos, const double* vel,
                    const double* mass, const double* h, const double* rho, const double* omega,
                    const double* pressure, const double* u, const double* c_s,
                    const double* alpha, const double* grad_v, const int64_t* offset,
                    const int64_t* index, int64_t nrows, const int64_t* rows, int kernel_id,
                    double beta, double alpha_u, int cond_signal, int closeness, double eta_crit,
                    double eta_fold, int gate, double* acc, double* dudt, double* vsig_max,
                    double* vheat, double* cheat, void* stream);

/* gradients_numba (sim/sph.py:883-902): corrected div v, |curl v| and d(div v)/dt of `rows`
 * (all when NULL; results in rows order) from velocities and accelerations over the given
 * lists. */
NB_API int nb_gradients(nb_ctx* ctx, int64_t n, const double* pos, const double* vel,
                 const double* acc, const double* mass, const double* h, const int64_t* offset,
                 const int64_t* index, int64_t nrows, const int64_t* rows, int kernel_id,
                 double* div_v, double* curl_v, double* ddivv_dt, void* stream);

/* velocity_gradients_numba (sim/sph.py:827-846): out (n, 3, 3) = dv^i/dx^j at the particles of
 * `rows` (all when NULL); the other entries of out are left as they are. */
NB_API int nb_velocity_gradients(nb_ctx* ctx, int64_t n, const double* pos, const double* vel,
                          const double* mass, const double* h, const int64_t* offset,
                          const int64_t* index, int64_t nrows, const int64_t* rows,
                          int kernel_id, double* out, void* stream);

/* disc_forces_numba (sim/sph.py:1120-1137). */
NB_API int nb_disc_forces(nb_ctx* ctx, int64_t n, const double* pos, const double* vel,
                   const double* mass, const double* h, const double* rho, const double* omega,
                   const double* c_s, double alpha_av, const int64_t* offset, const int64_t* index,
                   int64_t nrows, const int64_t* rows, int kernel_id, double* acc, double* dudt,
                   void* stream);

/* glf_step_many (sim/integrator.py:188-198): dt (n) or, when dt is NULL, dt_scalar for all.
 * iters: iterations, or -1 / -2 / -3 for a failed particle (status NB_ERR_GLF_*). */
NB_API int nb_glf_step_many(nb_ctx* ctx, int64_t n, const double* x, const double* p, const double* dt,
                     double dt_scalar, double* x1, double* p1, int64_t* iters, void* stream);

/* integrate_orbit (sim/integrator.py:220-298): norb test-particle orbits (state0: norb x 6 = x, p)
 * on the tick timeline (tick = dt_max / 2^40) to tick n_end, one GLF step per record; eta > 0:
 * quantized adaptive steps eta r^1.5, else fixed dt_max.  Outputs per orbit o at offset
 * o * max_records: t_out, s_out (x 6), it_out; nrec[o] = records or a negative code (-1/-2/-3 GLF
 * failures, -4 level beyond K_MAX, -5 max_records too small). */
NB_API int nb_integrate_orbit(nb_ctx* ctx, int norb, const double* state0, double dt_max, double eta,
                              int64_t n_end, int64_t max_records, double* t_out, double* s_out,
                              int64_t* it_out, int64_t* nrec, void* stream);

/* gn_v_from_p_nb (sim/fastphys.py:35-42) and gn_p_from_v (physics/gravity.py:66-77). */
NB_API int nb_gn_v_from_p(nb_ctx* ctx, int64_t n, const double* x, const double* p, double* v, void* stream);
NB_API int nb_gn_p_from_v(nb_ctx* ctx, int64_t n, const double* x, const double* v, double* p, void* stream);

/* beta_cool (physics/cooling.py:33-40), elementwise. */
NB_API int nb_beta_cool(nb_ctx* ctx, int64_t n, const double* u, const double* u_floor, const double* dt,
                 const double* t_cool, double* out, void* stream);

/* Exact bremsstrahlung cooling at fixed rho over dt (no reference counterpart; the law is
 * documented in cooling.cuh).  dt NULL: dt_scalar for all. */
NB_API int nb_brems_cool(nb_ctx* ctx, int64_t n, const double* u, const double* rho, const double* dt,
                  double dt_scalar, const nb_params* prm, double* out, void* stream);

/* eos_state (sim/hydro.py:121-139) with prm->eos: pressure and sound speed (code units) of n
 * particles; for gas + radiation (gasrad_state_nb, sim/fastphys.py:45-102) also T [K] and
 * beta_gas (T and beta may be NULL; other equations of state write 0 and 1). */
NB_API int nb_eos(nb_ctx* ctx, int64_t n, const double* rho, const double* u, const nb_params* prm,
                  double* P, double* c_s, double* T, double* beta, void* stream);

/* Ledger sums (sim/coupled.py:261-270) into out[9] on the host: sum m (H + u), sum m |H|,
 * angular momentum (3), momentum (3), mass. */
NB_API int nb_ledger(nb_ctx* ctx, int64_t n, const double* x, const double* p, const double* u,
              const double* mass, double* out, void* stream);

/* ---------------------------------------------------------------- learned cooling
 * MLP 3 -> 64 -> 64 -> 64 (SiLU) -> 1 predicting the fraction of u - u_floor one step removes.
 * Weights: a flat float32 vector of NB_MLP_NPARAM (W1 64x3, b1, W2 64x64, b2, W3 64x64, b3,
 * W4 1x64, b4), held per device by the library. */
#define NB_MLP_NPARAM 8641
/* n training samples, log-uniform over the hull, labelled by the exact integrator: X (n, 3)
 * scaled inputs, Y (n) labels, U (n, 3) code-unit (u, rho, dt) or NULL. */
NB_API int nb_mlp_data(nb_ctx* ctx, int64_t n, uint64_t seed, const nb_mlp_params* mp, float* X,
                       float* Y, double* U, void* stream);
/* Mean squared error of one batch and its gradient (device g, NB_MLP_NPARAM) at weights w,
 * with the forward pass rounding the weights to BF16 as inference does. */
NB_API int nb_mlp_grad(nb_ctx* ctx, int64_t batch, const float* X, const float* Y, const float* w,
                       float* g, double* loss, void* stream);
/* Train the device's network from scratch: n_samples fresh samples, Adam, cosine-decayed
 * learning rate; loss_hist (host, epochs) gets each epoch's last-batch loss (may be NULL). */
NB_API int nb_mlp_train(nb_ctx* ctx, const nb_mlp_params* mp, int64_t n_samples, int64_t batch,
                        int epochs, double lr, uint64_t seed, float* loss_hist, void* stream);
/* Copy the device's weights out (w_out, device) and/or replace them (w_in, device). */
NB_API int nb_mlp_weights(nb_ctx* ctx, float* w_out, const float* w_in, void* stream);
/* Cooling of n particles by the network with exact fallback (dt NULL: dt_scalar for all);
 * mode (optional, int8): 0 exact/no cooling, 1 network, 2 fallback. */
NB_API int nb_mlp_cool(nb_ctx* ctx, int64_t n, const double* u, const double* rho, const double* dt,
                       double dt_scalar, const nb_mlp_params* mp, double* u_out, int8_t* mode,
                       void* stream);
/* out[5] = max and rms of |du_net - du_exact| / u over the judged samples, judged count,
 * network results, fallbacks (accumulated since the last reset; reset != 0 clears). */
NB_API int nb_mlp_stats(nb_ctx* ctx, double* out, int reset);

/* ---------------------------------------------------------------- step runtime
 * The reference's step entry points (sim/coupled.py:198-258, sim/blocks.py:455-563) on device
 * state.  The list cache (and its reuse test, sim/sph.py:62-147) lives in the context. */
NB_API int nb_coupled_initialise(nb_ctx* ctx, nb_state* st, const nb_params* prm, void* stream);
NB_API int nb_coupled_step(nb_ctx* ctx, nb_state* st, const nb_params* prm, double dt, void* stream);
NB_API int nb_coupled_stable_dt(nb_ctx* ctx, nb_state* st, const nb_params* prm, double* dt_out,
                         void* stream);
NB_API int nb_block_initialise(nb_ctx* ctx, nb_state* st, const nb_params* prm, void* stream);
NB_API int nb_block_advance(nb_ctx* ctx, nb_state* st, const nb_params* prm, int64_t* rows_out,
                     void* stream);
/* A system step split for removal with removal_sync (sim/blocks.py:502-563, 566-627):
 * nb_block_advance_split does the step up to and including the closing kicks and leaves the
 * evaluation's velocities (n x 3) and predicted energies (n) in v_eval_out / u_eval_out; the
 * caller removes particles (renumbering rows and state); nb_block_finish recomputes the forces
 * of rows at v_eval / u_eval when redo != 0 (the switch not advanced), then chooses their levels
 * and opens their next steps.  nb_block_wake_doomed (sim/blocks.py:593-627): with doomed (n,
 * caller order) the particles whose next step ends beyond a removal radius, cuts the running
 * steps of their list neighbours among and around rows to end with theirs (st->woken counts
 * them). */
NB_API int nb_block_advance_split(nb_ctx* ctx, nb_state* st, const nb_params* prm,
                           int64_t* rows_out, double* v_eval_out, double* u_eval_out,
                           void* stream);
NB_API int nb_block_finish(nb_ctx* ctx, nb_state* st, const nb_params* prm, int64_t nrows,
                    const int64_t* rows, int redo, const double* v_eval, const double* u_eval,
                    void* stream);
NB_API int nb_block_wake_doomed(nb_ctx* ctx, nb_state* st, int64_t nrows, const int64_t* rows,
                         const uint8_t* doomed, void* stream);
/* Re-open the steps just opened so they land on n_stop (sim/blocks.py:722-734, run's prologue). */
NB_API int nb_block_land(nb_ctx* ctx, nb_state* st, const nb_params* prm, void* stream);

/* ---------------------------------------------------------------- allocation-free variant
 * No counterpart in the reference.  nb_density_noalloc is nb_density for callers that cannot
 * allocate device memory (a host framework that owns the device allocator, or a run that must
 * not allocate once planned): it takes no context and allocates nothing.  Its scratch (the packed
 * positions) is a fixed device array of NB_NOALLOC_MAX_N particles, 8 MiB, held by every GPU
 * that loads the library until exit; larger n returns NB_ERR_INPUT.  The first call on a device
 * looks up that array's device address (cudaGetSymbolAddress), so make it before any stream
 * capture.  All calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller.  offset (n + 1) and index must describe lists over [0, n), and with
 * rows given, 0 <= nrows <= n and every rows[k] in [0, n): the call does not read them back to
 * check, and an index at or beyond n would read entries of the shared array left by an earlier
 * call (stale positions) instead of failing.  nrows beyond n or negative returns NB_ERR_INPUT.
 * Messages of failed calls: nb_noalloc_last_error (per host thread). */
#define NB_NOALLOC_MAX_N 262144
NB_API int nb_density_noalloc(int64_t n, const double* pos, const double* mass,
                              const double* h_start, const double* h_search,
                              const int64_t* offset, const int64_t* index, int64_t nrows,
                              const int64_t* rows, int kernel_id, double eta, double tol,
                              double h_max, double* h_out, double* rho, double* omega,
                              int64_t* iters, int64_t* flags, void* stream);
NB_API const char* nb_noalloc_last_error(void);

/* ---------------------------------------------------------------- grid deposition
 * Particle -> render grid deposition (render/gasgrid.py:316-597): fields (m, m T, m T^4, m v)
 * of each particle to the cells whose centres lie inside its support, weights f(q) V_c
 * normalised to 1, or trilinear weights when fewer than 8 centres are inside; acc (cells x 6,
 * cell index (i * nth + j) * nph + k, zeroed by the call) receives the sums, *outside the mass
 * beyond the grid and *n_trilinear the fallback count (the call synchronises its stream).
 * nb_deposit_log: the log-spherical grid (render/gasgrid.py:52-83) with its theta / phi
 * cell-centre tables sin th_j, cos th_j, cos th_j1 - cos th_j2, cos ph_k, sin ph_k
 * (render/gasgrid.py:688-692); kernel_id 0 cubic, 1 Wendland C4. */
NB_API int nb_deposit_log(nb_ctx* ctx, int64_t n, const double* x, const double* h,
                   const double* m, const double* t, const double* v, double r_min, double dlnr,
                   double dth, double dph, int nr, int nth, int nph, int kernel_id,
                   const double* sth, const double* cth, const double* dcth, const double* cph,
                   const double* sph, double* acc, double* outside, int64_t* n_trilinear,
                   void* stream);
/* nb_deposit_box: a Cartesian box of nb^3 cells of edge dx from the corner (x0, y0, z0)
 * (render/gasgrid.py:534-597, 811-825). */
NB_API int nb_deposit_box(nb_ctx* ctx, int64_t n, const double* x, const double* h,
                   const double* m, const double* t, const double* v, double x0, double y0,
                   double z0, double dx, int nb, int kernel_id, double* acc, double* outside,
                   int64_t* n_trilinear, void* stream);
/* _finish (render/gasgrid.py:293-313): mass (float64), rho, mass-weighted T, emission-weighted
 * T and mass-weighted v (float32) per cell from acc; vol[cell / cells_per_volume] is a cell's
 * volume (nph for the log grid's (nr, nth) volumes, ncell for a box's single volume). */
NB_API int nb_grid_finish(nb_ctx* ctx, int64_t ncell, const double* acc, const double* vol,
                   int64_t cells_per_volume, double* mass, float* rho, float* t_mass,
                   float* t_em, float* vel, void* stream);
/* refine_sums (render/gasgrid.py:757-788): coarse log-grid sums (nrc, nthc, nphc, 6) with
 * their (nrc, nthc) volumes -> fine sums (nr, nth, nph, 6) written to out, rescaled to the
 * coarse mass; the coarsening (cr, ct, cp) must divide the fine grid. */
NB_API int nb_refine_sums(nb_ctx* ctx, const double* acc_c, const double* vol_c, int nrc,
                   int nthc, int nphc, const double* vol_f, int nr, int nth, int nph, int cr,
                   int ct, int cp, double* out, void* stream);

/* Live kernel timing with CUDA events on the launching stream: nb_profile(ctx, 1) resets and
 * starts, nb_profile_read fills out[36] = for each of {list build, density, forces, gravity
 * flow, touched-set marks, level choice (limiter, wake-up, opening), cooling, equation of state,
 * gradients (switch and reconstruction)}: (milliseconds, launches, rows or particles processed,
 * pair evaluations). */
NB_API int nb_profile(nb_ctx* ctx, int on);
NB_API int nb_profile_read(nb_ctx* ctx, double* out);

/* Drop the cached neighbour lists (the next density call rebuilds them). */
NB_API int nb_reset_cache(nb_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* NEBULA_B200_H */
