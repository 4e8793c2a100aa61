// The engine context behind the C-ABI: device workspace that grows on demand and is reused,
// the cached neighbour lists of the last build, and error reporting.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdio>
#include <cstring>

#include "common.cuh"
#include "../../include/nebula_b200.h"

namespace nbk {

constexpr int MAX_LEVELS = 16;

// Symmetric lists of the last build, in sorted (Hilbert-curve) order: row k belongs to the particle
// perm[k] of the caller's order; entries are sorted positions.
struct Lists {
  int64_t n = 0, total = 0;
  int64_t gen = 0;              // builds so far (the sorted order changes with every build)
  int32_t* perm = nullptr;      // sorted position -> caller index
  int32_t* inv_perm = nullptr;  // caller index -> sorted position
  double4* spos = nullptr;      // sorted (x, y, z, h_search)
  int64_t* off = nullptr;       // n + 1
  int32_t* idx = nullptr;       // total
};

struct Engine;

// Cached lists of the last build: positions and search radii they were built with
// (sim/sph.py:62-82, NeighbourCache).
struct Cache {
  bool valid = false;
  int64_t n = 0;
  double* x_ref = nullptr;
  double* hs = nullptr;
  int64_t cap = 0;
};

// Per-particle scratch of the step runtime (caller order unless noted).
struct Workspace {
  Cache cache;
  int64_t cap = 0;
  double *d_a = nullptr, *d_b = nullptr, *d_c = nullptr, *d_hg = nullptr, *d_hs = nullptr,
         *d_heff = nullptr, *d_hlim = nullptr, *d_disp = nullptr, *d_P = nullptr,
         *d_cs = nullptr, *d_vsig = nullptr, *d_ddudt = nullptr, *d_dm = nullptr,
         *d_tmp = nullptr, *d_uh = nullptr;
  double *v_flow = nullptr, *v_pred = nullptr, *v_eval = nullptr, *v_dacc = nullptr,
         *v_tmp = nullptr;  // (n, 3)
  double4 *pk0 = nullptr, *pk1 = nullptr, *pk2 = nullptr, *pk3 = nullptr;  // sorted packs
  float4* pk32 = nullptr;
  float* f_mass = nullptr;  // sorted masses as floats (FP32 density)
  float4 *pf1 = nullptr, *pf2 = nullptr, *pf3 = nullptr;  // FP32 packs of the force pass
  int64_t *rows = nullptr, *rows_s = nullptr, *rows2 = nullptr, *iters = nullptr,
          *flags = nullptr, *need = nullptr, *i_tmp = nullptr, *pairs = nullptr,
          *i_lvl = nullptr, *i_tmp2 = nullptr;
  uint8_t *m_rows = nullptr, *m_done = nullptr, *m_need = nullptr, *m_tmp = nullptr,
          *m_x = nullptr, *m_sorted = nullptr, *m_smark = nullptr;
  int32_t *i32a = nullptr, *i32b = nullptr;
  double* dk_b = nullptr;
  unsigned long long *tk_key0 = nullptr, *tk_key1 = nullptr;  // top-k candidates (reuse test)
  int32_t *tk_idx0 = nullptr, *tk_idx1 = nullptr;
  int* d_int = nullptr;
  int64_t* d_i64 = nullptr;
  int* h_int = nullptr;
  int64_t* h_i64 = nullptr;
  double* h_dbl = nullptr;
  int64_t* h_scal = nullptr;  // host copy of d_scal_i[0..8) and d_scal[0] (one read for all three)
  // W.rows (the active rows of the current step) changes version whenever it is rewritten; the
  // sorted copy in rows_s is kept while the rows and the lists stay the same
  int64_t rows_ver = 0, rs_ver = -1, rs_gen = -1, rs_n = -1, rs_count = 0;
  // the rows' interacting entries in E.tidx / i32a, written by the force pass of these rows
  // (rows version, lists generation, row count), for the level choice that follows
  int64_t tight_ver = -1, tight_gen = -1, tight_n = -1;
  // checks whose results are read at the next host synchronisation instead of a round trip of
  // their own: the device error word, the flow's worst iteration code (d_scal_i[0]) and a
  // radiated-energy sum (d_scal[0]) to add to *pend_erad
  bool pend_err = false, pend_glf = false;
  double* pend_erad = nullptr;
  int64_t* pend_woken = nullptr;  // the level choice's wake-up count (d_scal_i[2]) to add here
  double* d_scal = nullptr;    // = (double*)(d_scal_i + 8): one allocation, read in one copy
  int64_t* d_scal_i = nullptr;
  // switch and velocity reconstruction only (allocated on first use): sorted accelerations and
  // the sorted velocity gradients (9 per particle; float copy for the FP32 force pass)
  int64_t gcap = 0;
  double4* pk4 = nullptr;
  double* gvel = nullptr;
  float* gvel32 = nullptr;
  int ensure(Engine& E, int64_t n);
  int ensure_grad(Engine& E, int64_t n);
  void release();
};

// Live timing of the main kernels with CUDA events on the launching stream (off by default).
// Event pairs are recorded into a pool and read only when the profile is read (or the pool is
// full), and pair counts are summed on the device, so profiling adds no host synchronisation to
// the steps it times.
enum ProfCat {
  PROF_LISTS = 0, PROF_DENSITY = 1, PROF_FORCES = 2, PROF_FLOW = 3, PROF_MARKS = 4,
  PROF_LEVELS = 5, PROF_COOL = 6, PROF_EOS = 7, PROF_GRAD = 8, PROF_NCAT = 9
};
struct Prof {
  static constexpr int POOL = 1024;
  bool on = false;
  cudaEvent_t ev[2 * POOL] = {};
  int cat[POOL] = {};
  int used = 0;        // event pairs recorded and not yet read
  bool open = false;   // a begin() without its end()
  double ms[PROF_NCAT] = {0};
  int64_t launches[PROF_NCAT] = {0};
  double units[PROF_NCAT] = {0};   // rows (density, forces, flow) or particles (lists)
  double pairs[PROF_NCAT] = {0};   // host-known counts (lists: entries written)
  unsigned long long* d_pairs = nullptr;  // device-summed counts (density, forces)
  int ensure();
  void begin(cudaStream_t st) {
    if (!on) return;
    if (used == POOL) flush();
    if (ensure() != 0) return;
    cudaEventRecord(ev[2 * used], st);
    open = true;
  }
  void end(int c, cudaStream_t st, double u, double pr) {
    if (!on || !open) return;
    cudaEventRecord(ev[2 * used + 1], st);
    cat[used] = c;
    used += 1;
    open = false;
    launches[c] += 1;
    units[c] += u;
    pairs[c] += pr;
  }
  // waits for the recorded pairs and adds their times
  void flush() {
    for (int k = 0; k < used; ++k) {
      float t = 0.f;
      cudaEventSynchronize(ev[2 * k + 1]);
      cudaEventElapsedTime(&t, ev[2 * k], ev[2 * k + 1]);
      ms[cat[k]] += t;
    }
    used = 0;
  }
  void release() {
    for (int k = 0; k < 2 * POOL; ++k)
      if (ev[k]) cudaEventDestroy(ev[k]);
    if (d_pairs) cudaFree(d_pairs);
  }
};

struct Engine {
  int device = 0;
  Prof prof;
  int* d_err = nullptr;
  int* h_err = nullptr;  // pinned
  char last_error[512] = {0};
  int64_t cap_n = 0, cap_nodes = 0, cap_list = 0, cap_sort = 0;
  double* bbox_part = nullptr;
  double* bbox = nullptr;
  uint64_t* keys_a = nullptr;
  uint64_t* keys_b = nullptr;
  int32_t* vals_a = nullptr;
  int64_t* counts = nullptr;
  double4* node_lo = nullptr;
  double4* node_hi = nullptr;
  double4* sub_lo = nullptr;  // sub-leaf boxes
  double4* sub_hi = nullptr;
  int64_t cap_sub = 0;
  void* cub_tmp = nullptr;
  size_t cub_bytes = 0;
  int64_t* sort_keys = nullptr;
  // particle -> grid deposition: spatial sort keys / indices (double buffers) and the gathered
  // particle data (9 doubles per particle)
  unsigned long long *dep_k0 = nullptr, *dep_k1 = nullptr;
  int32_t *dep_i0 = nullptr, *dep_i1 = nullptr;
  double* dep_buf = nullptr;
  int64_t dep_cap = 0;
  int ensure_deposit(int64_t n);
  int64_t list_slots = 0, cand_slots = 0;  // resident warps of the persistent list passes
  int32_t* tidx = nullptr;  // interacting entries of the active rows, in the lists' layout
  int64_t cap_tidx = 0;
  // list build: the longest row of the last build [0], the passes' work counters [2, 3] and the
  // candidate and batch cursors [4, 5]
  unsigned long long* d_rowmax = nullptr;
  // list build: per query leaf the start of its candidate list and of its masks and its number
  // of candidate sub-leaves; the candidate lists and the tests' hit masks (32 per batch)
  int64_t *leaf_cbase = nullptr, *leaf_bbase = nullptr;
  int32_t* leaf_ncand = nullptr;
  int64_t cap_leaf = 0;
  int32_t* cands = nullptr;
  int64_t cap_cands = 0;
  uint32_t* masks = nullptr;
  int64_t cap_masks = 0;
  int64_t last_cands = 0, last_batches = 0;
  int ensure_leaves(int64_t m);
  int ensure_tiles(int64_t ncand, int64_t nbatch);
  int64_t* h_build = nullptr;  // pinned: total entries and longest row of the last build
  double* red = nullptr;      // reduction partials (doubles)
  double* h_red = nullptr;    // pinned host copy of small reductions
  Lists lists;
  Workspace ws;

  int ensure_n(int64_t n);
  int ensure_nodes(int64_t m);
  int grow2(int64_t m);
  int ensure_sub(int64_t m);
  int ensure_list_capacity(int64_t m);
  int ensure_sort_keys(int64_t m);
  int ensure_tight(int64_t m);
  int ensure_cub(size_t bytes);
  void release();
};

size_t cub_bytes_needed(int64_t n, int64_t m);
struct MlpHull;
// learned cooling (mlp.cu): u_out = cooled u of n particles (dt per particle or dt_scalar)
int mlp_cool(Engine& E, int64_t n, const double* u, const double* rho, const double* dt,
             double dt_scalar, const struct ::nb_mlp_params* mp, double* u_out, int8_t* mode,
             cudaStream_t st);
int build_lists(Engine& E, int64_t n, const double* pos, const double* hs, cudaStream_t st);
int export_lists_offsets(Engine& E, int64_t* off_out, cudaStream_t st);
int build_cells(Engine& E, int64_t n, const double* pos, const double* lo, const double* inv_cell,
                const int64_t* ncell, int64_t* start, int64_t* order, cudaStream_t st);
int cell_geometry(Engine& E, int64_t n, const double* pos, const double* h, double* lo,
                  double* inv_cell, int64_t* ncell, cudaStream_t st);
int export_lists(Engine& E, int64_t* off_out, int64_t* idx_out, cudaStream_t st);

inline int set_host_error(Engine& E, const char* msg) {
  std::snprintf(E.last_error, sizeof(E.last_error), "%s", msg);
  return -1;
}

int check_device_error(Engine& E, cudaStream_t st);

}  // namespace nbk

struct nb_ctx {
  nbk::Engine E;
};

#define NB_CUDA(call)                                                                        \
  do {                                                                                       \
    cudaError_t _e = (call);                                                                 \
    if (_e != cudaSuccess) {                                                                 \
      std::snprintf(E.last_error, sizeof(E.last_error), "CUDA error %s at %s:%d: %s",        \
                    cudaGetErrorName(_e), __FILE__, __LINE__, cudaGetErrorString(_e));       \
      return -2;                                                                             \
    }                                                                                        \
  } while (0)

#define NB_TRY(expr)        \
  do {                      \
    int _r = (expr);        \
    if (_r != 0) return _r; \
  } while (0)
