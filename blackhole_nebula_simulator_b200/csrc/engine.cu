// The step runtime: list cache with the reference's reuse test, density for given rows with the
// search-doubling loop, the fused EOS + force pass, and the shared-step and block-step drivers.
//
// State arrays stay in the caller's particle order.  Each list build sorts the particles in
// Hilbert-curve order; the pair passes read packed copies in that order (coalesced, cache-friendly) and
// scatter their results back to the caller's order.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <cmath>
#include <vector>

#include "../../include/nebula_b200.h"
#include "common.cuh"
#include "cooling.cuh"
#include "engine.cuh"
#include "eos.cuh"
#include "gravity.cuh"
#include "sph.cuh"
#include "steps.cuh"

namespace nbk {

// the reuse test looks at the TOPK = 65 largest displacements (its fast sets hold at most 64)
constexpr int TOPK = 65;
constexpr int TOPK_CHUNK = 2048;

// ---------------------------------------------------------------- workspace
template <typename T>
static int grow(Engine& E, T*& p, int64_t& cap, int64_t want) {
  if (want <= cap && p) return 0;
  int64_t c = std::max<int64_t>(want + want / 4, 1024);
  if (p) cudaFree(p);
  p = nullptr;
  NB_CUDA(cudaMalloc((void**)&p, sizeof(T) * (size_t)c));
  cap = c;
  return 0;
}

int Engine::ensure_cub(size_t bytes) {
  Engine& E = *this;
  if (bytes <= cub_bytes && cub_tmp) return 0;
  if (cub_tmp) cudaFree(cub_tmp);
  cub_tmp = nullptr;
  size_t b = bytes + bytes / 4 + 4096;
  NB_CUDA(cudaMalloc(&cub_tmp, b));
  cub_bytes = b;
  return 0;
}

int Engine::ensure_n(int64_t n) {
  Engine& E = *this;
  if (!d_err) {
    NB_CUDA(cudaMalloc((void**)&d_err, sizeof(int) * 4));
    NB_CUDA(cudaMemset(d_err, 0, sizeof(int) * 4));
    NB_CUDA(cudaMallocHost((void**)&h_err, sizeof(int) * 4));
    NB_CUDA(cudaMalloc((void**)&bbox, sizeof(double) * 8));
    NB_CUDA(cudaMallocHost((void**)&h_red, sizeof(double) * 64));
    NB_CUDA(cudaMalloc((void**)&d_rowmax, 8 * sizeof(unsigned long long)));
    NB_CUDA(cudaMallocHost((void**)&h_build, sizeof(int64_t) * 2));
  }
  if (n <= cap_n && keys_a) return 0;
  int64_t c = std::max<int64_t>(n + n / 4, 1024);
  auto fr = [](void* p) {
    if (p) cudaFree(p);
  };
  fr(bbox_part); fr(keys_a); fr(keys_b); fr(vals_a); fr(counts); fr(red);
  fr(lists.perm); fr(lists.inv_perm); fr(lists.spos); fr(lists.off);
  NB_CUDA(cudaMalloc((void**)&bbox_part, sizeof(double) * 6 * 1184));
  NB_CUDA(cudaMalloc((void**)&keys_a, sizeof(uint64_t) * c));
  NB_CUDA(cudaMalloc((void**)&keys_b, sizeof(uint64_t) * c));
  NB_CUDA(cudaMalloc((void**)&vals_a, sizeof(int32_t) * c));
  NB_CUDA(cudaMalloc((void**)&counts, sizeof(int64_t) * (c + 1)));
  NB_CUDA(cudaMalloc((void**)&red, sizeof(double) * 16 * 1184));
  NB_CUDA(cudaMalloc((void**)&lists.perm, sizeof(int32_t) * c));
  NB_CUDA(cudaMalloc((void**)&lists.inv_perm, sizeof(int32_t) * c));
  NB_CUDA(cudaMalloc((void**)&lists.spos, sizeof(double4) * c));
  NB_CUDA(cudaMalloc((void**)&lists.off, sizeof(int64_t) * (c + 1)));
  cap_n = c;
  lists.n = 0;
  return ensure_cub(cub_bytes_needed(c, 0));
}

int Prof::ensure() {
  if (ev[0]) return 0;
  for (int k = 0; k < 2 * POOL; ++k)
    if (cudaEventCreate(&ev[k]) != cudaSuccess) return -2;
  if (cudaMalloc((void**)&d_pairs, sizeof(unsigned long long) * PROF_NCAT) != cudaSuccess) return -2;
  if (cudaMemset(d_pairs, 0, sizeof(unsigned long long) * PROF_NCAT) != cudaSuccess) return -2;
  return 0;
}

int Engine::ensure_nodes(int64_t m) { return grow2(m); }

int Engine::grow2(int64_t m) {
  Engine& E = *this;
  if (m <= cap_nodes && node_lo) return 0;
  int64_t c = std::max<int64_t>(m + m / 4, 256);
  if (node_lo) cudaFree(node_lo);
  if (node_hi) cudaFree(node_hi);
  NB_CUDA(cudaMalloc((void**)&node_lo, sizeof(double4) * c));
  NB_CUDA(cudaMalloc((void**)&node_hi, sizeof(double4) * c));
  cap_nodes = c;
  return 0;
}

int Engine::ensure_sub(int64_t m) {
  Engine& E = *this;
  if (m <= cap_sub && sub_lo) return 0;
  int64_t c = std::max<int64_t>(m + m / 4, 256);
  if (sub_lo) cudaFree(sub_lo);
  if (sub_hi) cudaFree(sub_hi);
  NB_CUDA(cudaMalloc((void**)&sub_lo, sizeof(double4) * c));
  NB_CUDA(cudaMalloc((void**)&sub_hi, sizeof(double4) * c));
  cap_sub = c;
  return 0;
}

int Engine::ensure_list_capacity(int64_t m) {
  Engine& E = *this;
  NB_TRY(grow(E, lists.idx, cap_list, std::max<int64_t>(m, 1)));
  return 0;
}

int Engine::ensure_tight(int64_t m) {
  Engine& E = *this;
  return grow(E, tidx, cap_tidx, std::max<int64_t>(m, 1));
}

int Engine::ensure_leaves(int64_t m) {
  Engine& E = *this;
  if (m <= cap_leaf && leaf_cbase) return 0;
  int64_t c = 0;
  NB_TRY(grow(E, leaf_cbase, c, m));
  c = 0;
  NB_TRY(grow(E, leaf_bbase, c, m));
  c = 0;
  NB_TRY(grow(E, leaf_ncand, c, m));
  cap_leaf = c;
  return 0;
}

int Engine::ensure_tiles(int64_t ncand, int64_t nbatch) {
  Engine& E = *this;
  NB_TRY(grow(E, cands, cap_cands, std::max<int64_t>(ncand, 1)));
  return grow(E, masks, cap_masks, std::max<int64_t>(nbatch * 32, 32));
}

int Engine::ensure_deposit(int64_t n) {
  Engine& E = *this;
  if (n > dep_cap || !dep_buf) {
    void* ps[] = {dep_k0, dep_k1, dep_i0, dep_i1, dep_buf};
    for (void* p : ps)
      if (p) cudaFree(p);
    dep_k0 = dep_k1 = nullptr;
    dep_i0 = dep_i1 = nullptr;
    dep_buf = nullptr;
    const int64_t c = std::max<int64_t>(n + n / 4, 1024);
    NB_CUDA(cudaMalloc((void**)&dep_k0, sizeof(unsigned long long) * c));
    NB_CUDA(cudaMalloc((void**)&dep_k1, sizeof(unsigned long long) * c));
    NB_CUDA(cudaMalloc((void**)&dep_i0, sizeof(int32_t) * c));
    NB_CUDA(cudaMalloc((void**)&dep_i1, sizeof(int32_t) * c));
    NB_CUDA(cudaMalloc((void**)&dep_buf, sizeof(double) * 9 * c));
    dep_cap = c;
  }
  size_t b = 0;
  cub::DeviceRadixSort::SortPairs((void*)nullptr, b, (unsigned long long*)nullptr,
                                  (unsigned long long*)nullptr, (int32_t*)nullptr,
                                  (int32_t*)nullptr, (int)dep_cap);
  return ensure_cub(b);
}

int Engine::ensure_sort_keys(int64_t m) {
  Engine& E = *this;
  NB_TRY(grow(E, sort_keys, cap_sort, m));
  return ensure_cub(cub_bytes_needed(cap_n, m));
}

void Engine::release() {
  void* ps[] = {dep_k0, dep_k1, dep_i0, dep_i1, dep_buf, d_err, bbox, bbox_part, keys_a, keys_b, vals_a, counts, node_lo, node_hi, sub_lo, sub_hi,
                cub_tmp, sort_keys, red, lists.perm, lists.inv_perm, lists.spos, lists.off,
                lists.idx, d_rowmax, tidx, leaf_cbase, leaf_bbase, leaf_ncand, cands, masks};
  for (void* p : ps)
    if (p) cudaFree(p);
  if (h_err) cudaFreeHost(h_err);
  if (h_build) cudaFreeHost(h_build);
  prof.release();
  if (h_red) cudaFreeHost(h_red);
  ws.release();
}

int check_device_error(Engine& E, cudaStream_t st) {
  NB_CUDA(cudaMemcpyAsync(E.h_err, E.d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  NB_CUDA(host_sync(st));
  E.ws.pend_err = false;  // this read covers a deferred check of the same word
  NB_CUDA(cudaGetLastError());
  int code = E.h_err[0];
  if (code == 0) return 0;
  NB_CUDA(cudaMemsetAsync(E.d_err, 0, sizeof(int), st));
  const char* msg = "device error";
  int ret = NB_ERR_INPUT;
  switch (code) {
    case ERR_LIST_OVERFLOW: msg = "neighbour list longer than counted"; ret = -3; break;
    case ERR_TRAVERSAL_STACK: msg = "tree traversal stack exhausted"; ret = -3; break;
    case ERR_BAD_INDEX: msg = "index outside [0, n)"; ret = NB_ERR_INPUT; break;
    case ERR_NONPOSITIVE_U: msg = "non-positive internal energy"; ret = NB_ERR_NONPOSITIVE_U; break;
    case ERR_LEVEL: msg = "a particle needs a level beyond K_MAX = 40"; ret = NB_ERR_LEVEL; break;
    case ERR_LIMITER: msg = "level limiter did not settle"; ret = -3; break;
    case ERR_DT: msg = "time steps must be positive"; ret = NB_ERR_DT; break;
    case ERR_EOS_RANGE: msg = "u outside the EOS bracket [1, 1e13] K"; ret = NB_ERR_EOS_RANGE; break;
    case ERR_EOS_CONVERGE: msg = "gas + radiation EOS: temperature did not converge"; ret = NB_ERR_EOS; break;
  }
  std::snprintf(E.last_error, sizeof(E.last_error), "%s", msg);
  return ret;
}

// ---------------------------------------------------------------- small kernels
__global__ void k_mask_rows(int64_t nrows, const int64_t* __restrict__ rows, int64_t n,
                            uint8_t* __restrict__ mask, int* err) {
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= nrows) return;
  int64_t i = rows[q];
  if (i < 0 || i >= n) {
    set_error(err, ERR_BAD_INDEX);
    return;
  }
  mask[i] = 1;
}

// mask in sorted order from a caller-order mask
__global__ void k_sorted_mask(int64_t n, const int32_t* __restrict__ perm, const uint8_t* __restrict__ m,
                              uint8_t* __restrict__ ms) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < n) ms[k] = m[perm[k]];
}

__global__ void k_pack_sorted_f4(int64_t n, const int32_t* __restrict__ perm,
                                 const double* __restrict__ a, const double* __restrict__ b,
                                 const double* __restrict__ c, const double* __restrict__ d,
                                 int vec3, float4* __restrict__ out) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  int64_t i = perm[k];
  if (vec3)  // a: (n, 3) vector, b: scalar
    out[k] = make_float4((float)a[3 * i], (float)a[3 * i + 1], (float)a[3 * i + 2],
                         b ? (float)b[i] : 0.f);
  else
    out[k] = make_float4(a ? (float)a[i] : 0.f, b ? (float)b[i] : 0.f, c ? (float)c[i] : 0.f,
                         d ? (float)d[i] : 0.f);
}

// h_search = min(min(h_guess, h_max) * skin, cap) (sim/sph.py:373)
__global__ void k_hsearch(int64_t n, const double* __restrict__ hg, double h_max, double skin,
                          double* __restrict__ hs) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  hs[i] = fmin(hg[i], h_max) * skin;
}

// The displacements since the last build, and their largest value into *dmax (as the bits of a
// non-negative double, which order like the values; *dmax starts at 0).
__global__ void __launch_bounds__(NB_THREADS) k_disp(int64_t n, const double* __restrict__ x,
                                                     const double* __restrict__ xr,
                                                     double* __restrict__ disp,
                                                     unsigned long long* __restrict__ dmax) {
  __shared__ unsigned long long wmax[NB_THREADS / 32];
  const unsigned FULL = 0xffffffffu;
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  unsigned long long key = 0ull;
  if (i < n) {
    double dx = x[3 * i] - xr[3 * i], dy = x[3 * i + 1] - xr[3 * i + 1], dz = x[3 * i + 2] - xr[3 * i + 2];
    const double d = sqrt(dx * dx + dy * dy + dz * dz);
    disp[i] = d;
    key = (unsigned long long)__double_as_longlong(d);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long v = __shfl_xor_sync(FULL, key, o);
    key = v > key ? v : key;
  }
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = key;
  __syncthreads();
  if (threadIdx.x < 32) {
    key = threadIdx.x < NB_THREADS / 32 ? wmax[threadIdx.x] : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long v = __shfl_xor_sync(FULL, key, o);
      key = v > key ? v : key;
    }
    if (threadIdx.x == 0) atomicMax(dmax, key);
  }
}

// The TOPK largest displacements with their indices, in descending order and, among equal values,
// ascending index (the order of a stable descending sort).  Each block sorts a chunk of
// TOPK_CHUNK candidates (cub::BlockRadixSort, stable) and keeps its first TOPK; passes repeat
// over the kept candidates until one block remains.  Keys are the displacement's bits + 1
// (non-negative doubles order like their bits), 0 marks padding, which sorts after every value.
template <bool FIRST>
__global__ void __launch_bounds__(256) k_topk(int64_t count, const double* __restrict__ disp,
                                              const unsigned long long* __restrict__ key_in,
                                              const int32_t* __restrict__ idx_in,
                                              unsigned long long* __restrict__ key_out,
                                              int32_t* __restrict__ idx_out) {
  using Sort = cub::BlockRadixSort<unsigned long long, 256, TOPK_CHUNK / 256, int32_t>;
  __shared__ typename Sort::TempStorage tmp;
  constexpr int ITEMS = TOPK_CHUNK / 256;
  unsigned long long k[ITEMS];
  int32_t v[ITEMS];
  const int64_t base = (int64_t)blockIdx.x * TOPK_CHUNK + (int64_t)threadIdx.x * ITEMS;
#pragma unroll
  for (int t = 0; t < ITEMS; ++t) {
    int64_t g = base + t;
    if (g < count) {
      k[t] = FIRST ? (unsigned long long)__double_as_longlong(disp[g]) + 1ull : key_in[g];
      v[t] = FIRST ? (int32_t)g : idx_in[g];
    } else {
      k[t] = 0ull;
      v[t] = -1;
    }
  }
  Sort(tmp).SortDescending(k, v);
#pragma unroll
  for (int t = 0; t < ITEMS; ++t) {
    int r = threadIdx.x * ITEMS + t;
    if (r < TOPK) {
      key_out[(int64_t)blockIdx.x * TOPK + r] = k[t];
      idx_out[(int64_t)blockIdx.x * TOPK + r] = v[t];
    }
  }
}

__global__ void k_topk_out(int top, const unsigned long long* __restrict__ key,
                           const int32_t* __restrict__ idx, double* __restrict__ val_out,
                           int32_t* __restrict__ idx_out) {
  int r = threadIdx.x;
  if (r >= top) return;
  val_out[r] = __longlong_as_double((long long)(key[r] - 1ull));
  idx_out[r] = idx[r];
}

// h_eff = hs - (disp + d_rest)/2; fail if a row has h_eff <= h_guess/2 or another particle
// h_guess > h_eff (sim/sph.py:134-138).  Also fills h_lim (rows: h_eff, others: h_guess).
__global__ void k_reuse_test(int64_t n, const double* __restrict__ hs, const double* __restrict__ disp,
                             const double* __restrict__ d_rest_p, const double* __restrict__ hg,
                             const uint8_t* __restrict__ is_row, double* __restrict__ h_eff,
                             double* __restrict__ h_lim, int* __restrict__ fail) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double d_rest = *d_rest_p;  // the largest displacement outside the fast set
  double he = hs[i] - 0.5 * (disp[i] + d_rest);
  h_eff[i] = he;
  bool row = is_row[i];
  h_lim[i] = row ? he : hg[i];
  bool bad = row ? !(he > 0.5 * hg[i]) : !(hg[i] <= he);
  if (bad) atomicOr(fail, 1);
}

// sim/sph.py:85-111: every particle k within 2 max(h_lim_j, h_lim_k) of a fast particle j must be
// in j's list.  One block per fast particle; binary search in the (sorted) row.
__global__ void k_fast_complete(int64_t n, int nfast, const int32_t* __restrict__ fast,
                                const double* __restrict__ x, const double* __restrict__ h_lim,
                                const int32_t* __restrict__ inv_perm, const int64_t* __restrict__ off,
                                const int32_t* __restrict__ idx, int* __restrict__ fail) {
  int q = blockIdx.x;
  if (q >= nfast) return;
  int64_t j = fast[q];
  int64_t row = inv_perm[j];
  int64_t lo = off[row], hi = off[row + 1];
  double xj0 = x[3 * j], xj1 = x[3 * j + 1], xj2 = x[3 * j + 2];
  for (int64_t k = threadIdx.x; k < n; k += blockDim.x) {
    double d2 = d2_exact(x[3 * k] - xj0, x[3 * k + 1] - xj1, x[3 * k + 2] - xj2);
    double rr = 2.0 * fmax(h_lim[j], h_lim[k]);
    if (d2 <= rr * rr) {
      int32_t key = inv_perm[k];
      int64_t a = lo, b = hi;
      while (a < b) {
        int64_t m = (a + b) >> 1;
        if (idx[m] < key)
          a = m + 1;
        else
          b = m;
      }
      if (a >= hi || idx[a] != key) atomicOr(fail, 1);
    }
  }
}

// sorted packs for the pair passes
__global__ void k_pack_sorted(int64_t n, const int32_t* __restrict__ perm,
                              const double* __restrict__ x, const double* __restrict__ w,
                              double4* __restrict__ out) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  int64_t i = perm[k];
  out[k] = make_double4(x[3 * i], x[3 * i + 1], x[3 * i + 2], w ? w[i] : 0.0);
}

// the density pass's per-particle inputs in sorted order (masses also as floats when asked)
__global__ void k_gather_density(int64_t n, const int32_t* __restrict__ perm,
                                 const double* __restrict__ mass, const double* __restrict__ h0,
                                 const double* __restrict__ hs, double* __restrict__ mass_s,
                                 double* __restrict__ h0_s, double* __restrict__ hs_s,
                                 float* __restrict__ massf_s) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int32_t i = perm[k];
  const double m = mass[i];
  mass_s[k] = m;
  h0_s[k] = h0[i];
  hs_s[k] = hs[i];
  if (massf_s) massf_s[k] = (float)m;
}

__global__ void k_to_float(int64_t n, const double* __restrict__ a, float* __restrict__ out) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < n) out[k] = (float)a[k];
}

__global__ void k_pack_sorted4(int64_t n, const int32_t* __restrict__ perm, const double* __restrict__ a,
                               const double* __restrict__ b, const double* __restrict__ c,
                               const double* __restrict__ d, double4* __restrict__ out) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  int64_t i = perm[k];
  out[k] = make_double4(a ? a[i] : 0.0, b ? b[i] : 0.0, c ? c[i] : 0.0, d ? d[i] : 0.0);
}

// FP32 positions: the cell of a uniform grid (edge `cell`, at most 1024 per axis, corner lo) and
// the float offset from the cell centre, as two float4 per particle: (offset, mass) and (cell
// coordinates as exact floats, h); mass and h 0 when not given.
__device__ __forceinline__ void pos32_record(const double* __restrict__ x, int64_t i,
                                             const double* __restrict__ box6, float w0, float w1,
                                             float4* __restrict__ out) {
  double span = fmax(fmax(box6[3] - box6[0], box6[4] - box6[1]), box6[5] - box6[2]);
  const double cell = fmax(span / 1000.0, 1e-30);
  int c[3];
  float o[3];
  for (int a = 0; a < 3; ++a) {
    double t = (x[3 * i + a] - box6[a]) / cell;
    int ci = (int)floor(t);
    ci = min(max(ci, 0), 1023);
    c[a] = ci;
    o[a] = (float)(x[3 * i + a] - (box6[a] + (ci + 0.5) * cell));
  }
  out[0] = make_float4(o[0], o[1], o[2], w0);
  out[1] = make_float4((float)c[0], (float)c[1], (float)c[2], w1);
}

__global__ void k_pack_sorted32(int64_t n, const int32_t* __restrict__ perm,
                                const double* __restrict__ x, const double* __restrict__ m,
                                const double* __restrict__ h, const double* __restrict__ box6,
                                float4* __restrict__ out) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  int64_t i = perm[k];
  pos32_record(x, i, box6, m ? (float)m[i] : 0.0f, h ? (float)h[i] : 0.0f, out + 2 * k);
}

// The FP32 density pass's sorted inputs in one pass: k_gather_density's mass, h_start and
// h_search, and the position records (offset, m) (cell, 0).
__global__ void k_pack_density32(int64_t n, const int32_t* __restrict__ perm,
                                 const double* __restrict__ x, const double* __restrict__ mass,
                                 const double* __restrict__ h0, const double* __restrict__ hs,
                                 const double* __restrict__ box6, double* __restrict__ mass_s,
                                 double* __restrict__ h0_s, double* __restrict__ hs_s,
                                 float4* __restrict__ pk32) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int32_t i = perm[k];
  const double m = mass[i];
  mass_s[k] = m;
  h0_s[k] = h0[i];
  hs_s[k] = hs[i];
  pos32_record(x, i, box6, (float)m, 0.0f, pk32 + 2 * k);
}

// The FP32 force pass's sorted inputs in one pass (the switch and the reconstruction off): the
// position records (offset, m) (cell, h), the records (v, m), (h, rho, omega, P), (u, c_s, alpha)
// and, when pk0 is given, the double (x, h) of the exact band test; with `only`, the records of
// its particles alone.
__global__ void k_pack_force32(int64_t n, const int32_t* __restrict__ perm,
                               const double* __restrict__ x, const double* __restrict__ m,
                               const double* __restrict__ h, const double* __restrict__ box6,
                               const double* __restrict__ vel, const double* __restrict__ rho,
                               const double* __restrict__ omega, const double* __restrict__ P,
                               const double* __restrict__ u, const double* __restrict__ cs,
                               const double* __restrict__ alpha, const uint8_t* __restrict__ only,
                               float4* __restrict__ pk32, float4* __restrict__ pf1,
                               float4* __restrict__ pf2, float4* __restrict__ pf3,
                               double4* __restrict__ pk0) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int64_t i = perm[k];
  if (only && !only[i]) return;  // a record the pass does not read
  const double hi = h[i];
  const float mi = (float)m[i];
  pos32_record(x, i, box6, mi, (float)hi, pk32 + 2 * k);
  pf1[k] = make_float4((float)vel[3 * i], (float)vel[3 * i + 1], (float)vel[3 * i + 2], mi);
  pf2[k] = make_float4((float)hi, (float)rho[i], (float)omega[i], (float)P[i]);
  pf3[k] = make_float4((float)u[i], (float)cs[i], alpha ? (float)alpha[i] : 0.f, 0.f);
  if (pk0) pk0[k] = make_double4(x[3 * i], x[3 * i + 1], x[3 * i + 2], hi);
}

// the configured EOS (sim/hydro.py:119-139) for every particle, or for the particles of `mask`
// when one is given; u <= 0 is an error
__global__ void k_eos(int64_t n, const double* __restrict__ rho, const double* __restrict__ u,
                      const uint8_t* __restrict__ mask, EosParams ep, double* __restrict__ P,
                      double* __restrict__ cs, int* err) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (mask && !mask[i]) return;
  double ui = u[i];
  if (!(ui > 0.0)) {
    set_error(err, ERR_NONPOSITIVE_U);
    return;
  }
  double p, c, t, b;
  eos_point(ep, rho[i], ui, p, c, t, b, err);
  P[i] = p;
  cs[i] = c;
}

EosParams eos_of(const nb_params* prm) {
  EosParams ep;
  ep.kind = prm->eos;
  ep.gamma = prm->gamma;
  ep.rho_si = prm->eos_rho_si;
  ep.u_si = prm->eos_u_si;
  ep.a1 = prm->eos_a1;
  ep.kb_mu = prm->eos_a1 / 1.5;
  ep.a_rad = prm->eos_a_rad;
  return ep;
}

// after the force pass: add the disc viscosity, nu, alpha and v_sig of the rows
__global__ void k_combine_rows(int64_t nrows, const int64_t* __restrict__ rows, int use_visc,
                               double disc_alpha_av,
                               const double* __restrict__ dacc, const double* __restrict__ ddudt,
                               const double* __restrict__ cs, const double* __restrict__ h,
                               const double* __restrict__ vsig_f, double* __restrict__ acc,
                               double* __restrict__ dudt, double* __restrict__ vsig,
                               double* __restrict__ nu, double* __restrict__ disk_heating) {
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= nrows) return;
  int64_t i = rows[q];
  if (disc_alpha_av > 0) {
    for (int c = 0; c < 3; ++c) acc[3 * i + c] += dacc[3 * i + c];
    dudt[i] += ddudt[i];
    if (disk_heating) disk_heating[i] = ddudt[i];
    if (nu) nu[i] = disc_alpha_av * cs[i] * h[i] / 10.0;
  }
  vsig[i] = use_visc ? vsig_f[i] : cs[i];
}

// touched sets over curve-ordered rows: pk holds sorted (x, y, z, h) of the current state (read
// only with `tight`).  Marks go to a mask in sorted order, where a row's neighbours lie close
// together; k_unsort_marks moves them to the caller's order in one pass.  Eight lanes per row,
// each taking every eighth list entry.
__global__ void k_mark_s(int64_t nrows, const int64_t* __restrict__ rows_s,
                         const int64_t* __restrict__ off, const int32_t* __restrict__ idx, int tight,
                         const double4* __restrict__ pk, uint8_t* __restrict__ mark_s) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t q = t >> 3;
  const int gl = (int)(t & 7);
  if (q >= nrows) return;
  int64_t k = rows_s[q];
  if (gl == 0) mark_s[k] = 1;
  double4 me = tight ? pk[k] : make_double4(0, 0, 0, 0);
  for (int64_t e = off[k] + gl; e < off[k + 1]; e += 8) {
    int32_t js = ld_stream(idx + e);
    if (tight) {
      double4 o = pk[js];
      double d2 = d2_exact(o.x - me.x, o.y - me.y, o.z - me.z);
      double rr = 2.0 * fmax(me.w, o.w);
      if (!(d2 < rr * rr)) continue;
    }
    mark_s[js] = 1;
  }
}

// The same touched set read the other way round (the lists are symmetric): particle k is touched
// if it is a row or a row is among its own entries.  Eight lanes per particle scan its list until
// one of them meets a row, and the mark goes straight to the caller's order.  Cheaper than
// scattering marks when a large share of the particles are rows.
// With `tight`, only rows within 2 max(h_k, h_row) count (pk: sorted (x, h)), the same exact
// test k_mark_s makes from the row's side (the squared differences do not depend on the sign).
__global__ void k_mark_gather(int64_t n, const int64_t* __restrict__ off,
                              const int32_t* __restrict__ idx, const uint8_t* __restrict__ row_s,
                              const int32_t* __restrict__ perm, int tight,
                              const double4* __restrict__ pk, uint8_t* __restrict__ mark) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t k = t >> 3;
  const int gl = (int)(t & 7), g = (int)((threadIdx.x & 31) >> 3);
  const bool live = k < n;
  if (!__any_sync(0xffffffffu, live)) return;  // warp-uniform
  bool hit = live && row_s[k];
  const double4 me = tight && live ? pk[k] : make_double4(0, 0, 0, 0);
  const int64_t e0 = live ? off[k] : 0, e1 = live ? off[k + 1] : 0;
  for (int64_t b = e0; ; b += 8) {
    unsigned grp = (__ballot_sync(0xffffffffu, hit) >> (8 * g)) & 0xffu;
    bool more = grp == 0 && b < e1;  // this particle still unresolved
    if (!__any_sync(0xffffffffu, more)) {
      hit = grp != 0;
      break;
    }
    if (more && b + gl < e1) {
      const int32_t j = ld_stream(idx + b + gl);
      bool near = row_s[j];
      if (near && tight) {
        const double4 o = pk[j];
        const double d2 = d2_exact(o.x - me.x, o.y - me.y, o.z - me.z);
        const double rr = 2.0 * fmax(me.w, o.w);
        near = d2 < rr * rr;
      }
      hit = hit || near;
    }
  }
  if (live && gl == 0 && hit) mark[perm[k]] = 1;
}

__global__ void k_unsort_marks(int64_t n, const int32_t* __restrict__ perm,
                               const uint8_t* __restrict__ mark_s, uint8_t* __restrict__ mark) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < n && mark_s[k]) mark[perm[k]] = 1;
}

__global__ void k_mask_and_not(int64_t n, const uint8_t* __restrict__ a, const uint8_t* __restrict__ b,
                               uint8_t* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = a[i] && !b[i];
}

__global__ void k_mask_or(int64_t n, const uint8_t* __restrict__ a, uint8_t* __restrict__ b) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  b[i] = b[i] | a[i];
}

// rows with flag 2 (FLAG_SEARCH_TOO_SMALL): double their search; every row restarts from its h
// (sim/sph.py:378-386)
__global__ void k_grow(int64_t nrows, const int64_t* __restrict__ rows, const int64_t* __restrict__ flags,
                       const double* __restrict__ h_res, double* __restrict__ hs,
                       double* __restrict__ hg, int* __restrict__ count) {
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= nrows) return;
  int64_t i = rows[q];
  if (flags[i] == 2) {
    hs[i] = hs[i] * 2.0;
    atomicAdd(count, 1);
  }
  hg[i] = h_res[i];
}

__global__ void k_count_flag2(int64_t nrows, const int64_t* __restrict__ rows,
                              const int64_t* __restrict__ flags, int* __restrict__ count) {
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= nrows) return;
  if (flags[rows[q]] == 2) atomicAdd(count, 1);
}

__global__ void k_max_rows(int64_t nrows, const int64_t* __restrict__ rows, const double* __restrict__ a,
                           double* __restrict__ b) {
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= nrows) return;
  int64_t i = rows[q];
  b[i] = fmax(b[i], a[i]);
}

// ---------------------------------------------------------------- cache + density
int Workspace::ensure(Engine& E, int64_t n) {
  if (n <= cap && d_a) return 0;
  release();
  int64_t c = std::max<int64_t>(n + n / 4, 1024);
  double** dd[] = {&d_a, &d_b, &d_c, &d_hg, &d_hs, &d_heff, &d_hlim, &d_disp, &d_P, &d_cs,
                   &d_vsig, &d_ddudt, &d_dm, &d_tmp, &d_uh};
  for (double** p : dd) NB_CUDA(cudaMalloc((void**)p, sizeof(double) * c));
  double** d3[] = {&v_flow, &v_pred, &v_eval, &v_dacc, &v_tmp};
  for (double** p : d3) NB_CUDA(cudaMalloc((void**)p, sizeof(double) * 3 * c));
  double4** d4[] = {&pk0, &pk1, &pk2, &pk3};
  for (double4** p : d4) NB_CUDA(cudaMalloc((void**)p, sizeof(double4) * c));
  NB_CUDA(cudaMalloc((void**)&pk32, sizeof(float4) * 2 * c));
  NB_CUDA(cudaMalloc((void**)&f_mass, sizeof(float) * c));
  float4** f4s[] = {&pf1, &pf2, &pf3};
  for (float4** p : f4s) NB_CUDA(cudaMalloc((void**)p, sizeof(float4) * c));
  int64_t** i8[] = {&rows, &rows_s, &rows2, &iters, &flags, &need, &i_tmp, &pairs, &i_lvl, &i_tmp2};
  for (int64_t** p : i8) NB_CUDA(cudaMalloc((void**)p, sizeof(int64_t) * (c + 1)));
  uint8_t** u1[] = {&m_rows, &m_done, &m_need, &m_tmp, &m_x, &m_sorted, &m_smark};
  for (uint8_t** p : u1) NB_CUDA(cudaMalloc((void**)p, c));
  NB_CUDA(cudaMalloc((void**)&i32a, sizeof(int32_t) * c));
  NB_CUDA(cudaMalloc((void**)&i32b, sizeof(int32_t) * c));
  NB_CUDA(cudaMalloc((void**)&dk_b, sizeof(double) * c));
  const int64_t tk = (c / TOPK_CHUNK + 2) * TOPK;
  NB_CUDA(cudaMalloc((void**)&tk_key0, sizeof(unsigned long long) * tk));
  NB_CUDA(cudaMalloc((void**)&tk_key1, sizeof(unsigned long long) * tk));
  NB_CUDA(cudaMalloc((void**)&tk_idx0, sizeof(int32_t) * tk));
  NB_CUDA(cudaMalloc((void**)&tk_idx1, sizeof(int32_t) * tk));
  NB_CUDA(cudaMalloc((void**)&d_int, sizeof(int) * 16));
  NB_CUDA(cudaMalloc((void**)&d_i64, sizeof(int64_t) * 16));
  NB_CUDA(cudaMallocHost((void**)&h_int, sizeof(int) * 16));
  NB_CUDA(cudaMallocHost((void**)&h_i64, sizeof(int64_t) * 16));
  NB_CUDA(cudaMallocHost((void**)&h_dbl, sizeof(double) * 80));
  NB_CUDA(cudaMalloc((void**)&d_scal_i, sizeof(int64_t) * 16));
  d_scal = reinterpret_cast<double*>(d_scal_i + 8);
  NB_CUDA(cudaMallocHost((void**)&h_scal, sizeof(int64_t) * 16));
  cap = c;
  if (cache.cap < c) {
    if (cache.x_ref) cudaFree(cache.x_ref);
    if (cache.hs) cudaFree(cache.hs);
    NB_CUDA(cudaMalloc((void**)&cache.x_ref, sizeof(double) * 3 * c));
    NB_CUDA(cudaMalloc((void**)&cache.hs, sizeof(double) * c));
    cache.cap = c;
    cache.valid = false;
  }
  size_t need = cub_bytes_needed(c, 0);
  size_t a = 0;
  cub::DeviceRadixSort::SortPairsDescending((void*)nullptr, a, (double*)nullptr, (double*)nullptr,
                                            (int32_t*)nullptr, (int32_t*)nullptr, (int)c);
  size_t b = 0;
  cub::DeviceReduce::Min((void*)nullptr, b, (int64_t*)nullptr, (int64_t*)nullptr, (int)c);
  size_t d = 0;
  cub::DeviceReduce::Sum((void*)nullptr, d, (double*)nullptr, (double*)nullptr, (int)c);
  return E.ensure_cub(std::max(std::max(need, a), std::max(b, d)) + 4096);
}

int Workspace::ensure_grad(Engine& E, int64_t n) {
  if (n <= gcap && gvel) return 0;
  if (pk4) cudaFree(pk4);
  if (gvel) cudaFree(gvel);
  if (gvel32) cudaFree(gvel32);
  pk4 = nullptr;
  gvel = nullptr;
  gvel32 = nullptr;
  gcap = 0;
  const int64_t c = std::max<int64_t>(cap, n);
  NB_CUDA(cudaMalloc((void**)&pk4, sizeof(double4) * c));
  NB_CUDA(cudaMalloc((void**)&gvel, sizeof(double) * 9 * c));
  NB_CUDA(cudaMalloc((void**)&gvel32, sizeof(float) * 9 * c));
  gcap = c;
  return 0;
}

void Workspace::release() {
  void* ps[] = {pk4, gvel, gvel32, d_a, d_b, d_c, d_hg, d_hs, d_heff, d_hlim, d_disp, d_P, d_cs, d_vsig, d_ddudt,
                d_dm, d_tmp, d_uh, v_flow, v_pred, v_eval, v_dacc, v_tmp, pk0, pk1, pk2, pk3, pk32,
                pf1, pf2, pf3, m_x, m_sorted, m_smark, f_mass,
                rows, rows_s, rows2, iters, flags, need, i_tmp, pairs, i_lvl, i_tmp2, m_rows, m_done, m_need,
                m_tmp, i32a, i32b, dk_b, d_int, d_i64, tk_key0, tk_key1, tk_idx0, tk_idx1, d_scal_i};
  for (void* p : ps)
    if (p) cudaFree(p);
  if (h_int) cudaFreeHost(h_int);
  if (h_i64) cudaFreeHost(h_i64);
  if (h_dbl) cudaFreeHost(h_dbl);
  if (h_scal) cudaFreeHost(h_scal);
  *this = Workspace{cache};
}

// sum of a[rows] into E.ws.h_i64[0] (profiling only)
// profile: add a[rows] into the device counter of category `cat` (no host synchronisation)
__global__ void k_prof_sum_rows(int64_t nrows, const int64_t* __restrict__ rows,
                                const int64_t* __restrict__ a, unsigned long long* __restrict__ acc) {
  __shared__ unsigned long long s[NB_THREADS / 32];
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  unsigned long long v = q < nrows ? (unsigned long long)a[rows[q]] : 0ull;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < NB_THREADS / 32; ++w) t += s[w];
    atomicAdd(acc, t);
  }
}

static void prof_pairs(Engine& E, int cat, int64_t nrows, const int64_t* rows, const int64_t* a,
                       cudaStream_t st) {
  if (nrows <= 0 || E.prof.ensure() != 0) return;
  count_launch(), k_prof_sum_rows<<<grid_for(nrows), NB_THREADS, 0, st>>>(nrows, rows, a, E.prof.d_pairs + cat);
}

// The selection's count must equal the number of rows (the rows are distinct indices in
// [0, n)); otherwise flag an input error and fill the tail with a valid index, so no pass reads
// past the selected entries.
__global__ void k_rows_count_check(int64_t nrows, const int64_t* __restrict__ count,
                                   int64_t* __restrict__ rows_s, int* err) {
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t c = *count;
  if (q == 0 && c != nrows) set_error(err, ERR_BAD_INDEX);
  if (q < nrows && q >= c) rows_s[q] = c > 0 ? rows_s[0] : 0;
}

// The rows (caller order) as sorted positions in ascending curve order, into W.rows_s; the
// pair passes then walk neighbouring particles in neighbouring threads.  The rows are distinct
// (they come from a selection or are all particles), so their count is known without reading
// the selection's back; a mismatch is reported through the device error word.
static int rows_sorted(Engine& E, int64_t n, int64_t nrows, const int64_t* rows, int64_t* count,
                       cudaStream_t st) {
  Workspace& W = E.ws;
  const bool active = rows == W.rows;
  if (active && W.rs_ver == W.rows_ver && W.rs_gen == E.lists.gen && W.rs_n == nrows) {
    *count = W.rs_count;  // the active rows, sorted already on these lists
    return 0;
  }
  NB_CUDA(cudaMemsetAsync(W.m_x, 0, n, st));
  count_launch(), k_mask_rows<<<grid_for(nrows), NB_THREADS, 0, st>>>(nrows, rows, n, W.m_x, E.d_err);
  count_launch(), k_sorted_mask<<<grid_for(n), NB_THREADS, 0, st>>>(n, E.lists.perm, W.m_x, W.m_sorted);
  size_t tmp = E.cub_bytes;
  NB_CUDA(cub::DeviceSelect::Flagged(E.cub_tmp, tmp, thrust::counting_iterator<int64_t>(0), W.m_sorted,
                                     W.rows_s, W.d_i64 + 4, (int)n, st));
  count_launch(), k_rows_count_check<<<grid_for(nrows), NB_THREADS, 0, st>>>(nrows, W.d_i64 + 4, W.rows_s, E.d_err);
  W.pend_err = true;
  *count = nrows;
  W.rs_ver = active ? W.rows_ver : -1;
  W.rs_gen = E.lists.gen;
  W.rs_n = nrows;
  W.rs_count = *count;
  return 0;
}

// Pending checks: copy their device words next to the caller's own read (before its
// synchronisation), then act on them (after it).
int pending_enqueue(Engine& E, cudaStream_t st) {
  Workspace& W = E.ws;
  if (W.pend_err) NB_CUDA(cudaMemcpyAsync(E.h_err, E.d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  // the flow's worst iteration code (d_scal_i[0]), the wake-up count (d_scal_i[2]) and the
  // radiated energy (d_scal[0] = word 8 of the same allocation) in one copy
  if (W.pend_glf || W.pend_erad || W.pend_woken)
    NB_CUDA(cudaMemcpyAsync(W.h_scal, W.d_scal_i, sizeof(int64_t) * 9, cudaMemcpyDeviceToHost, st));
  return 0;
}

int pending_finish(Engine& E, cudaStream_t st) {
  Workspace& W = E.ws;
  if (W.pend_erad) {
    *W.pend_erad += reinterpret_cast<const double*>(W.h_scal)[8];
    W.pend_erad = nullptr;
  }
  if (W.pend_woken) {
    *W.pend_woken += W.h_scal[2];
    W.pend_woken = nullptr;
  }
  if (W.pend_glf) {
    W.pend_glf = false;
    int64_t worst = W.h_scal[0];
    if (worst < 0) {
      const char* msg = worst == -1   ? "stage 1 (p_half) did not converge in 10 iterations: time step too large"
                        : worst == -2 ? "stage 2 (x1) did not converge in 10 iterations: time step too large"
                                      : "particle inside r = 2.5";
      std::snprintf(E.last_error, sizeof(E.last_error), "%s", msg);
      W.pend_err = false;
      return worst == -1 ? NB_ERR_GLF_P_HALF : worst == -2 ? NB_ERR_GLF_X1 : NB_ERR_GLF_RADIUS;
    }
  }
  if (W.pend_err) {
    W.pend_err = false;
    if (E.h_err[0] != 0) return check_device_error(E, st);  // maps the code (and clears it)
  }
  return 0;
}

// the pending checks on their own (at the end of a step entry point)
int pending_flush(Engine& E, cudaStream_t st) {
  Workspace& W = E.ws;
  if (!W.pend_err && !W.pend_glf && !W.pend_erad && !W.pend_woken) return 0;
  NB_TRY(pending_enqueue(E, st));
  NB_CUDA(host_sync(st));
  return pending_finish(E, st);
}

static int read_int(Engine& E, int* d, int* out, cudaStream_t st) {
  NB_CUDA(cudaMemcpyAsync(E.ws.h_int, d, sizeof(int), cudaMemcpyDeviceToHost, st));
  NB_TRY(pending_enqueue(E, st));
  NB_CUDA(host_sync(st));
  *out = E.ws.h_int[0];
  return pending_finish(E, st);
}

// Density pass of `rows` on the current lists with the given search radii; results into the
// caller-order arrays h_out, rho, omega and the scratch flags/iters.
static int density_on_lists(Engine& E, int64_t n, const double* x, const double* mass,
                            const double* h_start, const double* h_search, int64_t nrows,
                            const int64_t* rows, const nb_params* prm, double* h_out,
                            double* rho, double* omega, cudaStream_t st) {
  Workspace& W = E.ws;
  Lists& L = E.lists;
  if (nrows == 0) return 0;
  int64_t ns = 0;
  NB_TRY(rows_sorted(E, n, nrows, rows, &ns, st));
  DensityParams dp{prm->kernel_id, prm->cnorm, prm->eta, prm->tol, prm->h_max};
  if (prm->precision == 1) {
    // grid over the box of the last list build (cells clamp to it; the edge is derived on the
    // device, so no host round trip)
    count_launch(), k_pack_density32<<<grid_for(n), NB_THREADS, 0, st>>>(
        n, L.perm, x, mass, h_start, h_search, E.bbox, W.d_a, W.d_b, W.d_c, W.pk32);
    E.prof.begin(st);
    launch_density32<int32_t>(nrows, W.rows_s, W.pk32, E.bbox, W.d_a, W.d_b, W.d_c, L.off,
                              L.idx, dp, L.perm, h_out, rho, omega, W.iters, W.flags,
                              E.prof.on ? W.pairs : nullptr, st);
  } else {
    count_launch(), k_gather_density<<<grid_for(n), NB_THREADS, 0, st>>>(
        n, L.perm, mass, h_start, h_search, W.d_a, W.d_b, W.d_c, nullptr);
    count_launch(), k_pack_sorted<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, x, nullptr, W.pk0);
    E.prof.begin(st);
    launch_density64<int32_t>(nrows, W.rows_s, W.pk0, W.d_a, W.d_b, W.d_c, L.off, L.idx, dp,
                              L.perm, h_out, rho, omega, W.iters, W.flags,
                              E.prof.on ? W.pairs : nullptr, st);
  }
  if (E.prof.on) {
    // kernel evaluations inside the support (pair evaluations summed over every Newton sum)
    E.prof.end(PROF_DENSITY, st, (double)nrows, 0.0);
    prof_pairs(E, PROF_DENSITY, nrows, rows, W.pairs, st);
  }
  NB_CUDA(cudaGetLastError());
  return 0;
}

// The first reuse test (no fast set: the largest displacement outside it is the largest of
// all, reduced into W.dk_b[0] by the displacement pass) for the rows of `mask`; its failure
// flag goes to *fail (zeroed here), read by the caller with its next round trip.  hg_in: the
// caller's h guesses, copied to W.d_hg for the tests and the solve (null: W.d_hg holds them).
int reuse_first_test(Engine& E, int64_t n, const double* x, const double* hg_in,
                     const uint8_t* mask, int* fail, cudaStream_t st) {
  Workspace& W = E.ws;
  Cache& C = W.cache;
  if (hg_in) NB_CUDA(cudaMemcpyAsync(W.d_hg, hg_in, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  NB_CUDA(cudaMemsetAsync(W.dk_b, 0, sizeof(double), st));
  count_launch(), k_disp<<<grid_for(n), NB_THREADS, 0, st>>>(n, x, C.x_ref, W.d_disp,
                                                            reinterpret_cast<unsigned long long*>(W.dk_b));
  NB_CUDA(cudaMemsetAsync(fail, 0, sizeof(int), st));
  count_launch(), k_reuse_test<<<grid_for(n), NB_THREADS, 0, st>>>(n, C.hs, W.d_disp, W.dk_b, W.d_hg, mask,
                                                   W.d_heff, W.d_hlim, fail);
  return 0;
}

// sim/sph.py:117-147 (_reuse_limits): returns 1 with W.d_heff filled if the cached lists are
// provably complete for the search limits h_eff, else 0.  first_fail: the first test's outcome
// when it ran already (reuse_first_test), -1 to run it here.
static int reuse_limits(Engine& E, int64_t n, const double* x, const uint8_t* mask,
                        int first_fail, int* ok, cudaStream_t st) {
  Workspace& W = E.ws;
  Cache& C = W.cache;
  *ok = 0;
  if (first_fail < 0) {
    NB_TRY(reuse_first_test(E, n, x, nullptr, mask, W.d_int, st));
    NB_TRY(read_int(E, W.d_int, &first_fail, st));
  }
  if (!first_fail) {
    *ok = 1;
    return 0;
  }
  // the largest displacements (descending; ties by index) into W.dk_b / W.i32b for the fast sets
  {
    int64_t count = n;
    unsigned long long *kin = nullptr, *kout = W.tk_key0;
    int32_t *iin = nullptr, *iout = W.tk_idx0;
    bool first = true;
    while (true) {
      int64_t nb = (count + TOPK_CHUNK - 1) / TOPK_CHUNK;
      if (first)
        count_launch(), k_topk<true><<<(unsigned)nb, 256, 0, st>>>(count, W.d_disp, nullptr, nullptr, kout, iout);
      else
        count_launch(), k_topk<false><<<(unsigned)nb, 256, 0, st>>>(count, nullptr, kin, iin, kout, iout);
      first = false;
      count = nb * TOPK;
      if (nb == 1) break;
      kin = kout;
      iin = iout;
      kout = (kout == W.tk_key0) ? W.tk_key1 : W.tk_key0;
      iout = (iout == W.tk_idx0) ? W.tk_idx1 : W.tk_idx0;
    }
    count_launch(), k_topk_out<<<1, 128, 0, st>>>((int)std::min<int64_t>(n, TOPK), kout, iout, W.dk_b, W.i32b);
  }
  int top = (int)std::min<int64_t>(n, TOPK);
  static const int FAST[] = {1, 2, 4, 8, 16, 32, 64};  // no fast set: tested above
  for (int nf : FAST) {
    if (nf >= top) break;
    NB_CUDA(cudaMemsetAsync(W.d_int, 0, sizeof(int), st));
    count_launch(), k_reuse_test<<<grid_for(n), NB_THREADS, 0, st>>>(n, C.hs, W.d_disp, W.dk_b + nf, W.d_hg, mask,
                                                     W.d_heff, W.d_hlim, W.d_int);
    int fail = 0;
    NB_TRY(read_int(E, W.d_int, &fail, st));
    if (fail) continue;
    NB_CUDA(cudaMemsetAsync(W.d_int, 0, sizeof(int), st));
    count_launch(), k_fast_complete<<<nf, NB_THREADS, 0, st>>>(n, nf, W.i32b, x, W.d_hlim, E.lists.inv_perm,
                                               E.lists.off, E.lists.idx, W.d_int);
    NB_TRY(read_int(E, W.d_int, &fail, st));
    if (!fail) {
      *ok = 1;
      return 0;
    }
  }
  return 0;
}

// sim/sph.py:329-387 (compute_density) for `rows` (caller order, W.rows is NOT used here): reuse
// the cached lists while provably complete, else rebuild with search h_guess * skin and double
// the search of rows whose root lies beyond it, up to 12 rounds.  h (in/out, caller order) is the
// guess for every particle; rows get their solved h, and rho / omega.
int compute_density(Engine& E, int64_t n, const double* x, const double* mass, double* h,
                    double* rho, double* omega, int64_t nrows, const int64_t* rows,
                    const nb_params* prm, int64_t* builds, int64_t* reuses, cudaStream_t st,
                    const uint8_t* rows_mask, int first_fail) {
  Workspace& W = E.ws;
  Cache& C = W.cache;
  NB_TRY(W.ensure(E, n));
  const uint8_t* mask = rows_mask;
  if (first_fail < 0) {
    NB_CUDA(cudaMemsetAsync(W.m_rows, 0, n, st));
    count_launch(), k_mask_rows<<<grid_for(nrows), NB_THREADS, 0, st>>>(nrows, rows, n, W.m_rows, E.d_err);
    NB_CUDA(cudaMemcpyAsync(W.d_hg, h, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    mask = W.m_rows;
  }
  if (C.valid && C.n == n && n > 0 && E.lists.n == n) {
    int ok = 0;
    NB_TRY(reuse_limits(E, n, x, mask, first_fail, &ok, st));
    if (ok) {
      NB_TRY(density_on_lists(E, n, x, mass, W.d_hg, W.d_heff, nrows, rows, prm, h, rho, omega, st));
      NB_CUDA(cudaMemsetAsync(W.d_int, 0, sizeof(int), st));
      count_launch(), k_count_flag2<<<grid_for(nrows), NB_THREADS, 0, st>>>(nrows, rows, W.flags, W.d_int);
      int grow_n = 0;
      W.pend_err = true;  // the density's error word comes back with the count
      NB_TRY(read_int(E, W.d_int, &grow_n, st));
      if (grow_n == 0) {
        *reuses += 1;
        return 0;
      }
      count_launch(), k_max_rows<<<grid_for(nrows), NB_THREADS, 0, st>>>(nrows, rows, h, W.d_hg);
    }
  }
  count_launch(), k_hsearch<<<grid_for(n), NB_THREADS, 0, st>>>(n, W.d_hg, prm->h_max, prm->skin, W.d_hs);
  for (int round = 0; round < 12; ++round) {
    NB_TRY(build_lists(E, n, x, W.d_hs, st));
    *builds += 1;
    NB_TRY(density_on_lists(E, n, x, mass, W.d_hg, W.d_hs, nrows, rows, prm, h, rho, omega, st));
    NB_CUDA(cudaMemsetAsync(W.d_int, 0, sizeof(int), st));
    count_launch(), k_grow<<<grid_for(nrows), NB_THREADS, 0, st>>>(nrows, rows, W.flags, h, W.d_hs, W.d_hg, W.d_int);
    int grow_n = 0;
    W.pend_err = true;  // the build's and the density's error word comes back with the count
    NB_TRY(read_int(E, W.d_int, &grow_n, st));
    if (grow_n == 0) {
      NB_CUDA(cudaMemcpyAsync(C.x_ref, x, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, st));
      NB_CUDA(cudaMemcpyAsync(C.hs, W.d_hs, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
      C.valid = true;
      C.n = n;
      return 0;
    }
  }
  std::snprintf(E.last_error, sizeof(E.last_error),
                "smoothing lengths kept outgrowing the neighbour search");
  return NB_ERR_SEARCH;
}

int mark_rows(Engine& E, int64_t nrows, const int64_t* rows, int tight, const double* x,
              const double* h, uint8_t* mark, cudaStream_t st) {
  if (nrows <= 0) return 0;
  Lists& L = E.lists;
  Workspace& W = E.ws;
  int64_t n = L.n, ns = 0;
  NB_TRY(rows_sorted(E, n, nrows, rows, &ns, st));
  if (tight) count_launch(), k_pack_sorted<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, x, h, W.pk0);
  if (nrows * 4 > n) {
    // most particles are rows: each particle looks for a row among its own entries (the lists
    // are symmetric) and stops at the first; W.m_sorted holds the rows' sorted mask
    count_launch(), k_mark_gather<<<grid_for(n * 8), NB_THREADS, 0, st>>>(n, L.off, L.idx, W.m_sorted, L.perm,
                                                                        tight, W.pk0, mark);
    return 0;
  }
  NB_CUDA(cudaMemsetAsync(W.m_smark, 0, n, st));
  count_launch(), k_mark_s<<<grid_for(ns * 8), NB_THREADS, 0, st>>>(ns, W.rows_s, L.off, L.idx, tight,
                                                               W.pk0, W.m_smark);
  count_launch(), k_unsort_marks<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, W.m_smark, mark);
  return 0;
}

int sorted_rows(Engine& E, int64_t nrows, const int64_t* rows, int64_t* ns, cudaStream_t st) {
  return rows_sorted(E, E.lists.n, nrows, rows, ns, st);
}

int sorted_rows_and_pack(Engine& E, int64_t nrows, const int64_t* rows, const double* x,
                         const double* h, int64_t* ns, cudaStream_t st) {
  Lists& L = E.lists;
  Workspace& W = E.ws;
  int64_t n = L.n;
  NB_TRY(rows_sorted(E, n, nrows, rows, ns, st));
  count_launch(), k_pack_sorted<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, x, h, W.pk0);
  return 0;
}

void mask_and_not(int64_t n, const uint8_t* a, const uint8_t* b, uint8_t* out, cudaStream_t st) {
  if (n > 0) count_launch(), k_mask_and_not<<<grid_for(n), NB_THREADS, 0, st>>>(n, a, b, out);
}

void mask_or(int64_t n, const uint8_t* a, uint8_t* b, cudaStream_t st) {
  if (n > 0) count_launch(), k_mask_or<<<grid_for(n), NB_THREADS, 0, st>>>(n, a, b);
}

int select_mask(Engine& E, int64_t n, const uint8_t* mask, int64_t* out, int64_t* count,
                cudaStream_t st, int64_t* also) {
  Workspace& W = E.ws;
  size_t tmp = E.cub_bytes;
  NB_CUDA(cub::DeviceSelect::Flagged(E.cub_tmp, tmp, thrust::counting_iterator<int64_t>(0), mask, out,
                                     W.d_i64, (int)n, st));
  // the count, and W.d_i64[1] when the caller left a value there to read with it
  NB_CUDA(cudaMemcpyAsync(W.h_i64, W.d_i64, sizeof(int64_t) * (also ? 2 : 1), cudaMemcpyDeviceToHost, st));
  NB_TRY(pending_enqueue(E, st));
  NB_CUDA(host_sync(st));
  *count = W.h_i64[0];
  if (also) *also = W.h_i64[1];
  return pending_finish(E, st);
}

// Fused EOS + force pass for `rows` (caller order) with interacting pairs only (the tightened
// lists of sim/neighbours.py:284-323, tested on the fly).  Writes a_hydro, dudt, vsig_max,
// visc_heating (and nu) at the rows.  P and c_s go to W.d_P / W.d_cs: for every particle with the
// ideal gas, and with an iterative EOS for the particles of `touched` (every particle when null),
// a superset of the rows and their interacting neighbours.
int engine_forces(Engine& E, nb_state* s, const double* vel, const double* u, int64_t nrows,
                  const int64_t* rows, const nb_params* prm, const uint8_t* touched,
                  const ShockStep& sk, cudaStream_t st) {
  Workspace& W = E.ws;
  Lists& L = E.lists;
  int64_t n = s->n;
  const uint8_t* eos_mask = prm->eos == 0 ? nullptr : touched;
  E.prof.begin(st);
  count_launch(), k_eos<<<grid_for(n), NB_THREADS, 0, st>>>(n, s->rho, u, eos_mask, eos_of(prm), W.d_P, W.d_cs, E.d_err);
  E.prof.end(PROF_EOS, st, (double)n, 0.0);
  W.pend_err = true;  // the EOS's and the force pass's error word, read at the step's end
  if (nrows == 0) return 0;
  int64_t ns = 0;
  NB_TRY(rows_sorted(E, n, nrows, rows, &ns, st));
  const bool sw_on = prm->viscosity && prm->visc_switch && sk.switch_on;
  const bool recon = prm->viscosity && prm->recon;
  // FP32 without the switch and the reconstruction: every sorted input in one pass below, for
  // the touched particles only when they hold every list entry of the rows and are few
  const bool fused_pack = prm->precision == 1 && !sw_on && !recon;
  const bool sparse_pack = fused_pack && touched && sk.touched_covers_lists && nrows * 8 < n;
  if (prm->precision == 1 && !fused_pack) {
    count_launch(), k_pack_sorted_f4<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, vel, s->mass, nullptr, nullptr, 1, W.pf1);
    count_launch(), k_pack_sorted_f4<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, s->h, s->rho, s->omega, W.d_P, 0, W.pf2);
  }
  if (prm->precision != 1 || sw_on || recon) {
    // FP64 packs (the FP32 form needs them only for the gradient passes)
    count_launch(), k_pack_sorted<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, vel, s->mass, W.pk1);
    count_launch(), k_pack_sorted4<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, s->h, s->rho, s->omega, W.d_P, W.pk2);
  }
  if (sw_on || recon) {
    NB_TRY(W.ensure_grad(E, n));
    count_launch(), k_pack_sorted<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, s->x, s->h, W.pk0);
  }
  if (sw_on || recon) {
    // Cullen-Dehnen switch (sim/blocks.py:261-266, sim/coupled.py:159-162): corrected gradients
    // of the rows over their interacting pairs with the previous accelerations, then alpha of
    // the rows advanced over their step; velocity gradients for the reconstruction: block
    // steps, every touched particle over its untightened cached list (sim/blocks.py:271-278),
    // shared steps, every particle over its interacting pairs (sim/coupled.py:164-168).  One
    // pass for both; W.m_sorted holds the rows' sorted mask (rows_sorted above).
    if (sw_on)
      count_launch(), k_pack_sorted<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, s->a_hydro, nullptr, W.pk4);
    GradOut go;
    go.gv = W.gvel;
    go.alpha = s->alpha;
    go.cs = W.d_cs;
    go.h = s->h;
    go.dt = sk.dt;
    go.n_beg = sk.n_beg;
    go.n_end = sk.n_end;
    go.tick = sk.tick;
    E.prof.begin(st);
    launch_shock_gradients(n, W.pk0, W.pk1, W.pk2, W.pk4, L.off, L.idx, prm->kernel_id,
                           prm->cnorm, recon ? 1 : 0, sk.recon_full,
                           sk.recon_full ? touched : nullptr, sw_on ? W.m_sorted : nullptr,
                           L.perm, go, st);
    E.prof.end(PROF_GRAD, st, (double)n, 0.0);
    if (recon && prm->precision == 1)
      count_launch(), k_to_float<<<grid_for(9 * n), NB_THREADS, 0, st>>>(9 * n, W.gvel, W.gvel32);
  }
  if (prm->precision == 1) {
    if (!fused_pack)
      count_launch(), k_pack_sorted_f4<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, u, W.d_cs, s->alpha, nullptr, 0, W.pf3);
  } else
    count_launch(), k_pack_sorted4<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, u, W.d_cs, s->alpha, nullptr, W.pk3);
  ForceParams fp{};
  fp.kid = prm->kernel_id;
  fp.cnorm = prm->cnorm;
  fp.use_sph = 1;
  fp.use_visc = prm->viscosity;
  fp.use_cond = prm->viscosity && prm->conductivity;
  fp.cond_signal = prm->cond_signal;
  fp.beta = prm->beta;
  fp.alpha_u = prm->alpha_u;
  fp.use_disc = prm->disc_alpha_av > 0;
  fp.disc_alpha_av = prm->disc_alpha_av;
  fp.tighten = 1;
  const bool want_tight = sk.want_tight && prm->limiter && rows == W.rows;
  W.tight_ver = -1;
  // the FP32 form without the reconstruction walks the lists in a launch of its own that writes
  // the interacting entries, and sums the pairs from them in a second launch (they are also
  // the limiter's entries when it wants them, decided exactly in the FP32 test's band)
  const bool split = prm->precision == 1 && !recon;
  if (want_tight || split) {
    NB_TRY(E.ensure_tight(L.total));
    fp.tidx = E.tidx;
    fp.tcnt = W.i32a;
  }
  if (want_tight && prm->precision == 1) {
    if (!fused_pack) count_launch(), k_pack_sorted<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, s->x, s->h, W.pk0);
    fp.pos64 = W.pk0;
  }
  if (recon) {
    fp.use_recon = 1;
    fp.closeness = prm->recon_closeness;
    fp.gate = prm->recon_gate;
    fp.eta_crit = prm->recon_eta_crit;
    fp.eta_fold = prm->recon_eta_fold;
    fp.gv64 = W.gvel;
    fp.gv32 = W.gvel32;
  }
  ForceOut fo;
  fo.acc = s->a_hydro;
  fo.dudt = s->dudt;
  fo.vsig = W.d_vsig;
  fo.vheat = s->visc_heating;
  fo.cheat = s->cond_heating;
  fo.dacc = W.v_dacc;
  fo.ddudt = W.d_ddudt;
  fo.pairs = W.pairs;
  if (prm->precision == 1) {
    if (fused_pack)
      count_launch(), k_pack_force32<<<grid_for(n), NB_THREADS, 0, st>>>(
          n, L.perm, s->x, s->mass, s->h, E.bbox, vel, s->rho, s->omega, W.d_P, u, W.d_cs, s->alpha,
          sparse_pack ? touched : nullptr, W.pk32, W.pf1, W.pf2, W.pf3, want_tight ? W.pk0 : nullptr);
    else
      count_launch(), k_pack_sorted32<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, s->x, s->mass, s->h, E.bbox, W.pk32);
    E.prof.begin(st);
    launch_forces32<int32_t>(nrows, W.rows_s, W.pk32, E.bbox, W.pf1, W.pf2, W.pf3, L.off,
                             L.idx, fp, L.perm, fo, st);
  } else {
    count_launch(), k_pack_sorted<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, s->x, nullptr, W.pk0);
    E.prof.begin(st);
    launch_forces64<int32_t>(nrows, W.rows_s, W.pk0, W.pk1, W.pk2, W.pk3, L.off, L.idx, fp,
                             L.perm, fo, st);
  }
  if (want_tight) {
    W.tight_ver = W.rows_ver;
    W.tight_gen = L.gen;
    W.tight_n = nrows;
  }
  if (E.prof.on) {
    E.prof.end(PROF_FORCES, st, (double)nrows, 0.0);
    // interacting pairs of the rows (written per row by the kernel)
    prof_pairs(E, PROF_FORCES, nrows, rows, W.pairs, st);
  }
  count_launch(), k_combine_rows<<<grid_for(nrows), NB_THREADS, 0, st>>>(
      nrows, rows, prm->viscosity, prm->disc_alpha_av, W.v_dacc, W.d_ddudt, W.d_cs, s->h,
      W.d_vsig, s->a_hydro, s->dudt, s->vsig_max, s->nu, s->disk_heating);
  NB_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace nbk
