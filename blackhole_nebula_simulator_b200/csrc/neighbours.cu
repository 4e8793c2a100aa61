// Neighbour lists on the GPU: particles sorted along a Hilbert curve, an implicit 8-ary tree of boxes over
// leaves of 32 consecutive sorted particles, and a warp-per-leaf traversal that writes exact
// symmetric lists.
//
// The set is the reference's (sim/neighbours.py:240-281, find_neighbours_numba):
//     N(i) = { j : r_ij^2 < (2 h_i)^2  or  r_ij^2 < (2 h_j)^2 },  i itself included,
// with r_ij^2 = dx*dx + dy*dy + dz*dz, dx = x_j - x_i, evaluated in double with the reference's
// rounding (no fused multiply-add), so the lists are identical bit for bit.  The tree only
// prunes: a node is skipped when the distance between its box and the query leaf's box is at
// least 2 max(h_query_max, h_node_max) (with a 1e-12 relative margin on the safe side), which
// can never drop a pair the test above accepts.
//
// Rows come out in sorted (curve) order with each row's entries in ascending sorted index.
#include <cub/cub.cuh>

#include "common.cuh"
#include "engine.cuh"

namespace nbk {

static constexpr int LEAF = 32;
static constexpr int SUB = 8;  // sub-leaf: the unit each lane tests its own sphere against
static constexpr int FAN = 8;
static constexpr int STACK = 96;
static constexpr int QCAP = 24;  // sub-leaves a lane queues before the warp flushes
// entries of the fixed-width row scratch of the one-pass build (int32, 24 GiB); larger builds
// count first and fill second
static constexpr double ELL_MAX_ENTRIES = 6.0 * 1024 * 1024 * 1024;

// ---------------------------------------------------------------- bounding box
__global__ void k_bbox_partial(int64_t n, const double* __restrict__ pos, double* __restrict__ part) {
  __shared__ double s[6][NB_THREADS];
  double mn[3] = {1e308, 1e308, 1e308}, mx[3] = {-1e308, -1e308, -1e308};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    for (int c = 0; c < 3; ++c) {
      double v = pos[3 * i + c];
      mn[c] = fmin(mn[c], v);
      mx[c] = fmax(mx[c], v);
    }
  }
  for (int c = 0; c < 3; ++c) {
    s[c][threadIdx.x] = mn[c];
    s[3 + c][threadIdx.x] = mx[c];
  }
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int c = 0; c < 3; ++c) {
        s[c][threadIdx.x] = fmin(s[c][threadIdx.x], s[c][threadIdx.x + w]);
        s[3 + c][threadIdx.x] = fmax(s[3 + c][threadIdx.x], s[3 + c][threadIdx.x + w]);
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < 6; ++c) part[6 * blockIdx.x + c] = s[c][0];
}

__global__ void k_bbox_final(int nb, const double* __restrict__ part, double* __restrict__ box6) {
  __shared__ double s[6][NB_THREADS];
  double r[6] = {1e308, 1e308, 1e308, -1e308, -1e308, -1e308};
  for (int b = threadIdx.x; b < nb; b += blockDim.x)
    for (int c = 0; c < 3; ++c) {
      r[c] = fmin(r[c], part[6 * b + c]);
      r[3 + c] = fmax(r[3 + c], part[6 * b + 3 + c]);
    }
  for (int c = 0; c < 6; ++c) s[c][threadIdx.x] = r[c];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int c = 0; c < 3; ++c) {
        s[c][threadIdx.x] = fmin(s[c][threadIdx.x], s[c][threadIdx.x + w]);
        s[3 + c][threadIdx.x] = fmax(s[3 + c][threadIdx.x], s[3 + c][threadIdx.x + w]);
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < 6; ++c) box6[c] = s[c][0];
}

// ---------------------------------------------------------------- curve keys
__device__ __forceinline__ uint64_t spread21(uint64_t v) {
  v &= 0x1fffffull;
  v = (v | (v << 32)) & 0x1f00000000ffffull;
  v = (v | (v << 16)) & 0x1f0000ff0000ffull;
  v = (v | (v << 8)) & 0x100f00f00f00f00full;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}

// Hilbert index of a point on the 2^21 grid over the bounding box: J. Skilling's transform
// ("Programming the Hilbert curve", AIP Conf. Proc. 707, 2004) from axes to the transposed
// index, then the three coordinates' bits interleaved (first axis most significant).  Runs of
// consecutive particles along the Hilbert curve have tighter boxes than Morton runs (fewer jumps
// between distant octants), so leaves and sub-leaves prune better.
__device__ __forceinline__ uint64_t hilbert_key(uint32_t x0, uint32_t x1, uint32_t x2) {
  uint32_t X[3] = {x0, x1, x2};
  const uint32_t M = 1u << 20;
  for (uint32_t Q = M; Q > 1; Q >>= 1) {
    const uint32_t P = Q - 1;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      if (X[i] & Q) {
        X[0] ^= P;  // invert the low bits of the first axis
      } else {
        uint32_t t = (X[0] ^ X[i]) & P;  // exchange the low bits of axes 0 and i
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  X[1] ^= X[0];  // Gray encode
  X[2] ^= X[1];
  uint32_t t = 0;
  for (uint32_t Q = M; Q > 1; Q >>= 1)
    if (X[2] & Q) t ^= Q - 1;
  X[0] ^= t;
  X[1] ^= t;
  X[2] ^= t;
  return (spread21(X[0]) << 2) | (spread21(X[1]) << 1) | spread21(X[2]);
}

__global__ void k_curve_keys(int64_t n, const double* __restrict__ pos,
                             const double* __restrict__ box6, uint64_t* __restrict__ keys,
                             int32_t* __restrict__ vals) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double span = fmax(fmax(box6[3] - box6[0], box6[4] - box6[1]), box6[5] - box6[2]);
  double scale = span > 0 ? 2097151.0 / span : 0.0;
  uint32_t q[3];
  for (int c = 0; c < 3; ++c) {
    double t = (pos[3 * i + c] - box6[c]) * scale;
    t = fmin(fmax(t, 0.0), 2097151.0);
    q[c] = (uint32_t)t;
  }
  keys[i] = hilbert_key(q[0], q[1], q[2]);
  vals[i] = (int32_t)i;
}

__global__ void k_gather_sorted(int64_t n, const int32_t* __restrict__ perm,
                                const double* __restrict__ pos, const double* __restrict__ hs,
                                double4* __restrict__ spos, int32_t* __restrict__ inv_perm) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  int32_t i = perm[k];
  spos[k] = make_double4(pos[3 * (int64_t)i], pos[3 * (int64_t)i + 1], pos[3 * (int64_t)i + 2], hs[i]);
  inv_perm[i] = (int32_t)k;
}

// ---------------------------------------------------------------- tree of boxes
__global__ void k_leaf_boxes(int64_t n, int64_t nleaf, const double4* __restrict__ spos,
                             double4* __restrict__ lo, double4* __restrict__ hi) {
  int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (l >= nleaf) return;
  int64_t a = l * LEAF, b = min(a + LEAF, n);
  double4 mn = make_double4(1e308, 1e308, 1e308, 0.0), mx = make_double4(-1e308, -1e308, -1e308, 0.0);
  for (int64_t k = a; k < b; ++k) {
    double4 p = spos[k];
    mn.x = fmin(mn.x, p.x);
    mn.y = fmin(mn.y, p.y);
    mn.z = fmin(mn.z, p.z);
    mx.x = fmax(mx.x, p.x);
    mx.y = fmax(mx.y, p.y);
    mx.z = fmax(mx.z, p.z);
    mn.w = fmax(mn.w, p.w);  // lo.w carries the largest h of the node
  }
  lo[l] = mn;
  hi[l] = mx;
}

// Boxes (and largest h) of the sub-leaves of SUB consecutive sorted particles.
__global__ void k_sub_boxes(int64_t n, int64_t nsub, const double4* __restrict__ spos,
                            double4* __restrict__ lo, double4* __restrict__ hi) {
  int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (l >= nsub) return;
  int64_t a = l * SUB, b = min(a + SUB, n);
  double4 mn = make_double4(1e308, 1e308, 1e308, 0.0), mx = make_double4(-1e308, -1e308, -1e308, 0.0);
  for (int64_t k = a; k < b; ++k) {
    double4 p = spos[k];
    mn.x = fmin(mn.x, p.x);
    mn.y = fmin(mn.y, p.y);
    mn.z = fmin(mn.z, p.z);
    mx.x = fmax(mx.x, p.x);
    mx.y = fmax(mx.y, p.y);
    mx.z = fmax(mx.z, p.z);
    mn.w = fmax(mn.w, p.w);
  }
  lo[l] = mn;
  hi[l] = mx;
}

__global__ void k_level_up(int64_t nchild, int64_t nparent, const double4* __restrict__ clo,
                           const double4* __restrict__ chi, double4* __restrict__ plo,
                           double4* __restrict__ phi) {
  int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= nparent) return;
  double4 mn = make_double4(1e308, 1e308, 1e308, 0.0), mx = make_double4(-1e308, -1e308, -1e308, 0.0);
  for (int64_t c = p * FAN; c < min((p + 1) * FAN, nchild); ++c) {
    double4 a = clo[c], b = chi[c];
    mn.x = fmin(mn.x, a.x);
    mn.y = fmin(mn.y, a.y);
    mn.z = fmin(mn.z, a.z);
    mn.w = fmax(mn.w, a.w);
    mx.x = fmax(mx.x, b.x);
    mx.y = fmax(mx.y, b.y);
    mx.z = fmax(mx.z, b.z);
  }
  plo[p] = mn;
  phi[p] = mx;
}

struct TreeView {
  const double4* lo;
  const double4* hi;
  int64_t level_off[MAX_LEVELS + 1];
  int64_t level_size[MAX_LEVELS];
  int nlevels;
};

__device__ __forceinline__ double box_gap2(double4 alo, double4 ahi, double4 blo, double4 bhi) {
  double gx = fmax(fmax(blo.x - ahi.x, alo.x - bhi.x), 0.0);
  double gy = fmax(fmax(blo.y - ahi.y, alo.y - bhi.y), 0.0);
  double gz = fmax(fmax(blo.z - ahi.z, alo.z - bhi.z), 0.0);
  return gx * gx + gy * gy + gz * gz;
}

__device__ __forceinline__ double point_gap2(double x, double y, double z, double4 blo, double4 bhi) {
  double gx = fmax(fmax(blo.x - x, x - bhi.x), 0.0);
  double gy = fmax(fmax(blo.y - y, y - bhi.y), 0.0);
  double gz = fmax(fmax(blo.z - z, z - bhi.z), 0.0);
  return gx * gx + gy * gy + gz * gz;
}

// The rows of one query leaf of LEAF consecutive sorted particles, one lane per particle.  The
// warp walks the tree of boxes with an explicit stack in shared memory (entries (level << 40) |
// index; children pushed highest first, so candidate leaves are reached in ascending order).  At
// each candidate leaf every lane tests its own search sphere against the leaf's sub-leaves and
// queues the ones it reaches (shared memory, per lane, in ascending order); the warp flushes the
// queues in lockstep, each lane walking its own sub-leaves' particles, so every row comes out
// sorted.
// PASS 0 counts each row's entries; PASS 1 writes them at off[k]; PASS 2 writes them into a
// fixed-width slot of row_cap entries at k * row_cap and counts them.  Returns the row length.
template <int PASS>
__device__ __forceinline__ int64_t leaf_rows(int64_t leaf, int64_t n, const TreeView& tv,
                                             const double4* __restrict__ slo,
                                             const double4* __restrict__ shi,
                                             const double4* __restrict__ spos,
                                             int64_t* __restrict__ counts,
                                             const int64_t* __restrict__ off,
                                             int32_t* __restrict__ idx, int64_t row_cap,
                                             int64_t* stack, int32_t (*queue)[32], int lane,
                                             int* err) {
  int64_t k = leaf * LEAF + lane;
  bool valid = k < n;
  double4 me = valid ? spos[k] : make_double4(0, 0, 0, 0);
  double ri = 2.0 * me.w;
  double r2i = __dmul_rn(ri, ri);
  const double4 qlo = tv.lo[leaf], qhi = tv.hi[leaf];
  const double qh = qlo.w;
  int64_t m = 0, base = 0, cap = 0;
  if (PASS == 1 && valid) {
    base = off[k];
    cap = off[k + 1] - base;
  }
  if (PASS == 2) {
    base = k * row_cap;
    cap = row_cap;
  }
  int qn = 0;  // this lane's queued sub-leaves
  auto flush = [&]() {
    int qmax = qn;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) qmax = max(qmax, __shfl_xor_sync(0xffffffffu, qmax, o));
    for (int t = 0; t < qmax; ++t) {
      if (t < qn) {
        int64_t sb = (int64_t)queue[t][lane] * SUB;
        int64_t se = min(sb + SUB, n);
        for (int64_t j = sb; j < se; ++j) {
          double4 c = spos[j];
          double d2 = d2_exact(c.x - me.x, c.y - me.y, c.z - me.z);
          double rj = 2.0 * c.w;
          if (d2 < r2i || d2 < __dmul_rn(rj, rj)) {
            if (PASS == 1) {
              if (m < cap)
                idx[base + m] = (int32_t)j;
              else
                set_error(err, ERR_LIST_OVERFLOW);
            } else if (PASS == 2) {
              if (m < cap) idx[base + m] = (int32_t)j;  // longer rows are redone in CSR
            }
            m += 1;
          }
        }
      }
    }
    __syncwarp();
    qn = 0;
  };
  int sp = 0;
  __syncwarp();
  if (lane == 0) stack[0] = ((int64_t)(tv.nlevels - 1) << 40);
  sp = 1;
  __syncwarp();
  while (sp > 0) {
    int64_t e = stack[sp - 1];
    __syncwarp();
    sp -= 1;
    int lvl = (int)(e >> 40);
    int64_t node = e & ((1ll << 40) - 1);
    if (lvl == 0) {
      // candidate leaf: queue the sub-leaves this lane's sphere reaches
      int64_t s0 = node * (LEAF / SUB);
      int64_t s1 = min(s0 + LEAF / SUB, (n + SUB - 1) / SUB);
      bool near = valid;
      if (near) {
        // the leaf's own box first: a lane whose sphere misses it skips the sub-leaf tests
        const double4 llo = tv.lo[node], lhi = tv.hi[node];
        const double lreach = 2.0 * fmax(me.w, llo.w);
        near = point_gap2(me.x, me.y, me.z, llo, lhi) < lreach * lreach * (1.0 + 1e-12);
      }
      if (near) {
        for (int64_t sidx = s0; sidx < s1; ++sidx) {
          double4 blo = slo[sidx], bhi = shi[sidx];
          double reach = 2.0 * fmax(me.w, blo.w);
          if (point_gap2(me.x, me.y, me.z, blo, bhi) < reach * reach * (1.0 + 1e-12))
            queue[qn++][lane] = (int32_t)sidx;
        }
      }
      if (__any_sync(0xffffffffu, qn > QCAP - LEAF / SUB)) flush();
      continue;
    }
    int64_t c0 = node * FAN;
    int64_t csize = tv.level_size[lvl - 1];
    int64_t child = c0 + lane;
    bool hit = false;
    if (lane < FAN && child < csize) {
      int64_t g = tv.level_off[lvl - 1] + child;
      double4 blo = tv.lo[g], bhi = tv.hi[g];
      double reach = 2.0 * fmax(qh, blo.w);
      hit = box_gap2(qlo, qhi, blo, bhi) < reach * reach * (1.0 + 1e-12);
    }
    unsigned mask = __ballot_sync(0xffffffffu, hit);
    int nh = __popc(mask);
    if (sp + nh > STACK) {
      set_error(err, ERR_TRAVERSAL_STACK);
      break;
    }
    if (hit) {
      int above = __popc(mask & ~((2u << lane) - 1u));
      stack[sp + above] = ((int64_t)(lvl - 1) << 40) | child;
    }
    __syncwarp();
    sp += nh;
  }
  flush();
  if (PASS != 1 && valid) counts[k] = m;
  return valid ? m : 0;
}

// Persistent list kernel: each warp takes the next query leaf from `order` (heaviest first) until
// none is left, so a few slow leaves (sparse regions whose 32 curve-consecutive particles spread
// far) overlap with the rest instead of holding whole blocks.  PASS 2 also records the longest
// row in *rowmax.
template <int PASS>
__global__ void __launch_bounds__(NB_THREADS) k_lists_sub(int64_t n, int64_t nwork,
                                                          const int32_t* __restrict__ order,
                                                          unsigned long long* __restrict__ next,
                                                          TreeView tv,
                                                          const double4* __restrict__ slo,
                                                          const double4* __restrict__ shi,
                                                          const double4* __restrict__ spos,
                                                          int64_t* __restrict__ counts,
                                                          const int64_t* __restrict__ off,
                                                          int32_t* __restrict__ idx,
                                                          int64_t row_cap,
                                                          unsigned long long* __restrict__ rowmax,
                                                          int* err) {
  __shared__ int64_t stack_s[NB_THREADS / 32][STACK];
  __shared__ int32_t queue_s[NB_THREADS / 32][QCAP][32];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  int64_t* stack = stack_s[wib];
  int32_t(*queue)[32] = queue_s[wib];
  unsigned longest = 0;
  while (true) {
    unsigned long long w = 0;
    if (lane == 0) w = atomicAdd(next, 1ull);
    w = __shfl_sync(0xffffffffu, w, 0);
    if (w >= (unsigned long long)nwork) break;  // warp-uniform
    int64_t leaf = order[w];
    int64_t m = leaf_rows<PASS>(leaf, n, tv, slo, shi, spos, counts, off, idx, row_cap, stack,
                                queue, lane, err);
    longest = max(longest, (unsigned)m);
  }
  if (PASS == 2) {
    unsigned mx = __reduce_max_sync(0xffffffffu, longest);
    if (lane == 0) atomicMax(rowmax, (unsigned long long)mx);
  }
}

// Cost key of each query leaf for the heaviest-first order: the linear size of the region its
// traversal covers (box extent plus twice the largest search diameter), as descending-order bits.
__global__ void k_leaf_cost(int64_t nleaf, const double4* __restrict__ lo,
                            const double4* __restrict__ hi, uint32_t* __restrict__ key,
                            int32_t* __restrict__ id) {
  int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (l >= nleaf) return;
  double4 a = lo[l], b = hi[l];
  double ext = fmax(fmax(b.x - a.x, b.y - a.y), b.z - a.z);
  float c = (float)(ext + 4.0 * a.w);
  key[l] = ~__float_as_uint(c);  // non-negative floats order like their bits
  id[l] = (int32_t)l;
}

// Pack the fixed-width rows into CSR: warp per row, coalesced on both sides.  Rows longer than
// the width are left to the CSR pass over their leaves.
__global__ void k_pack_rows(int64_t n, int64_t row_cap, const int32_t* __restrict__ ell,
                            const int64_t* __restrict__ off, int32_t* __restrict__ idx) {
  int64_t k = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (k >= n) return;
  int64_t b = off[k], cnt = off[k + 1] - b;
  if (cnt > row_cap) return;
  const int32_t* src = ell + k * row_cap;
  for (int64_t t = lane; t < cnt; t += 32) idx[b + t] = src[t];
}

// Leaves holding a row longer than the width (unordered list; each is redone on its own).
__global__ void k_long_leaves(int64_t n, int64_t nleaf, const int64_t* __restrict__ counts,
                              int64_t row_cap, int32_t* __restrict__ out,
                              unsigned long long* __restrict__ nout) {
  int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (l >= nleaf) return;
  bool longer = false;
  for (int64_t k = l * LEAF; k < min((l + 1) * LEAF, n); ++k) longer |= counts[k] > row_cap;
  if (longer) out[atomicAdd(nout, 1ull)] = (int32_t)l;
}

// ---------------------------------------------------------------- export to original order
__global__ void k_export_counts(int64_t n, const int32_t* __restrict__ inv_perm,
                                const int64_t* __restrict__ off_s, int64_t* __restrict__ cnt_o) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int32_t k = inv_perm[i];
  cnt_o[i] = off_s[k + 1] - off_s[k];
}

__global__ void k_export_fill(int64_t n, const int32_t* __restrict__ perm,
                              const int64_t* __restrict__ off_s, const int32_t* __restrict__ idx_s,
                              const int64_t* __restrict__ off_o, int64_t* __restrict__ idx_o) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  int64_t i = perm[k];
  int64_t dst = off_o[i];
  for (int64_t e = off_s[k]; e < off_s[k + 1]; ++e) idx_o[dst++] = perm[idx_s[e]];
}

// ---------------------------------------------------------------- host orchestration
// Resident blocks of the persistent list kernel over the whole device (fewest of its variants).
static int list_kernel_slots(Engine& E) {
  if (E.list_slots > 0) return 0;
  int sms = 0, b0 = 0, b1 = 0, b2 = 0;
  NB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, E.device));
  NB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b0, k_lists_sub<0>, NB_THREADS, 0));
  NB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_lists_sub<1>, NB_THREADS, 0));
  NB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2, k_lists_sub<2>, NB_THREADS, 0));
  E.list_slots = (int64_t)sms * std::max(1, std::min(b0, std::min(b1, b2)));
  return 0;
}
int build_lists(Engine& E, int64_t n, const double* pos, const double* hs, cudaStream_t st) {
  NB_TRY(E.ensure_n(n));
  if (n == 0) {
    E.lists.n = 0;
    E.lists.total = 0;
    NB_CUDA(cudaMemsetAsync(E.lists.off, 0, sizeof(int64_t), st));
    return 0;
  }
  Lists& L = E.lists;
  L.gen += 1;
  E.prof.begin(st);
  // bounding box and Hilbert keys
  int nbb = (int)std::min<int64_t>(grid_for(n), 1184);
  count_launch(), k_bbox_partial<<<nbb, NB_THREADS, 0, st>>>(n, pos, E.bbox_part);
  count_launch(), k_bbox_final<<<1, NB_THREADS, 0, st>>>(nbb, E.bbox_part, E.bbox);
  count_launch(), k_curve_keys<<<grid_for(n), NB_THREADS, 0, st>>>(n, pos, E.bbox, E.keys_a, E.vals_a);
  // the top 48 of the 63 key bits (2^16 cells per axis over the box; within a cell the caller's
  // order): six radix passes instead of eight, and the leaves stay as compact
  size_t tmp = E.cub_bytes;
  NB_CUDA(cub::DeviceRadixSort::SortPairs(E.cub_tmp, tmp, E.keys_a, E.keys_b, E.vals_a, L.perm,
                                          (int)n, 15, 63, st));
  count_launch(), k_gather_sorted<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, pos, hs, L.spos, L.inv_perm);
  // tree
  int64_t nleaf = (n + LEAF - 1) / LEAF;
  TreeView tv;
  int64_t size = nleaf, offs = 0;
  int nl = 0;
  while (true) {
    tv.level_off[nl] = offs;
    tv.level_size[nl] = size;
    offs += size;
    nl += 1;
    if (size == 1 || nl == MAX_LEVELS) break;
    size = (size + FAN - 1) / FAN;
  }
  tv.level_off[nl] = offs;
  tv.nlevels = nl;
  if (tv.level_size[nl - 1] != 1) return set_host_error(E, "tree deeper than MAX_LEVELS");
  NB_TRY(E.ensure_nodes(offs));
  count_launch(), k_leaf_boxes<<<grid_for(nleaf), NB_THREADS, 0, st>>>(n, nleaf, L.spos, E.node_lo, E.node_hi);
  for (int l = 1; l < nl; ++l)
    count_launch(), k_level_up<<<grid_for(tv.level_size[l]), NB_THREADS, 0, st>>>(
        tv.level_size[l - 1], tv.level_size[l], E.node_lo + tv.level_off[l - 1],
        E.node_hi + tv.level_off[l - 1], E.node_lo + tv.level_off[l], E.node_hi + tv.level_off[l]);
  tv.lo = E.node_lo;
  tv.hi = E.node_hi;
  int64_t nsub = (n + SUB - 1) / SUB;
  NB_TRY(E.ensure_sub(nsub));
  count_launch(), k_sub_boxes<<<grid_for(nsub), NB_THREADS, 0, st>>>(n, nsub, L.spos, E.sub_lo, E.sub_hi);
  // query leaves heaviest first, for the persistent list kernel
  uint32_t* cost = reinterpret_cast<uint32_t*>(E.keys_a);
  uint32_t* cost_sorted = reinterpret_cast<uint32_t*>(E.keys_b);
  int32_t* order = reinterpret_cast<int32_t*>(E.keys_b) + E.cap_n;  // second half of keys_b
  count_launch(), k_leaf_cost<<<grid_for(nleaf), NB_THREADS, 0, st>>>(nleaf, E.node_lo, E.node_hi, cost, E.vals_a);
  tmp = 0;
  NB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, cost, cost_sorted, E.vals_a, order, (int)nleaf, 0, 32, st));
  NB_TRY(E.ensure_cub(tmp));
  tmp = E.cub_bytes;
  NB_CUDA(cub::DeviceRadixSort::SortPairs(E.cub_tmp, tmp, cost, cost_sorted, E.vals_a, order, (int)nleaf, 0, 32, st));
  NB_CUDA(cudaMemsetAsync(E.d_rowmax, 0, 4 * sizeof(unsigned long long), st));
  NB_TRY(list_kernel_slots(E));
  auto grid = [&](int64_t nwork) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((nwork * 32 + NB_THREADS - 1) / NB_THREADS, E.list_slots));
  };
  int64_t total = 0;
  if ((double)n * (double)E.row_cap <= ELL_MAX_ENTRIES) {
    // one traversal into fixed-width rows, scan, pack; the few rows longer than the width are
    // written straight into CSR by a second traversal over their leaves only
    NB_TRY(E.ensure_ell(n * E.row_cap));
    count_launch(), k_lists_sub<2><<<grid(nleaf), NB_THREADS, 0, st>>>(n, nleaf, order, E.d_rowmax + 2, tv, E.sub_lo, E.sub_hi, L.spos, E.counts, nullptr, E.ell, E.row_cap, E.d_rowmax, E.d_err);
    NB_CUDA(cudaMemsetAsync(L.off, 0, sizeof(int64_t), st));
    tmp = E.cub_bytes;
    NB_CUDA(cub::DeviceScan::InclusiveSum(E.cub_tmp, tmp, E.counts, L.off + 1, (int)n, st));
    NB_CUDA(cudaMemcpyAsync(E.h_build, L.off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    NB_CUDA(cudaMemcpyAsync(E.h_build + 1, E.d_rowmax, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    NB_CUDA(cudaStreamSynchronize(st));
    total = E.h_build[0];
    int64_t longest = E.h_build[1];
    NB_TRY(E.ensure_list_capacity(total));
    count_launch(), k_pack_rows<<<grid_for(n * 32), NB_THREADS, 0, st>>>(n, E.row_cap, E.ell, L.off, L.idx);
    if (longest > E.row_cap) {
      int32_t* leaves = reinterpret_cast<int32_t*>(E.keys_a);  // free after the order sort
      count_launch(), k_long_leaves<<<grid_for(nleaf), NB_THREADS, 0, st>>>(n, nleaf, E.counts, E.row_cap, leaves, E.d_rowmax + 1);
      NB_CUDA(cudaMemcpyAsync(E.h_build + 1, E.d_rowmax + 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
      NB_CUDA(cudaStreamSynchronize(st));
      int64_t nlong = E.h_build[1];
      count_launch(), k_lists_sub<1><<<grid(nlong), NB_THREADS, 0, st>>>(n, nlong, leaves, E.d_rowmax + 3, tv, E.sub_lo, E.sub_hi, L.spos, nullptr, L.off, L.idx, 0, nullptr, E.d_err);
    }
    // width for the next build: half as much again as this build's longest row (a redo of the
    // longest leaves costs far more than idle slots, which are never read), within the scratch
    // bound (rows beyond it take the CSR redo above)
    int64_t widest = std::min<int64_t>(1024, (int64_t)(ELL_MAX_ENTRIES / (double)n) / 32 * 32);
    E.row_cap = std::min<int64_t>(std::max<int64_t>((longest + longest / 2 + 31) / 32 * 32, 256), std::max<int64_t>(widest, 64));
  } else {
    // count, scan, fill
    count_launch(), k_lists_sub<0><<<grid(nleaf), NB_THREADS, 0, st>>>(n, nleaf, order, E.d_rowmax + 2, tv, E.sub_lo, E.sub_hi, L.spos, E.counts, nullptr, nullptr, 0, nullptr, E.d_err);
    NB_CUDA(cudaMemsetAsync(L.off, 0, sizeof(int64_t), st));
    tmp = E.cub_bytes;
    NB_CUDA(cub::DeviceScan::InclusiveSum(E.cub_tmp, tmp, E.counts, L.off + 1, (int)n, st));
    NB_CUDA(cudaMemcpyAsync(E.h_build, L.off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    NB_CUDA(cudaStreamSynchronize(st));
    total = E.h_build[0];
    NB_TRY(E.ensure_list_capacity(total));
    count_launch(), k_lists_sub<1><<<grid(nleaf), NB_THREADS, 0, st>>>(n, nleaf, order, E.d_rowmax + 3, tv, E.sub_lo, E.sub_hi, L.spos, nullptr, L.off, L.idx, 0, nullptr, E.d_err);
  }
  E.prof.end(PROF_LISTS, st, (double)n, (double)total);
  L.n = n;
  L.total = total;
  return check_device_error(E, st);
}

// Offsets (n + 1) of the last build's lists in the caller's order.
int export_lists_offsets(Engine& E, int64_t* off_out, cudaStream_t st) {
  Lists& L = E.lists;
  int64_t n = L.n;
  NB_CUDA(cudaMemsetAsync(off_out, 0, sizeof(int64_t), st));
  if (n == 0) return 0;
  count_launch(), k_export_counts<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.inv_perm, L.off, E.counts);
  size_t tmp = E.cub_bytes;
  NB_CUDA(cub::DeviceScan::InclusiveSum(E.cub_tmp, tmp, E.counts, off_out + 1, (int)n, st));
  return check_device_error(E, st);
}

// Entries of the last build's lists in the caller's order and numbering, each row ascending;
// off_out must hold the offsets from export_lists_offsets.
int export_lists(Engine& E, int64_t* off_out, int64_t* idx_out, cudaStream_t st) {
  Lists& L = E.lists;
  int64_t n = L.n;
  if (n == 0) return 0;
  size_t tmp = E.cub_bytes;
  count_launch(), k_export_fill<<<grid_for(n), NB_THREADS, 0, st>>>(n, L.perm, L.off, L.idx, off_out, idx_out);
  if (L.total > 0) {
    NB_TRY(E.ensure_sort_keys(L.total));
    NB_CUDA(cudaMemcpyAsync(E.sort_keys, idx_out, sizeof(int64_t) * L.total,
                            cudaMemcpyDeviceToDevice, st));
    tmp = E.cub_bytes;
    NB_CUDA(cub::DeviceSegmentedSort::SortKeys(E.cub_tmp, tmp, E.sort_keys, idx_out, L.total,
                                                (int)n, off_out, off_out + 1, st));
  }
  return check_device_error(E, st);
}

// ---------------------------------------------------------------- the reference's cell grid
// sim/neighbours.py:95-126 (_cell_of, _build_grid): per axis k = floor((x - lo) * inv_cell),
// clamped to [0, ncell - 1], cell = (cx * ny + cy) * nz + cz, and a stable counting sort of the
// particles by cell (start: ncell + 1 offsets, order: particles by cell, ascending index within a
// cell).  The subtraction and product round as the reference's (no fused multiply-add), so the
// assignment is the same bit for bit.  The lists above do not need these cells (their tree
// prunes with exact tests); this is the reference's cell assignment on its own, for callers and
// for the parity tests.
__global__ void k_cell_index(int64_t n, const double* __restrict__ pos, double lo0, double lo1,
                             double lo2, double ic0, double ic1, double ic2, int64_t n0,
                             int64_t n1, int64_t n2, uint32_t* __restrict__ cell,
                             int32_t* __restrict__ iota,
                             unsigned long long* __restrict__ per_cell) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double lo[3] = {lo0, lo1, lo2}, ic[3] = {ic0, ic1, ic2};
  const int64_t nc[3] = {n0, n1, n2};
  int64_t k[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double t = __dmul_rn(__dsub_rn(pos[3 * i + c], lo[c]), ic[c]);
    int64_t v = (int64_t)floor(t);
    k[c] = v < 0 ? 0 : (v >= nc[c] ? nc[c] - 1 : v);
  }
  const int64_t id = (k[0] * n1 + k[1]) * n2 + k[2];
  cell[i] = (uint32_t)id;
  iota[i] = (int32_t)i;
  atomicAdd(per_cell + id, 1ull);
}

__global__ void k_widen_order(int64_t n, const int32_t* __restrict__ src, int64_t* __restrict__ dst) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < n) dst[k] = src[k];
}

int build_cells(Engine& E, int64_t n, const double* pos, const double* lo, const double* inv_cell,
                const int64_t* ncell, int64_t* start, int64_t* order, cudaStream_t st) {
  const int64_t total = ncell[0] * ncell[1] * ncell[2];
  if (ncell[0] < 1 || ncell[1] < 1 || ncell[2] < 1 || total > (int64_t)INT32_MAX)
    return set_host_error(E, "cell counts must be positive and hold at most 2^31 cells");
  NB_TRY(E.ensure_n(std::max<int64_t>(n, 1)));
  NB_TRY(E.ensure_sort_keys(total));
  unsigned long long* per_cell = reinterpret_cast<unsigned long long*>(E.sort_keys);
  NB_CUDA(cudaMemsetAsync(per_cell, 0, sizeof(int64_t) * total, st));
  NB_CUDA(cudaMemsetAsync(start, 0, sizeof(int64_t), st));
  if (n > 0) {
    uint32_t* cell = reinterpret_cast<uint32_t*>(E.keys_a);
    uint32_t* cell_sorted = reinterpret_cast<uint32_t*>(E.keys_b);
    int32_t* by_cell = reinterpret_cast<int32_t*>(E.keys_b) + E.cap_n;  // second half of keys_b
    count_launch(), k_cell_index<<<grid_for(n), NB_THREADS, 0, st>>>(
        n, pos, lo[0], lo[1], lo[2], inv_cell[0], inv_cell[1], inv_cell[2], ncell[0], ncell[1],
        ncell[2], cell, E.vals_a, per_cell);
    int end_bit = 1;
    while (end_bit < 32 && (int64_t(1) << end_bit) < total) ++end_bit;
    size_t tmp = 0;
    NB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, cell, cell_sorted, E.vals_a, by_cell,
                                            (int)n, 0, end_bit, st));
    NB_TRY(E.ensure_cub(tmp));
    tmp = E.cub_bytes;
    // radix sort is stable: within a cell the particles keep ascending index, as the reference's
    // counting sort leaves them
    NB_CUDA(cub::DeviceRadixSort::SortPairs(E.cub_tmp, tmp, cell, cell_sorted, E.vals_a, by_cell,
                                            (int)n, 0, end_bit, st));
    count_launch(), k_widen_order<<<grid_for(n), NB_THREADS, 0, st>>>(n, by_cell, order);
  }
  size_t tmp = 0;
  const int64_t* counts = reinterpret_cast<const int64_t*>(per_cell);
  NB_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, counts, start + 1, (int)total, st));
  NB_TRY(E.ensure_cub(tmp));
  tmp = E.cub_bytes;
  NB_CUDA(cub::DeviceScan::InclusiveSum(E.cub_tmp, tmp, counts, start + 1, (int)total, st));
  return check_device_error(E, st);
}

// sim/neighbours.py:250-265 (find_neighbours_numba, no periodic box): lo = the smallest
// coordinates, cell = max(R_KERN * median(h) / 2, max(span) / 160, 1e-300), ncell = floor(span /
// cell) + 1 per axis, inv_cell = 1 / cell (host outputs; the call synchronises its stream).
int cell_geometry(Engine& E, int64_t n, const double* pos, const double* h, double* lo,
                  double* inv_cell, int64_t* ncell, cudaStream_t st) {
  if (n <= 0) return set_host_error(E, "the cell grid needs at least one particle");
  NB_TRY(E.ensure_n(n));
  int nbb = (int)std::min<int64_t>(grid_for(n), 1184);
  count_launch(), k_bbox_partial<<<nbb, NB_THREADS, 0, st>>>(n, pos, E.bbox_part);
  count_launch(), k_bbox_final<<<1, NB_THREADS, 0, st>>>(nbb, E.bbox_part, E.bbox);
  double* h_sorted = reinterpret_cast<double*>(E.keys_b);
  size_t tmp = 0;
  NB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp, h, h_sorted, (int)n, 0, 64, st));
  NB_TRY(E.ensure_cub(tmp));
  tmp = E.cub_bytes;
  NB_CUDA(cub::DeviceRadixSort::SortKeys(E.cub_tmp, tmp, h, h_sorted, (int)n, 0, 64, st));
  double box[6], mid[2];
  NB_CUDA(cudaMemcpyAsync(box, E.bbox, sizeof(box), cudaMemcpyDeviceToHost, st));
  NB_CUDA(cudaMemcpyAsync(mid, h_sorted + (n - 1) / 2, sizeof(double) * (n % 2 ? 1 : 2),
                          cudaMemcpyDeviceToHost, st));
  NB_CUDA(cudaStreamSynchronize(st));
  // numpy's median: the middle value, or the mean of the two middle values for even n
  const double median = n % 2 ? mid[0] : (mid[0] + mid[1]) / 2.0;
  double span[3], smax = 0.0;
  for (int c = 0; c < 3; ++c) {
    lo[c] = box[c];
    span[c] = box[3 + c] - box[c];
    smax = std::max(smax, span[c]);
  }
  const double cell = std::max(std::max(0.5 * 2.0 * median, smax / 160.0), 1e-300);
  for (int c = 0; c < 3; ++c) {
    ncell[c] = std::max<int64_t>((int64_t)std::floor(span[c] / cell) + 1, 1);
    inv_cell[c] = 1.0 / cell;
  }
  return check_device_error(E, st);
}

size_t cub_bytes_needed(int64_t n, int64_t m) {
  size_t a = 0, b = 0, c = 0, d = 0;
  cub::DeviceRadixSort::SortPairs((void*)nullptr, a, (uint64_t*)nullptr, (uint64_t*)nullptr,
                                  (int32_t*)nullptr, (int32_t*)nullptr, (int)n, 0, 63);
  cub::DeviceScan::InclusiveSum((void*)nullptr, b, (int64_t*)nullptr, (int64_t*)nullptr, (int)n);
  if (m > 0)
    cub::DeviceSegmentedSort::SortKeys((void*)nullptr, c, (int64_t*)nullptr, (int64_t*)nullptr,
                                       m, (int)n, (int64_t*)nullptr, (int64_t*)nullptr);
  cub::DeviceSelect::Flagged((void*)nullptr, d, (int64_t*)nullptr, (const uint8_t*)nullptr,
                             (int64_t*)nullptr, (int64_t*)nullptr, (int)n);
  return std::max(std::max(a, b), std::max(c, d)) + 256;
}

}  // namespace nbk
