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
#include <thrust/iterator/counting_iterator.h>

#include "common.cuh"
#include "engine.cuh"

namespace nbk {

static constexpr int LEAF = 32;
static constexpr int SUB = 8;  // sub-leaf: the unit of the candidate queue (4 per staged batch)
static constexpr int FAN = 8;
static constexpr int STACK = 96;

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

// The rows of one query leaf of LEAF consecutive sorted particles, one lane per particle, tested
// tile by tile.  The warp walks the tree of boxes with an explicit stack in shared memory (entries
// (level << 40) | index; children pushed highest first, so candidate leaves are reached in
// ascending order) and takes, in ascending order, the sub-leaves whose boxes lie within reach of
// the query leaf's box.  Every 4 of them (32 candidates) are staged in shared memory, one
// candidate per lane with coalesced loads, as float offsets from the query leaf's centre, and
// every lane tests its own particle against all 32: the whole warp stays busy on the same
// candidates, with no per-lane queues.
//
// The test is the reference's FP64 r^2 < (2 h_i)^2 or r^2 < (2 h_j)^2 decided in FP32 with a
// rigorous band.  With D the largest offset component of the query lanes and the staged batch
// and u = 2^-24, the offsets round with error <= u D, their differences with error <= 4 u D,
// and the float r^2 of a pair (three rounded squares and sums of terms <= 12 D^2) differs from
// the exact one by at most 84 u D^2; the float thresholds and their subtractions add at most
// 36 u D^2 for every threshold that can matter (r^2 <= 12 D^2).  With B = 192 u D^2 and the
// float threshold T lowered by B, q = fl(r^2 - (T - B)) < 0 is a certain hit (the sign of a
// rounded difference is exact, and r^2 + 84 u D^2 < T - B + 36 u D^2 < T) and q >= 2 B a
// certain miss (r^2 >= T - B + 2 B (1 - u) - 120 u D^2 > T); pairs in between are decided by
// the exact FP64 test (no fused multiply-add) from the double positions.  So the lists are the
// reference's bit for bit.
//
// Three passes share the traversal: k_lists_cand counts each query leaf's candidate sub-leaves
// (so every leaf gets its own slice of the candidate and mask buffers), k_lists_test runs the
// tests once, storing each lane's 32-bit hit mask per batch and its row's entry count, and
// k_lists_expand turns the masks into the CSR entries at the rows' offsets, each row ascending
// (batches come in ascending candidate order, a mask's bits from the lowest slot up).

constexpr float BAND_U = 192.0f / 16777216.0f;  // 192 u, u = 2^-24

// The query leaf's box, centre and largest search radius.
struct QueryLeaf {
  double4 lo, hi;
  double cx, cy, cz;
};

__device__ __forceinline__ QueryLeaf query_leaf(const TreeView& tv, int64_t leaf) {
  QueryLeaf q;
  q.lo = tv.lo[leaf];
  q.hi = tv.hi[leaf];
  q.cx = 0.5 * (q.lo.x + q.hi.x);
  q.cy = 0.5 * (q.lo.y + q.hi.y);
  q.cz = 0.5 * (q.lo.z + q.hi.z);
  return q;
}

// Walk the tree for one query leaf; on_subs(s0, mask) is called warp-uniformly for every
// candidate leaf with its first sub-leaf s0 and the ballot of its sub-leaves within reach of the
// query leaf's box (bit c: sub-leaf s0 + c), in ascending order.  Returns false if the stack
// overflowed.
template <typename F>
__device__ __forceinline__ bool walk_candidates(int64_t n, const TreeView& tv, const QueryLeaf& q,
                                                const double4* __restrict__ slo,
                                                const double4* __restrict__ shi,
                                                int64_t* stack, int lane, F&& on_subs) {
  const unsigned FULL = 0xffffffffu;
  const int64_t nsub = (n + SUB - 1) / SUB;
  const double qh = q.lo.w;
  int sp = 0;
  __syncwarp();
  if (lane == 0) stack[0] = ((int64_t)(tv.nlevels - 1) << 40);
  sp = 1;
  __syncwarp();
  while (sp > 0) {
    const int64_t e = stack[sp - 1];
    __syncwarp();
    sp -= 1;
    const int lvl = (int)(e >> 40);
    const int64_t node = e & ((1ll << 40) - 1);
    if (lvl == 0) {
      const int64_t s0 = node * (LEAF / SUB);
      const int64_t s1 = min(s0 + LEAF / SUB, nsub);
      bool near = false;
      if (lane < s1 - s0) {
        const double4 blo = slo[s0 + lane], bhi = shi[s0 + lane];
        const double reach = 2.0 * fmax(qh, blo.w);
        near = box_gap2(q.lo, q.hi, blo, bhi) < reach * reach * (1.0 + 1e-12);
      }
      const unsigned mk = __ballot_sync(FULL, near);
      if (mk) on_subs(s0, mk);
      continue;
    }
    const int64_t c0 = node * FAN;
    const int64_t csize = tv.level_size[lvl - 1];
    const int64_t child = c0 + lane;
    bool hit = false;
    if (lane < FAN && child < csize) {
      const int64_t g = tv.level_off[lvl - 1] + child;
      const double4 blo = tv.lo[g], bhi = tv.hi[g];
      const double reach = 2.0 * fmax(qh, blo.w);
      hit = box_gap2(q.lo, q.hi, blo, bhi) < reach * reach * (1.0 + 1e-12);
    }
    const unsigned mask = __ballot_sync(FULL, hit);
    const int nh = __popc(mask);
    if (sp + nh > STACK) return false;
    if (hit) {
      const int above = __popc(mask & ~((2u << lane) - 1u));
      stack[sp + above] = ((int64_t)(lvl - 1) << 40) | child;
    }
    __syncwarp();
    sp += nh;
  }
  return true;
}

// Pass 1: the candidate sub-leaves of each query leaf, in ascending order, into its own slice of
// the candidate buffer.  The walk goes level by level: the nodes within reach of the query box at
// one level (a frontier in shared memory, ascending) give the next level's nodes to test, 32 at
// a time, one per lane; the leaves within reach give the sub-leaves to test the same way, and the
// sub-leaves within reach are the leaf's candidate list (ascending, since every frontier is).  A
// frontier larger than its buffer sends the leaf to the depth-first walk instead, which counts
// first and writes in a second walk.  The leaf takes its slices of the candidate and mask
// buffers with two atomic adds (cand_at / batch_at, so slices of different leaves lie in any
// order).  A slice that would pass the buffers' capacity is not written; the host then grows the
// buffers from the cursors' final values and runs the pass again.
constexpr int CAND_WARPS = 4;
#ifndef CAND_SMEM
#define CAND_SMEM 1024  // entries of a frontier buffer
#endif

__global__ void __launch_bounds__(CAND_WARPS * 32) k_lists_cand(int64_t n, int64_t nwork,
                                                           const uint64_t* __restrict__ order,
                                                           unsigned long long* __restrict__ next,
                                                           TreeView tv,
                                                           const double4* __restrict__ slo,
                                                           const double4* __restrict__ shi,
                                                           unsigned long long* __restrict__ cand_at,
                                                           unsigned long long* __restrict__ batch_at,
                                                           int64_t cap_cands, int64_t cap_batches,
                                                           int32_t* __restrict__ cands,
                                                           int64_t* __restrict__ leaf_cbase,
                                                           int64_t* __restrict__ leaf_bbase,
                                                           int32_t* __restrict__ leaf_ncand,
                                                           int* err) {
  __shared__ int64_t stacks[CAND_WARPS][STACK];
  __shared__ int32_t fronts[CAND_WARPS][2][CAND_SMEM];
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  int64_t* stack = stacks[threadIdx.x >> 5];
  int32_t(*front)[CAND_SMEM] = fronts[threadIdx.x >> 5];
  const int64_t nsub = (n + SUB - 1) / SUB;
  while (true) {
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(next, 1ull);
    t = __shfl_sync(FULL, t, 0);
    if (t >= (unsigned long long)nwork) break;  // warp-uniform
    const int64_t leaf = (int64_t)(order[t] & 0xffffffffull);
    const QueryLeaf q = query_leaf(tv, leaf);
    const double qh = q.lo.w;
    // level by level from the root; `cur` holds the frontier (ascending node indices)
    int cur = 0, fn = 1;
    bool over = false;
    __syncwarp();
    if (lane == 0) front[0][0] = 0;
    __syncwarp();
    for (int lvl = tv.nlevels - 1; lvl >= 0 && !over; --lvl) {
      // children of the frontier: nodes of level lvl - 1, or at the leaves their sub-leaves
      const int fan = lvl > 0 ? FAN : LEAF / SUB;
      const int64_t csize = lvl > 0 ? tv.level_size[lvl - 1] : nsub;
      const int64_t coff = lvl > 0 ? tv.level_off[lvl - 1] : 0;
      const double4* clo = lvl > 0 ? tv.lo : slo;
      const double4* chi = lvl > 0 ? tv.hi : shi;
      const int total = fn * fan;
      int nn = 0;
      for (int c0 = 0; c0 < total; c0 += 32) {
        const int c = c0 + lane;
        bool hit = false;
        int32_t child = 0;
        if (c < total) {
          child = front[cur][c / fan] * fan + c % fan;
          if (child < csize) {
            const double4 blo = clo[coff + child], bhi = chi[coff + child];
            const double reach = 2.0 * fmax(qh, blo.w);
            hit = box_gap2(q.lo, q.hi, blo, bhi) < reach * reach * (1.0 + 1e-12);
          }
        }
        const unsigned mk = __ballot_sync(FULL, hit);
        if (nn + __popc(mk) > CAND_SMEM) {
          over = true;
          break;
        }
        if (hit) front[cur ^ 1][nn + __popc(mk & below)] = child;
        nn += __popc(mk);
      }
      __syncwarp();
      cur ^= 1;
      fn = nn;
    }
    int64_t count = fn;
    if (over) {
      // a frontier outgrew its buffer: the depth-first walk counts instead
      count = 0;
      if (!walk_candidates(n, tv, q, slo, shi, stack, lane,
                           [&](int64_t, unsigned mk) { count += __popc(mk); }))
        set_error(err, ERR_TRAVERSAL_STACK);
    }
    const int64_t nbat = (count + 3) / 4;
    unsigned long long cb = 0, bb = 0;
    if (lane == 0) {
      cb = atomicAdd(cand_at, (unsigned long long)count);
      bb = atomicAdd(batch_at, (unsigned long long)nbat);
    }
    cb = __shfl_sync(FULL, cb, 0);
    bb = __shfl_sync(FULL, bb, 0);
    const bool fits = (int64_t)cb + count <= cap_cands && (int64_t)bb + nbat <= cap_batches;
    if (fits) {
      if (!over) {
        for (int64_t c = lane; c < count; c += 32) cands[cb + c] = front[cur][c];
      } else {
        int64_t c2 = 0;
        walk_candidates(n, tv, q, slo, shi, stack, lane, [&](int64_t s0, unsigned mk) {
          const int pos = __popc(mk & below);
          if (((mk >> lane) & 1u) && c2 + pos < count) cands[cb + c2 + pos] = (int32_t)(s0 + lane);
          c2 += __popc(mk);
        });
      }
    }
    if (lane == 0) {
      leaf_cbase[leaf] = (int64_t)cb;
      leaf_bbase[leaf] = (int64_t)bb;
      leaf_ncand[leaf] = (int32_t)count;
    }
    __syncwarp();
  }
}

// Pass 2: the tests, on each leaf's candidate list.  Each batch's final hit masks go to
// masks[(batch base + b) * 32 + lane], the rows' entry counts to counts.
#ifndef TEST_BLOCKS_PER_SM
#define TEST_BLOCKS_PER_SM 3
#endif
__global__ void __launch_bounds__(NB_THREADS, TEST_BLOCKS_PER_SM) k_lists_test(int64_t n, int64_t nwork,
                                                           const uint64_t* __restrict__ order,
                                                           unsigned long long* __restrict__ next,
                                                           TreeView tv,
                                                           const double4* __restrict__ spos,
                                                           const int32_t* __restrict__ cands,
                                                           const int64_t* __restrict__ leaf_cbase,
                                                           const int64_t* __restrict__ leaf_bbase,
                                                           const int32_t* __restrict__ leaf_ncand,
                                                           uint32_t* __restrict__ masks,
                                                           int64_t* __restrict__ counts,
                                                           unsigned long long* __restrict__ rowmax,
                                                           int* err) {
  __shared__ float4 cand_s[NB_THREADS / 32][32];
  __shared__ int32_t cidx_s[NB_THREADS / 32][32];
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  float4* cand = cand_s[threadIdx.x >> 5];
  int32_t* cidx = cidx_s[threadIdx.x >> 5];
  unsigned longest = 0;
  while (true) {
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(next, 1ull);
    t = __shfl_sync(FULL, t, 0);
    if (t >= (unsigned long long)nwork) break;  // warp-uniform
    const int64_t leaf = (int64_t)(order[t] & 0xffffffffull);
    const QueryLeaf q = query_leaf(tv, leaf);
    const int64_t cbase = leaf_cbase[leaf], bbase = leaf_bbase[leaf];
    const int64_t ncand = leaf_ncand[leaf];
    const int64_t k = leaf * LEAF + lane;
    const bool valid = k < n;
    const double4 me = valid ? spos[k] : make_double4(0, 0, 0, 0);
    float mx = 1e30f, my = 1e30f, mz = 1e30f, Dl = 0.0f, r2i_f = -1.0f;
    const double ri = 2.0 * me.w;
    const double r2i = __dmul_rn(ri, ri);
    if (valid) {
      mx = (float)(me.x - q.cx);
      my = (float)(me.y - q.cy);
      mz = (float)(me.z - q.cz);
      Dl = fmaxf(fmaxf(fabsf(mx), fabsf(my)), fabsf(mz));
      r2i_f = (float)r2i;
    }
    // non-negative floats order like their bits
    const float Dq = __uint_as_float(__reduce_max_sync(FULL, __float_as_uint(Dl)));
    int64_t m = 0;
    for (int64_t b = 0; 4 * b < ncand; ++b) {
      // stage: slot = lane, candidate sub-leaf 4 b + lane / 8, particle lane % 8 of it
      const int64_t c = 4 * b + (lane >> 3);
      const int32_t sb = c < ncand ? cands[cbase + c] : -1;
      const int64_t j = (int64_t)sb * SUB + (lane & 7);
      float4 cc = make_float4(1e30f, 1e30f, 1e30f, 0.0f);
      float Dj = 0.0f;
      int32_t jj = -1;
      if (sb >= 0 && j < n) {
        const double4 p = spos[j];
        cc.x = (float)(p.x - q.cx);
        cc.y = (float)(p.y - q.cy);
        cc.z = (float)(p.z - q.cz);
        const double rj = 2.0 * p.w;
        cc.w = (float)(rj * rj);
        Dj = fmaxf(fmaxf(fabsf(cc.x), fabsf(cc.y)), fabsf(cc.z));
        jj = (int32_t)j;
      }
      const float D = fmaxf(Dq, __uint_as_float(__reduce_max_sync(FULL, __float_as_uint(Dj))));
      // offsets beyond float's comfortable range (never in code units): every pair exactly
      const bool wide = !(D < 1e15f);
      const float B = wide ? 0.0f : BAND_U * D * D;
      cc.w -= B;
      cand[lane] = cc;
      cidx[lane] = jj;
      __syncwarp();
      const float ri_lo = r2i_f - B, twoB = 2.0f * B;
      // q = r^2 - (threshold - B) of each candidate: its sign bit is a certain hit, shifted into
      // the mask (candidate 31 first, so bit tt is candidate tt); the smallest non-negative q
      // (signed floats' bits sort above every non-negative float's) tells whether any lies in
      // the band 0 <= q < 2B
      unsigned hit = 0u, closest = 0xffffffffu;
#pragma unroll
      for (int tt = 31; tt >= 0; --tt) {
        const float4 e = cand[tt];
        const float dx = e.x - mx, dy = e.y - my, dz = e.z - mz;
        const float q = fmaf(dz, dz, fmaf(dy, dy, dx * dx)) - fmaxf(e.w, ri_lo);
        hit = __funnelshift_l(__float_as_uint(q), hit, 1);
        closest = min(closest, __float_as_uint(q));
      }
      unsigned amb = 0u;
      if (wide) {
        hit = 0u;
        amb = __ballot_sync(FULL, jj >= 0);
      } else if (__any_sync(FULL, valid && closest < __float_as_uint(twoB))) {
        for (int tt = 0; tt < 32; ++tt) {
          const float4 e = cand[tt];
          const float dx = e.x - mx, dy = e.y - my, dz = e.z - mz;
          const float q = fmaf(dz, dz, fmaf(dy, dy, dx * dx)) - fmaxf(e.w, ri_lo);
          amb |= q >= 0.0f && q < twoB ? 1u << tt : 0u;
        }
      }
      if (!valid) hit = amb = 0u;
      if (__any_sync(FULL, amb != 0u)) {
        // the band: the reference's exact FP64 test from the double positions
        while (amb) {
          const int tt = __ffs(amb) - 1;
          amb &= amb - 1u;
          const double4 pj = spos[cidx[tt]];
          const double d2 = d2_exact(pj.x - me.x, pj.y - me.y, pj.z - me.z);
          const double rj = 2.0 * pj.w;
          if (d2 < r2i || d2 < __dmul_rn(rj, rj)) hit |= 1u << tt;
        }
      }
      masks[(bbase + b) * 32 + lane] = hit;
      m += __popc(hit);
      __syncwarp();  // the next batch overwrites the staged candidates
    }
    if (valid) counts[k] = m;
    longest = max(longest, valid ? (unsigned)m : 0u);
  }
  const unsigned mx = __reduce_max_sync(FULL, longest);
  if (lane == 0) atomicMax(rowmax, (unsigned long long)mx);
}

// Position of the k-th set bit (k from 0) of m, for k < popc(m): halving by population count.
__device__ __forceinline__ int nth_set_bit(uint32_t m, int k) {
  int p = 0;
  int c = __popc(m & 0xffffu);
  if (k >= c) { k -= c; p += 16; m >>= 16; }
  c = __popc(m & 0xffu);
  if (k >= c) { k -= c; p += 8; m >>= 8; }
  c = __popc(m & 0xfu);
  if (k >= c) { k -= c; p += 4; m >>= 4; }
  c = __popc(m & 0x3u);
  if (k >= c) { k -= c; p += 2; m >>= 2; }
  if (k >= (int)(m & 1u)) p += 1;
  return p;
}

// Pass 3: masks -> CSR entries.  One warp per query leaf.  The leaf's masks (all 32 rows) and
// candidate sub-leaves are staged in shared memory a chunk of batches at a time; then the warp
// takes the rows one after the other, 32 batches at a time with lane b on batch b: the batches'
// entry counts are scanned across the lanes, and the row's entries of those batches are written
// 32 at a time, lane s taking entry s: its batch is found by a binary search over the scanned
// counts, its candidate as the set bit of that rank in the batch's mask.  Every store writes up
// to 32 consecutive entries of one row, and each row's entries come out in ascending order
// (batches ascending, a mask's bits from the lowest slot up), contiguous from the row's offset.
//
// Warps per block and batches staged at a time: measured on the 4M torus (list build ms per
// build) 10.45 with 8 warps and 32 batches, 10.86 with 4 and 32, 11.35 with 4 and 64, 11.68
// with 2 and 64 (37.9 KB of shared memory per block for 8 x 32 and 4 x 64)
#ifndef EXPAND_WARPS
#define EXPAND_WARPS 8
#endif
#ifndef EXPAND_CHUNK
#define EXPAND_CHUNK 32
#endif
constexpr int EXPAND_STRIDE = 33;  // padded mask rows: lane b reading row r of batch b is conflict-free

__global__ void __launch_bounds__(EXPAND_WARPS * 32) k_lists_expand(int64_t n, int64_t nleaf,
                                                             const int32_t* __restrict__ cands,
                                                             const int64_t* __restrict__ leaf_cbase,
                                                             const int64_t* __restrict__ leaf_bbase,
                                                             const int32_t* __restrict__ leaf_ncand,
                                                             const uint32_t* __restrict__ masks,
                                                             const int64_t* __restrict__ off,
                                                             int32_t* __restrict__ idx, int* err) {
  __shared__ uint32_t msk_s[EXPAND_WARPS][EXPAND_CHUNK * EXPAND_STRIDE];
  __shared__ int32_t sub_s[EXPAND_WARPS][EXPAND_CHUNK * 4];
  const unsigned FULL = 0xffffffffu;
  const int64_t leaf = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (leaf >= nleaf) return;  // warp-uniform
  uint32_t* msk = msk_s[threadIdx.x >> 5];
  int32_t* sub = sub_s[threadIdx.x >> 5];
  const int64_t cbase = leaf_cbase[leaf], bbase = leaf_bbase[leaf];
  const int64_t ncand = leaf_ncand[leaf], nbat = (ncand + 3) / 4;
  const int64_t k0 = leaf * LEAF;
  const int rows = (int)(n - k0 < LEAF ? n - k0 : LEAF);
  // lane r keeps row r's running output position and its end
  int64_t pos = lane < rows ? off[k0 + lane] : 0;
  const int64_t stop = lane < rows ? off[k0 + lane + 1] : 0;
  for (int64_t c0 = 0; c0 < nbat; c0 += EXPAND_CHUNK) {
    const int nb = (int)(nbat - c0 < EXPAND_CHUNK ? nbat - c0 : EXPAND_CHUNK);
    __syncwarp();
    for (int e = lane; e < nb * 32; e += 32)
      msk[(e >> 5) * EXPAND_STRIDE + (e & 31)] = masks[(bbase + c0) * 32 + e];
    for (int e = lane; e < nb * 4; e += 32) {
      const int64_t c = 4 * c0 + e;
      sub[e] = c < ncand ? cands[cbase + c] : 0;
    }
    __syncwarp();
    for (int r = 0; r < rows; ++r) {
      int64_t at = __shfl_sync(FULL, pos, r);  // warp-uniform from here on
      const int64_t end = __shfl_sync(FULL, stop, r);
      for (int b0 = 0; b0 < nb; b0 += 32) {
        const uint32_t m = b0 + lane < nb ? msk[(b0 + lane) * EXPAND_STRIDE + r] : 0u;
        int incl = __popc(m);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(FULL, incl, o);
          if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(FULL, incl, 31);
        for (int base = 0; base < total; base += 32) {
          const int s = base + lane;
          // batch of entry s: the number of batches whose inclusive count is <= s (< 32 for
          // s < total; the probes stay within lanes 0..30)
          int j = 0;
#pragma unroll
          for (int step = 16; step > 0; step >>= 1)
            if (__shfl_sync(FULL, incl, j + step - 1) <= s) j += step;
          const uint32_t mb = __shfl_sync(FULL, m, j);
          const int first = __shfl_sync(FULL, incl, j) - __popc(mb);
          if (s < total) {
            const int t = nth_set_bit(mb, s - first);
            const int64_t w = at + s;
            if (w < end)
              idx[w] = sub[4 * (b0 + j) + (t >> 3)] * SUB + (t & 7);
            else
              set_error(err, ERR_LIST_OVERFLOW);
          }
        }
        at += total;
      }
      if (lane == r) pos = at;
    }
  }
  if (lane < rows && pos != stop) set_error(err, ERR_LIST_OVERFLOW);
}

// Order key of each query leaf: its cost class (the binary exponent of the linear size of the
// region its traversal covers, box extent plus twice the largest search diameter), heaviest
// first, then the leaf's curve position.
__global__ void k_leaf_cost(int64_t nleaf, const double4* __restrict__ lo,
                            const double4* __restrict__ hi, uint64_t* __restrict__ key) {
  int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (l >= nleaf) return;
  double4 a = lo[l], b = hi[l];
  double ext = fmax(fmax(b.x - a.x, b.y - a.y), b.z - a.z);
  float c = (float)(ext + 4.0 * a.w);
  const uint64_t cls = 255u - ((__float_as_uint(c) >> 23) & 255u);
  key[l] = (cls << 32) | (uint64_t)l;
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
// Synchronise the stream after a pass whose size the host needs next, and stop on a device
// error the pass raised (so no buffer is sized from a failed pass).
static int pending_check(Engine& E, cudaStream_t st) {
  NB_CUDA(cudaMemcpyAsync(E.h_err, E.d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  NB_CUDA(host_sync(st));
  if (E.h_err[0] != 0) return check_device_error(E, st);
  return 0;
}

// Resident blocks of the persistent list kernels over the whole device (fewest of the two).
static int list_kernel_slots(Engine& E) {
  if (E.list_slots > 0) return 0;
  int sms = 0, b0 = 0, b1 = 0;
  NB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, E.device));
  NB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b0, k_lists_cand, CAND_WARPS * 32, 0));
  NB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_lists_test, NB_THREADS, 0));
  // resident warps of each pass over the whole device
  E.list_slots = (int64_t)sms * std::max(1, b1) * (NB_THREADS / 32);
  E.cand_slots = (int64_t)sms * std::max(1, b0) * CAND_WARPS;
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
  // query leaves by cost class, heaviest first, each class in curve order
  uint64_t* cost = E.keys_a;
  uint64_t* order = E.keys_b;
  count_launch(), k_leaf_cost<<<grid_for(nleaf), NB_THREADS, 0, st>>>(nleaf, E.node_lo, E.node_hi, cost);
  tmp = 0;
  NB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp, cost, order, (int)nleaf, 0, 40, st));
  NB_TRY(E.ensure_cub(tmp));
  tmp = E.cub_bytes;
  NB_CUDA(cub::DeviceRadixSort::SortKeys(E.cub_tmp, tmp, cost, order, (int)nleaf, 0, 40, st));
  NB_TRY(list_kernel_slots(E));
  // persistent passes: at most one warp per query leaf, at most the resident warps
  const unsigned grid = (unsigned)std::max<int64_t>(
      1, std::min<int64_t>(nleaf, E.list_slots) / (NB_THREADS / 32));
  const unsigned cand_grid = (unsigned)std::max<int64_t>(
      1, std::min<int64_t>(nleaf, E.cand_slots) / CAND_WARPS);
  // candidate lists of the query leaves, each in its own slice of the buffers (sized from the
  // last build's totals; a pass that outgrows them is run again with buffers of its size)
  NB_TRY(E.ensure_leaves(nleaf));
  NB_TRY(E.ensure_tiles(E.last_cands > 0 ? E.last_cands + E.last_cands / 4 : nleaf * 512,
                        E.last_batches > 0 ? E.last_batches + E.last_batches / 4 : nleaf * 128));
  for (int attempt = 0;; ++attempt) {
    NB_CUDA(cudaMemsetAsync(E.d_rowmax, 0, 8 * sizeof(unsigned long long), st));
    count_launch(), k_lists_cand<<<cand_grid, CAND_WARPS * 32, 0, st>>>(
        n, nleaf, order, E.d_rowmax + 2, tv, E.sub_lo, E.sub_hi, E.d_rowmax + 4, E.d_rowmax + 5,
        E.cap_cands, E.cap_masks / 32, E.cands, E.leaf_cbase, E.leaf_bbase, E.leaf_ncand, E.d_err);
    NB_CUDA(cudaMemcpyAsync(E.h_build, E.d_rowmax + 4, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    NB_TRY(pending_check(E, st));
    const int64_t ncand = E.h_build[0], nbatch = E.h_build[1];
    E.last_cands = ncand;
    E.last_batches = nbatch;
    if (ncand <= E.cap_cands && nbatch <= E.cap_masks / 32) break;
    if (attempt > 0) return set_host_error(E, "list build: candidate buffers outgrown twice");
    NB_TRY(E.ensure_tiles(ncand + ncand / 4, nbatch + nbatch / 4));
  }
  // the tests, once: hit masks per batch and lane, entries per row
  count_launch(), k_lists_test<<<grid, NB_THREADS, 0, st>>>(n, nleaf, order, E.d_rowmax + 3, tv, L.spos, E.cands, E.leaf_cbase, E.leaf_bbase, E.leaf_ncand, E.masks, E.counts, E.d_rowmax, E.d_err);
  NB_CUDA(cudaMemsetAsync(L.off, 0, sizeof(int64_t), st));
  tmp = E.cub_bytes;
  NB_CUDA(cub::DeviceScan::InclusiveSum(E.cub_tmp, tmp, E.counts, L.off + 1, (int)n, st));
  NB_CUDA(cudaMemcpyAsync(E.h_build, L.off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  NB_CUDA(cudaMemcpyAsync(E.h_build + 1, E.d_rowmax, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  NB_TRY(pending_check(E, st));
  const int64_t total = E.h_build[0];
  NB_TRY(E.ensure_list_capacity(total));
  // masks -> entries at the rows' offsets
  count_launch(), k_lists_expand<<<grid_for(nleaf * 32, EXPAND_WARPS * 32), EXPAND_WARPS * 32, 0, st>>>(
      n, nleaf, E.cands, E.leaf_cbase, E.leaf_bbase, E.leaf_ncand, E.masks, L.off, L.idx, E.d_err);
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
  NB_CUDA(host_sync(st));
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
  size_t e = 0;
  cub::DeviceSelect::Flagged((void*)nullptr, e, thrust::counting_iterator<int64_t>(0),
                             (const uint8_t*)nullptr, (int64_t*)nullptr, (int64_t*)nullptr, (int)n);
  return std::max(std::max(std::max(a, b), std::max(c, d)), e) + 256;
}

}  // namespace nbk
