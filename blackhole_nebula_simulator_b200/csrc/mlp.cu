// The learned bremsstrahlung cooling step: data generation labelled by the exact integrator,
// training by hand-written forward / backward / Adam kernels, and the fused inference kernel on
// the BF16 tensor cores with an exact fallback.
//
// Training runs in FP32 with the weights rounded to BF16 in every forward pass (the rounding the
// inference kernel applies), and the straight-through gradient.  Inference (k_mlp_cool) keeps
// BF16 weights in shared memory and runs each layer as mma.sync m16n8k16 BF16 x BF16 -> FP32
// tiles: a warp carries 16 particles through all four layers in registers (the accumulator
// layout of one layer is the A-operand layout of the next).  Activations are split into a BF16
// high part and a BF16 remainder (two MMAs per tile), so only the weights are rounded to BF16.
// The 3 inputs occupy columns 0-2 (high parts) and 3-5 (remainders) of the first layer's K = 16.
#include <cuda_bf16.h>

#include <cmath>
#include <vector>

#include "../../include/nebula_b200.h"
#include "common.cuh"
#include "cooling.cuh"
#include "engine.cuh"
#include "mlp.cuh"

namespace nbk {

// ---------------------------------------------------------------- random numbers
__device__ __forceinline__ uint64_t splitmix(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}
__device__ __forceinline__ double uniform01(uint64_t seed, uint64_t i, int k) {
  uint64_t r = splitmix(seed * 0x100000001b3ull + i * 4ull + (uint64_t)k);
  return (double)(r >> 11) * (1.0 / 9007199254740992.0);
}

// Training samples: log-uniform rho [g/cm^3], T [K], dt [s] over the hull, labelled with the
// exact integrator's f.  Stored scaled (X) with their code-unit values (U: u, rho, dt).
__global__ void k_mlp_data(int64_t n, uint64_t seed, BremsParams bp, MlpHull hl,
                           float* __restrict__ X, float* __restrict__ Y, double* __restrict__ U) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double lr = hl.lrho_lo + (hl.lrho_hi - hl.lrho_lo) * uniform01(seed, i, 0);
  double lt = hl.lt_lo + (hl.lt_hi - hl.lt_lo) * uniform01(seed, i, 1);
  double ld = hl.ldt_lo + (hl.ldt_hi - hl.ldt_lo) * uniform01(seed, i, 2);
  double rho = pow(10.0, lr) / hl.rho_unit_cgs;
  double u = pow(10.0, lt) / bp.tfac;
  double dt = pow(10.0, ld) / hl.t_unit_s;
  float x[3];
  mlp_inputs(u, rho, dt, bp, hl, x);
  X[3 * i] = x[0];
  X[3 * i + 1] = x[1];
  X[3 * i + 2] = x[2];
  Y[i] = mlp_label(u, rho, dt, bp);
  if (U) {
    U[3 * i] = u;
    U[3 * i + 1] = rho;
    U[3 * i + 2] = dt;
  }
}

__global__ void k_mlp_init(uint64_t seed, float* __restrict__ w) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= MLP_NPARAM) return;
  float fan_in = p < MLP_B1 ? (float)MLP_IN : (float)MLP_H;
  bool bias = (p >= MLP_B1 && p < MLP_W2) || (p >= MLP_B2 && p < MLP_W3) ||
              (p >= MLP_B3 && p < MLP_W4) || p == MLP_B4;
  float a = sqrtf(3.0f / fan_in);  // uniform with variance 1/fan_in
  float r = (float)uniform01(seed, (uint64_t)p, 3) * 2.0f - 1.0f;
  w[p] = bias ? 0.0f : a * r;
}

__device__ __forceinline__ float bf16r(float w) { return __bfloat162float(__float2bfloat16(w)); }

// ---------------------------------------------------------------- training kernels
// Z = A W^T + b (W rounded to BF16), A_out = SiLU(Z) (identity for the last layer)
__global__ void k_fwd(int64_t B, int in, int out, const float* __restrict__ A, const float* __restrict__ W,
                      const float* __restrict__ b, float* __restrict__ Z, float* __restrict__ Aout, int act) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= B * out) return;
  int64_t s = t / out;
  int o = (int)(t % out);
  float z = b[o];
  for (int i = 0; i < in; ++i) z = fmaf(bf16r(W[o * in + i]), A[s * in + i], z);
  Z[t] = z;
  Aout[t] = act == 1 ? silu(z) : (act == 2 ? 1.0f / (1.0f + __expf(-z)) : z);
}

// the output is f = sigmoid(z4); loss = mean (f - label)^2: dZ4 = 2 (f - label) f (1 - f) / B
__global__ void k_loss(int64_t B, const float* __restrict__ y, const float* __restrict__ lab,
                       float* __restrict__ dz, float* __restrict__ se) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= B) return;
  float f = y[s];
  float d = f - lab[s];
  dz[s] = 2.0f * d * f * (1.0f - f) / (float)B;
  se[s] = d * d;
}

// dA_in = dZ W (W rounded as in the forward pass); then optionally dZ_in = dA_in * SiLU'(Z_in)
__global__ void k_bwd_in(int64_t B, int in, int out, const float* __restrict__ dZ,
                         const float* __restrict__ W, const float* __restrict__ Zin,
                         float* __restrict__ dZin) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= B * in) return;
  int64_t s = t / in;
  int i = (int)(t % in);
  float g = 0.0f;
  for (int o = 0; o < out; ++o) g = fmaf(dZ[s * out + o], bf16r(W[o * in + i]), g);
  dZin[t] = g * dsilu(Zin[t]);
}

// partial weight and bias gradients of one chunk of samples: P[c][o][in + 1]
constexpr int WG_CHUNK = 256;
__global__ void k_wgrad(int64_t B, int in, int out, const float* __restrict__ dZ,
                        const float* __restrict__ A, float* __restrict__ part) {
  int c = blockIdx.x;
  int64_t s0 = (int64_t)c * WG_CHUNK, s1 = min(s0 + WG_CHUNK, B);
  int npar = out * (in + 1);
  for (int q = threadIdx.x; q < npar; q += blockDim.x) {
    int o = q / (in + 1), i = q % (in + 1);
    float g = 0.0f;
    if (i < in) {
      for (int64_t s = s0; s < s1; ++s) g = fmaf(dZ[s * out + o], A[s * in + i], g);
    } else {
      for (int64_t s = s0; s < s1; ++s) g += dZ[s * out + o];
    }
    part[(int64_t)c * npar + q] = g;
  }
}

// sum the chunk partials in chunk order into the flat gradient (W block then bias block)
__global__ void k_wgrad_reduce(int nchunk, int in, int out, const float* __restrict__ part,
                               float* __restrict__ gW, float* __restrict__ gb) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  int npar = out * (in + 1);
  if (q >= npar) return;
  float g = 0.0f;
  for (int c = 0; c < nchunk; ++c) g += part[(int64_t)c * npar + q];
  int o = q / (in + 1), i = q % (in + 1);
  if (i < in)
    gW[o * in + i] = g;
  else
    gb[o] = g;
}

__global__ void k_adam(int n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  float gp = g[p];
  float mp = b1 * m[p] + (1.0f - b1) * gp;
  float vp = b2 * v[p] + (1.0f - b2) * gp * gp;
  m[p] = mp;
  v[p] = vp;
  w[p] -= lr * (mp / c1) / (sqrtf(vp / c2) + eps);
}

__global__ void k_sum_f(int64_t n, const float* __restrict__ a, double* __restrict__ out) {
  __shared__ double s[NB_THREADS];
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) acc += a[i];
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0];
}

// ---------------------------------------------------------------- one forward + backward
struct MlpBuffers {
  int64_t cap = 0;
  float *Z1 = nullptr, *A1 = nullptr, *Z2 = nullptr, *A2 = nullptr, *Z3 = nullptr, *A3 = nullptr,
        *Y = nullptr, *Yd = nullptr, *dY = nullptr, *se = nullptr, *dZ3 = nullptr, *dZ2 = nullptr,
        *dZ1 = nullptr, *dZ4 = nullptr, *part = nullptr;
  double* red = nullptr;
  void release() {
    float* ps[] = {Z1, A1, Z2, A2, Z3, A3, Y, Yd, dY, se, dZ3, dZ2, dZ1, dZ4, part};
    for (float* p : ps)
      if (p) cudaFree(p);
    if (red) cudaFree(red);
    *this = MlpBuffers{};
  }
};

static int mlp_buffers(Engine& E, MlpBuffers& M, int64_t B) {
  if (B <= M.cap) return 0;
  M.release();
  float** f64[] = {&M.Z1, &M.A1, &M.Z2, &M.A2, &M.Z3, &M.A3, &M.dZ3, &M.dZ2, &M.dZ1};
  for (float** p : f64) NB_CUDA(cudaMalloc((void**)p, sizeof(float) * B * MLP_H));
  float** f1[] = {&M.Y, &M.Yd, &M.dY, &M.se, &M.dZ4};
  for (float** p : f1) NB_CUDA(cudaMalloc((void**)p, sizeof(float) * B));
  int64_t nchunk = (B + WG_CHUNK - 1) / WG_CHUNK;
  NB_CUDA(cudaMalloc((void**)&M.part, sizeof(float) * nchunk * MLP_H * (MLP_H + 1)));
  NB_CUDA(cudaMalloc((void**)&M.red, sizeof(double) * 4));
  M.cap = B;
  return 0;
}

// Forward and backward of one batch (X: B x 3, labels: B) at weights w: gradient into g (P),
// mean squared error into *loss (host).
static int mlp_grad(Engine& E, MlpBuffers& M, int64_t B, const float* X, const float* lab,
                    const float* w, float* g, double* loss, cudaStream_t st) {
  NB_TRY(mlp_buffers(E, M, B));
  const int T = NB_THREADS;
  auto G = [&](int64_t n) { return grid_for(n, T); };
  count_launch(), k_fwd<<<G(B * MLP_H), T, 0, st>>>(B, MLP_IN, MLP_H, X, w + MLP_W1, w + MLP_B1, M.Z1, M.A1, 1);
  count_launch(), k_fwd<<<G(B * MLP_H), T, 0, st>>>(B, MLP_H, MLP_H, M.A1, w + MLP_W2, w + MLP_B2, M.Z2, M.A2, 1);
  count_launch(), k_fwd<<<G(B * MLP_H), T, 0, st>>>(B, MLP_H, MLP_H, M.A2, w + MLP_W3, w + MLP_B3, M.Z3, M.A3, 1);
  count_launch(), k_fwd<<<G(B), T, 0, st>>>(B, MLP_H, 1, M.A3, w + MLP_W4, w + MLP_B4, M.Yd, M.Y, 2);
  count_launch(), k_loss<<<G(B), T, 0, st>>>(B, M.Y, lab, M.dZ4, M.se);
  int nchunk = (int)((B + WG_CHUNK - 1) / WG_CHUNK);
  // layer 4
  count_launch(), k_wgrad<<<nchunk, T, 0, st>>>(B, MLP_H, 1, M.dZ4, M.A3, M.part);
  count_launch(), k_wgrad_reduce<<<G(MLP_H + 1), T, 0, st>>>(nchunk, MLP_H, 1, M.part, g + MLP_W4, g + MLP_B4);
  count_launch(), k_bwd_in<<<G(B * MLP_H), T, 0, st>>>(B, MLP_H, 1, M.dZ4, w + MLP_W4, M.Z3, M.dZ3);
  // layer 3
  count_launch(), k_wgrad<<<nchunk, T, 0, st>>>(B, MLP_H, MLP_H, M.dZ3, M.A2, M.part);
  count_launch(), k_wgrad_reduce<<<G(MLP_H * (MLP_H + 1)), T, 0, st>>>(nchunk, MLP_H, MLP_H, M.part, g + MLP_W3, g + MLP_B3);
  count_launch(), k_bwd_in<<<G(B * MLP_H), T, 0, st>>>(B, MLP_H, MLP_H, M.dZ3, w + MLP_W3, M.Z2, M.dZ2);
  // layer 2
  count_launch(), k_wgrad<<<nchunk, T, 0, st>>>(B, MLP_H, MLP_H, M.dZ2, M.A1, M.part);
  count_launch(), k_wgrad_reduce<<<G(MLP_H * (MLP_H + 1)), T, 0, st>>>(nchunk, MLP_H, MLP_H, M.part, g + MLP_W2, g + MLP_B2);
  count_launch(), k_bwd_in<<<G(B * MLP_H), T, 0, st>>>(B, MLP_H, MLP_H, M.dZ2, w + MLP_W2, M.Z1, M.dZ1);
  // layer 1
  count_launch(), k_wgrad<<<nchunk, T, 0, st>>>(B, MLP_IN, MLP_H, M.dZ1, X, M.part);
  count_launch(), k_wgrad_reduce<<<G(MLP_H * (MLP_IN + 1)), T, 0, st>>>(nchunk, MLP_IN, MLP_H, M.part, g + MLP_W1, g + MLP_B1);
  if (loss) {
    count_launch(), k_sum_f<<<1, NB_THREADS, 0, st>>>(B, M.se, M.red);
    double h = 0;
    NB_CUDA(cudaMemcpyAsync(&h, M.red, sizeof(double), cudaMemcpyDeviceToHost, st));
    NB_CUDA(host_sync(st));
    *loss = h / (double)B;
  }
  NB_CUDA(cudaGetLastError());
  return 0;
}

// ---------------------------------------------------------------- fused inference
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// split a pair of floats into BF16 high parts and BF16 remainders
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
  __nv_bfloat16 ah = __float2bfloat16(a), bh = __float2bfloat16(b);
  float ar = a - __bfloat162float(ah), br = b - __bfloat162float(bh);
  __nv_bfloat162 h;
  h.x = ah;
  h.y = bh;
  hi = *reinterpret_cast<uint32_t*>(&h);
  lo = pack_bf16(ar, br);
}

__device__ __forceinline__ void mma16816(float& d0, float& d1, float& d2, float& d3, uint32_t a0,
                                         uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d0), "+f"(d1), "+f"(d2), "+f"(d3)
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Shared-memory image of the network: BF16 weights (row = output unit, K contiguous), FP32 biases.
struct MlpSmem {
  __nv_bfloat16 w1[MLP_H][16];     // cols 0-2 and 3-5: W1 (high parts and remainders share W1)
  __nv_bfloat16 w2[MLP_H][MLP_H];
  __nv_bfloat16 w3[MLP_H][MLP_H];
  __nv_bfloat16 w4[8][MLP_H];      // row 0: W4
  float b1[MLP_H], b2[MLP_H], b3[MLP_H], b4;
};

__device__ void mlp_load_smem(MlpSmem& S, const float* __restrict__ w) {
  for (int q = threadIdx.x; q < MLP_H * 16; q += blockDim.x) {
    int o = q / 16, k = q % 16;
    float v = k < 3 ? w[MLP_W1 + o * 3 + k] : (k < 6 ? w[MLP_W1 + o * 3 + k - 3] : 0.0f);
    S.w1[o][k] = __float2bfloat16(v);
  }
  for (int q = threadIdx.x; q < MLP_H * MLP_H; q += blockDim.x) {
    S.w2[q / MLP_H][q % MLP_H] = __float2bfloat16(w[MLP_W2 + q]);
    S.w3[q / MLP_H][q % MLP_H] = __float2bfloat16(w[MLP_W3 + q]);
  }
  for (int q = threadIdx.x; q < 8 * MLP_H; q += blockDim.x)
    S.w4[q / MLP_H][q % MLP_H] = __float2bfloat16(q < MLP_H ? w[MLP_W4 + q] : 0.0f);
  for (int q = threadIdx.x; q < MLP_H; q += blockDim.x) {
    S.b1[q] = w[MLP_B1 + q];
    S.b2[q] = w[MLP_B2 + q];
    S.b3[q] = w[MLP_B3 + q];
  }
  if (threadIdx.x == 0) S.b4 = w[MLP_B4];
}

__device__ __forceinline__ uint32_t ld2(const __nv_bfloat16* p) {
  return *reinterpret_cast<const uint32_t*>(p);
}

// SiLU for inference: the reciprocal of 1 + e^-z by the fast approximate division (within 2
// ulp; the training pass uses the IEEE division, a difference far below the BF16 rounding of the
// activations that follows)
__device__ __forceinline__ float silu_inf(float z) { return __fdividef(z, 1.0f + __expf(-z)); }

// One hidden layer on tensor cores: in (hi, lo) fragments for 4 k-steps -> out fragments.
__device__ __forceinline__ void mlp_hidden(const __nv_bfloat16 (*W)[MLP_H], const float* bias,
                                           const uint32_t ahi[4][4], const uint32_t alo[4][4],
                                           uint32_t ohi[4][4], uint32_t olo[4][4], int g, int t) {
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    float c0 = bias[j * 8 + 2 * t], c1 = bias[j * 8 + 2 * t + 1];
    float d0 = c0, d1 = c1, d2 = c0, d3 = c1;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      uint32_t b0 = ld2(&W[j * 8 + g][kk * 16 + 2 * t]);
      uint32_t b1 = ld2(&W[j * 8 + g][kk * 16 + 8 + 2 * t]);
      mma16816(d0, d1, d2, d3, ahi[kk][0], ahi[kk][1], ahi[kk][2], ahi[kk][3], b0, b1);
      mma16816(d0, d1, d2, d3, alo[kk][0], alo[kk][1], alo[kk][2], alo[kk][3], b0, b1);
    }
    d0 = silu_inf(d0);
    d1 = silu_inf(d1);
    d2 = silu_inf(d2);
    d3 = silu_inf(d3);
    // n-tile j is half of the next layer's k-step j/2: rows g (regs 0/2) and g+8 (regs 1/3)
    int kk = j >> 1, hsel = (j & 1) * 2;
    split2(d0, d1, ohi[kk][hsel], olo[kk][hsel]);
    split2(d2, d3, ohi[kk][hsel + 1], olo[kk][hsel + 1]);
  }
}

// Cooling of n particles over dt (per particle, code units) at fixed rho: the network's f where
// the inputs lie inside the hull and the a-posteriori bracket holds, else the exact integrator.
// mode_out (optional): 0 exact (at or below the floor, or not cooled), 1 network, 2 fallback.
// judge: every judge-th network result is compared with the exact one (|du_mlp - du_exact| / u
// accumulated as max and sum of squares in stats[0..1], count in stats[2]).
#ifndef MLP_BLOCKS_PER_SM
// resident blocks per SM: 4 (128 registers, 48 B spilled) measured 0.936 ms per 4M torus step
// against 0.996 with 5 (96 registers, 208 B spilled) and 0.992 with 3
#define MLP_BLOCKS_PER_SM 4
#endif
__global__ void __launch_bounds__(128, MLP_BLOCKS_PER_SM) k_mlp_cool(int64_t n, const double* __restrict__ u_in,
                                                  const double* __restrict__ rho,
                                                  const double* __restrict__ dt, double dt_scalar,
                                                  const float* __restrict__ w, BremsParams bp,
                                                  MlpHull hl, int judge, double* __restrict__ u_out,
                                                  int8_t* __restrict__ mode_out,
                                                  unsigned long long* __restrict__ counts,
                                                  double* __restrict__ stats) {
  __shared__ MlpSmem S;
  mlp_load_smem(S, w);
  __syncthreads();
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int warps = blockDim.x >> 5;
  int64_t wid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int64_t nwarps = (int64_t)gridDim.x * warps;
  unsigned long long n_mlp = 0, n_fb = 0;
  double j_e2 = 0.0, j_n = 0.0, j_max = 0.0;  // judged errors of this thread (summed per warp)
  for (int64_t base = wid * 32; base < n; base += nwarps * 32) {
    // lane l: the scaled inputs and, after the two tiles below, the network's f of particle
    // base + l; the tensor tiles take rows 0-15 (lanes 0-15's inputs) and then rows 16-31
    int64_t me = base + lane;
    bool have = me < n;
    double u = have ? u_in[me] : 1.0, r = have ? rho[me] : 1.0;
    double d = have ? (dt ? dt[me] : dt_scalar) : 1.0;
    float x[3] = {0.f, 0.f, 0.f};
    bool inside = have && mlp_inputs(u, r, d, bp, hl, x);
    bool hot = have && (bp.tfac * u > bp.t_floor) && d > 0;
    float f_a = 0.f, f_b = 0.f;
#pragma unroll 1
    for (int tile = 0; tile < 2; ++tile) {
      // layer 1 (K = 16: x high parts in cols 0-2, remainders in cols 3-5)
      float xr[2][3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        xr[0][c] = __shfl_sync(0xffffffffu, x[c], 16 * tile + g);
        xr[1][c] = __shfl_sync(0xffffffffu, x[c], 16 * tile + g + 8);
      }
      uint32_t a[4] = {0u, 0u, 0u, 0u};
#pragma unroll
      for (int rr = 0; rr < 2; ++rr) {
        float hi0 = __bfloat162float(__float2bfloat16(xr[rr][0]));
        float hi1 = __bfloat162float(__float2bfloat16(xr[rr][1]));
        float hi2 = __bfloat162float(__float2bfloat16(xr[rr][2]));
        float c6[6] = {hi0, hi1, hi2, xr[rr][0] - hi0, xr[rr][1] - hi1, xr[rr][2] - hi2};
        // a0/a1: cols 2t, 2t+1 of rows g / g+8 (a2, a3: cols 8+ are zero)
        float e0 = 2 * t < 6 ? c6[2 * t] : 0.f, e1 = 2 * t + 1 < 6 ? c6[2 * t + 1] : 0.f;
        a[rr] = pack_bf16(e0, e1);
      }
      uint32_t h1hi[4][4], h1lo[4][4];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        float c0 = S.b1[j * 8 + 2 * t], c1 = S.b1[j * 8 + 2 * t + 1];
        float d0 = c0, d1 = c1, d2 = c0, d3 = c1;
        uint32_t b0 = ld2(&S.w1[j * 8 + g][2 * t]);
        uint32_t b1 = ld2(&S.w1[j * 8 + g][8 + 2 * t]);
        mma16816(d0, d1, d2, d3, a[0], a[1], a[2], a[3], b0, b1);
        d0 = silu_inf(d0);
        d1 = silu_inf(d1);
        d2 = silu_inf(d2);
        d3 = silu_inf(d3);
        int kk = j >> 1, hsel = (j & 1) * 2;
        split2(d0, d1, h1hi[kk][hsel], h1lo[kk][hsel]);
        split2(d2, d3, h1hi[kk][hsel + 1], h1lo[kk][hsel + 1]);
      }
      uint32_t h2hi[4][4], h2lo[4][4];
      mlp_hidden(S.w2, S.b2, h1hi, h1lo, h2hi, h2lo, g, t);
      mlp_hidden(S.w3, S.b3, h2hi, h2lo, h1hi, h1lo, g, t);
      // output layer: one n-tile, only column 0 is real
      float o0 = S.b4, o1 = 0.f, o2 = S.b4, o3 = 0.f;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        uint32_t b0 = ld2(&S.w4[g][kk * 16 + 2 * t]);
        uint32_t b1 = ld2(&S.w4[g][kk * 16 + 8 + 2 * t]);
        mma16816(o0, o1, o2, o3, h1hi[kk][0], h1hi[kk][1], h1hi[kk][2], h1hi[kk][3], b0, b1);
        mma16816(o0, o1, o2, o3, h1lo[kk][0], h1lo[kk][1], h1lo[kk][2], h1lo[kk][3], b0, b1);
      }
      // lanes with t == 0 hold f of rows g (o0) and g + 8 (o2) of the tile; lane l takes row l % 16
      float f_lo = __shfl_sync(0xffffffffu, o0, (lane & 7) * 4);
      float f_hi = __shfl_sync(0xffffffffu, o2, ((lane & 7)) * 4);
      const float f_row = (lane & 15) < 8 ? f_lo : f_hi;
      if (tile == 0)
        f_a = f_row;
      else
        f_b = f_row;
    }
    const float f = lane < 16 ? f_a : f_b;
    if (have) {
      double un;
      int mode = 0;
      if (!hot) {
        un = u;
      } else {
        bool ok = inside;
        // the network predicts the logit f; its sigmoid in float (1e-7 of u, far inside the
        // acceptance test below, which judges the u it implies)
        double ff = (double)(1.0f / (1.0f + __expf(-f)));
        double um = u - ff * (u - bp.u_floor);
        if (ok) {
          // a-posteriori acceptance: the cooling rate r(u) grows with T, so the exact step du_e
          // satisfies dt r(u_e) <= du_e <= dt r(u).  If du_m lies within tol of
          // [dt r(u_m), dt r(u)], then |du_m - du_e| <= dt (r(u) - r(u_m)) + tol; accept only
          // when that bound is <= 2 tol.  A prediction at the floor is accepted only when even
          // the floor's rate dt r(u_floor) removes all of u - u_floor (then the exact step ends
          // at the floor too).
          double du = u - um;
          double tol = hl.check_tol * u;
          double r_hi = d * fabs(brems_rate(u, r, bp));
          if (ff >= 1.0 - 1e-6) {
            double r_f = d * fabs(brems_rate(bp.u_floor * (1.0 + 1e-12), r, bp));
            ok = r_f >= u - bp.u_floor;
            um = bp.u_floor;
          } else {
            double r_lo = d * fabs(brems_rate(um, r, bp));
            ok = du >= r_lo - tol && du <= r_hi + tol && (r_hi - r_lo) <= tol;
          }
        }
        if (ok) {
          un = um;
          mode = 1;
          n_mlp++;
          if (judge > 0 && stats && (me % judge) == 0) {
            double ue = brems_cool_one(u, r, d, bp);
            double e = fabs(um - ue) / u;
            j_e2 += e * e;
            j_n += 1.0;
            j_max = fmax(j_max, e);
          }
        } else {
          un = brems_cool_one(u, r, d, bp);
          mode = 2;
          n_fb++;
        }
      }
      u_out[me] = un;
      if (mode_out) mode_out[me] = (int8_t)mode;
    }
  }
  // one atomic per warp for the counts and the judged statistics
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    n_mlp += __shfl_xor_sync(0xffffffffu, n_mlp, o);
    n_fb += __shfl_xor_sync(0xffffffffu, n_fb, o);
    j_e2 += __shfl_xor_sync(0xffffffffu, j_e2, o);
    j_n += __shfl_xor_sync(0xffffffffu, j_n, o);
    j_max = fmax(j_max, __shfl_xor_sync(0xffffffffu, j_max, o));
  }
  if (lane == 0) {
    if (counts) {
      atomicAdd(&counts[0], n_mlp);
      atomicAdd(&counts[1], n_fb);
    }
    if (stats && j_n > 0.0) {
      atomicAdd(&stats[1], j_e2);
      atomicAdd(&stats[2], j_n);
      // non-negative doubles order like their bits
      atomicMax((unsigned long long*)&stats[0], (unsigned long long)__double_as_longlong(j_max));
    }
  }
}

// ---------------------------------------------------------------- host side
struct MlpState {
  float* w = nullptr;  // trained FP32 weights (device, MLP_NPARAM)
  double* stats = nullptr;  // judge statistics (device, 3)
  unsigned long long* counts = nullptr;  // (device, 2)
  MlpBuffers buf;
};

static MlpState g_mlp_state[64];

MlpHull hull_of(const nb_mlp_params* mp) {
  MlpHull h;
  h.rho_unit_cgs = mp->rho_unit_cgs;
  h.t_unit_s = mp->t_unit_s;
  h.lrho_lo = mp->lrho_lo;
  h.lrho_hi = mp->lrho_hi;
  h.lt_lo = mp->lt_lo;
  h.lt_hi = mp->lt_hi;
  h.ldt_lo = mp->ldt_lo;
  h.ldt_hi = mp->ldt_hi;
  h.check_tol = mp->check_tol;
  return h;
}

BremsParams brems_of_mlp(const nb_mlp_params* mp) {
  BremsParams b;
  b.tfac = mp->tfac;
  b.b = mp->b;
  b.kappa = mp->kappa;
  b.u_floor = mp->u_floor;
  b.t_floor = mp->t_floor;
  return b;
}

int mlp_state(Engine& E, MlpState** out) {
  MlpState& M = g_mlp_state[E.device & 63];
  if (!M.w) {
    NB_CUDA(cudaMalloc((void**)&M.w, sizeof(float) * MLP_NPARAM));
    NB_CUDA(cudaMemset(M.w, 0, sizeof(float) * MLP_NPARAM));
    NB_CUDA(cudaMalloc((void**)&M.stats, sizeof(double) * 3));
    NB_CUDA(cudaMemset(M.stats, 0, sizeof(double) * 3));
    NB_CUDA(cudaMalloc((void**)&M.counts, sizeof(unsigned long long) * 2));
    NB_CUDA(cudaMemset(M.counts, 0, sizeof(unsigned long long) * 2));
  }
  *out = &M;
  return 0;
}

int mlp_train(Engine& E, const nb_mlp_params* mp, int64_t nsamp, int64_t batch, int epochs,
              double lr, uint64_t seed, float* loss_hist, cudaStream_t st) {
  MlpState* M;
  NB_TRY(mlp_state(E, &M));
  BremsParams bp = brems_of_mlp(mp);
  MlpHull hl = hull_of(mp);
  float *X = nullptr, *Y = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  NB_CUDA(cudaMalloc((void**)&X, sizeof(float) * 3 * nsamp));
  NB_CUDA(cudaMalloc((void**)&Y, sizeof(float) * nsamp));
  NB_CUDA(cudaMalloc((void**)&g, sizeof(float) * MLP_NPARAM));
  NB_CUDA(cudaMalloc((void**)&m, sizeof(float) * MLP_NPARAM));
  NB_CUDA(cudaMalloc((void**)&v, sizeof(float) * MLP_NPARAM));
  NB_CUDA(cudaMemsetAsync(m, 0, sizeof(float) * MLP_NPARAM, st));
  NB_CUDA(cudaMemsetAsync(v, 0, sizeof(float) * MLP_NPARAM, st));
  count_launch(), k_mlp_data<<<grid_for(nsamp), NB_THREADS, 0, st>>>(nsamp, seed, bp, hl, X, Y, nullptr);
  count_launch(), k_mlp_init<<<grid_for(MLP_NPARAM), NB_THREADS, 0, st>>>(seed ^ 0x5bd1e995ull, M->w);
  int64_t nb = nsamp / batch;
  int64_t step = 0;
  int rc = 0;
  for (int ep = 0; ep < epochs && rc == 0; ++ep) {
    double ep_loss = 0.0;
    // cosine decay of the learning rate over the run
    for (int64_t bi = 0; bi < nb && rc == 0; ++bi) {
      double frac = (double)step / (double)(epochs * nb);
      float lr_t = (float)(lr * 0.5 * (1.0 + cos(M_PI * frac)) + 1e-6);
      double loss = 0;
      bool want = (bi == nb - 1) && loss_hist;
      rc = mlp_grad(E, M->buf, batch, X + 3 * bi * batch, Y + bi * batch, M->w, g,
                    want ? &loss : nullptr, st);
      step += 1;
      float c1 = 1.0f - powf(0.9f, (float)step), c2 = 1.0f - powf(0.999f, (float)step);
      count_launch(), k_adam<<<grid_for(MLP_NPARAM), NB_THREADS, 0, st>>>(MLP_NPARAM, M->w, g, m, v, lr_t, 0.9f,
                                                           0.999f, 1e-8f, c1, c2);
      if (want) ep_loss = loss;
    }
    if (loss_hist) loss_hist[ep] = (float)ep_loss;
  }
  host_sync(st);
  cudaFree(X);
  cudaFree(Y);
  cudaFree(g);
  cudaFree(m);
  cudaFree(v);
  if (rc) return rc;
  NB_CUDA(cudaGetLastError());
  return 0;
}

int mlp_cool(Engine& E, int64_t n, const double* u, const double* rho, const double* dt,
             double dt_scalar, const nb_mlp_params* mp, double* u_out, int8_t* mode,
             cudaStream_t st) {
  if (n <= 0) return 0;
  MlpState* M;
  NB_TRY(mlp_state(E, &M));
  int blocks = (int)std::min<int64_t>((n + 127) / 128, 148 * 16);
  count_launch(), k_mlp_cool<<<blocks, 128, 0, st>>>(n, u, rho, dt, dt_scalar, M->w, brems_of_mlp(mp),
                                                     hull_of(mp), mp->judge, u_out, mode, M->counts,
                                                     M->stats);
  NB_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace nbk

using nbk::Engine;

namespace {
int begin_mlp(nb_ctx* ctx) {
  if (!ctx) return NB_ERR_INPUT;
  Engine& E = ctx->E;
  E.last_error[0] = 0;
  NB_CUDA(cudaSetDevice(E.device));
  return 0;
}
}  // namespace

extern "C" {

int nb_mlp_data(nb_ctx* ctx, int64_t n, uint64_t seed, const nb_mlp_params* mp, float* X,
                float* Y, double* U, void* stream) {
  NB_TRY(begin_mlp(ctx));
  Engine& E = ctx->E;
  if (n > 0)
    nbk::count_launch(), nbk::k_mlp_data<<<nbk::grid_for(n), NB_THREADS, 0, (cudaStream_t)stream>>>(
        n, seed, nbk::brems_of_mlp(mp), nbk::hull_of(mp), X, Y, U);
  NB_CUDA(cudaGetLastError());
  return 0;
}

int nb_mlp_grad(nb_ctx* ctx, int64_t batch, const float* X, const float* Y, const float* w, float* g,
                double* loss, void* stream) {
  NB_TRY(begin_mlp(ctx));
  nbk::MlpState* M;
  NB_TRY(nbk::mlp_state(ctx->E, &M));
  return nbk::mlp_grad(ctx->E, M->buf, batch, X, Y, w, g, loss, (cudaStream_t)stream);
}

int nb_mlp_train(nb_ctx* ctx, const nb_mlp_params* mp, int64_t n_samples, int64_t batch,
                 int epochs, double lr, uint64_t seed, float* loss_hist, void* stream) {
  NB_TRY(begin_mlp(ctx));
  Engine& E = ctx->E;
  if (batch <= 0 || n_samples < batch || epochs <= 0)
    return nbk::set_host_error(E, "nb_mlp_train: need 0 < batch <= n_samples and epochs > 0"),
           NB_ERR_INPUT;
  return nbk::mlp_train(E, mp, n_samples, batch, epochs, lr, seed, loss_hist, (cudaStream_t)stream);
}

int nb_mlp_weights(nb_ctx* ctx, float* w_out, const float* w_in, void* stream) {
  NB_TRY(begin_mlp(ctx));
  Engine& E = ctx->E;
  nbk::MlpState* M;
  NB_TRY(nbk::mlp_state(E, &M));
  cudaStream_t st = (cudaStream_t)stream;
  if (w_out) NB_CUDA(cudaMemcpyAsync(w_out, M->w, sizeof(float) * nbk::MLP_NPARAM, cudaMemcpyDeviceToDevice, st));
  if (w_in) NB_CUDA(cudaMemcpyAsync(M->w, w_in, sizeof(float) * nbk::MLP_NPARAM, cudaMemcpyDeviceToDevice, st));
  NB_CUDA(nbk::host_sync(st));
  return 0;
}

int nb_mlp_cool(nb_ctx* ctx, int64_t n, const double* u, const double* rho, const double* dt,
                double dt_scalar, const nb_mlp_params* mp, double* u_out, int8_t* mode, void* stream) {
  NB_TRY(begin_mlp(ctx));
  return nbk::mlp_cool(ctx->E, n, u, rho, dt, dt_scalar, mp, u_out, mode, (cudaStream_t)stream);
}

int nb_mlp_stats(nb_ctx* ctx, double* out, int reset) {
  NB_TRY(begin_mlp(ctx));
  Engine& E = ctx->E;
  nbk::MlpState* M;
  NB_TRY(nbk::mlp_state(E, &M));
  double s[3];
  unsigned long long c[2];
  NB_CUDA(cudaDeviceSynchronize());
  NB_CUDA(cudaMemcpy(s, M->stats, sizeof(s), cudaMemcpyDeviceToHost));
  NB_CUDA(cudaMemcpy(c, M->counts, sizeof(c), cudaMemcpyDeviceToHost));
  out[0] = s[0];
  out[1] = s[2] > 0 ? sqrt(s[1] / s[2]) : 0.0;
  out[2] = s[2];
  out[3] = (double)c[0];
  out[4] = (double)c[1];
  if (reset) {
    NB_CUDA(cudaMemset(M->stats, 0, sizeof(s)));
    NB_CUDA(cudaMemset(M->counts, 0, sizeof(c)));
  }
  return 0;
}

}  // extern "C"
