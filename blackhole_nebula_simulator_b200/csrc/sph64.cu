// FP64 instantiations of the pair passes (compiled without fused multiply-add: the FP64 path
// rounds like the reference).
#include "sph_impl.cuh"

namespace nbk {

template <typename I>
void launch_density64(int64_t nrows, const int64_t* rows, const double4* pos, const double* mass,
                      const double* h_start, const double* h_search, const int64_t* off,
                      const I* idx, DensityParams prm, const int32_t* out_map, double* h_out,
                      double* rho, double* omega, int64_t* iters, int64_t* flags, int64_t* work,
                      cudaStream_t st) {
  if (nrows <= 0) return;
  Pos64 geo{pos};
  count_launch(), k_density_thread<double, Pos64, I><<<grid_for(nrows), NB_THREADS, 0, st>>>(
      nrows, rows, geo, mass, h_start, h_search, off, idx, prm, out_map, h_out, rho, omega, iters,
      flags, work);
}

template <typename I>
void launch_forces64(int64_t nrows, const int64_t* rows, const double4* pos, const double4* vm,
                     const double4* hydro, const double4* aux, const int64_t* off, const I* idx,
                     ForceParams prm, const int32_t* out_map, ForceOut out, cudaStream_t st) {
  if (nrows <= 0) return;
  Pos64 geo{pos};
  if (prm.use_recon && prm.use_visc)
    count_launch(), k_forces_g<double, Pos64, I, double4, true><<<grid_for(nrows * 8), NB_THREADS, 0, st>>>(
        nrows, rows, geo, vm, hydro, aux, off, idx, prm, out_map, out);
  else
    count_launch(), k_forces_g<double, Pos64, I, double4, false><<<grid_for(nrows * 8), NB_THREADS, 0, st>>>(
        nrows, rows, geo, vm, hydro, aux, off, idx, prm, out_map, out);
}

template <typename I>
void launch_gradients(int64_t nrows, const int64_t* rows, const double4* pos, const double4* vm,
                      const double4* hydro, const double4* acc, const int64_t* off, const I* idx,
                      GradParams prm, const int32_t* out_map, GradOut out, cudaStream_t st) {
  if (nrows <= 0) return;
  Pos64 geo{pos};
  if (acc)
    count_launch(), k_gradients<I, true><<<grid_for(nrows * 8), NB_THREADS, 0, st>>>(
        nrows, rows, geo, vm, hydro, acc, off, idx, prm, out_map, out);
  else
    count_launch(), k_gradients<I, false><<<grid_for(nrows * 8), NB_THREADS, 0, st>>>(
        nrows, rows, geo, vm, hydro, acc, off, idx, prm, out_map, out);
}

void launch_shock_gradients(int64_t n, const double4* pos, const double4* vm,
                            const double4* hydro, const double4* acc, const int64_t* off,
                            const int32_t* idx, int kid, double cnorm, int recon, int recon_full,
                            const uint8_t* live_mask, const uint8_t* row_sorted,
                            const int32_t* perm, GradOut out, cudaStream_t st) {
  if (n <= 0) return;
  Pos64 geo{pos};
  if (row_sorted)
    count_launch(), k_shock_grad<int32_t, true><<<grid_for(n * 8), NB_THREADS, 0, st>>>(
        n, geo, vm, hydro, acc, off, idx, kid, cnorm, recon, recon_full, live_mask, row_sorted,
        perm, out);
  else
    count_launch(), k_shock_grad<int32_t, false><<<grid_for(n * 8), NB_THREADS, 0, st>>>(
        n, geo, vm, hydro, acc, off, idx, kid, cnorm, recon, recon_full, live_mask, row_sorted,
        perm, out);
}

template void launch_gradients<int64_t>(int64_t, const int64_t*, const double4*, const double4*,
                                        const double4*, const double4*, const int64_t*,
                                        const int64_t*, GradParams, const int32_t*, GradOut,
                                        cudaStream_t);
template void launch_gradients<int32_t>(int64_t, const int64_t*, const double4*, const double4*,
                                        const double4*, const double4*, const int64_t*,
                                        const int32_t*, GradParams, const int32_t*, GradOut,
                                        cudaStream_t);

template void launch_density64<int64_t>(int64_t, const int64_t*, const double4*, const double*,
                                        const double*, const double*, const int64_t*,
                                        const int64_t*, DensityParams, const int32_t*, double*,
                                        double*, double*, int64_t*, int64_t*, int64_t*,
                                        cudaStream_t);
template void launch_density64<int32_t>(int64_t, const int64_t*, const double4*, const double*,
                                        const double*, const double*, const int64_t*,
                                        const int32_t*, DensityParams, const int32_t*, double*,
                                        double*, double*, int64_t*, int64_t*, int64_t*,
                                        cudaStream_t);
template void launch_forces64<int64_t>(int64_t, const int64_t*, const double4*, const double4*,
                                       const double4*, const double4*, const int64_t*,
                                       const int64_t*, ForceParams, const int32_t*, ForceOut,
                                       cudaStream_t);
template void launch_forces64<int32_t>(int64_t, const int64_t*, const double4*, const double4*,
                                       const double4*, const double4*, const int64_t*,
                                       const int32_t*, ForceParams, const int32_t*, ForceOut,
                                       cudaStream_t);

// ---------------------------------------------------------------- packing (caller order)
__global__ void k_pack_pos(int64_t n, const double* __restrict__ pos, const double* __restrict__ w,
                           double4* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = make_double4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], w ? w[i] : 0.0);
}

__global__ void k_pack4(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                        const double* __restrict__ c, const double* __restrict__ d,
                        double4* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = make_double4(a ? a[i] : 0.0, b ? b[i] : 0.0, c ? c[i] : 0.0, d ? d[i] : 0.0);
}

__global__ void k_pack_vm(int64_t n, const double* __restrict__ vel, const double* __restrict__ m,
                          double4* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = make_double4(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2], m[i]);
}


void pack_pos(int64_t n, const double* pos, const double* w, double4* out, cudaStream_t st) {
  if (n > 0) count_launch(), k_pack_pos<<<grid_for(n), NB_THREADS, 0, st>>>(n, pos, w, out);
}
void pack4(int64_t n, const double* a, const double* b, const double* c, const double* d,
           double4* out, cudaStream_t st) {
  if (n > 0) count_launch(), k_pack4<<<grid_for(n), NB_THREADS, 0, st>>>(n, a, b, c, d, out);
}
void pack_vm(int64_t n, const double* vel, const double* m, double4* out, cudaStream_t st) {
  if (n > 0) count_launch(), k_pack_vm<<<grid_for(n), NB_THREADS, 0, st>>>(n, vel, m, out);
}

}  // namespace nbk
