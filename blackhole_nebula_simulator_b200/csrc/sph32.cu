// FP32 instantiations of the pair passes (fused multiply-add allowed: the FP32 path is judged
// against the FP64 oracle by its stated tolerance, not bit for bit).
#include "sph_impl.cuh"

namespace nbk {

template <typename I>
void launch_density32(int64_t nrows, const int64_t* rows, const float4* pos, const double* box6,
                      const double* mass, const double* h_start, const double* h_search,
                      const int64_t* off, const I* idx, DensityParams prm, const int32_t* out_map,
                      double* h_out, double* rho, double* omega, int64_t* iters, int64_t* flags,
                      int64_t* work, cudaStream_t st) {
  if (nrows <= 0) return;
  Pos32 geo{pos, 0.f, box6};
  count_launch(), k_density<float, Pos32, I><<<grid_for((nrows + 3) / 4 * 32, DENSITY_THREADS), DENSITY_THREADS, 0, st>>>(
      nrows, rows, geo, mass, h_start, h_search, off, idx, prm, out_map, h_out, rho, omega, iters,
      flags, work);
}

template <typename I>
void launch_forces32(int64_t nrows, const int64_t* rows, const float4* pos, const double* box6,
                     const float4* vm, const float4* hydro, const float4* aux,
                     const int64_t* off, const I* idx, ForceParams prm, const int32_t* out_map,
                     ForceOut out, cudaStream_t st) {
  if (nrows <= 0) return;
  Pos32 geo{pos, 0.f, box6};
  if (prm.use_recon && prm.use_visc) {
    count_launch(), k_forces_g<float, Pos32, I, float4, true><<<grid_for(nrows * 8), NB_THREADS, 0, st>>>(
        nrows, rows, geo, vm, hydro, aux, off, idx, prm, out_map, out);
  } else if (prm.tidx && prm.tcnt) {
    // the walk, then the pairs from its entries
    count_launch(), k_forces_g<float, Pos32, I, float4, false, 1><<<grid_for(nrows * 8), NB_THREADS, 0, st>>>(
        nrows, rows, geo, vm, hydro, aux, off, idx, prm, out_map, out);
    count_launch(), k_forces_g<float, Pos32, I, float4, false, 2><<<grid_for(nrows * 8), NB_THREADS, 0, st>>>(
        nrows, rows, geo, vm, hydro, aux, off, idx, prm, out_map, out);
  } else {
    count_launch(), k_forces_g<float, Pos32, I, float4, false><<<grid_for(nrows * 8), NB_THREADS, 0, st>>>(
        nrows, rows, geo, vm, hydro, aux, off, idx, prm, out_map, out);
  }
}


template void launch_density32<int32_t>(int64_t, const int64_t*, const float4*, const double*,
                                        const double*, const double*, const double*,
                                        const int64_t*, const int32_t*, DensityParams,
                                        const int32_t*, double*, double*, double*, int64_t*,
                                        int64_t*, int64_t*, cudaStream_t);
template void launch_forces32<int32_t>(int64_t, const int64_t*, const float4*, const double*,
                                       const float4*, const float4*, const float4*,
                                       const int64_t*, const int32_t*, ForceParams,
                                       const int32_t*, ForceOut, cudaStream_t);

}  // namespace nbk
