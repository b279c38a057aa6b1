/*
 * hm_vpipes_step_tma.cu - instances of k_vp_step_tma (the previous step's
 * advection and this step's flow, water and erosion in one TMA-staged
 * tile, hm_vpipes_tiled.cuh) for every option word of the erosion steps,
 * and their launcher.  A translation unit of its own so the instances
 * compile in parallel with the rest of the library.
 */
#include <cuda_runtime.h>

#include "hm_internal.h"
#include "hm_vpipes_tiled.cuh"

namespace hm
{

namespace
{
template <bool M, int F> struct StepKernel
{
  static auto fn() { return &k_vp_step_tma<M, F>; }
};
} // namespace

int launch_step_tma(const FweIo &io, const FweMaps &maps, const AdvMaps &am, const VpConst &c, VpScalars *sc,
                    double *partials, dim3 grid, cudaStream_t s)
{
  return step_dispatch<StepKernel>(io.maintain != 0, fwe_flags(io, c), [&](auto kernel) -> int {
    kernel<<<grid, FT_NT, 0, s>>>(io, maps, am, c, sc, partials);
    HM_LAUNCH_CHECK("k_vp_step_tma");
    return HM_OK;
  });
}

} // namespace hm
