/*
 * hm_vpipes_step_cp_async.cu - instances of k_vp_step (the previous step's
 * advection and this step's flow, water and erosion in one cp.async-staged
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
template <bool M, int F> struct StepCpKernel
{
  static auto fn() { return &k_vp_step<M, F>; }
};
} // namespace

int launch_step_cp_async(const FweIo &io, const float *u_prev, const float *v_prev, const VpConst &c, VpScalars *sc,
                         double *partials, dim3 grid, cudaStream_t s)
{
  return step_dispatch<StepCpKernel>(io.maintain != 0, fwe_flags(io, c), [&](auto kernel) -> int {
    kernel<<<grid, FT_NT, 0, s>>>(io, u_prev, v_prev, c, sc, partials);
    HM_LAUNCH_CHECK("k_vp_step");
    return HM_OK;
  });
}

} // namespace hm
