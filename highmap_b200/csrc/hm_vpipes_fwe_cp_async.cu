/*
 * hm_vpipes_fwe_cp_async.cu - instances of k_vp_fwe (flow, water and
 * erosion of one virtual-pipes step over cp.async-staged tiles,
 * hm_vpipes_tiled.cuh) for every option word, and their launcher.  Kept in
 * a translation unit of its own so the instances compile in parallel with
 * the rest of the library.
 */
#include <cuda_runtime.h>

#include "hm_internal.h"
#include "hm_vpipes_tiled.cuh"

namespace hm
{

namespace
{
template <bool M, int F> struct CpAsyncKernel
{
  static auto fn() { return &k_vp_fwe<M, F>; }
};
} // namespace

int launch_fwe_cp_async(const FweIo &io, const VpConst &c, VpScalars *sc, double *partials, dim3 grid,
                        cudaStream_t s)
{
  return fwe_dispatch<CpAsyncKernel>(io.maintain != 0, fwe_flags(io, c), [&](auto kernel) -> int {
    kernel<<<grid, FT_NT, 0, s>>>(io, c, sc, partials);
    HM_LAUNCH_CHECK("k_vp_fwe");
    return HM_OK;
  });
}

} // namespace hm
