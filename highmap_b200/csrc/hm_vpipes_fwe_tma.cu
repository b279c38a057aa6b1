/*
 * hm_vpipes_fwe_tma.cu - instances of k_vp_fwe_tma (flow, water and
 * erosion of one virtual-pipes step over TMA-staged tiles,
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
template <bool M, int F> struct TmaKernel
{
  static auto fn() { return &k_vp_fwe_tma<M, F>; }
};
} // namespace

int launch_fwe_tma(const FweIo &io, const FweMaps &maps, const VpConst &c, VpScalars *sc, double *partials,
                   dim3 grid, cudaStream_t s)
{
  return fwe_dispatch<TmaKernel>(io.maintain != 0, fwe_flags(io, c), [&](auto kernel) -> int {
    kernel<<<grid, FT_NT, 0, s>>>(io, maps, c, sc, partials);
    HM_LAUNCH_CHECK("k_vp_fwe_tma");
    return HM_OK;
  });
}

} // namespace hm
