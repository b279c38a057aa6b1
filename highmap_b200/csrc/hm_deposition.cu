/*
 * hm_deposition.cu - sediment_deposition on sm_100a: a caller that chains
 * short thermal solves.
 *
 * Replaces HighMap/src/erosion/deposition.cpp:19-66: sediment is laid
 * down in `iterations` equal layers; after each layer, terrain + sediment
 * is settled by thermal_subiterations steps of thermal erosion (talus map,
 * no bedrock, then the border extrapolation, as hmap::gpu::thermal) and
 * the sediment becomes max(settled - terrain, 0) (std::max, range.cpp:
 * 253-261).  The reference re-uploads and downloads the grids around every
 * thermal call; here the terrain, the sediment and the settling grid stay
 * in HBM and each layer is two elementwise kernels around thermal_core.
 */
#include <cuda_runtime.h>

#include "hm_internal.h"
#include "hm_thermal.h"

namespace hm
{

namespace
{

/* sediment of the previous layer (from the settled grid, or 0 on the
 * first), plus one layer; the grid to settle = terrain + sediment */
__global__ void k_dep_layer(const float *__restrict__ z, float *__restrict__ smap, float *__restrict__ ztot,
                            float step, int first, size_t n)
{
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
  {
    float s = 0.f;
    if (!first)
    {
      const float d = __fsub_rn(ztot[k], z[k]);
      s = d < 0.f ? 0.f : d;
    }
    s = __fadd_rn(s, step);
    smap[k] = s;
    ztot[k] = __fadd_rn(z[k], s);
  }
}

/* last layer's sediment; z = z + sediment, blended with the input where a
 * mask is given (lerp, math.cpp:183-195) */
__global__ void k_dep_final(float *__restrict__ z, const float *__restrict__ ztot, const float *__restrict__ mask,
                            float *__restrict__ depo, int settled, size_t n)
{
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
  {
    float s = 0.f;
    if (settled)
    {
      const float d = __fsub_rn(ztot[k], z[k]);
      s = d < 0.f ? 0.f : d;
    }
    const float zf = __fadd_rn(z[k], s);
    if (mask)
    {
      const float m = mask[k];
      z[k] = __fadd_rn(__fmul_rn(z[k], __fsub_rn(1.f, m)), __fmul_rn(zf, m));
    }
    else
      z[k] = zf;
    if (depo) depo[k] = s;
  }
}

} // namespace

size_t deposition_scratch_floats(int nx, int ny)
{
  /* sediment, the grid to settle, and thermal_core's workspace */
  return 2 * align_up((size_t)nx * ny, 64) + thermal_scratch_floats(nx, ny, false);
}

int deposition_core(int device, float *z, int nx, int ny, const float *talus, float max_deposition, int iterations,
                    int thermal_subiterations, float *depo, const float *mask, float *scratch, cudaStream_t s)
{
  const size_t n = (size_t)nx * ny;
  const size_t na = align_up(n, 64);
  float       *smap = scratch, *ztot = scratch + na, *tws = scratch + 2 * na;
  /* deposition_step = max_deposition / (int)iterations (deposition.cpp:26) */
  const float step = max_deposition / (float)iterations;
  for (int it = 0; it < iterations; it++)
  {
    k_dep_layer<<<592, 256, 0, s>>>(z, smap, ztot, step, it == 0, n);
    HM_LAUNCH_CHECK("k_dep_layer");
    int rc = thermal_core(device, ztot, nx, ny, talus, 0.f, thermal_subiterations, nullptr, nullptr, nullptr, nullptr,
                          tws, s);
    if (rc) return rc;
  }
  k_dep_final<<<592, 256, 0, s>>>(z, ztot, mask, depo, iterations > 0, n);
  HM_LAUNCH_CHECK("k_dep_final");
  return HM_OK;
}

} // namespace hm
