/*
 * hm_snow.cu - the post-filter of snow_simulation on sm_100a: the snow
 * cover settled by masked thermal erosion of terrain + snow.
 *
 * Replaces HighMap/src/hydrology/snow_simulation.cpp:140-152 and the
 * clamp_min(s, 0) that follows it:
 *   mask = clamp_max_smooth(s / snow_depth, 1), k = 0.2 (range.cpp:98-110,
 *          default of range.hpp:195);
 *   z_w  = z + s;
 *   talus = ratio * gradient_norm(z_w) (gradient.cpp:124-135 with
 *          gradient_x / gradient_y, gradient.cpp:182-215: 0.5 (a(i+1) -
 *          a(i-1)) inside, one-sided differences on the edges; the norm is
 *          sqrt(dx dx + dy dy) in fp32, math.cpp:142-151);
 *   thermal(z_w, &mask, talus, iterations) (thermal_core, masked);
 *   s = max(z_w - z, 0).
 * One kernel builds the mask, z_w and the talus map (the talus of a cell
 * re-forms z_w of its four neighbours from z and s, bit-identical to the
 * stored values), thermal_core runs the steps and the blend, and one
 * kernel forms the new snow depth.
 */
#include <cuda_runtime.h>

#include "hm_internal.h"
#include "hm_thermal.h"

namespace hm
{

namespace
{

constexpr int SN_NT = 256;
constexpr int SN_GRID = 148 * 8;

__device__ __forceinline__ float zw_at(const float *__restrict__ z, const float *__restrict__ s, size_t k)
{
  return __fadd_rn(z[k], s[k]);
}

__global__ void __launch_bounds__(SN_NT) k_snow_prep(const float *__restrict__ z,
                                                     const float *__restrict__ s,
                                                     float *__restrict__ mask,
                                                     float *__restrict__ zw,
                                                     float *__restrict__ talus,
                                                     int nx,
                                                     int ny,
                                                     float snow_depth,
                                                     float ratio)
{
  const size_t n = (size_t)nx * ny;
  for (size_t k = blockIdx.x * (size_t)SN_NT + threadIdx.x; k < n; k += (size_t)gridDim.x * SN_NT)
  {
    const int j = (int)(k / (size_t)nx), i = (int)(k - (size_t)j * nx);
    /* clamp_max_smooth(x, 1, 0.2): min(x, 1) - h^3 k / 6 with
     * h = max(k - |x - 1|, 0) / k (std::max / std::min order) */
    const float x = __fdiv_rn(s[k], snow_depth);
    const float kk = 0.2f;
    const float a = __fsub_rn(kk, fabsf(__fsub_rn(x, 1.f)));
    const float h = __fdiv_rn(a < 0.f ? 0.f : a, kk);
    const float lo = 1.f < x ? 1.f : x;
    mask[k] = __fsub_rn(lo, __fdiv_rn(__fmul_rn(__fmul_rn(__fmul_rn(h, h), h), kk), 6.f));
    zw[k] = zw_at(z, s, k);
    float dx, dy;
    if (i == 0) dx = __fsub_rn(zw_at(z, s, k + 1), zw_at(z, s, k));
    else if (i == nx - 1) dx = __fsub_rn(zw_at(z, s, k), zw_at(z, s, k - 1));
    else dx = __fmul_rn(0.5f, __fsub_rn(zw_at(z, s, k + 1), zw_at(z, s, k - 1)));
    if (j == 0) dy = __fsub_rn(zw_at(z, s, k + nx), zw_at(z, s, k));
    else if (j == ny - 1) dy = __fsub_rn(zw_at(z, s, k), zw_at(z, s, k - nx));
    else dy = __fmul_rn(0.5f, __fsub_rn(zw_at(z, s, k + nx), zw_at(z, s, k - nx)));
    talus[k] = __fmul_rn(ratio, __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy))));
  }
}

/* s = max(z_w - z, 0) (clamp_min: x > 0 ? x : 0) */
__global__ void __launch_bounds__(SN_NT) k_snow_final(const float *__restrict__ z, const float *__restrict__ zw,
                                                      float *__restrict__ s, size_t n)
{
  for (size_t k = blockIdx.x * (size_t)SN_NT + threadIdx.x; k < n; k += (size_t)gridDim.x * SN_NT)
  {
    const float d = __fsub_rn(zw[k], z[k]);
    s[k] = d > 0.f ? d : 0.f;
  }
}

} // namespace

size_t snow_scratch_floats(int nx, int ny)
{
  /* mask, z_w, talus map, and thermal_core's two grids (masked solve) */
  return 3 * align_up((size_t)nx * ny, 64) + thermal_scratch_floats(nx, ny, true);
}

int snow_post_filter_core(int device, const float *z, float *s, int nx, int ny, float snow_depth, int iterations,
                          float ratio, float *scratch, cudaStream_t st)
{
  const size_t n = (size_t)nx * ny;
  const size_t na = align_up(n, 64);
  float       *mask = scratch, *zw = scratch + na, *talus = scratch + 2 * na, *tws = scratch + 3 * na;
  k_snow_prep<<<SN_GRID, SN_NT, 0, st>>>(z, s, mask, zw, talus, nx, ny, snow_depth, ratio);
  HM_LAUNCH_CHECK("k_snow_prep");
  int rc = thermal_core(device, zw, nx, ny, talus, 0.f, iterations, nullptr, nullptr, mask, nullptr, tws, st);
  if (rc) return rc;
  k_snow_final<<<SN_GRID, SN_NT, 0, st>>>(z, zw, s, n);
  HM_LAUNCH_CHECK("k_snow_final");
  return HM_OK;
}

} // namespace hm
