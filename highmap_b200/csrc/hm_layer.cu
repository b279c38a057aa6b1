/*
 * hm_layer.cu - sediment_layer on sm_100a: thermal erosion whose talus is
 * derived from the terrain's own slopes, with an optional smoothing
 * post-filter.
 *
 * Replaces HighMap/src/erosion/deposition.cpp:68-113:
 *   1. g = gradient_talus(z) (HighMap/src/gradient/gradient.cpp:217-243);
 *      where g > talus_upper_limit the cell's talus becomes
 *      4 (g - limit) + limit and its filter mask 0, elsewhere the talus is
 *      talus_layer and the mask 1;
 *   2. thermal erosion with that talus map (no bedrock) and its deposition
 *      map max(z - z_in, 0), as hmap::gpu::thermal (thermal_core);
 *   3. with the post-filter: z = z_in + deposition; the mask is smoothed
 *      by hmap::laplace (filters.cpp:290-324 with the defaults sigma 0.125,
 *      3 steps, filters.hpp:573-598), then z = lerp(z, laplace(z), mask)
 *      (apply_with_mask, operator.hpp:405-418).
 * All of it stays on the device: one kernel for the slope and the talus
 * preparation, thermal_core, then six one-step filter launches and a blend.
 *
 * gradient_talus in the reference is an in-place sweep from a zeroed grid:
 * for odd i, d = |z(i) - z(i+1)|, t(i) = max(t(i), d), t(i-1) =
 * max(t(i-1), t(i)), t(i+1) = d; then the same over rows for odd j.  Its
 * result is a closed form of a few neighbour differences per cell
 * (layer_slope below), so each cell is computed independently:
 *   row pass, h(i):  odd i < nx-1  -> max(0, d(i));
 *                    odd i = nx-1  -> 0 (never visited);
 *                    even i, i+1 < nx-1 -> max(d(i-1) or 0 at i = 0, max(0, d(i+1)));
 *                    even i, only i-1 visited -> d(i-1);  else 0.
 *   column pass on h: odd j < ny-1 -> max(h(j), e(j));  odd j = ny-1 -> h(j);
 *                    even j, j+1 < ny-1 -> max(j = 0 ? h(0) : e(j-1), max(h(j+1), e(j+1)));
 *                    even j, only j-1 visited -> e(j-1);  else h(j),
 * with d(i) = |z(i, j) - z(i+1, j)|, e(j) = |z(i, j) - z(i, j+1)| and
 * max(a, b) = a < b ? b : a (std::max, NaN-faithful).
 */
#include <cuda_runtime.h>

#include "hm_internal.h"
#include "hm_thermal.h"

namespace hm
{

namespace
{

constexpr int LY_NT = 256;
constexpr int LY_GRID = 148 * 8;

__device__ __forceinline__ float std_max(float a, float b) { return a < b ? b : a; }

__device__ __forceinline__ float dx_abs(const float *__restrict__ z, int nx, int i, int j)
{
  const size_t k = (size_t)j * nx + i;
  return fabsf(__fsub_rn(z[k], z[k + 1]));
}

__device__ __forceinline__ float dy_abs(const float *__restrict__ z, int nx, int i, int j)
{
  const size_t k = (size_t)j * nx + i;
  return fabsf(__fsub_rn(z[k], z[k + nx]));
}

/* row pass of gradient_talus at (i, j) */
__device__ __forceinline__ float row_pass(const float *__restrict__ z, int nx, int i, int j)
{
  if (i & 1) return i < nx - 1 ? std_max(0.f, dx_abs(z, nx, i, j)) : 0.f;
  if (i + 1 < nx - 1) return std_max(i == 0 ? 0.f : dx_abs(z, nx, i - 1, j), std_max(0.f, dx_abs(z, nx, i + 1, j)));
  if (i >= 1) return dx_abs(z, nx, i - 1, j); /* i - 1 odd and < nx - 1 */
  return 0.f;
}

/* gradient_talus at (i, j): the column pass over the row pass */
__device__ __forceinline__ float layer_slope(const float *__restrict__ z, int nx, int ny, int i, int j)
{
  if (j & 1) return j < ny - 1 ? std_max(row_pass(z, nx, i, j), dy_abs(z, nx, i, j)) : row_pass(z, nx, i, j);
  if (j + 1 < ny - 1)
  {
    const float prev = j == 0 ? row_pass(z, nx, i, 0) : dy_abs(z, nx, i, j - 1);
    return std_max(prev, std_max(row_pass(z, nx, i, j + 1), dy_abs(z, nx, i, j + 1)));
  }
  if (j >= 1) return dy_abs(z, nx, i, j - 1);
  return row_pass(z, nx, i, j);
}

/* talus map and filter mask from the slope (deposition.cpp:82-92) */
__global__ void __launch_bounds__(LY_NT) k_layer_prep(const float *__restrict__ z,
                                                      const float *__restrict__ talus_layer,
                                                      const float *__restrict__ upper,
                                                      float *__restrict__ talus_ref,
                                                      float *__restrict__ fmask,
                                                      int nx,
                                                      int ny)
{
  const size_t n = (size_t)nx * ny;
  for (size_t k = blockIdx.x * (size_t)LY_NT + threadIdx.x; k < n; k += (size_t)gridDim.x * LY_NT)
  {
    const int   j = (int)(k / (size_t)nx), i = (int)(k - (size_t)j * nx);
    const float g = layer_slope(z, nx, ny, i, j);
    const float u = upper[k];
    if (g > u)
    {
      fmask[k] = 0.f;
      talus_ref[k] = __fadd_rn(__fmul_rn(4.f, __fsub_rn(g, u)), u);
    }
    else
    {
      fmask[k] = 1.f;
      talus_ref[k] = talus_layer[k];
    }
  }
}

/* z = z_in + deposition */
__global__ void __launch_bounds__(LY_NT) k_layer_add(float *__restrict__ z, const float *__restrict__ z0,
                                                     const float *__restrict__ depo, size_t n)
{
  for (size_t k = blockIdx.x * (size_t)LY_NT + threadIdx.x; k < n; k += (size_t)gridDim.x * LY_NT)
    z[k] = __fadd_rn(z0[k], depo[k]);
}

/* one step of hmap::laplace from a into b: b = a + sigma (sum of the 8
 * clamped neighbours - 8 a), the sum accumulated from +0 in the
 * reference's loop order (dj outer, di inner) */
__global__ void __launch_bounds__(LY_NT) k_laplace_step(const float *__restrict__ a, float *__restrict__ b, int nx,
                                                        int ny, float sigma)
{
  const size_t n = (size_t)nx * ny;
  for (size_t k = blockIdx.x * (size_t)LY_NT + threadIdx.x; k < n; k += (size_t)gridDim.x * LY_NT)
  {
    const int    j = (int)(k / (size_t)nx), i = (int)(k - (size_t)j * nx);
    const int    im = i > 0 ? i - 1 : 0, ip = i < nx - 1 ? i + 1 : nx - 1;
    const size_t rm = (size_t)(j > 0 ? j - 1 : 0) * nx, r0 = (size_t)j * nx, rp = (size_t)(j < ny - 1 ? j + 1 : ny - 1) * nx;
    float        sum = 0.f;
    sum = __fadd_rn(sum, a[rm + im]);
    sum = __fadd_rn(sum, a[rm + i]);
    sum = __fadd_rn(sum, a[rm + ip]);
    sum = __fadd_rn(sum, a[r0 + im]);
    sum = __fadd_rn(sum, a[r0 + ip]);
    sum = __fadd_rn(sum, a[rp + im]);
    sum = __fadd_rn(sum, a[rp + i]);
    sum = __fadd_rn(sum, a[rp + ip]);
    const float c = a[k];
    const float delta = __fsub_rn(sum, __fmul_rn(8.f, c));
    b[k] = __fadd_rn(c, __fmul_rn(sigma, delta));
  }
}

/* z = lerp(z, smoothed, mask) (math.cpp:183-195) */
__global__ void __launch_bounds__(LY_NT) k_layer_blend(float *__restrict__ z, const float *__restrict__ smooth,
                                                       const float *__restrict__ mask, size_t n)
{
  for (size_t k = blockIdx.x * (size_t)LY_NT + threadIdx.x; k < n; k += (size_t)gridDim.x * LY_NT)
  {
    const float m = mask[k];
    z[k] = __fadd_rn(__fmul_rn(z[k], __fsub_rn(1.f, m)), __fmul_rn(smooth[k], m));
  }
}

/* `steps` laplace steps of the grid in *cur, ping-ponging with `spare`;
 * *cur ends on the buffer that holds the result */
int laplace_steps(float **cur, float *spare, int nx, int ny, float sigma, int steps, cudaStream_t s)
{
  float *a = *cur, *b = spare;
  for (int it = 0; it < steps; it++)
  {
    k_laplace_step<<<LY_GRID, LY_NT, 0, s>>>(a, b, nx, ny, sigma);
    HM_LAUNCH_CHECK("k_laplace_step");
    float *t = a;
    a = b;
    b = t;
  }
  *cur = a;
  return HM_OK;
}

} // namespace

size_t layer_scratch_floats(int nx, int ny)
{
  /* talus map, mask, input copy, deposition, and thermal_core's two grids */
  return 4 * align_up((size_t)nx * ny, 64) + thermal_scratch_floats(nx, ny, true);
}

int layer_core(int device, float *z, int nx, int ny, const float *talus_layer, const float *talus_upper_limit,
               int iterations, bool post_filter, float *depo, float *scratch, cudaStream_t s)
{
  const size_t n = (size_t)nx * ny;
  const size_t na = align_up(n, 64);
  float       *talus_ref = scratch, *fmask = scratch + na, *z0 = scratch + 2 * na, *dmap = scratch + 3 * na;
  float       *tws = scratch + 4 * na;
  float       *map = depo ? depo : dmap;

  k_layer_prep<<<LY_GRID, LY_NT, 0, s>>>(z, talus_layer, talus_upper_limit, talus_ref, fmask, nx, ny);
  HM_LAUNCH_CHECK("k_layer_prep");
  if (post_filter) HM_CUDA_TRY(cudaMemcpyAsync(z0, z, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
  int rc = thermal_core(device, z, nx, ny, talus_ref, 0.f, iterations, nullptr, map, nullptr, nullptr, tws, s);
  if (rc || !post_filter) return rc;

  k_layer_add<<<LY_GRID, LY_NT, 0, s>>>(z, z0, map, n);
  HM_LAUNCH_CHECK("k_layer_add");
  /* the mask, smoothed with the talus map's buffer as the spare */
  float *m = fmask;
  if ((rc = laplace_steps(&m, talus_ref, nx, ny, 0.125f, 3, s))) return rc;
  /* a smoothed copy of z: the first step from z into the input copy's
   * buffer, the other two between it and thermal_core's first grid */
  k_laplace_step<<<LY_GRID, LY_NT, 0, s>>>(z, z0, nx, ny, 0.125f);
  HM_LAUNCH_CHECK("k_laplace_step");
  float *zs = z0;
  if ((rc = laplace_steps(&zs, tws, nx, ny, 0.125f, 2, s))) return rc;
  k_layer_blend<<<LY_GRID, LY_NT, 0, s>>>(z, zs, m, n);
  HM_LAUNCH_CHECK("k_layer_blend");
  return HM_OK;
}

} // namespace hm
