/*
 * hm_sibling.cu - the sibling talus stencils of thermal erosion on sm_100a:
 * thermal_ridge, thermal_scree, thermal_schott, thermal_olsen,
 * thermal_flatten, thermal_inflate and thermal_rib.
 *
 * Replaces the drivers of HighMap/src/erosion/thermal_gpu.cpp:154-396 and
 * the in-place OpenCL kernels thermal_ridge.cl, thermal_scree.cl,
 * thermal_schott.cl, thermal_olsen.cl, thermal_flatten.cl,
 * thermal_inflate.cl and thermal_rib.cl (Jacobi form: every read sees
 * step t, except a work-item's reads of its own cell, which see its own
 * earlier writes).  After the steps, the thermal finish pass: border
 * extrapolation (3 cells deep for rib), the deposition map (|z - z0| for
 * ridge and schott, max(z - z0, 0) for scree, none for the others) and
 * the mask blend.
 *
 * Kernels: the 3 x 3 rules (ridge, scree, schott, inflate, rib) run as
 * cell rules of the thermal warp sweeps; olsen and flatten, which read the
 * neighbours of their neighbours, on k_sibling_step, a 32 x 8 tile per CTA
 * with a 2-cell halo of z in shared memory, one cell per thread.  Arithmetic is explicitly rounded, one rounding per
 * operation as the reference's fp32 text; division by the diagonal
 * distance 1.414f is the exact Markstein form of hm_thermal_math.cuh.
 */
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "hm_internal.h"
#include "hm_thermal.h"
#include "hm_thermal_math.cuh"
#include "hm_thermal_sweep.cuh"

namespace hm
{

namespace
{

constexpr int SB_TX = 32, SB_TY = 8, SB_H = 2; /* tile and halo */

/* smoothstep3 and almost_unit_identity (_common_math.cl:20-23,111-114) */
__device__ __forceinline__ float smoothstep3(float x)
{
  return __fmul_rn(__fmul_rn(x, x), __fsub_rn(3.f, __fmul_rn(2.f, x)));
}
__device__ __forceinline__ float almost_unit_identity(float x)
{
  return __fmul_rn(__fmul_rn(__fsub_rn(2.f, x), x), x);
}
__device__ __forceinline__ float clamp01(float x) { return fminf(fmaxf(x, 0.f), 1.f); }

/* hash21u (_common_rand.cl:19-26) */
__device__ __forceinline__ unsigned hash21u(unsigned x, unsigned y)
{
  unsigned h = x * 0x8da6b343u ^ y * 0xd8163841u;
  h ^= h >> 13;
  h *= 0x85ebca6bu;
  h ^= h >> 16;
  return h;
}

/* HMAP_DI / HMAP_DJ (erosion.hpp:21-22) + 1, packed two bits per direction:
 * a direction chosen at run time is decoded with shifts instead of an
 * indexed local array */
constexpr unsigned DI1 = 0xA094u, DJ1 = 0x8849u;
__host__ __device__ constexpr int di8(int k) { return (int)((DI1 >> (2 * k)) & 3u) - 1; }
__host__ __device__ constexpr int dj8(int k) { return (int)((DJ1 >> (2 * k)) & 3u) - 1; }

/* (val - other) / c for c = 1 or 1.414 */
__device__ __forceinline__ float slope(float val, float other, bool diag)
{
  const float d = __fsub_rn(val, other);
  return diag ? div_by_diag(d) : d;
}

/* The 3 x 3 rules as cell rules of the warp sweeps (hm_thermal_sweep.cuh);
 * neighbours in the reference's loop order w, s, n, e, nw, sw, ne, se
 * (HMAP_DI / HMAP_DJ), distance 1.414 for the diagonals. */
template <int RULE>
struct SiblingRule
{
  static constexpr bool EXTRA = RULE == HM_SCREE; /* zmax */
  __device__ static __forceinline__ float cell(float c, float w, float s, float n, float e, float nw, float sw,
                                               float ne, float se, float t, float zmax, bool, float intensity)
  {
    const float z8[8] = {w, s, n, e, nw, sw, ne, se};
    if (RULE == HM_SCHOTT)
    {
      int up = 0, down = 0;
#pragma unroll
      for (int k = 0; k < 8; k++)
      {
        const float dz = slope(c, z8[k], k >= 4);
        if (dz > t)
          down++;
        else if (dz < -t)
          up++;
      }
      return __fadd_rn(c, __fmul_rn(__fmul_rn(intensity, t), (float)(up - down)));
    }
    if (RULE == HM_RIB)
    {
      /* thermal_rib.cl: z -= the least |slope| to a neighbour */
      float delta_min = FLT_MAX;
#pragma unroll
      for (int k = 0; k < 8; k++) delta_min = fminf(delta_min, fabsf(slope(c, z8[k], k >= 4)));
      return __fsub_rn(c, delta_min);
    }
    /* ridge sums the slopes down to the neighbours, scree and inflate the
     * slopes up */
    float sum = 0.f, slope_max = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++)
    {
      const float dz = slope(c, z8[k], k >= 4);
      if (RULE == HM_RIDGE ? dz > 0.f : dz < 0.f) sum = __fadd_rn(sum, dz);
      slope_max = fmaxf(slope_max, fabsf(dz));
    }
    float amp = smoothstep3(clamp01(__fsub_rn(1.f, __fdiv_rn(t, slope_max))));
    if (RULE == HM_SCREE) amp = __fmul_rn(amp, almost_unit_identity(clamp01(__fsub_rn(1.f, __fdiv_rn(c, zmax)))));
    return __fadd_rn(c, __fmul_rn(__fmul_rn(0.25f, __fsub_rn(t, __fmul_rn(0.5f, sum))), amp));
  }
};

constexpr int SS_NT = 256, SS2_NT = 128, SS_H = 16; /* as the thermal sweeps */

template <int RULE>
__global__ void __launch_bounds__(SS_NT)
    k_sibling_sweep(const float *__restrict__ a, float *__restrict__ b, int nx, int ny, const float *__restrict__ talus,
                    const float *__restrict__ zmax, float intensity)
{
  const int wx = (blockIdx.x * (SS_NT / 32) + (threadIdx.x >> 5)) * 32;
  if (wx >= nx) return; /* the whole warp */
  const int y0 = blockIdx.y * SS_H;
  thermal_sweep_warp<RULE != HM_RIB, SiblingRule<RULE>>(a, b, nx, ny, talus, 0.f, zmax, 0, wx, y0,
                                                         min(ny, y0 + SS_H), intensity);
}

template <int RULE>
__global__ void __launch_bounds__(SS2_NT)
    k_sibling_sweep2(const float *__restrict__ a, float *__restrict__ b, int nx, int ny,
                     const float *__restrict__ talus, const float *__restrict__ zmax, float intensity)
{
  const int wx = (blockIdx.x * (SS2_NT / 32) + (threadIdx.x >> 5)) * 64;
  if (wx >= nx) return; /* the whole warp */
  const int y0 = blockIdx.y * SS_H;
  thermal_sweep2_warp<RULE != HM_RIB, SiblingRule<RULE>>(a, b, nx, ny, talus, 0.f, zmax, 0, wx, y0,
                                                          min(ny, y0 + SS_H), intensity);
}

/* thermal_olsen and thermal_flatten: radius-2 reads, a shared-memory tile
 * per CTA (intensity: flatten's sigma_inf, p1 its sigma_sup) */
template <int RULE>
__global__ void __launch_bounds__(SB_TX *SB_TY)
    k_sibling_step(const float *__restrict__ a,
                   float *__restrict__ b,
                   int nx,
                   int ny,
                   const float *__restrict__ talus,
                   const float *__restrict__ zmax,
                   float intensity,
                   float p1)
{
  __shared__ float t[SB_TY + 2 * SB_H][SB_TX + 2 * SB_H];
  const int x0 = blockIdx.x * SB_TX, y0 = blockIdx.y * SB_TY;
  const int tid = threadIdx.y * SB_TX + threadIdx.x;
  for (int e = tid; e < (SB_TY + 2 * SB_H) * (SB_TX + 2 * SB_H); e += SB_TX * SB_TY)
  {
    const int ly = e / (SB_TX + 2 * SB_H), lx = e - ly * (SB_TX + 2 * SB_H);
    const int gx = min(max(x0 - SB_H + lx, 0), nx - 1), gy = min(max(y0 - SB_H + ly, 0), ny - 1);
    t[ly][lx] = __ldg(a + (size_t)gy * nx + gx);
  }
  __syncthreads();
  /* flatten: the steepest descent of every cell of the tile and its 1-cell
   * ring, once per cell (see below) */
  __shared__ float    fm[RULE == HM_FLATTEN ? SB_TY + 2 : 1][SB_TX + 2];
  __shared__ unsigned fk[RULE == HM_FLATTEN ? SB_TY + 2 : 1][SB_TX + 2];
  if (RULE == HM_FLATTEN)
  {
    for (int e = tid; e < (SB_TY + 2) * (SB_TX + 2); e += SB_TX * SB_TY)
    {
      const int   ly = e / (SB_TX + 2), lx = e - ly * (SB_TX + 2);
      const float zp = t[ly + 1][lx + 1];
      float       dz[8], m = 0.f;
#pragma unroll
      for (int k = 0; k < 8; k++)
      {
        dz[k] = slope(zp, t[ly + 1 + dj8(k)][lx + 1 + di8(k)], k >= 4);
        if (dz[k] > m) m = dz[k];
      }
      unsigned mask = 0u;
#pragma unroll
      for (int k = 0; k < 8; k++)
        if (m > 0.f && dz[k] == m) mask |= 1u << k;
      fm[ly][lx] = m;
      fk[ly][lx] = mask;
    }
    __syncthreads();
  }
  const int i = x0 + threadIdx.x, j = y0 + threadIdx.y;
  if (i >= nx || j >= ny) return;
  const size_t idx = (size_t)j * nx + i;
  /* z at (i + dx, j + dy), |dx|, |dy| <= 2 */
  auto zat = [&](int dx, int dy) -> float { return t[threadIdx.y + SB_H + dy][threadIdx.x + SB_H + dx]; };
  const int di[8] = {-1, 0, 0, 1, -1, -1, 1, 1};
  const int dj[8] = {0, 1, -1, 0, -1, 1, -1, 1};

  if (RULE == HM_OLSEN)
  {
    /* apply_boundaries_buffer(z, i, j, nx, ny, 3), _common_index.cl:134-152 */
    const int bw = 3;
    if (!(i >= bw && i < nx - bw && j >= bw && j < ny - bw))
    {
      const int ci = min(max(i, bw), nx - bw - 1), cj = min(max(j, bw), ny - bw - 1);
      b[idx] = __ldg(a + (size_t)cj * nx + ci);
      return;
    }
    const float    c2 = 1.414213562f;
    float          self = zat(0, 0);
    const float    talus_ref = __ldg(talus + idx);
    const unsigned shift = hash21u((unsigned)i, (unsigned)j) & 7u;
    for (int k = 0; k < 8; ++k)
    {
      const int s = (k + (int)shift) & 7;
      const int gx = di8(s), gy = dj8(s); /* neighbour offset */
      float     dsum = 0.f, dmax = 0.f, dz[8];
#pragma unroll
      for (int p = 0; p < 8; ++p)
      {
        const int   px = gx + di[p], py = gy + dj[p];
        const float zp = (px == 0 && py == 0) ? self : zat(px, py);
        dz[p] = __fsub_rn(zat(gx, gy), zp);
        if (dz[p] > __fmul_rn(talus_ref, p < 4 ? 1.f : c2))
        {
          dsum = __fadd_rn(dsum, dz[p]);
          dmax = fmaxf(dmax, dz[p]);
        }
      }
      if (dmax > 0.f)
      {
#pragma unroll
        for (int p = 0; p < 8; ++p)
          if (gx + di[p] == 0 && gy + dj[p] == 0)
          {
            const float cp = p < 4 ? 1.f : c2;
            const float amount =
                __fdiv_rn(__fmul_rn(__fmul_rn(0.25f, __fsub_rn(dmax, __fmul_rn(talus_ref, cp))), dz[p]), dsum);
            self = __fadd_rn(self, amount);
          }
      }
    }
    b[idx] = self;
    return;
  }

  if (RULE == HM_FLATTEN)
  {
    /* apply_boundaries_buffer(z, i, j, nx, ny, 2), _common_index.cl:134-152 */
    const int bw = 2;
    if (!(i >= bw && i < nx - bw && j >= bw && j < ny - bw))
    {
      const int ci = min(max(i, bw), nx - bw - 1), cj = min(max(j, bw), ny - bw - 1);
      b[idx] = __ldg(a + (size_t)cj * nx + ci);
      return;
    }
    /* thermal_flatten.cl visits the neighbours from a rotating start
     * (i + j) % 8 and keeps the first strict maximum.  The cell loses
     * sigma_inf (below its talus) or sigma_sup (above) times its steepest
     * descent, and gains half of each neighbour's steepest descent that
     * points at it and lies below that neighbour's talus.  A steepest
     * descent's value does not depend on the visiting order; its direction
     * does, through ties only: the first of the tied directions in this
     * cell's rotated order.  So each cell's maximum and the mask of
     * directions reaching it come from the table above, and the rotation is
     * applied to the mask here (the kernel text evaluates the 64 slopes for
     * every cell). */
    const int   rot = (i + j) % 8;
    const int   ty = threadIdx.y + 1, tx = threadIdx.x + 1; /* this cell in the table */
    const float zc = zat(0, 0);
    const float tc = __ldg(talus + idx);
    const float slope_min = __fdiv_rn(0.f, (float)nx);
    const float dmax = fm[ty][tx];
    float       delta = 0.f;
    const float excess = fmaxf(__fsub_rn(dmax, slope_min), 0.f);
    if (dmax < tc) delta = __fsub_rn(delta, __fmul_rn(intensity, excess));
    if (dmax > tc) delta = __fsub_rn(delta, __fmul_rn(p1, excess));
    for (int n = 0; n < 8; ++n)
    {
      const int      k = (n + rot) & 7;
      const int      px = -di8(k), py = -dj8(k);
      const unsigned mask = fk[ty + py][tx + px];
      if (!mask) continue; /* no descent: the kernel text's ka = -1 */
      const unsigned r = ((mask >> rot) | (mask << (8 - rot))) & 0xffu;
      const int      ka = (__ffs(r) - 1 + rot) & 7;
      const float    dm = fm[ty + py][tx + px];
      if (ka == k && dm < __ldg(talus + (size_t)(j + py) * nx + (i + px))) delta = __fadd_rn(delta, __fmul_rn(0.5f, dm));
    }
    b[idx] = __fadd_rn(zc, delta);
    return;
  }

  /* apply_boundaries, _common_index.cl:106-132: x edges first, then y */
  if (i == 0) { b[idx] = zat(1, 0); return; }
  if (i == nx - 1) { b[idx] = zat(-1, 0); return; }
  if (j == 0) { b[idx] = zat(0, 1); return; }
  if (j == ny - 1) { b[idx] = zat(0, -1); return; }
  const float val = zat(0, 0);
  const float tv = __ldg(talus + idx);
  if (RULE == HM_SCHOTT)
  {
    int up = 0, down = 0;
#pragma unroll
    for (int k = 0; k < 8; k++)
    {
      const float dz = slope(val, zat(di[k], dj[k]), k >= 4);
      if (dz > tv)
        down++;
      else if (dz < -tv)
        up++;
    }
    b[idx] = __fadd_rn(val, __fmul_rn(__fmul_rn(intensity, tv), (float)(up - down)));
    return;
  }
  float sum = 0.f, slope_max = 0.f;
#pragma unroll
  for (int k = 0; k < 8; k++)
  {
    const float dz = slope(val, zat(di[k], dj[k]), k >= 4);
    if (RULE == HM_RIDGE ? dz > 0.f : dz < 0.f) sum = __fadd_rn(sum, dz);
    slope_max = fmaxf(slope_max, fabsf(dz));
  }
  float amp = smoothstep3(clamp01(__fsub_rn(1.f, __fdiv_rn(tv, slope_max))));
  if (RULE == HM_SCREE)
    amp = __fmul_rn(amp, almost_unit_identity(clamp01(__fsub_rn(1.f, __fdiv_rn(val, __ldg(zmax + idx))))));
  b[idx] = __fadd_rn(val, __fmul_rn(__fmul_rn(0.25f, __fsub_rn(tv, __fmul_rn(0.5f, sum))), amp));
}

} // namespace

int sibling_check_args(int rule, const float *z, int nx, int ny, const float *talus, const float *zmax, int iterations)
{
  if (rule < HM_RIDGE || rule > HM_RIB) return fail(HM_ERR_INVALID_ARGUMENT, "thermal stencil: unknown rule");
  if (!z) return fail(HM_ERR_INVALID_ARGUMENT, "thermal stencil: z is NULL");
  if (!talus && rule != HM_RIB) return fail(HM_ERR_INVALID_ARGUMENT, "thermal stencil: talus is NULL");
  if (rule == HM_SCREE && !zmax) return fail(HM_ERR_INVALID_ARGUMENT, "thermal_scree: zmax is NULL");
  /* olsen's border is 3 cells wide; flatten's 2; rib extrapolates 3 deep */
  const int nmin = rule == HM_OLSEN ? 7 : (rule == HM_FLATTEN || rule == HM_RIB ? 5 : 3);
  if (nx < nmin || ny < nmin)
    return fail(HM_ERR_INVALID_ARGUMENT, rule == HM_OLSEN   ? "thermal_olsen: nx and ny must be >= 7"
                                         : nmin == 5        ? "thermal_flatten / thermal_rib: nx and ny must be >= 5"
                                                            : "thermal stencil: nx and ny must be >= 3");
  if ((long long)nx * (long long)ny > (1ll << 34))
    return fail(HM_ERR_INVALID_ARGUMENT, "thermal stencil: grid larger than 2^34 cells");
  if (iterations < 0) return fail(HM_ERR_INVALID_ARGUMENT, "thermal stencil: iterations < 0");
  return HM_OK;
}

int sibling_core(int device, int rule, float *z, int nx, int ny, const float *talus, const float *zmax,
                 float intensity, int iterations, float *depo, const float *mask, float *scratch_buf,
                 cudaStream_t s, float p1)
{
  const size_t n = (size_t)nx * ny;
  float       *tmp = scratch_buf;
  float       *z0 = scratch_buf + align_up(n, 64);
  const bool   want_depo = depo && rule <= HM_SCHOTT;
  if (want_depo || mask) HM_CUDA_TRY(cudaMemcpyAsync(z0, z, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
  const dim3   grid((nx + SB_TX - 1) / SB_TX, (ny + SB_TY - 1) / SB_TY), block(SB_TX, SB_TY);
  const float *src = z;
  float       *dst = tmp;
  auto al8 = [](const void *p) { return ((uintptr_t)p & 7u) == 0; };
  const bool pairs = nx % 2 == 0 && al8(z) && al8(tmp) && al8(talus) && (rule != HM_SCREE || al8(zmax));
  const dim3 g2((nx + 2 * SS2_NT - 1) / (2 * SS2_NT), (ny + SS_H - 1) / SS_H);
  const dim3 g1((nx + SS_NT - 1) / SS_NT, (ny + SS_H - 1) / SS_H);
  for (int it = 0; it < iterations; it++)
  {
#define HM_SIB_SWEEP(R)                                                                                                \
  if (pairs) k_sibling_sweep2<R><<<g2, SS2_NT, 0, s>>>(src, dst, nx, ny, talus, zmax, intensity);                       \
  else k_sibling_sweep<R><<<g1, SS_NT, 0, s>>>(src, dst, nx, ny, talus, zmax, intensity);
    switch (rule)
    {
    case HM_RIDGE: HM_SIB_SWEEP(HM_RIDGE) break;
    case HM_SCREE: HM_SIB_SWEEP(HM_SCREE) break;
    case HM_SCHOTT: HM_SIB_SWEEP(HM_SCHOTT) break;
    case HM_INFLATE: HM_SIB_SWEEP(HM_INFLATE) break;
    case HM_RIB: HM_SIB_SWEEP(HM_RIB) break;
    case HM_FLATTEN: k_sibling_step<HM_FLATTEN><<<grid, block, 0, s>>>(src, dst, nx, ny, talus, zmax, intensity, p1); break;
    default: k_sibling_step<HM_OLSEN><<<grid, block, 0, s>>>(src, dst, nx, ny, talus, zmax, intensity, p1);
    }
#undef HM_SIB_SWEEP
    HM_LAUNCH_CHECK("k_sibling_step");
    const float *t = src;
    src = dst;
    dst = const_cast<float *>(t);
  }
  if (src != z) HM_CUDA_TRY(cudaMemcpyAsync(z, src, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
  return thermal_finish(device, z, nx, ny, z0, want_depo ? depo : nullptr, mask, s, rule != HM_SCREE,
                        rule == HM_RIB ? 3 : 1);
}

} // namespace hm
