/*
 * hm_thermal.cu - talus thermal erosion on sm_100a.
 *
 * Replaces the host loop of HighMap/src/erosion/thermal_gpu.cpp:17-96 and
 * the OpenCL kernels thermal / thermal_with_bedrock
 * (HighMap/src/gpu_opencl/kernels/thermal.cl:26-100).
 *
 * Device data: z, talus and bedrock stay in HBM for the whole call; steps
 * ping-pong between z and one workspace grid (Jacobi).  After the steps:
 * extrapolate_borders (HighMap/src/boundary/boundary.cpp:19-41) on the
 * outer ring, then, when asked, the deposition map max(z - z0, 0)
 * (HighMap/src/range/range.cpp:253-262) and the mask blend
 * lerp(z0, z, mask) (HighMap/include/highmap/operator.hpp:405-418).
 *
 * Kernels
 *   k_thermal_sweep2  one step per launch: a warp walks down rows of 64
 *                     columns (two per lane), neighbours by warp shuffles;
 *                     reads z, talus and bedrock once, writes z: 12 B/cell
 *                     (16 B with bedrock).  Even nx, 8-byte aligned grids.
 *   k_thermal_sweep   the same with one column per lane (any grid).
 *   k_thermal_tb      up to 8 steps per launch (temporal blocking): a
 *                     strip of columns streams down the grid; each time
 *                     level keeps a 4-row ring in shared memory, so HBM
 *                     sees the 12/16 B of one step per T steps.
 *   k_extrapolate     the outer ring, one block.
 *   k_thermal_final   deposition map and mask blend, elementwise.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "hm_internal.h"
#include "hm_thermal.h"
#include "hm_thermal_math.cuh"
#include "hm_thermal_sweep.cuh"
#include "hm_tune.h"

namespace hm
{

__device__ __forceinline__ int clamp_col(int g, int n) { return g < 0 ? 0 : (g > n - 1 ? n - 1 : g); }

/* ------------------------------------------------------------------ */
/* one step per launch, column sweep                                  */
/* ------------------------------------------------------------------ */

constexpr int SW_NT = 256; /* 8 warps; a warp owns 32 columns              */
constexpr int SW_H = 16;   /* output rows per CTA (a multiple of SW_P)      */

/* One Jacobi step, a warp per 32 columns and SW_H rows
 * (hm_thermal_sweep.cuh). */
template <bool TMAP, int BED>
__global__ void __launch_bounds__(SW_NT)
    k_thermal_sweep(const float *__restrict__ a,
                    float *__restrict__ b,
                    int nx,
                    int ny,
                    const float *__restrict__ talus,
                    float talus_value,
                    const float *__restrict__ bedrock,
                    int first)
{
  const int wx = (blockIdx.x * (SW_NT / 32) + (threadIdx.x >> 5)) * 32;
  if (wx >= nx) return; /* the whole warp: no CTA barrier in this kernel */
  const int y0 = blockIdx.y * SW_H;
  thermal_sweep_warp<TMAP, TalusExchange<BED>>(a, b, nx, ny, talus, talus_value, bedrock, first, wx, y0, min(ny, y0 + SW_H));
}

/* One Jacobi step, a warp per 64 columns (two per lane) and SW_H rows
 * (hm_thermal_sweep.cuh); even nx, 8-byte aligned grids. */
constexpr int S2_NT = 128; /* 4 warps; a warp owns 64 columns */

template <bool TMAP, int BED>
__global__ void __launch_bounds__(S2_NT)
    k_thermal_sweep2(const float *__restrict__ a,
                     float *__restrict__ b,
                     int nx,
                     int ny,
                     const float *__restrict__ talus,
                     float talus_value,
                     const float *__restrict__ bedrock,
                     int first)
{
  const int wx = (blockIdx.x * (S2_NT / 32) + (threadIdx.x >> 5)) * 64;
  if (wx >= nx) return; /* the whole warp: no CTA barrier in this kernel */
  const int y0 = blockIdx.y * SW_H;
  thermal_sweep2_warp<TMAP, TalusExchange<BED>>(a, b, nx, ny, talus, talus_value, bedrock, first, wx, y0, min(ny, y0 + SW_H));
}

/* ------------------------------------------------------------------ */
/* several steps per launch (temporal blocking)                       */
/* ------------------------------------------------------------------ */

constexpr int TB_TPB = 256; /* strip width in columns, one thread each      */
constexpr int TB_TMAX = 8;  /* most steps one launch advances                */

__device__ __forceinline__ void tb_cp_async4(float *smem, const float *gmem)
{
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}

/* T Jacobi steps of a column strip in one pass down the rows.
 *
 * Thread t owns global column gi = x0 - T + t of a strip of TPB columns
 * (W = TPB - 2T output columns), and the CTA owns output rows [y0, y1).
 * Level 0 is the input z, staged row by row into an 8-row ring with
 * cp.async; level k (1 <= k < T) keeps a 4-row ring.  Iteration r loads
 * row r and computes, for every level k, row r - 1 - 2k from rows
 * r - 2 - 2k .. r - 2k of level k - 1, all finished in earlier iterations;
 * one __syncthreads per iteration publishes them.  Level T goes straight
 * to the output grid.  Level k is needed on rows [y0 - (T-k), y1 + T-k)
 * and is correct on columns [k, TPB - k) of the strip, so the T halo
 * columns each side cover the shrinking valid region.
 *
 * Each cell follows the rule of the one-step kernel (border copy, then
 * the talus exchange with bedrock), so T steps here are bit-identical to
 * T one-step launches. */
template <bool TMAP, int BED>
__global__ void __launch_bounds__(TB_TPB)
    k_thermal_tb(const float *__restrict__ a,
                 float *__restrict__ b,
                 int nx,
                 int ny,
                 const float *__restrict__ talus,
                 float talus_value,
                 const float *__restrict__ bedrock,
                 int T,
                 int H,
                 int it0)
{
  __shared__ float lv0[8][TB_TPB];
  __shared__ float lvk[TB_TMAX - 1][4][TB_TPB];

  const int  tid = threadIdx.x;
  const int  W = TB_TPB - 2 * T;
  const int  x0 = blockIdx.x * W;
  const int  gi = x0 - T + tid;
  const bool in_grid = gi >= 0 && gi < nx;
  const int  gic = clamp_col(gi, nx);
  const int  y0 = blockIdx.y * H;
  const int  y1 = min(ny, y0 + H);
  const int  lw = max(tid - 1, 0), le = min(tid + 1, TB_TPB - 1);
  const bool out_col = tid >= T && tid < T + W && gi < nx;
  const int  load_lo = max(0, y0 - T), load_hi = min(ny - 1, y1 - 1 + T);

  for (int r = y0 - T; r <= y1 + 2 * T; ++r)
  {
    if (r >= load_lo && r <= load_hi && in_grid) tb_cp_async4(&lv0[r & 7][tid], a + (size_t)r * nx + gi);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");

#pragma unroll
    for (int k = 1; k <= TB_TMAX; k++)
    {
      if (k > T) break;
      const int j = r - 1 - 2 * k;
      if (j < max(0, y0 - (T - k)) || j > min(ny - 1, y1 - 1 + (T - k))) continue;
      /* rows j-1, j, j+1 of level k-1 */
      const float *pn, *pc, *ps;
      if (k == 1)
      {
        pn = lv0[(j - 1) & 7];
        pc = lv0[j & 7];
        ps = lv0[(j + 1) & 7];
      }
      else
      {
        pn = lvk[k - 2][(j - 1) & 3];
        pc = lvk[k - 2][j & 3];
        ps = lvk[k - 2][(j + 1) & 3];
      }
      float out;
      /* apply_boundaries, _common_index.cl:106-132 */
      if (gi == 0) out = pc[le];
      else if (gi == nx - 1) out = pc[lw];
      else if (j == 0) out = ps[tid];
      else if (j == ny - 1) out = pn[tid];
      else
      {
        const size_t q = (size_t)j * nx + gic;
        const float  t = TMAP ? __ldg(talus + q) : talus_value;
        const float  zb = BED != BED_NONE ? __ldg(bedrock + q) : 0.f;
        out = thermal_cell<BED>(pc[tid], pc[lw], ps[tid], pn[tid], pc[le], pn[lw], ps[lw], pn[le], ps[le], t, zb,
                                it0 + k == 1);
      }
      if (k == T)
      {
        if (out_col && j >= y0 && j < y1) b[(size_t)j * nx + gi] = out;
      }
      else
        lvk[k - 1][j & 3][tid] = out;
    }
    __syncthreads();
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

/* ------------------------------------------------------------------ */
/* borders and finalisation                                           */
/* ------------------------------------------------------------------ */

/* extrapolate_borders(z, 1, 0): columns first, then rows, as the loops of
 * boundary.cpp:26-40 order them (the row pass reads the column pass's
 * corner values). */
__global__ void __launch_bounds__(1024) k_extrapolate(float *z, int nx, int ny)
{
  for (int j = threadIdx.x; j < ny; j += blockDim.x)
  {
    float *r = z + (size_t)j * nx;
    r[0] = __fsub_rn(__fmul_rn(2.f, r[1]), r[2]);
    r[nx - 1] = __fsub_rn(__fmul_rn(2.f, r[nx - 2]), r[nx - 3]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nx; i += blockDim.x)
  {
    z[i] = __fsub_rn(__fmul_rn(2.f, z[(size_t)nx + i]), z[(size_t)2 * nx + i]);
    size_t l = (size_t)(ny - 1) * nx + i;
    z[l] = __fsub_rn(__fmul_rn(2.f, z[l - nx]), z[l - 2 * (size_t)nx]);
  }
}

/* extrapolate_borders(z, nb, 0) for nb > 1 (boundary.cpp:19-41): per row,
 * for k = nb-1 .. 0, column k from columns k+1, k+2, then column nx-1-k
 * from its two inward neighbours; then the same per column over the rows.
 * One thread walks one row (then one column) in the reference's order, so
 * rows narrower than 2 nb + 2, where the two sides meet, match too. */
__global__ void __launch_bounds__(1024) k_extrapolate_n(float *z, int nx, int ny, int nb)
{
  for (int j = threadIdx.x; j < ny; j += blockDim.x)
  {
    float *r = z + (size_t)j * nx;
    for (int k = nb - 1; k > -1; k--)
    {
      r[k] = __fsub_rn(__fmul_rn(2.f, r[k + 1]), r[k + 2]);
      r[nx - 1 - k] = __fsub_rn(__fmul_rn(2.f, r[nx - 2 - k]), r[nx - 3 - k]);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nx; i += blockDim.x)
    for (int k = nb - 1; k > -1; k--)
    {
      z[(size_t)k * nx + i] = __fsub_rn(__fmul_rn(2.f, z[(size_t)(k + 1) * nx + i]), z[(size_t)(k + 2) * nx + i]);
      z[(size_t)(ny - 1 - k) * nx + i] =
          __fsub_rn(__fmul_rn(2.f, z[(size_t)(ny - 2 - k) * nx + i]), z[(size_t)(ny - 3 - k) * nx + i]);
    }
}

__global__ void k_thermal_final(float *__restrict__ z,
                                const float *__restrict__ z0,
                                float *__restrict__ depo,
                                const float *__restrict__ mask,
                                size_t n,
                                int depo_abs)
{
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
  {
    float r = z[k];
    float o = z0[k];
    if (depo)
    {
      float dz = __fsub_rn(r, o);
      depo[k] = depo_abs ? fabsf(dz) : (dz > 0.f ? dz : 0.f);
    }
    if (mask)
    {
      float m = mask[k];
      z[k] = __fadd_rn(__fmul_rn(o, __fsub_rn(1.f, m)), __fmul_rn(r, m));
    }
  }
}

/* ------------------------------------------------------------------ */
/* host side                                                          */
/* ------------------------------------------------------------------ */

static int num_sms(int device)
{
  static int cached[64] = {0};
  if (device >= 0 && device < 64 && cached[device]) return cached[device];
  int n = 0;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
  if (n <= 0) n = 148;
  if (device >= 0 && device < 64) cached[device] = n;
  return n;
}

/* kernel bedrock mode: auto (bed = z0) or the caller's bedrock grid */
static int kernel_bed_mode(const float *bed, int bed_mode, bool auto_bed)
{
  if (auto_bed) return BED_AUTO;
  return bed ? (bed_mode == HM_BEDROCK_LITERAL ? BED_LITERAL : BED_INTENDED) : BED_NONE;
}

/* one Jacobi step: the column-pair sweep where the grid allows 8-byte
 * access (even nx, 8-byte aligned grids), else the one-column sweep */
template <bool TMAP, int BED>
static void launch_step(const float *a, float *b, int nx, int ny, const float *talus, float tv,
                        const float *bed, int first, cudaStream_t s)
{
  auto al8 = [](const void *p) { return ((uintptr_t)p & 7u) == 0; };
  if (nx % 2 == 0 && al8(a) && al8(b) && (!TMAP || al8(talus)) && (BED == BED_NONE || al8(bed)))
  {
    dim3 grid((nx + 2 * S2_NT - 1) / (2 * S2_NT), (ny + SW_H - 1) / SW_H);
    k_thermal_sweep2<TMAP, BED><<<grid, S2_NT, 0, s>>>(a, b, nx, ny, talus, tv, bed, first);
    return;
  }
  dim3 grid((nx + SW_NT - 1) / SW_NT, (ny + SW_H - 1) / SW_H);
  k_thermal_sweep<TMAP, BED><<<grid, SW_NT, 0, s>>>(a, b, nx, ny, talus, tv, bed, first);
}

template <bool TMAP>
static void step_dispatch_t(const float *a, float *b, int nx, int ny, const float *talus, float tv,
                            const float *bed, int mode, int first, cudaStream_t s)
{
  switch (mode)
  {
  case BED_NONE: launch_step<TMAP, BED_NONE>(a, b, nx, ny, talus, tv, bed, first, s); break;
  case BED_INTENDED: launch_step<TMAP, BED_INTENDED>(a, b, nx, ny, talus, tv, bed, first, s); break;
  case BED_LITERAL: launch_step<TMAP, BED_LITERAL>(a, b, nx, ny, talus, tv, bed, first, s); break;
  default: launch_step<TMAP, BED_AUTO>(a, b, nx, ny, talus, tv, bed, first, s); break;
  }
}

static void step_dispatch(const float *a, float *b, int nx, int ny, const float *talus, float tv,
                          const float *bed, int mode, int first, cudaStream_t s)
{
  if (talus) step_dispatch_t<true>(a, b, nx, ny, talus, tv, bed, mode, first, s);
  else step_dispatch_t<false>(a, b, nx, ny, talus, tv, bed, mode, first, s);
}

/* post-processing of a finished thermal solve (z holds the last step):
 * border extrapolation (nbuffer cells deep), then the deposition map (max(z - z0, 0), or
 * |z - z0| with depo_abs) and the mask blend when asked (z0 = the input
 * heights) */
int thermal_finish(int device, float *z, int nx, int ny, const float *z0, float *depo, const float *mask,
                   cudaStream_t s, bool depo_abs, int nbuffer)
{
  if (nbuffer > 1)
  {
    k_extrapolate_n<<<1, 1024, 0, s>>>(z, nx, ny, nbuffer);
    HM_LAUNCH_CHECK("k_extrapolate_n");
  }
  else
  {
    k_extrapolate<<<1, 1024, 0, s>>>(z, nx, ny);
    HM_LAUNCH_CHECK("k_extrapolate");
  }
  if (depo || mask)
  {
    k_thermal_final<<<num_sms(device) * 8, 256, 0, s>>>(z, z0, depo, mask, (size_t)nx * ny, depo_abs ? 1 : 0);
    HM_LAUNCH_CHECK("k_thermal_final");
  }
  return HM_OK;
}

template <bool TMAP, int BED>
static void launch_tb(const float *a, float *b, int nx, int ny, const float *talus, float tv, const float *bed,
                      int T, int H, int it0, cudaStream_t s)
{
  const int W = TB_TPB - 2 * T;
  dim3      grid((nx + W - 1) / W, (ny + H - 1) / H);
  k_thermal_tb<TMAP, BED><<<grid, TB_TPB, 0, s>>>(a, b, nx, ny, talus, tv, bed, T, H, it0);
}

template <bool TMAP>
static void tb_dispatch_t(const float *a, float *b, int nx, int ny, const float *talus, float tv, const float *bed,
                          int mode, int T, int H, int it0, cudaStream_t s)
{
  switch (mode)
  {
  case BED_NONE: launch_tb<TMAP, BED_NONE>(a, b, nx, ny, talus, tv, bed, T, H, it0, s); break;
  case BED_INTENDED: launch_tb<TMAP, BED_INTENDED>(a, b, nx, ny, talus, tv, bed, T, H, it0, s); break;
  case BED_LITERAL: launch_tb<TMAP, BED_LITERAL>(a, b, nx, ny, talus, tv, bed, T, H, it0, s); break;
  default: launch_tb<TMAP, BED_AUTO>(a, b, nx, ny, talus, tv, bed, T, H, it0, s); break;
  }
}

static void tb_dispatch(const float *a, float *b, int nx, int ny, const float *talus, float tv, const float *bed,
                        int mode, int T, int H, int it0, cudaStream_t s)
{
  if (talus) tb_dispatch_t<true>(a, b, nx, ny, talus, tv, bed, mode, T, H, it0, s);
  else tb_dispatch_t<false>(a, b, nx, ny, talus, tv, bed, mode, T, H, it0, s);
}

static int g_tb_rows = 0; /* output rows per CTA of the blocked kernel; 0 = built-in */

/* steps per launch when the caller leaves the choice to the library and
 * the grid's size class is not tuned */
static int g_tb_default = 1;

int thermal_check_args(const float *z, int nx, int ny, int iterations, const hm_thermal_options *o)
{
  if (!z) return fail(HM_ERR_INVALID_ARGUMENT, "thermal: z is NULL");
  if (nx < 3 || ny < 3) return fail(HM_ERR_INVALID_ARGUMENT, "thermal: nx and ny must be >= 3");
  if ((long long)nx * (long long)ny > (1ll << 34))
    return fail(HM_ERR_INVALID_ARGUMENT, "thermal: grid larger than 2^34 cells");
  if (iterations < 0) return fail(HM_ERR_INVALID_ARGUMENT, "thermal: iterations < 0");
  if (o && o->bedrock_mode != HM_BEDROCK_INTENDED && o->bedrock_mode != HM_BEDROCK_LITERAL)
    return fail(HM_ERR_INVALID_ARGUMENT, "thermal: unknown bedrock_mode");
  if (o && o->time_block < 0) return fail(HM_ERR_INVALID_ARGUMENT, "thermal: time_block < 0");
  return HM_OK;
}

size_t thermal_scratch_floats(int nx, int ny, bool need_z0)
{
  size_t n = align_up((size_t)nx * ny, 64);
  return n * (need_z0 ? 2 : 1);
}

int thermal_core(int device,
                 float *z,
                 int nx,
                 int ny,
                 const float *talus,
                 float talus_value,
                 int iterations,
                 const float *bedrock,
                 float *depo,
                 const float *mask,
                 const hm_thermal_options *opts,
                 float *scratch_buf,
                 cudaStream_t s,
                 bool auto_bed)
{
  hm_thermal_options o;
  hm_thermal_default_options(&o);
  if (opts) o = *opts;
  const size_t n = (size_t)nx * ny;
  const bool   need_z0 = depo || mask || auto_bed;
  float       *tmp = scratch_buf;
  float       *z0 = need_z0 ? scratch_buf + align_up(n, 64) : nullptr;
  (void)device;

  if (need_z0) HM_CUDA_TRY(cudaMemcpyAsync(z0, z, n * sizeof(float), cudaMemcpyDeviceToDevice, s));

  /* steps per launch: 1 runs the one-step kernel, 2..8 the blocked kernel.
   * 0 takes the tuned choice for this grid (thermal_pick_block), else one
   * step per launch, the faster of the two on B200 at 4096^2 when untuned
   * (both are bound by the issue rate of the exact arithmetic, not by
   * HBM). */
  int tb = o.time_block;
  int rows = g_tb_rows;
  if (tb == 0)
  {
    TuneEntry e;
    if (tuned_thermal(nx, ny, &e))
    {
      tb = e.block;
      if (rows == 0) rows = e.rows;
    }
    else
      tb = g_tb_default;
  }
  if (tb > TB_TMAX) tb = TB_TMAX;
  if (rows <= 0) rows = 128;
  /* auto-bedrock reads the input heights as its bedrock */
  const int    mode = kernel_bed_mode(bedrock, o.bedrock_mode, auto_bed);
  const float *bed = auto_bed ? z0 : bedrock;
  const float *src = z;
  float       *dst = tmp;
  for (int done = 0; done < iterations;)
  {
    const int T = (iterations - done < tb) ? iterations - done : tb;
    if (tb == 1)
    {
      step_dispatch(src, dst, nx, ny, talus, talus_value, bed, mode, done == 0, s);
      HM_LAUNCH_CHECK("k_thermal_sweep");
    }
    else
    {
      tb_dispatch(src, dst, nx, ny, talus, talus_value, bed, mode, T, rows, done, s);
      HM_LAUNCH_CHECK("k_thermal_tb");
    }
    done += T;
    const float *t = src;
    src = dst;
    dst = const_cast<float *>(t);
  }
  if (src != z) HM_CUDA_TRY(cudaMemcpyAsync(z, src, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
  return thermal_finish(device, z, nx, ny, z0, depo, mask, s);
}

} // namespace hm

extern "C" int hm_thermal_set_launch(int rows)
{
  hm::clear_error();
  if (rows != 0 && (rows < 8 || rows > 4096))
    return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_thermal_set_launch: rows must be 0 or in [8, 4096]");
  hm::g_tb_rows = rows;
  return HM_OK;
}

extern "C" void hm_thermal_default_options(hm_thermal_options *opts)
{
  if (!opts) return;
  opts->bedrock_mode = HM_BEDROCK_INTENDED;
  opts->time_block = 0;
}
