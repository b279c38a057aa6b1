/*
 * hm_vpipes_tiled.cuh - one virtual-pipes step as two kernels over 2-D
 * tiles.
 *
 *   k_vp_fwe     flow (hydraulic_vpipes.cl:5-69), water (:71-116) and
 *                erosion (:118-184) of a TX x TY tile.  z and the depth are
 *                staged with a 2-cell halo, sediment and the old fluxes with
 *                a 1-cell halo (loads clamped to the grid, so every raw
 *                neighbour read is the reference's clamp-to-edge read); the
 *                flow pass runs on the tile plus a 1-cell ring into shared
 *                memory, then water and erosion run on the tile.  Writes z',
 *                the evaporated depth, the new fluxes, the eroded sediment
 *                s1 and the velocity.
 *   k_vp_advect  advection (:186-211): s = bilinear(s1, x - dt u), a gather
 *                from s1 in global memory, so the footprint may lie
 *                anywhere.
 *   k_vp_step(_tma)  every step after the first: the previous step's
 *                advection and this step's flow, water and erosion in one
 *                tile.  Besides z, d and the fluxes it stages the previous
 *                step's u and v (1-cell halo) and s1 (a 4-cell halo); each
 *                cell of the tile and its ring gathers its advected sediment
 *                from the staged s1, or from s1 in global memory where the
 *                back-traced sample falls outside the staged box (s1 of the
 *                previous step is complete in memory, so that read is exact
 *                and needs no replay).  One kernel per step; the last step's
 *                advection runs as k_vp_advect after the loop.  k_vp_step
 *                stages by cp.async: clamped 4-byte copies, or whole box
 *                rows in 16-byte copies where the boxes lie inside a grid
 *                whose rows are 16-byte aligned (a quarter of the copies,
 *                no index clamps: 9 % instead of 27 % behind the TMA form
 *                at 2048^2).
 *
 * HBM traffic per cell and step: 7 fields read and 9 written by k_vp_fwe,
 * 3 read (plus the gather, mostly L2) and 1 written by k_vp_advect: 80 B;
 * k_vp_step reads and writes 9 fields: 72 B.  Every read of a step comes
 * from the old state copy or from the previous step's s1 / u / v
 * (double-buffered), never from a grid the step writes, so tiles need no
 * ordering between them.
 */
#ifndef HM_VPIPES_TILED_CUH
#define HM_VPIPES_TILED_CUH

#include "hm_reduce.cuh"
#include "hm_vpipes_fused.cuh"
#include "hm_vpipes_math.cuh"
#include "hm_tma.cuh"

namespace hm
{

constexpr int FT_TX = 32, FT_TY = 16;          /* output tile                 */
constexpr int FT_NT = 256;                     /* threads per CTA             */
constexpr int FT_W2 = FT_TX + 4, FT_H2 = FT_TY + 4; /* z, depth region (halo 2) */
constexpr int FT_W1 = FT_TX + 2, FT_H1 = FT_TY + 2; /* s, fluxes region (halo 1) */

/* Step options as kernel template flags.  FWE_GENERIC kernels read every
 * option from FweIo / VpConst at run time; the others have pipe length 1
 * and discharge exponent 1 built in and the three bits below fixed, so
 * the branches on options vanish from the cell loops (about 6 % of the
 * step at 4096^2).  Both forms compute the same bits. */
constexpr int FWE_DIFF = 1;      /* flux diffusion                     */
constexpr int FWE_RAINMAP = 2;   /* a rain map scales rain and top-up   */
constexpr int FWE_RAINSTEP = 4;  /* rain added every step               */
constexpr int FWE_GENERIC = 8;   /* options read at run time            */
constexpr int FWE_RTOPTS = 32;   /* diffusion, rain map and per-step rain read at run time,
                                  * pipe length 1 and exponent 1 built in (the batched form) */
constexpr int FWE_FLOWONLY = 16; /* flow and water passes only (flow_simulation): no
                                  * erosion, terrain fixed, writes depth and fluxes */

/* Resident CTAs per SM the step kernels are compiled for.  The erosion
 * forms take five (at most 48 registers, 5 x 34 KB of shared memory): 40
 * warps per SM issuing outrun four CTAs of the unconstrained 52-register
 * code although a few words then spill.  The flow-only form
 * (flow_simulation) fits 40 registers, six CTAs per SM; a looser bound
 * lets the compiler take 46 and costs the sixth CTA (5 % slower). */
constexpr int fwe_min_blocks(int flags) { return (flags & FWE_FLOWONLY) ? 6 : 5; }

/* Shared-memory layout of the staged fields, one for both staging modes.
 * Every array row covers the 40 columns x0-4 .. x0+35 (a TMA box must start
 * on a 16-byte boundary, so the boxes start at x0-4), column c holding
 * global column x0-4+c.  z and d hold rows y0-2 .. y0+17 (region 2: the
 * tile and a 2-cell halo), s, the old fluxes fo and the new fluxes fn rows
 * y0-1 .. y0+16 (region 1: a 1-cell halo).  The tile's own columns sit at
 * 4 .. 35, so cell pairs (2k, 2k+1) of the tile are 8-byte aligned in
 * every array.  Each staged array is padded to 20 rows so every box starts
 * 128-byte aligned. */
constexpr int FW = 40;

/* rows of the staged s1 box of k_vp_step(_tma): y0-4 .. y0+19 (region 1
 * and a reach of 2.5 cells for the bilinear taps of its cells) */
constexpr int FS_H = FT_TY + 8;

/* k_vp_step(_tma)'s staging of the previous step's velocity (region 1, in
 * rows padded to 20) and eroded sediment (rows y0-4 .. y0+19); dead once
 * the advected sediment is in FweSmem::s, so it shares memory with the new
 * fluxes of the flow pass */
struct AdvStage
{
  alignas(128) float u[FT_H2][FW];
  alignas(128) float v[FT_H2][FW];
  alignas(128) float s1[FS_H][FW];
};

struct FweSmem
{
  alignas(128) float z[FT_H2][FW];
  alignas(128) float d[FT_H2][FW];
  alignas(128) float s[FT_H2][FW];
  alignas(128) float fo[4][FT_H2][FW];
  union alignas(128)
  {
    float    fn[4][FT_H1][FW];
    AdvStage adv;
  };
  uint64_t bar;
  uint64_t bar2; /* k_vp_step_tma: the second group of boxes */
};
static_assert(sizeof(AdvStage) <= sizeof(float) * 4 * FT_H1 * FW, "advect-in staging fits the new-flux arrays");

/* the step's grids: old state in, new state out, plus this step's s1, u, v */
struct FweIo
{
  VpState      in;
  VpStateOut   out; /* out.s unused here (k_vp_advect writes it) */
  float       *s1, *u, *v;
  const float *rain;
  int          parity;
  int          maintain, diffusion, pl_one, kexp_one;
  float       *u_out, *v_out; /* last step: velocity outputs, nullable */
  int          vec;           /* nx even and every output 8-byte aligned: pair stores */
  int          flow_only;     /* flow_simulation step (FWE_FLOWONLY kernels) */
  int          stage16;       /* nx a multiple of 4 and every staged grid 16-byte aligned: a tile whose
                               * boxes lie inside the grid may stage them in 16-byte copies */
  unsigned     tma_extra_tx;  /* bytes a TMA tile's barrier expects beyond its boxes: 0, or the
                               * test hook's count, which makes every tile's wait run out */
  const float *s1_prev;       /* k_vp_step(_tma): the previous step's eroded sediment */
};

/* tensor maps of the seven input fields of one step (TMA staging):
 * z and d with a 40 x 20 box, s and the fluxes with a 40 x 18 box */
struct FweMaps
{
  CUtensorMap z, d, s, fl, fr, ft, fb;
};

/* tensor maps of the previous step's velocity and eroded sediment
 * (k_vp_step_tma): u and v with a 40 x 18 box, s1 with a 40 x 24 box */
struct AdvMaps
{
  CUtensorMap u, v, s1;
};

/* bytes the seven TMA boxes deliver */
constexpr unsigned FWE_TMA_BYTES = 4u * 40u * (2u * FT_H2 + 5u * FT_H1);
/* bytes the nine boxes of k_vp_step_tma deliver: group A (the previous
 * step's u, v and s1, and the stored depth), on which the advection and
 * the depth pass run while group B (z and the four old fluxes) is still
 * arriving */
constexpr unsigned STEP_TMA_BYTES = 4u * 40u * (2u * FT_H2 + 6u * FT_H1 + FS_H);
constexpr unsigned STEP_TMA_BYTES_A = 4u * 40u * (FT_H2 + 2u * FT_H1 + FS_H);
constexpr unsigned STEP_TMA_BYTES_B = 4u * 40u * (FT_H2 + 4u * FT_H1);
static_assert(STEP_TMA_BYTES_A + STEP_TMA_BYTES_B == STEP_TMA_BYTES, "the two groups are the nine boxes");

/* cp.async staging: z, d on the halo-2 region; s and old fluxes on the
 * halo-1 region; loads clamped to the grid, so every raw neighbour read is
 * the reference's clamp-to-edge read */
__device__ __forceinline__ void fwe_stage_cp_async(const FweIo &io, int nx, int ny, int x0, int y0, FweSmem &sm)
{
  const int tid = threadIdx.x;
  for (int e = tid; e < FT_W2 * FT_H2; e += FT_NT)
  {
    const int    ly = e / FT_W2, lx = e - ly * FT_W2;
    const size_t k = (size_t)clampi(y0 - 2 + ly, 0, ny - 1) * nx + clampi(x0 - 2 + lx, 0, nx - 1);
    cp_async4(&sm.z[ly][lx + 2], io.in.z + k);
    cp_async4(&sm.d[ly][lx + 2], io.in.d + k);
  }
  for (int e = tid; e < FT_W1 * FT_H1; e += FT_NT)
  {
    const int    ly = e / FT_W1, lx = e - ly * FT_W1;
    const size_t k = (size_t)clampi(y0 - 1 + ly, 0, ny - 1) * nx + clampi(x0 - 1 + lx, 0, nx - 1);
    cp_async4(&sm.s[ly][lx + 3], io.in.s + k);
    cp_async4(&sm.fo[0][ly][lx + 3], io.in.fl + k);
    cp_async4(&sm.fo[1][ly][lx + 3], io.in.fr + k);
    cp_async4(&sm.fo[2][ly][lx + 3], io.in.ft + k);
    cp_async4(&sm.fo[3][ly][lx + 3], io.in.fb + k);
  }
  cp_async_commit();
  cp_async_wait<0>();
}

/* cp.async staging of a folded step (k_vp_step): z, d (region 2) and the
 * old fluxes (region 1) clamped to the grid as fwe_stage_cp_async stages
 * them, the previous step's u and v on region 1 and s1 on columns x0-4 ..
 * x0+35, rows y0-4 .. y0+19, the last three at in-grid cells only (they
 * are read nowhere else).  io.u, io.v are this step's outputs; the
 * previous step's velocity comes in as u_prev, v_prev. */
__device__ __forceinline__ void fwe_stage_cp_async_step(const FweIo &io, const float *u_prev, const float *v_prev,
                                                        int nx, int ny, int x0, int y0, FweSmem &sm)
{
  const int tid = threadIdx.x;
  for (int e = tid; e < FT_W2 * FT_H2; e += FT_NT)
  {
    const int    ly = e / FT_W2, lx = e - ly * FT_W2;
    const size_t k = (size_t)clampi(y0 - 2 + ly, 0, ny - 1) * nx + clampi(x0 - 2 + lx, 0, nx - 1);
    cp_async4(&sm.z[ly][lx + 2], io.in.z + k);
    cp_async4(&sm.d[ly][lx + 2], io.in.d + k);
  }
  for (int e = tid; e < FT_W1 * FT_H1; e += FT_NT)
  {
    const int    ly = e / FT_W1, lx = e - ly * FT_W1;
    const int    gx = x0 - 1 + lx, gy = y0 - 1 + ly;
    const size_t k = (size_t)clampi(gy, 0, ny - 1) * nx + clampi(gx, 0, nx - 1);
    cp_async4(&sm.fo[0][ly][lx + 3], io.in.fl + k);
    cp_async4(&sm.fo[1][ly][lx + 3], io.in.fr + k);
    cp_async4(&sm.fo[2][ly][lx + 3], io.in.ft + k);
    cp_async4(&sm.fo[3][ly][lx + 3], io.in.fb + k);
    if (gx >= 0 && gx < nx && gy >= 0 && gy < ny)
    {
      cp_async4(&sm.adv.u[ly][lx + 3], u_prev + k);
      cp_async4(&sm.adv.v[ly][lx + 3], v_prev + k);
    }
  }
  for (int e = tid; e < FW * FS_H; e += FT_NT)
  {
    const int ly = e / FW, lx = e - ly * FW;
    const int gx = x0 - 4 + lx, gy = y0 - 4 + ly;
    if (gx >= 0 && gx < nx && gy >= 0 && gy < ny) cp_async4(&sm.adv.s1[ly][lx], io.s1_prev + (size_t)gy * nx + gx);
  }
  cp_async_commit();
  cp_async_wait<0>();
}

/* the boxes of k_vp_step's staging (rows y0-4 .. y0+19, columns x0-4 ..
 * x0+35) lie inside the grid, and the grids allow 16-byte copies */
__device__ __forceinline__ bool stage16_tile(const FweIo &io, int nx, int ny, int x0, int y0)
{
  return io.stage16 != 0 && x0 >= 4 && y0 >= 4 && x0 + FW - 4 <= nx && y0 + FS_H - 4 <= ny;
}

__device__ __forceinline__ void cp_async16(float *smem, const float *gmem)
{
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

/* fwe_stage_cp_async_step for a tile whose boxes lie inside the grid
 * (stage16_tile): whole 40-column box rows in 16-byte copies, about a
 * quarter of the copies and none of the index clamps.  The same cells land
 * at the same places (and the box columns that the clamped form leaves
 * unwritten, which no pass reads). */
__device__ __forceinline__ void fwe_stage_cp_async16_step(const FweIo &io, const float *u_prev, const float *v_prev,
                                                          int nx, int x0, int y0, FweSmem &sm)
{
  constexpr int Q = FW / 4; /* 16-byte copies per box row */
  const int     tid = threadIdx.x;
  for (int e = tid; e < Q * FT_H2; e += FT_NT)
  {
    const int    ly = e / Q, c = 4 * (e - ly * Q);
    const size_t k = (size_t)(y0 - 2 + ly) * nx + (x0 - 4 + c);
    cp_async16(&sm.z[ly][c], io.in.z + k);
    cp_async16(&sm.d[ly][c], io.in.d + k);
  }
  for (int e = tid; e < Q * FT_H1; e += FT_NT)
  {
    const int    ly = e / Q, c = 4 * (e - ly * Q);
    const size_t k = (size_t)(y0 - 1 + ly) * nx + (x0 - 4 + c);
    cp_async16(&sm.fo[0][ly][c], io.in.fl + k);
    cp_async16(&sm.fo[1][ly][c], io.in.fr + k);
    cp_async16(&sm.fo[2][ly][c], io.in.ft + k);
    cp_async16(&sm.fo[3][ly][c], io.in.fb + k);
    cp_async16(&sm.adv.u[ly][c], u_prev + k);
    cp_async16(&sm.adv.v[ly][c], v_prev + k);
  }
  for (int e = tid; e < Q * FS_H; e += FT_NT)
  {
    const int ly = e / Q, c = 4 * (e - ly * Q);
    cp_async16(&sm.adv.s1[ly][c], io.s1_prev + (size_t)(y0 - 4 + ly) * nx + (x0 - 4 + c));
  }
  cp_async_commit();
  cp_async_wait<0>();
}

/* Clamp-to-edge rebuild of the staged fields on a tile that touches the
 * grid's edge (TMA boxes read zeros outside the grid): z and d on region 2,
 * the old fluxes and, WITH_S, the sediment on region 1.  The clamped cell
 * is always inside the box; the edge test depends only on the tile, so the
 * barrier inside it is uniform. */
template <bool WITH_S>
__device__ __forceinline__ void fwe_fix_edges(int nx, int ny, int x0, int y0, FweSmem &sm)
{
  const int tid = threadIdx.x;
  if (x0 - 2 < 0 || x0 + FT_TX + 2 > nx || y0 - 2 < 0 || y0 + FT_TY + 2 > ny)
  {
    /* region 2: columns x0-2 .. x0+33 at smem 2 .. 37, rows y0-2 .. y0+17 */
    for (int e = tid; e < FT_W2 * FT_H2; e += FT_NT)
    {
      const int ly = e / FT_W2, lx = e - ly * FT_W2;
      const int gx = x0 - 2 + lx, gy = y0 - 2 + ly;
      if (gx >= 0 && gx < nx && gy >= 0 && gy < ny) continue;
      const int cy = clampi(gy, 0, ny - 1) - (y0 - 2), cx = clampi(gx, 0, nx - 1) - (x0 - 4);
      sm.z[ly][lx + 2] = sm.z[cy][cx];
      sm.d[ly][lx + 2] = sm.d[cy][cx];
    }
    /* region 1: columns x0-1 .. x0+32 at smem 3 .. 36, rows y0-1 .. y0+16 */
    for (int e = tid; e < FT_W1 * FT_H1; e += FT_NT)
    {
      const int ly = e / FT_W1, lx = e - ly * FT_W1;
      const int gx = x0 - 1 + lx, gy = y0 - 1 + ly;
      if (gx >= 0 && gx < nx && gy >= 0 && gy < ny) continue;
      const int cy = clampi(gy, 0, ny - 1) - (y0 - 1), cx = clampi(gx, 0, nx - 1) - (x0 - 4);
      if (WITH_S) sm.s[ly][lx + 3] = sm.s[cy][cx];
#pragma unroll
      for (int f = 0; f < 4; f++) sm.fo[f][ly][lx + 3] = sm.fo[f][cy][cx];
    }
    /* the copies read in-grid cells that the depth pass rewrites in place */
    __syncthreads();
  }
}

/* TMA staging: thread 0 arms the barrier and issues the seven box loads;
 * every thread waits (bounded).  Boxes read zeros outside the grid, so on
 * tiles that touch the grid's edge the cells outside are then overwritten
 * with their clamp-to-edge values (the clamped cell is always inside the
 * box; the edge test depends only on the tile, so the barrier inside it is
 * uniform).  Returns false, uniformly across the CTA, if the loads did not
 * complete in time. */
__device__ __forceinline__ bool fwe_stage_tma(const FweMaps &maps, int nx, int ny, int x0, int y0, FweSmem &sm,
                                              unsigned extra_tx)
{
  const int tid = threadIdx.x;
  if (tid == 0)
  {
    mbar_init(&sm.bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (tid == 0)
  {
    mbar_arrive_expect_tx(&sm.bar, FWE_TMA_BYTES + extra_tx);
    tma_load_2d(&sm.z[0][0], &maps.z, x0 - 4, y0 - 2, &sm.bar);
    tma_load_2d(&sm.d[0][0], &maps.d, x0 - 4, y0 - 2, &sm.bar);
    tma_load_2d(&sm.s[0][0], &maps.s, x0 - 4, y0 - 1, &sm.bar);
    tma_load_2d(&sm.fo[0][0][0], &maps.fl, x0 - 4, y0 - 1, &sm.bar);
    tma_load_2d(&sm.fo[1][0][0], &maps.fr, x0 - 4, y0 - 1, &sm.bar);
    tma_load_2d(&sm.fo[2][0][0], &maps.ft, x0 - 4, y0 - 1, &sm.bar);
    tma_load_2d(&sm.fo[3][0][0], &maps.fb, x0 - 4, y0 - 1, &sm.bar);
  }
  bool ok = mbar_wait_bounded(&sm.bar, 0);
  if (!ok) ok = mbar_wait_bounded(&sm.bar, 0); /* loads still in flight: give them a second window */
  if (!__syncthreads_and(ok)) return false;
  fwe_fix_edges<true>(nx, ny, x0, y0, sm);
  return true;
}

/* TMA staging of k_vp_step_tma in two groups on two barriers.  Group A:
 * the previous step's u and v (region 1), its s1 (rows y0-4 .. y0+19) and
 * the stored depth d (region 2), waited for here.  Group B: z (region 2)
 * and the old fluxes (region 1), waited for by fwe_wait_tma_step_b after
 * the advection and the depth pass have run on group A, so those overlap
 * its arrival.  Returns false, uniformly across the CTA, if group A did
 * not complete in time; group B's loads are then given their own windows
 * to land before the CTA leaves. */
__device__ __forceinline__ bool fwe_stage_tma_step(const FweMaps &maps, const AdvMaps &am, int x0, int y0,
                                                   FweSmem &sm, unsigned extra_tx)
{
  const int tid = threadIdx.x;
  if (tid == 0)
  {
    mbar_init(&sm.bar, 1);
    mbar_init(&sm.bar2, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (tid == 0)
  {
    mbar_arrive_expect_tx(&sm.bar, STEP_TMA_BYTES_A + extra_tx);
    tma_load_2d(&sm.adv.u[0][0], &am.u, x0 - 4, y0 - 1, &sm.bar);
    tma_load_2d(&sm.adv.v[0][0], &am.v, x0 - 4, y0 - 1, &sm.bar);
    tma_load_2d(&sm.adv.s1[0][0], &am.s1, x0 - 4, y0 - 4, &sm.bar);
    tma_load_2d(&sm.d[0][0], &maps.d, x0 - 4, y0 - 2, &sm.bar);
    mbar_arrive_expect_tx(&sm.bar2, STEP_TMA_BYTES_B);
    tma_load_2d(&sm.z[0][0], &maps.z, x0 - 4, y0 - 2, &sm.bar2);
    tma_load_2d(&sm.fo[0][0][0], &maps.fl, x0 - 4, y0 - 1, &sm.bar2);
    tma_load_2d(&sm.fo[1][0][0], &maps.fr, x0 - 4, y0 - 1, &sm.bar2);
    tma_load_2d(&sm.fo[2][0][0], &maps.ft, x0 - 4, y0 - 1, &sm.bar2);
    tma_load_2d(&sm.fo[3][0][0], &maps.fb, x0 - 4, y0 - 1, &sm.bar2);
  }
  bool ok = mbar_wait_bounded(&sm.bar, 0);
  if (!ok) ok = mbar_wait_bounded(&sm.bar, 0); /* loads still in flight: give them a second window */
  if (__syncthreads_and(ok)) return true;
  if (!mbar_wait_bounded(&sm.bar2, 0)) mbar_wait_bounded(&sm.bar2, 0);
  return false;
}

/* Group B of k_vp_step_tma's boxes (bounded wait), then the clamp-to-edge
 * rebuild of z, d and the old fluxes on edge tiles.  It runs after the
 * depth pass, so the rebuild copies depths already brought to the start
 * of the step, which are the depths of the clamped cells.  The sediment
 * needs no rebuild: it is advected at clamped cells, and u, v and s1 are
 * only read at in-grid cells.  false, uniformly across the CTA, if the
 * group did not complete in time. */
__device__ __forceinline__ bool fwe_wait_tma_step_b(int nx, int ny, int x0, int y0, FweSmem &sm)
{
  bool ok = mbar_wait_bounded(&sm.bar2, 0);
  if (!ok) ok = mbar_wait_bounded(&sm.bar2, 0);
  if (!__syncthreads_and(ok)) return false;
  fwe_fix_edges<false>(nx, ny, x0, y0, sm);
  return true;
}

/* Advected sediment of the tile and its ring (region 1) into sm.s:
 * s(i, j) = bilinear(s1, (i - dt u, j - dt v)) with the previous step's u,
 * v and s1, exactly as k_vp_advect evaluates it.  A ring cell outside the
 * grid takes the value of its clamp-to-edge cell (the reference's
 * clamped read of s there), so it is computed at that cell.  Taps inside
 * the staged s1 box (columns x0-4 .. x0+35, rows y0-4 .. y0+19) read shared
 * memory, the rest s1 in global memory.  INNER: region 1 lies inside the
 * grid, so no cell is clamped. */
/* advected sediment of one region-1 cell: column gx, row gy of the grid
 * (clamped), at shared-memory row l and column cc */
__device__ __forceinline__ void advect_cell(const VpConst &c, const float *__restrict__ s1g, int x0, int y0, int gx,
                                            int gy, int l, int cc, FweSmem &sm)
{
  const int   nx = c.nx, ny = c.ny;
  const float uu = sm.adv.u[gy - (y0 - 1)][gx - (x0 - 4)];
  const float vv = sm.adv.v[gy - (y0 - 1)][gx - (x0 - 4)];
  const float x = fsub((float)gx, fmul(c.dt, uu));
  const float y = fsub((float)gy, fmul(c.dt, vv));
  if (x >= 0.5f && x < c.xhi && y >= 0.5f && y < c.yhi)
  {
    /* The sample point lies inside the texel centres: the mirror of
     * linear_tap returns the coordinate itself, floor(x - 0.5) lies in
     * [0, nx - 2], so i0 needs no clamp and i1 = i0 + 1 (rows likewise).
     * The same rounded operations as linear_tap, without the identities. */
    Tap         tp;
    const float xm = fsub(x, 0.5f), ym = fsub(y, 0.5f);
    const float fx = floorf(xm), fy = floorf(ym);
    tp.a = fsub(xm, fx);
    tp.b = fsub(ym, fy);
    tp.i0 = (int)fx;
    tp.j0 = (int)fy;
    tp.i1 = tp.i0 + 1;
    tp.j1 = tp.j0 + 1;
    const int bi = tp.i0 - (x0 - 4), bj = tp.j0 - (y0 - 4);
    float     g00, g10, g01, g11;
    if ((unsigned)bi < (unsigned)(FW - 1) && (unsigned)bj < (unsigned)(FS_H - 1))
    {
      const float *r = &sm.adv.s1[bj][bi];
      g00 = r[0];
      g10 = r[1];
      g01 = r[FW];
      g11 = r[FW + 1];
    }
    else
    {
      const float *r = s1g + (size_t)tp.j0 * nx + tp.i0;
      g00 = __ldg(r);
      g10 = __ldg(r + 1);
      g01 = __ldg(r + nx);
      g11 = __ldg(r + nx + 1);
    }
    sm.s[l][cc] = blend(tp, g00, g10, g01, g11);
    return;
  }
  const Tap t = linear_tap(x, y, nx, ny);
  const int bi0 = t.i0 - (x0 - 4), bi1 = t.i1 - (x0 - 4);
  const int   bj0 = t.j0 - (y0 - 4), bj1 = t.j1 - (y0 - 4);
  float       g00, g10, g01, g11;
  if (bi0 >= 0 && bi1 < FW && bj0 >= 0 && bj1 < FS_H)
  {
    g00 = sm.adv.s1[bj0][bi0];
    g10 = sm.adv.s1[bj0][bi1];
    g01 = sm.adv.s1[bj1][bi0];
    g11 = sm.adv.s1[bj1][bi1];
  }
  else
  {
    const size_t r0 = (size_t)t.j0 * nx, r1 = (size_t)t.j1 * nx;
    g00 = __ldg(s1g + r0 + t.i0);
    g10 = __ldg(s1g + r0 + t.i1);
    g01 = __ldg(s1g + r1 + t.i0);
    g11 = __ldg(s1g + r1 + t.i1);
  }
  sm.s[l][cc] = blend(t, g00, g10, g01, g11);
}

/* rows of region 1 one thread advects */
constexpr int ADV_ROWS = 3;

/* Thread t < 204 takes column 3 + t % 34 of region 1 and its rows
 * ADV_ROWS (t / 34) .. + ADV_ROWS - 1: the column's index work is shared
 * and its gathers are in flight together (2 % fewer instructions per step
 * than one cell per loop item). */
template <bool INNER>
__device__ __forceinline__ void advect_region1(const VpConst &c, const float *__restrict__ s1g, int x0, int y0,
                                               FweSmem &sm)
{
  static_assert(FT_H1 % ADV_ROWS == 0, "region 1 splits into whole row groups");
  const int t = threadIdx.x;
  if (t >= FT_W1 * (FT_H1 / ADV_ROWS)) return;
  const int cc = 3 + t % FT_W1, l0 = ADV_ROWS * (t / FT_W1);
  int       gx = x0 - 4 + cc;
  if (!INNER) gx = clampi(gx, 0, c.nx - 1);
#pragma unroll
  for (int r = 0; r < ADV_ROWS; r++)
  {
    int gy = y0 - 1 + l0 + r;
    if (!INNER) gy = clampi(gy, 0, c.ny - 1);
    advect_cell(c, s1g, x0, y0, gx, gy, l0 + r, cc, sm);
  }
}

__device__ __forceinline__ float2 lds2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ void   sts2(float *p, float a, float b) { *reinterpret_cast<float2 *>(p) = make_float2(a, b); }

/* Store the values of a cell pair (columns gx, gx + 1 of row offset k = the
 * pair's first cell): one 8-byte store when both cells are in the grid and
 * the grids allow it, else one or two 4-byte stores. */
__device__ __forceinline__ void st_pair(float *p, size_t k, float a, float b, bool second, bool vec)
{
  if (second && vec)
    *reinterpret_cast<float2 *>(p + k) = make_float2(a, b);
  else
  {
    p[k] = a;
    if (second) p[k + 1] = b;
  }
}

/* One tile of the step on staged fields, two adjacent cells per thread:
 * depth at the start of the step, flow on the tile plus a 1-cell ring into
 * shared memory, then water and erosion on the tile, which also store the
 * tile's new fluxes.  A pair reads its centre values as 8-byte words and
 * shares its inner neighbours, so a cell costs about half the shared-memory
 * and store instructions of one cell per thread; the arithmetic of each
 * cell is unchanged.  INNER: the tile and its 2-cell halo lie inside the
 * grid and the outputs take pair stores (fwe_inner_tile), so every edge
 * clamp and store-width test below is known to be the identity / true and
 * drops out; the cells' values are the same either way.  mid() runs
 * between the depth pass and the flow pass (uniformly across the CTA); if
 * it returns false the tile computes and stores nothing (a staging
 * timeout) but still takes part in the volume sum. */
/* fwe_compute's hook between the depth pass and the flow pass: nothing
 * to wait for */
struct NoMid
{
  __device__ bool operator()() const { return true; }
};

template <bool MAINTAIN, int F, bool INNER = false, class Mid = NoMid>
__device__ __forceinline__ void fwe_compute(const FweIo &io, const VpConst &c, VpScalars *sc, double *partials,
                                            int bx, int by, int nbx, int nby, FweSmem &sm, Mid mid = Mid())
{
  static_assert(FT_TX == 32 && FT_TY == 16 && FT_NT == 256, "one cell pair per thread in the water pass");
  constexpr bool GEN = (F & FWE_GENERIC) != 0;
  constexpr bool RT = GEN || (F & FWE_RTOPTS) != 0;
  constexpr bool FLOW_ONLY = (F & FWE_FLOWONLY) != 0;
  const int      tid = threadIdx.x;
  const int      nx = c.nx, ny = c.ny;
  const int      x0 = bx * FT_TX, y0 = by * FT_TY;
  const float    add = MAINTAIN ? sc->add[io.parity] : 0.f;
  const float    rvol = MAINTAIN ? sc->rvol : 1.f;
  const bool     rain_step = RT ? c.rps != 0.f : (F & FWE_RAINSTEP) != 0;
  const bool     rain_map = RT ? io.rain != nullptr : (F & FWE_RAINMAP) != 0;
  const bool     diffusion = RT ? io.diffusion != 0 : (F & FWE_DIFF) != 0;
  const bool     pl_one = GEN ? io.pl_one != 0 : true;
  const bool     kexp_one = GEN ? io.kexp_one != 0 : true;

  /* stored depth -> depth at the start of the step, region 2 (columns
   * x0-2 .. x0+33 = smem 2 .. 37), 18 pairs per row */
  for (int e = tid; e < 18 * FT_H2; e += FT_NT)
  {
    const int q = e / 18, cc = 2 + 2 * (e - q * 18);
    float2    dd = lds2(&sm.d[q][cc]);
    float     r0 = 1.f, r1 = 1.f;
    if (rain_map)
    {
      const size_t row = (size_t)clampi(y0 - 2 + q, 0, ny - 1) * nx;
      r0 = __ldg(io.rain + row + clampi(x0 - 4 + cc, 0, nx - 1));
      r1 = __ldg(io.rain + row + clampi(x0 - 3 + cc, 0, nx - 1));
    }
    if (rain_step)
    {
      dd.x = depth_d1<MAINTAIN, true>(dd.x, r0, add, rvol, c.rps);
      dd.y = depth_d1<MAINTAIN, true>(dd.y, r1, add, rvol, c.rps);
    }
    else
    {
      dd.x = depth_d1<MAINTAIN, false>(dd.x, r0, add, rvol, c.rps);
      dd.y = depth_d1<MAINTAIN, false>(dd.y, r1, add, rvol, c.rps);
    }
    sts2(&sm.d[q][cc], dd.x, dd.y);
  }
  __syncthreads();

  double part = 0.0;
  if (mid())
  {
    /* flow pass on region 1 (columns x0-1 .. x0+32 = smem 3 .. 36, rows
     * y0-1 .. y0+16): items 0 .. 287 are the 16 pairs (smem 4 .. 35) of each
     * of the 18 rows, items 288 .. 323 the two ring columns 3 and 36 */
    auto flow1 = [&](float zc, float dc, float zw, float dw, float ze, float de, float zs, float ds, float zn,
                     float dn, float &fl, float &fr, float &ft, float &fb) {
      if (diffusion)
      {
        if (pl_one) flow_cell<true, true>(c, zc, dc, zw, dw, ze, de, zs, ds, zn, dn, fl, fr, ft, fb);
        else flow_cell<true, false>(c, zc, dc, zw, dw, ze, de, zs, ds, zn, dn, fl, fr, ft, fb);
      }
      else
      {
        if (pl_one) flow_cell<false, true>(c, zc, dc, zw, dw, ze, de, zs, ds, zn, dn, fl, fr, ft, fb);
        else flow_cell<false, false>(c, zc, dc, zw, dw, ze, de, zs, ds, zn, dn, fl, fr, ft, fb);
      }
    };
    for (int e = tid; e < 16 * FT_H1 + 2 * FT_H1; e += FT_NT)
    {
      if (e < 16 * FT_H1)
      {
        const int    l = e >> 4, cc = 4 + 2 * (e & 15), q = l + 1;
        const float2 zc = lds2(&sm.z[q][cc]), dc = lds2(&sm.d[q][cc]);
        const float2 zn = lds2(&sm.z[q - 1][cc]), dn = lds2(&sm.d[q - 1][cc]);
        const float2 zs = lds2(&sm.z[q + 1][cc]), ds = lds2(&sm.d[q + 1][cc]);
        const float  zw = sm.z[q][cc - 1], dw = sm.d[q][cc - 1], ze = sm.z[q][cc + 2], de = sm.d[q][cc + 2];
        float2       fl = lds2(&sm.fo[0][l][cc]), fr = lds2(&sm.fo[1][l][cc]), ft = lds2(&sm.fo[2][l][cc]),
               fb = lds2(&sm.fo[3][l][cc]);
        flow1(zc.x, dc.x, zw, dw, zc.y, dc.y, zs.x, ds.x, zn.x, dn.x, fl.x, fr.x, ft.x, fb.x);
        flow1(zc.y, dc.y, zc.x, dc.x, ze, de, zs.y, ds.y, zn.y, dn.y, fl.y, fr.y, ft.y, fb.y);
        sts2(&sm.fn[0][l][cc], fl.x, fl.y);
        sts2(&sm.fn[1][l][cc], fr.x, fr.y);
        sts2(&sm.fn[2][l][cc], ft.x, ft.y);
        sts2(&sm.fn[3][l][cc], fb.x, fb.y);
      }
      else
      {
        const int r = e - 16 * FT_H1, l = r >> 1, cc = (r & 1) ? 36 : 3, q = l + 1;
        float     fl = sm.fo[0][l][cc], fr = sm.fo[1][l][cc], ft = sm.fo[2][l][cc], fb = sm.fo[3][l][cc];
        flow1(sm.z[q][cc], sm.d[q][cc], sm.z[q][cc - 1], sm.d[q][cc - 1], sm.z[q][cc + 1], sm.d[q][cc + 1],
              sm.z[q + 1][cc], sm.d[q + 1][cc], sm.z[q - 1][cc], sm.d[q - 1][cc], fl, fr, ft, fb);
        sm.fn[0][l][cc] = fl;
        sm.fn[1][l][cc] = fr;
        sm.fn[2][l][cc] = ft;
        sm.fn[3][l][cc] = fb;
      }
    }
    __syncthreads();

    /* water and erosion on the tile: thread t takes row t / 16 and the pair
     * of tile columns 2 (t % 16), 2 (t % 16) + 1 */
    const int ty = tid >> 4, pk = tid & 15;
    const int gy = y0 + ty, gx = x0 + 2 * pk;
    const int cc = 4 + 2 * pk; /* smem column of the first cell */
    if (INNER || (gx < nx && gy < ny))
    {
      const bool second = INNER || gx + 1 < nx;
      const int  l = ty + 1, q = ty + 2;
      /* flux neighbours: rows and columns clamped to the grid (new fluxes are
       * derived: outside the grid they are the edge cell's own values) */
      const int  ln = INNER ? ty : clampi(gy - 1, 0, ny - 1) - (y0 - 1);
      const int  ls = INNER ? ty + 2 : clampi(gy + 1, 0, ny - 1) - (y0 - 1);
      const int  cw0 = INNER || gx > 0 ? cc - 1 : cc;          /* west of the first cell  */
      const int  ce0 = second ? cc + 1 : cc;                   /* east of the first cell  */
      const int  ce1 = INNER || gx + 2 < nx ? cc + 2 : cc + 1; /* east of the second cell */
      const float2 flc = lds2(&sm.fn[0][l][cc]), frc = lds2(&sm.fn[1][l][cc]), ftc = lds2(&sm.fn[2][l][cc]),
                   fbc = lds2(&sm.fn[3][l][cc]);
      const float2 ftn = lds2(&sm.fn[2][ln][cc]), fbs = lds2(&sm.fn[3][ls][cc]);
      const float  frw0 = sm.fn[1][l][cw0], fle0 = sm.fn[0][l][ce0], fle1 = sm.fn[0][l][ce1];
      const float2 d1 = lds2(&sm.d[q][cc]);
      float        d2a, ua, va, d2b, ub, vb;
      if (pl_one)
      {
        water_cell<true>(c, d1.x, flc.x, frc.x, ftc.x, fbc.x, frw0, fle0, ftn.x, fbs.x, d2a, ua, va);
        water_cell<true>(c, d1.y, flc.y, frc.y, ftc.y, fbc.y, frc.x, fle1, ftn.y, fbs.y, d2b, ub, vb);
      }
      else
      {
        water_cell<false>(c, d1.x, flc.x, frc.x, ftc.x, fbc.x, frw0, fle0, ftn.x, fbs.x, d2a, ua, va);
        water_cell<false>(c, d1.y, flc.y, frc.y, ftc.y, fbc.y, frc.x, fle1, ftn.y, fbs.y, d2b, ub, vb);
      }
      const size_t k = (size_t)gy * nx + gx;
      const bool   vec = INNER || io.vec != 0;
      if (FLOW_ONLY)
      {
        /* flow_simulation: the depth after the water pass is the next step's
         * depth as it is (no evaporation, no erosion; the terrain is fixed) */
        st_pair(io.out.fl, k, flc.x, flc.y, second, vec);
        st_pair(io.out.fr, k, frc.x, frc.y, second, vec);
        st_pair(io.out.ft, k, ftc.x, ftc.y, second, vec);
        st_pair(io.out.fb, k, fbc.x, fbc.y, second, vec);
        st_pair(io.out.d, k, d2a, d2b, second, vec);
        (void)ua, (void)ub, (void)va, (void)vb;
      }
      else
      {
        const float dea = fmul(d2a, c.keep), deb = fmul(d2b, c.keep);
        /* what the water pass produced, stored before the erosion arithmetic
         * so its registers are free there (the stores go through generic
         * pointers, so the compiler keeps them after the shared-memory loads
         * that follow them in the source: their order decides what stays
         * live; 48 registers without spills, 2.5 % faster than storing after
         * erosion) */
        st_pair(io.out.fl, k, flc.x, flc.y, second, vec);
        st_pair(io.out.fr, k, frc.x, frc.y, second, vec);
        st_pair(io.out.ft, k, ftc.x, ftc.y, second, vec);
        st_pair(io.out.fb, k, fbc.x, fbc.y, second, vec);
        st_pair(io.out.d, k, dea, deb, second, vec);
        st_pair(io.u, k, ua, ub, second, vec);
        st_pair(io.v, k, va, vb, second, vec);
        if (io.u_out)
        {
          st_pair(io.u_out, k, ua, ub, second, vec);
          st_pair(io.v_out, k, va, vb, second, vec);
        }
        const float2 zc = lds2(&sm.z[q][cc]), zn = lds2(&sm.z[q - 1][cc]), zs = lds2(&sm.z[q + 1][cc]);
        const float  zw = sm.z[q][cc - 1], ze = sm.z[q][cc + 2];
        const float2 s0 = lds2(&sm.s[l][cc]), sn = lds2(&sm.s[l - 1][cc]), ss = lds2(&sm.s[l + 1][cc]);
        const float  sw = sm.s[l][cc - 1], se = sm.s[l][cc + 2];
        float        zoa, soa, zob, sob;
        if (kexp_one)
        {
          erosion_cell<true>(c, zc.x, s0.x, zw, zc.y, zn.x, zs.x, sw, s0.y, sn.x, ss.x, d2a, ua, va, zoa, soa);
          erosion_cell<true>(c, zc.y, s0.y, zc.x, ze, zn.y, zs.y, s0.x, se, sn.y, ss.y, d2b, ub, vb, zob, sob);
        }
        else
        {
          erosion_cell<false>(c, zc.x, s0.x, zw, zc.y, zn.x, zs.x, sw, s0.y, sn.x, ss.x, d2a, ua, va, zoa, soa);
          erosion_cell<false>(c, zc.y, s0.y, zc.x, ze, zn.y, zs.y, s0.x, se, sn.y, ss.y, d2b, ub, vb, zob, sob);
        }
        st_pair(io.out.z, k, zoa, zob, second, vec);
        st_pair(io.s1, k, soa, sob, second, vec);
        part = (double)dea;
        if (second) part += (double)deb;
      }
    }
  }

  if (MAINTAIN)
  {
    const float v0 = sc->v0;
    float      *outp = &sc->add[io.parity ^ 1];
    grid_sum_commit<FT_NT>(part, partials, &sc->ticket, (unsigned)(nbx * nby), (unsigned)(by * nbx + bx),
                           [&](double total) { *outp = fsub(v0, (float)total); });
  }
}

/* the tile at (x0, y0) and its 2-cell halo lie inside the grid, and the
 * outputs take pair stores: fwe_compute's INNER form applies */
__device__ __forceinline__ bool fwe_inner_tile(const FweIo &io, int nx, int ny, int x0, int y0)
{
  return io.vec != 0 && x0 >= 2 && x0 + FT_TX + 2 <= nx && y0 >= 2 && y0 + FT_TY + 2 <= ny;
}

template <bool MAINTAIN, int F>
__global__ void __launch_bounds__(FT_NT, fwe_min_blocks(F)) k_vp_fwe(FweIo io, VpConst c, VpScalars *sc, double *partials)
{
  __shared__ FweSmem sm;
  fwe_stage_cp_async(io, c.nx, c.ny, blockIdx.x * FT_TX, blockIdx.y * FT_TY, sm);
  __syncthreads();
  if (fwe_inner_tile(io, c.nx, c.ny, blockIdx.x * FT_TX, blockIdx.y * FT_TY))
    fwe_compute<MAINTAIN, F, true>(io, c, sc, partials, blockIdx.x, blockIdx.y, gridDim.x, gridDim.y, sm);
  else
    fwe_compute<MAINTAIN, F>(io, c, sc, partials, blockIdx.x, blockIdx.y, gridDim.x, gridDim.y, sm);
}

/* The same step with the input tiles fetched by TMA.  A tile whose loads
 * time out sets bit 0 of sc->error and writes nothing; with the volume
 * top-up it still takes part in the grid-wide sum (adding zero) so the
 * last block's finish is not left waiting for it. */
template <bool MAINTAIN, int F>
__global__ void __launch_bounds__(FT_NT, fwe_min_blocks(F))
    k_vp_fwe_tma(FweIo io, const __grid_constant__ FweMaps maps, VpConst c, VpScalars *sc, double *partials)
{
  __shared__ FweSmem sm;
  if (!fwe_stage_tma(maps, c.nx, c.ny, blockIdx.x * FT_TX, blockIdx.y * FT_TY, sm, io.tma_extra_tx))
  {
    if (threadIdx.x == 0) atomicOr(&sc->error, 1u);
    if (MAINTAIN)
    {
      const float v0 = sc->v0;
      float      *outp = &sc->add[io.parity ^ 1];
      grid_sum_commit<FT_NT>(0.0, partials, &sc->ticket, gridDim.x * gridDim.y,
                             blockIdx.y * gridDim.x + blockIdx.x,
                             [&](double total) { *outp = fsub(v0, (float)total); });
    }
    return;
  }
  if (fwe_inner_tile(io, c.nx, c.ny, blockIdx.x * FT_TX, blockIdx.y * FT_TY))
    fwe_compute<MAINTAIN, F, true>(io, c, sc, partials, blockIdx.x, blockIdx.y, gridDim.x, gridDim.y, sm);
  else
    fwe_compute<MAINTAIN, F>(io, c, sc, partials, blockIdx.x, blockIdx.y, gridDim.x, gridDim.y, sm);
}

/* A step after the first with cp.async staging (grids the TMA rules
 * exclude): the previous step's advection and this step's flow, water and
 * erosion in one tile; u_prev, v_prev and io.s1_prev hold the previous
 * step's velocity and eroded sediment. */
template <bool MAINTAIN, int F>
__global__ void __launch_bounds__(FT_NT, fwe_min_blocks(F))
    k_vp_step(FweIo io, const float *__restrict__ u_prev, const float *__restrict__ v_prev, VpConst c,
              VpScalars *sc, double *partials)
{
  __shared__ FweSmem sm;
  const int x0 = blockIdx.x * FT_TX, y0 = blockIdx.y * FT_TY;
  if (stage16_tile(io, c.nx, c.ny, x0, y0)) fwe_stage_cp_async16_step(io, u_prev, v_prev, c.nx, x0, y0, sm);
  else fwe_stage_cp_async_step(io, u_prev, v_prev, c.nx, c.ny, x0, y0, sm);
  __syncthreads();
  /* the advected sediment is written here and read after fwe_compute's
   * first barrier */
  if (fwe_inner_tile(io, c.nx, c.ny, x0, y0))
  {
    advect_region1<true>(c, io.s1_prev, x0, y0, sm);
    fwe_compute<MAINTAIN, F, true>(io, c, sc, partials, blockIdx.x, blockIdx.y, gridDim.x, gridDim.y, sm);
  }
  else
  {
    advect_region1<false>(c, io.s1_prev, x0, y0, sm);
    fwe_compute<MAINTAIN, F>(io, c, sc, partials, blockIdx.x, blockIdx.y, gridDim.x, gridDim.y, sm);
  }
}

/* The same with the nine input boxes fetched by TMA in two groups (am
 * holds the maps of the previous step's u, v and s1).  Timeouts as
 * k_vp_fwe_tma. */
template <bool MAINTAIN, int F>
__global__ void __launch_bounds__(FT_NT, fwe_min_blocks(F))
    k_vp_step_tma(FweIo io, const __grid_constant__ FweMaps maps, const __grid_constant__ AdvMaps am, VpConst c,
                  VpScalars *sc, double *partials)
{
  __shared__ FweSmem sm;
  const int x0 = blockIdx.x * FT_TX, y0 = blockIdx.y * FT_TY;
  if (!fwe_stage_tma_step(maps, am, x0, y0, sm, io.tma_extra_tx))
  {
    if (threadIdx.x == 0) atomicOr(&sc->error, 1u);
    if (MAINTAIN)
    {
      const float v0 = sc->v0;
      float      *outp = &sc->add[io.parity ^ 1];
      grid_sum_commit<FT_NT>(0.0, partials, &sc->ticket, gridDim.x * gridDim.y,
                             blockIdx.y * gridDim.x + blockIdx.x,
                             [&](double total) { *outp = fsub(v0, (float)total); });
    }
    return;
  }
  /* group B (z, fluxes) arrives during the advection and the depth pass */
  auto group_b = [&]() {
    if (fwe_wait_tma_step_b(c.nx, c.ny, x0, y0, sm)) return true;
    if (threadIdx.x == 0) atomicOr(&sc->error, 1u);
    return false;
  };
  if (fwe_inner_tile(io, c.nx, c.ny, x0, y0))
  {
    advect_region1<true>(c, io.s1_prev, x0, y0, sm);
    fwe_compute<MAINTAIN, F, true>(io, c, sc, partials, blockIdx.x, blockIdx.y, gridDim.x, gridDim.y, sm, group_b);
  }
  else
  {
    advect_region1<false>(c, io.s1_prev, x0, y0, sm);
    fwe_compute<MAINTAIN, F>(io, c, sc, partials, blockIdx.x, blockIdx.y, gridDim.x, gridDim.y, sm, group_b);
  }
}

/* Launch one k_vp_fwe (tma false) or k_vp_fwe_tma (maps != NULL) step on
 * stream s with the kernel specialised for the step's options
 * (hm_vpipes_fwe_cp_async.cu, hm_vpipes_fwe_tma.cu). */
int launch_fwe_cp_async(const FweIo &io, const VpConst &c, VpScalars *sc, double *partials, dim3 grid,
                        cudaStream_t s);
int launch_fwe_tma(const FweIo &io, const FweMaps &maps, const VpConst &c, VpScalars *sc, double *partials,
                   dim3 grid, cudaStream_t s);
/* Launch one k_vp_step_tma step (hm_vpipes_step_tma.cu); io.s1_prev and am
 * hold the previous step's s1, u and v. */
int launch_step_tma(const FweIo &io, const FweMaps &maps, const AdvMaps &am, const VpConst &c, VpScalars *sc,
                    double *partials, dim3 grid, cudaStream_t s);
/* Launch one k_vp_step (cp.async staging, hm_vpipes_step_cp_async.cu). */
int launch_step_cp_async(const FweIo &io, const float *u_prev, const float *v_prev, const VpConst &c, VpScalars *sc,
                         double *partials, dim3 grid, cudaStream_t s);

/* Two steps t, t+1 (t >= 1, no volume top-up) in one launch of k_vp_tb2
 * (hm_vpipes_tb.cu): the grids it reads and the grids it writes. */
struct TbIo
{
  VpState      in;                        /* state before step t (z, d, fluxes)          */
  const float *s1_prev, *u_prev, *v_prev; /* step t-1's eroded sediment and velocity      */
  const float *rain;                      /* nullable                                    */
  VpStateOut   out;                       /* state after step t+1 (z, d, fluxes)         */
  float       *s1, *u, *v;                /* step t+1's eroded sediment and velocity      */
  float       *u_out, *v_out;             /* velocity outputs when t+1 is the last step, nullable */
  int          diffusion, pl_one, kexp_one;
};
int launch_vp_tb2(const TbIo &io, const VpConst &c, cudaStream_t s);

/* tensor maps of one state copy (hm_vpipes.cu); false if the grid or the
 * buffers do not meet the TMA rules (row pitch and bases 16-byte aligned,
 * boxes no larger than the grid) */
bool fwe_maps(const VpFields &f, int nx, int ny, FweMaps *m);
/* tensor maps of one copy of s1, u, v for k_vp_step_tma; false as above */
bool adv_maps(const float *u, const float *v, const float *s1, int nx, int ny, AdvMaps *m);

/* template flags of a step's options */
inline int fwe_flags(const FweIo &io, const VpConst &c)
{
  if (io.flow_only) return FWE_FLOWONLY | (io.diffusion ? FWE_DIFF : 0);
  if (!io.pl_one || !io.kexp_one) return FWE_GENERIC;
  return (io.diffusion ? FWE_DIFF : 0) | (io.rain ? FWE_RAINMAP : 0) | (c.rps != 0.f ? FWE_RAINSTEP : 0);
}

/* The same for the erosion steps only (no flow-only words). */
template <template <bool, int> class K, class Launch>
int step_dispatch(bool maintain, int f, Launch launch)
{
#define HM_STEP_CASE(FF)                                                                                               \
  case FF: return maintain ? launch(K<true, FF>::fn()) : launch(K<false, FF>::fn());
  switch (f)
  {
    HM_STEP_CASE(0)
    HM_STEP_CASE(1)
    HM_STEP_CASE(2)
    HM_STEP_CASE(3)
    HM_STEP_CASE(4)
    HM_STEP_CASE(5)
    HM_STEP_CASE(6)
    HM_STEP_CASE(7)
  default: return maintain ? launch(K<true, FWE_GENERIC>::fn()) : launch(K<false, FWE_GENERIC>::fn());
  }
#undef HM_STEP_CASE
}

/* Launch the kernel K<MAINTAIN, F> for run-time (maintain, f), f one of
 * the eight fixed-option words or FWE_GENERIC; `launch` receives the
 * kernel's address. */
template <template <bool, int> class K, class Launch>
int fwe_dispatch(bool maintain, int f, Launch launch)
{
#define HM_FWE_CASE(FF)                                                                                                \
  case FF: return maintain ? launch(K<true, FF>::fn()) : launch(K<false, FF>::fn());
  switch (f)
  {
    HM_FWE_CASE(0)
    HM_FWE_CASE(1)
    HM_FWE_CASE(2)
    HM_FWE_CASE(3)
    HM_FWE_CASE(4)
    HM_FWE_CASE(5)
    HM_FWE_CASE(6)
    HM_FWE_CASE(7)
    HM_FWE_CASE(FWE_FLOWONLY)
    HM_FWE_CASE(FWE_FLOWONLY | FWE_DIFF)
  default: return maintain ? launch(K<true, FWE_GENERIC>::fn()) : launch(K<false, FWE_GENERIC>::fn());
  }
#undef HM_FWE_CASE
}

/* Advection over the grid: block x covers 256 columns, and each thread
 * takes ADV_R consecutive rows of its column at a time, so that the
 * velocity loads of all ADV_R rows, then all their 4 ADV_R gathers, are in
 * flight together (the pass is bound by the latency of these two dependent
 * rounds of loads). */
constexpr int ADV_R = 4;

/* Advection of rows jb .. jb+R-1 of column i (rows past the grid are
 * loaded clamped and not stored). */
template <int R>
__device__ __forceinline__ void advect_rows(const float *__restrict__ s1,
                                            const float *__restrict__ u,
                                            const float *__restrict__ v,
                                            float *__restrict__ s_out,
                                            const VpConst &c,
                                            int i,
                                            int jb)
{
  float uu[R], vv[R];
#pragma unroll
  for (int q = 0; q < R; q++)
  {
    const size_t k = (size_t)min(jb + q, c.ny - 1) * c.nx + i;
    uu[q] = __ldg(u + k);
    vv[q] = __ldg(v + k);
  }
  Tap   t[R];
  float g[R][4];
#pragma unroll
  for (int q = 0; q < R; q++)
  {
    const int    j = min(jb + q, c.ny - 1);
    const float  x = fsub((float)i, fmul(c.dt, uu[q]));
    const float  y = fsub((float)j, fmul(c.dt, vv[q]));
    t[q] = linear_tap(x, y, c.nx, c.ny);
    const size_t r0 = (size_t)t[q].j0 * c.nx, r1 = (size_t)t[q].j1 * c.nx;
    g[q][0] = __ldg(s1 + r0 + t[q].i0);
    g[q][1] = __ldg(s1 + r0 + t[q].i1);
    g[q][2] = __ldg(s1 + r1 + t[q].i0);
    g[q][3] = __ldg(s1 + r1 + t[q].i1);
  }
#pragma unroll
  for (int q = 0; q < R; q++)
    if (jb + q < c.ny) s_out[(size_t)(jb + q) * c.nx + i] = blend(t[q], g[q][0], g[q][1], g[q][2], g[q][3]);
}

template <int R>
__global__ void __launch_bounds__(256) k_vp_advect(const float *__restrict__ s1,
                                                    const float *__restrict__ u,
                                                    const float *__restrict__ v,
                                                    float *__restrict__ s_out,
                                                    VpConst c)
{
  const int i = blockIdx.x * 256 + threadIdx.x;
  if (i >= c.nx) return;
  for (int jb = blockIdx.y * R; jb < c.ny; jb += gridDim.y * R) advect_rows<R>(s1, u, v, s_out, c, i, jb);
}

} // namespace hm

#endif
