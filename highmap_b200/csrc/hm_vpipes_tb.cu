/*
 * hm_vpipes_tb.cu - two virtual-pipes steps per launch (temporal blocking).
 *
 * The reference advances one step per round of its four kernels
 * (HighMap/src/erosion/hydraulic_vpipes_gpu.cpp:59-170 around
 * HighMap/src/gpu_opencl/kernels/hydraulic_vpipes.cl:5-211).  k_vp_tb2
 * advances steps t and t + 1 of an output tile (32 x 16, or 16 x 8 on
 * small grids) in one CTA: the
 * state of step t is read once from HBM and only the state after step
 * t + 1 is written, half the traffic of two one-step launches, at the cost
 * of computing step t again on a halo that neighbouring tiles also compute.
 *
 * Regions around the tile (h = ring width, clipped to the grid):
 *   h = 6  z and the start depth d1 of step t;
 *   h = 5  the old fluxes, step t's flow (new fluxes, in place) and its
 *          advected sediment s_t = bilinear(s1_{t-1}, x - dt u_{t-1});
 *   h = 4  step t's water and erosion: z', the evaporated depth, s1_t,
 *          u_t, v_t;
 *   h = 2  step t + 1's start depth;
 *   h = 1  step t + 1's flow and its advected sediment s_{t+1}, gathered
 *          from s1_t: taps inside the h = 4 region read shared memory,
 *          taps beyond it (water faster than about 2.5 cells per step)
 *          recompute s1_t at that cell from step t's state in global
 *          memory (tb_s1_at), which no CTA writes during the launch;
 *   h = 0  step t + 1's water and erosion, written out.
 * Every value is computed at a cell inside the grid, and every neighbour
 * read is of the clamped neighbour (the reference's clamp-to-edge reads),
 * so a cell's values are the one-step kernels' bit for bit.  The region of
 * each pass lies one ring inside the region of the values it reads.
 *
 * Without the water-volume top-up only: the top-up of step t + 1 needs the
 * grid-wide sum of step t's depth.  Work per output cell-step against the
 * one-step tile: about 1.4x (step t on the halo), with generic cell loops
 * (one cell per loop item, options read at run time).  The autotuner times
 * it beside the one-step kernels and keeps it only where it is faster.
 */
#include <cuda_runtime.h>

#include "hm_internal.h"
#include "hm_vpipes_tiled.cuh"

namespace hm
{

constexpr int TB_NT = 256;              /* threads per CTA                     */
constexpr int TB_HX = 4;                /* ring of step t's eroded sediment     */
constexpr int TB_H1 = TB_HX + 1;        /* ring of step t's flow and advection  */
constexpr int TB_H2 = TB_HX + 2;        /* ring of step t's z and depth         */
/* Output tile TX x TY: 32 x 16, or 16 x 8 on grids with fewer than two
 * 32 x 16 tiles per SM, where a launch is one wave and its time is one
 * CTA's chain of dependent passes (a quarter of the cells per CTA, four
 * times the CTAs).  Shared-memory fields, each W x H floats over columns
 * x0-6 .. x0+TX+5 and rows y0-6 .. y0+TY+5. */
template <int TX, int TY>
struct TbShape
{
  static constexpr int    W = TX + 2 * TB_H2, H = TY + 2 * TB_H2, N = W * H;
  static constexpr size_t SMEM = 11 * (size_t)N * sizeof(float);
};
enum
{
  TB_Z,   /* z of step t                                        */
  TB_D,   /* d1 of step t, then the evaporated depth, then d1 of step t+1 */
  TB_FL,  /* fluxes: old, then step t's, then step t+1's         */
  TB_FR,
  TB_FT,
  TB_FB,
  TB_S,   /* advected sediment of step t, then of step t+1        */
  TB_ZN,  /* z after step t                                      */
  TB_S1N, /* eroded sediment of step t                           */
  TB_UN,  /* velocity of step t                                  */
  TB_VN,
  TB_NF
};
static_assert(TB_NF == 11, "TbShape::SMEM holds eleven fields");

/* Kernel option word: TB_DIFF flux diffusion; TB_GEN pipe length and
 * discharge exponent read at run time (without it both are 1, and
 * diffusion is TB_DIFF). */
constexpr int TB_DIFF = 1, TB_GEN = 2;

/* ---- per-cell passes ------------------------------------------------- */

__device__ __forceinline__ float tb_d1(const VpConst &c, const float *rain, float d, size_t k)
{
  if (c.rps == 0.f) return d;
  const float r = rain ? __ldg(rain + k) : 1.f;
  return fadd(d, fmul(c.rps, r));
}

template <int F>
__device__ __forceinline__ void tb_flow(const VpConst &c, const TbIo &io, float zc, float dc, float zw, float dw,
                                        float ze, float de, float zs, float ds, float zn, float dn, float &fl,
                                        float &fr, float &ft, float &fb)
{
  if (!(F & TB_GEN))
    flow_cell<(F & TB_DIFF) != 0, true>(c, zc, dc, zw, dw, ze, de, zs, ds, zn, dn, fl, fr, ft, fb);
  else if (io.diffusion)
  {
    if (io.pl_one) flow_cell<true, true>(c, zc, dc, zw, dw, ze, de, zs, ds, zn, dn, fl, fr, ft, fb);
    else flow_cell<true, false>(c, zc, dc, zw, dw, ze, de, zs, ds, zn, dn, fl, fr, ft, fb);
  }
  else
  {
    if (io.pl_one) flow_cell<false, true>(c, zc, dc, zw, dw, ze, de, zs, ds, zn, dn, fl, fr, ft, fb);
    else flow_cell<false, false>(c, zc, dc, zw, dw, ze, de, zs, ds, zn, dn, fl, fr, ft, fb);
  }
}

template <int F>
__device__ __forceinline__ void tb_water(const VpConst &c, const TbIo &io, float d1, float fl, float fr, float ft,
                                         float fb, float frw, float fle, float ftn, float fbs, float &d2, float &u,
                                         float &v)
{
  if (!(F & TB_GEN) || io.pl_one) water_cell<true>(c, d1, fl, fr, ft, fb, frw, fle, ftn, fbs, d2, u, v);
  else water_cell<false>(c, d1, fl, fr, ft, fb, frw, fle, ftn, fbs, d2, u, v);
}

template <int F>
__device__ __forceinline__ void tb_erosion(const VpConst &c, const TbIo &io, float zc, float sc, float zw, float ze,
                                           float zn, float zs, float sw, float se, float sn, float ss, float d2,
                                           float u, float v, float &zo, float &so)
{
  if (!(F & TB_GEN) || io.kexp_one) erosion_cell<true>(c, zc, sc, zw, ze, zn, zs, sw, se, sn, ss, d2, u, v, zo, so);
  else erosion_cell<false>(c, zc, sc, zw, ze, zn, zs, sw, se, sn, ss, d2, u, v, zo, so);
}

/* s1_prev advected to grid cell (gx, gy) with that cell's velocity, as
 * k_vp_advect evaluates it */
__device__ __forceinline__ float tb_advect(const VpConst &c, const float *__restrict__ s1, float uu, float vv, int gx,
                                           int gy)
{
  const float  x = fsub((float)gx, fmul(c.dt, uu));
  const float  y = fsub((float)gy, fmul(c.dt, vv));
  const Tap    t = linear_tap(x, y, c.nx, c.ny);
  const size_t r0 = (size_t)t.j0 * c.nx, r1 = (size_t)t.j1 * c.nx;
  return blend(t, __ldg(s1 + r0 + t.i0), __ldg(s1 + r0 + t.i1), __ldg(s1 + r1 + t.i0), __ldg(s1 + r1 + t.i1));
}

/* ---- step t's eroded sediment at one cell, from global memory -------- */

__device__ __forceinline__ size_t tb_k(const VpConst &c, int i, int j)
{
  return (size_t)clampi(j, 0, c.ny - 1) * c.nx + clampi(i, 0, c.nx - 1);
}

/* new fluxes of step t at grid cell (i, j) */
template <int F>
__device__ __forceinline__ void tb_flux_g(const TbIo &io, const VpConst &c, int i, int j, float &fl, float &fr,
                                          float &ft, float &fb)
{
  const float *z = io.in.z, *d = io.in.d;
  auto         zz = [&](int a, int b) { return __ldg(z + tb_k(c, a, b)); };
  auto         dd = [&](int a, int b) {
    const size_t k = tb_k(c, a, b);
    return tb_d1(c, io.rain, __ldg(d + k), k);
  };
  const size_t k = (size_t)j * c.nx + i;
  fl = __ldg(io.in.fl + k);
  fr = __ldg(io.in.fr + k);
  ft = __ldg(io.in.ft + k);
  fb = __ldg(io.in.fb + k);
  tb_flow<F>(c, io, zz(i, j), dd(i, j), zz(i - 1, j), dd(i - 1, j), zz(i + 1, j), dd(i + 1, j), zz(i, j + 1),
          dd(i, j + 1), zz(i, j - 1), dd(i, j - 1), fl, fr, ft, fb);
}

/* step t's advected sediment at grid cell (i, j) */
__device__ __forceinline__ float tb_sed_g(const TbIo &io, const VpConst &c, int i, int j)
{
  const size_t k = (size_t)j * c.nx + i;
  return tb_advect(c, io.s1_prev, __ldg(io.u_prev + k), __ldg(io.v_prev + k), i, j);
}

/* step t's eroded sediment s1_t at grid cell (i, j): its flow and the
 * flows of its four neighbours, its water pass, the advected sediment of it
 * and its neighbours and its erosion pass, from step t's state */
template <int F>
__device__ __noinline__ float tb_s1_at(const TbIo io, const VpConst c, int i, int j)
{
  const int im = clampi(i - 1, 0, c.nx - 1), ip = clampi(i + 1, 0, c.nx - 1);
  const int jm = clampi(j - 1, 0, c.ny - 1), jp = clampi(j + 1, 0, c.ny - 1);
  float     fl, fr, ft, fb, t0, t1, t2, frw, fle, ftn, fbs;
  tb_flux_g<F>(io, c, i, j, fl, fr, ft, fb);
  tb_flux_g<F>(io, c, im, j, t0, frw, t1, t2);
  tb_flux_g<F>(io, c, ip, j, fle, t0, t1, t2);
  tb_flux_g<F>(io, c, i, jm, t0, t1, ftn, t2);
  tb_flux_g<F>(io, c, i, jp, t0, t1, t2, fbs);
  const size_t k = (size_t)j * c.nx + i;
  float        d2, u, v;
  tb_water<F>(c, io, tb_d1(c, io.rain, __ldg(io.in.d + k), k), fl, fr, ft, fb, frw, fle, ftn, fbs, d2, u, v);
  const float *z = io.in.z;
  float        zo, so;
  tb_erosion<F>(c, io, __ldg(z + k), tb_sed_g(io, c, i, j), __ldg(z + tb_k(c, i - 1, j)), __ldg(z + tb_k(c, i + 1, j)),
             __ldg(z + tb_k(c, i, j - 1)), __ldg(z + tb_k(c, i, j + 1)), tb_sed_g(io, c, im, j),
             tb_sed_g(io, c, ip, j), tb_sed_g(io, c, i, jm), tb_sed_g(io, c, i, jp), d2, u, v, zo, so);
  return so;
}

/* ---- the kernel ------------------------------------------------------ */

/* the cells of the tile's ring of width h that lie inside the grid, and
 * the rounded reciprocal of the row width */
struct TbRegion
{
  int   xa, ya, w, cnt;
  float rw;
};

template <int TX, int TY>
__device__ __forceinline__ TbRegion tb_region(int x0, int y0, int h, int nx, int ny)
{
  const int xa = max(0, x0 - h), xb = min(nx - 1, x0 + TX - 1 + h);
  const int ya = max(0, y0 - h), yb = min(ny - 1, y0 + TY - 1 + h);
  const int w = xb - xa + 1;
  return TbRegion{xa, ya, w, w * (yb - ya + 1), __fdiv_rn(1.f, (float)w)};
}

/* grid cell of item e of region r: row e / w as (e + 0.5) * RN(1/w)
 * truncated, exact for every w < 64 and e < 4096 (checked exhaustively;
 * the regions have w <= 44 and at most 1232 cells) */
__device__ __forceinline__ void tb_cell(const TbRegion &r, int e, int &gx, int &gy)
{
  const int q = (int)__fmul_rn(__fadd_rn((float)e, 0.5f), r.rw);
  gx = r.xa + (e - q * r.w);
  gy = r.ya + q;
}

/* items of the first pass's advection loop whose loads are issued together */
constexpr int TB_AB = 2;

template <int F, int TX, int TY>
__global__ void __launch_bounds__(TB_NT, 4) k_vp_tb2(TbIo io, VpConst c)
{
  extern __shared__ __align__(16) float tb_sm[];
  using Sh = TbShape<TX, TY>;
  constexpr int N = Sh::N;
  float *const  Z = tb_sm + TB_Z * N, *const D = tb_sm + TB_D * N;
  float *const  FL = tb_sm + TB_FL * N, *const FR = tb_sm + TB_FR * N;
  float *const  FT = tb_sm + TB_FT * N, *const FB = tb_sm + TB_FB * N;
  float *const  S = tb_sm + TB_S * N, *const ZN = tb_sm + TB_ZN * N;
  float *const  S1N = tb_sm + TB_S1N * N, *const UN = tb_sm + TB_UN * N, *const VN = tb_sm + TB_VN * N;
  const int    nx = c.nx, ny = c.ny, tid = threadIdx.x;
  const int    x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const int    ox = x0 - TB_H2, oy = y0 - TB_H2;
  /* shared-memory index of grid cell (gx, gy) of the h <= 6 region */
  auto at = [&](int gx, int gy) { return (gy - oy) * Sh::W + (gx - ox); };
  /* indices of a cell and its clamped neighbours */
  struct Nb
  {
    int c, w, e, n, s;
  };
  auto nb = [&](int gx, int gy) {
    return Nb{at(gx, gy), at(max(gx - 1, 0), gy), at(min(gx + 1, nx - 1), gy), at(gx, max(gy - 1, 0)),
              at(gx, min(gy + 1, ny - 1))};
  };

  /* A: step t's z and start depth (h 6), old fluxes and advected sediment
   * (h 5); the advection takes TB_AB items at a time so that their
   * velocity loads, then their tap gathers, are in flight together */
  {
    const TbRegion r = tb_region<TX, TY>(x0, y0, TB_H2, nx, ny);
#pragma unroll 4
    for (int e = tid; e < r.cnt; e += TB_NT)
    {
      int gx, gy;
      tb_cell(r, e, gx, gy);
      const size_t k = (size_t)gy * nx + gx;
      const int    i = at(gx, gy);
      Z[i] = __ldg(io.in.z + k);
      D[i] = tb_d1(c, io.rain, __ldg(io.in.d + k), k);
    }
    const TbRegion r1 = tb_region<TX, TY>(x0, y0, TB_H1, nx, ny);
    for (int e0 = tid; e0 < r1.cnt; e0 += TB_AB * TB_NT)
    {
      int   gx[TB_AB], gy[TB_AB];
      float uu[TB_AB], vv[TB_AB];
#pragma unroll
      for (int q = 0; q < TB_AB; q++)
      {
        /* an item past the region repeats the last cell and is not stored */
        tb_cell(r1, min(e0 + q * TB_NT, r1.cnt - 1), gx[q], gy[q]);
        const size_t k = (size_t)gy[q] * nx + gx[q];
        uu[q] = __ldg(io.u_prev + k);
        vv[q] = __ldg(io.v_prev + k);
      }
      Tap   t[TB_AB];
      float g[TB_AB][4];
#pragma unroll
      for (int q = 0; q < TB_AB; q++)
      {
        const float x = fsub((float)gx[q], fmul(c.dt, uu[q]));
        const float y = fsub((float)gy[q], fmul(c.dt, vv[q]));
        t[q] = linear_tap(x, y, nx, ny);
        const size_t k0 = (size_t)t[q].j0 * nx, k1 = (size_t)t[q].j1 * nx;
        g[q][0] = __ldg(io.s1_prev + k0 + t[q].i0);
        g[q][1] = __ldg(io.s1_prev + k0 + t[q].i1);
        g[q][2] = __ldg(io.s1_prev + k1 + t[q].i0);
        g[q][3] = __ldg(io.s1_prev + k1 + t[q].i1);
      }
#pragma unroll
      for (int q = 0; q < TB_AB; q++)
        if (e0 + q * TB_NT < r1.cnt)
        {
          const size_t k = (size_t)gy[q] * nx + gx[q];
          const int    i = at(gx[q], gy[q]);
          S[i] = blend(t[q], g[q][0], g[q][1], g[q][2], g[q][3]);
          FL[i] = __ldg(io.in.fl + k);
          FR[i] = __ldg(io.in.fr + k);
          FT[i] = __ldg(io.in.ft + k);
          FB[i] = __ldg(io.in.fb + k);
        }
    }
  }
  __syncthreads();

  /* B: step t's flow (h 5); a cell reads only its own old fluxes */
  {
    const TbRegion r = tb_region<TX, TY>(x0, y0, TB_H1, nx, ny);
    for (int e = tid; e < r.cnt; e += TB_NT)
    {
      int gx, gy;
      tb_cell(r, e, gx, gy);
      const Nb  p = nb(gx, gy);
      float     fl = FL[p.c], fr = FR[p.c], ft = FT[p.c], fb = FB[p.c];
      tb_flow<F>(c, io, Z[p.c], D[p.c], Z[p.w], D[p.w], Z[p.e], D[p.e], Z[p.s], D[p.s], Z[p.n], D[p.n], fl, fr, ft, fb);
      FL[p.c] = fl;
      FR[p.c] = fr;
      FT[p.c] = ft;
      FB[p.c] = fb;
    }
  }
  __syncthreads();

  /* C: step t's water and erosion (h 4); the depth slot of a cell takes its
   * evaporated depth (only the cell itself reads its start depth here) */
  {
    const TbRegion r = tb_region<TX, TY>(x0, y0, TB_HX, nx, ny);
    for (int e = tid; e < r.cnt; e += TB_NT)
    {
      int gx, gy;
      tb_cell(r, e, gx, gy);
      const Nb  p = nb(gx, gy);
      float     d2, u, v, zo, so;
      tb_water<F>(c, io, D[p.c], FL[p.c], FR[p.c], FT[p.c], FB[p.c], FR[p.w], FL[p.e], FT[p.n], FB[p.s], d2, u, v);
      tb_erosion<F>(c, io, Z[p.c], S[p.c], Z[p.w], Z[p.e], Z[p.n], Z[p.s], S[p.w], S[p.e], S[p.n], S[p.s], d2, u, v, zo,
                 so);
      ZN[p.c] = zo;
      S1N[p.c] = so;
      UN[p.c] = u;
      VN[p.c] = v;
      D[p.c] = fmul(d2, c.keep);
    }
  }
  __syncthreads();

  /* D: step t+1's start depth (h 2) and advected sediment (h 1) */
  {
    const TbRegion r = tb_region<TX, TY>(x0, y0, 2, nx, ny);
    for (int e = tid; e < r.cnt; e += TB_NT)
    {
      int gx, gy;
      tb_cell(r, e, gx, gy);
      const int i = at(gx, gy);
      D[i] = tb_d1(c, io.rain, D[i], (size_t)gy * nx + gx);
    }
    /* s1_t at grid cell (ti, tj): shared memory inside the h 4 region,
     * else recomputed from step t's state */
    const int xlo = x0 - TB_HX, xhi = x0 + TX - 1 + TB_HX, ylo = y0 - TB_HX, yhi = y0 + TY - 1 + TB_HX;
    auto      s1t = [&](int ti, int tj) {
      return (ti >= xlo && ti <= xhi && tj >= ylo && tj <= yhi) ? S1N[at(ti, tj)] : tb_s1_at<F>(io, c, ti, tj);
    };
    const TbRegion r1 = tb_region<TX, TY>(x0, y0, 1, nx, ny);
    for (int e = tid; e < r1.cnt; e += TB_NT)
    {
      int gx, gy;
      tb_cell(r1, e, gx, gy);
      const int   i = at(gx, gy);
      const float x = fsub((float)gx, fmul(c.dt, UN[i]));
      const float y = fsub((float)gy, fmul(c.dt, VN[i]));
      const Tap   t = linear_tap(x, y, nx, ny);
      const float g00 = s1t(t.i0, t.j0), g10 = s1t(t.i1, t.j0), g01 = s1t(t.i0, t.j1), g11 = s1t(t.i1, t.j1);
      S[i] = blend(t, g00, g10, g01, g11);
    }
  }
  __syncthreads();

  /* E: step t+1's flow (h 1) on z after step t and the new start depth */
  {
    const TbRegion r = tb_region<TX, TY>(x0, y0, 1, nx, ny);
    for (int e = tid; e < r.cnt; e += TB_NT)
    {
      int gx, gy;
      tb_cell(r, e, gx, gy);
      const Nb  p = nb(gx, gy);
      float     fl = FL[p.c], fr = FR[p.c], ft = FT[p.c], fb = FB[p.c];
      tb_flow<F>(c, io, ZN[p.c], D[p.c], ZN[p.w], D[p.w], ZN[p.e], D[p.e], ZN[p.s], D[p.s], ZN[p.n], D[p.n], fl, fr, ft,
              fb);
      FL[p.c] = fl;
      FR[p.c] = fr;
      FT[p.c] = ft;
      FB[p.c] = fb;
    }
  }
  __syncthreads();

  /* F: step t+1's water and erosion on the tile, written out */
  {
    const TbRegion r = tb_region<TX, TY>(x0, y0, 0, nx, ny);
    for (int e = tid; e < r.cnt; e += TB_NT)
    {
      int gx, gy;
      tb_cell(r, e, gx, gy);
      const Nb     p = nb(gx, gy);
      const size_t k = (size_t)gy * nx + gx;
      float        d2, u, v, zo, so;
      const float  fl = FL[p.c], fr = FR[p.c], ft = FT[p.c], fb = FB[p.c];
      tb_water<F>(c, io, D[p.c], fl, fr, ft, fb, FR[p.w], FL[p.e], FT[p.n], FB[p.s], d2, u, v);
      tb_erosion<F>(c, io, ZN[p.c], S[p.c], ZN[p.w], ZN[p.e], ZN[p.n], ZN[p.s], S[p.w], S[p.e], S[p.n], S[p.s], d2, u,
                 v, zo, so);
      io.out.z[k] = zo;
      io.out.d[k] = fmul(d2, c.keep);
      io.out.fl[k] = fl;
      io.out.fr[k] = fr;
      io.out.ft[k] = ft;
      io.out.fb[k] = fb;
      io.s1[k] = so;
      io.u[k] = u;
      io.v[k] = v;
      if (io.u_out) io.u_out[k] = u;
      if (io.v_out) io.v_out[k] = v;
    }
  }
}

/* Launch k_vp_tb2 for steps t, t+1 (t >= 1, no volume top-up) on stream s. */
template <int TX, int TY>
static int launch_tb2_shape(const TbIo &io, const VpConst &c, cudaStream_t s)
{
  constexpr int SMEM = (int)TbShape<TX, TY>::SMEM;
  static bool   attr_set[64] = {};
  int           dev = 0;
  HM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64 || !attr_set[dev])
  {
    HM_CUDA_TRY(cudaFuncSetAttribute(k_vp_tb2<0, TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
    HM_CUDA_TRY(cudaFuncSetAttribute(k_vp_tb2<TB_DIFF, TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
    HM_CUDA_TRY(cudaFuncSetAttribute(k_vp_tb2<TB_GEN, TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
    if (dev >= 0 && dev < 64) attr_set[dev] = true;
  }
  const dim3 grid((c.nx + TX - 1) / TX, (c.ny + TY - 1) / TY);
  if (!io.pl_one || !io.kexp_one) k_vp_tb2<TB_GEN, TX, TY><<<grid, TB_NT, SMEM, s>>>(io, c);
  else if (io.diffusion) k_vp_tb2<TB_DIFF, TX, TY><<<grid, TB_NT, SMEM, s>>>(io, c);
  else k_vp_tb2<0, TX, TY><<<grid, TB_NT, SMEM, s>>>(io, c);
  HM_LAUNCH_CHECK("k_vp_tb2");
  return HM_OK;
}

/* Launch k_vp_tb2 for steps t, t+1 (t >= 1, no volume top-up) on stream s:
 * 16 x 8 tiles on grids with fewer than two 32 x 16 tiles per SM. */
int launch_vp_tb2(const TbIo &io, const VpConst &c, cudaStream_t s)
{
  static int sms[64] = {};
  int        dev = 0;
  HM_CUDA_TRY(cudaGetDevice(&dev));
  int n_sm = dev >= 0 && dev < 64 ? sms[dev] : 0;
  if (n_sm == 0)
  {
    HM_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
    if (dev >= 0 && dev < 64) sms[dev] = n_sm;
  }
  const long long big_tiles = (long long)((c.nx + 31) / 32) * ((c.ny + 15) / 16);
  if (big_tiles < 2LL * n_sm) return launch_tb2_shape<16, 8>(io, c, s);
  return launch_tb2_shape<32, 16>(io, c, s);
}

} // namespace hm
