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
 *
 * HBM traffic per cell and step: 7 fields read and 9 written by k_vp_fwe,
 * 3 read (plus the gather, mostly L2) and 1 written by k_vp_advect: 80 B.
 * Every read of the step comes from the old state copy or from this
 * step's s1 / u / v, never from a grid this step writes, so tiles need no
 * ordering between them.
 */
#ifndef HM_VPIPES_TILED_CUH
#define HM_VPIPES_TILED_CUH

#include "hm_reduce.cuh"
#include "hm_vpipes_fused.cuh"
#include "hm_vpipes_math.cuh"

namespace hm
{

constexpr int FT_TX = 32, FT_TY = 16;          /* output tile                 */
constexpr int FT_NT = 256;                     /* threads per CTA             */
constexpr int FT_W2 = FT_TX + 4, FT_H2 = FT_TY + 4; /* z, depth region (halo 2) */
constexpr int FT_W1 = FT_TX + 2, FT_H1 = FT_TY + 2; /* s, fluxes region (halo 1) */

struct FweSmem
{
  float z[FT_H2][FT_W2];
  float d[FT_H2][FT_W2];
  float s[FT_H1][FT_W1];
  float fo[4][FT_H1][FT_W1];
  float fn[4][FT_H1][FT_W1];
};

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
};

template <bool MAINTAIN>
__device__ __forceinline__ void fwe_tile(const FweIo &io, const VpConst &c, VpScalars *sc, double *partials,
                                         int bx, int by, int nbx, int nby, FweSmem &sm)
{
  static_assert(FT_TX == 32, "a lane is a column of the tile");
  const int   tid = threadIdx.x;
  const int   nx = c.nx, ny = c.ny;
  const int   x0 = bx * FT_TX, y0 = by * FT_TY;
  const float add = MAINTAIN ? sc->add[io.parity] : 0.f;
  const float rvol = MAINTAIN ? sc->rvol : 1.f;
  const bool  rain_step = c.rps != 0.f;

  /* stage: z, d on the halo-2 region; s and old fluxes on the halo-1 region */
  for (int e = tid; e < FT_W2 * FT_H2; e += FT_NT)
  {
    const int    ly = e / FT_W2, lx = e - ly * FT_W2;
    const size_t k = (size_t)clampi(y0 - 2 + ly, 0, ny - 1) * nx + clampi(x0 - 2 + lx, 0, nx - 1);
    cp_async4(&sm.z[ly][lx], io.in.z + k);
    cp_async4(&sm.d[ly][lx], io.in.d + k);
  }
  for (int e = tid; e < FT_W1 * FT_H1; e += FT_NT)
  {
    const int    ly = e / FT_W1, lx = e - ly * FT_W1;
    const size_t k = (size_t)clampi(y0 - 1 + ly, 0, ny - 1) * nx + clampi(x0 - 1 + lx, 0, nx - 1);
    cp_async4(&sm.s[ly][lx], io.in.s + k);
    cp_async4(&sm.fo[0][ly][lx], io.in.fl + k);
    cp_async4(&sm.fo[1][ly][lx], io.in.fr + k);
    cp_async4(&sm.fo[2][ly][lx], io.in.ft + k);
    cp_async4(&sm.fo[3][ly][lx], io.in.fb + k);
  }
  cp_async_commit();
  cp_async_wait<0>();
  /* stored depth -> depth at the start of the step (own elements) */
  for (int e = tid; e < FT_W2 * FT_H2; e += FT_NT)
  {
    const int   ly = e / FT_W2, lx = e - ly * FT_W2;
    float      &d = sm.d[ly][lx];
    const float rn = io.rain ? __ldg(io.rain + (size_t)clampi(y0 - 2 + ly, 0, ny - 1) * nx +
                                    clampi(x0 - 2 + lx, 0, nx - 1))
                             : 1.f;
    d = rain_step ? depth_d1<MAINTAIN, true>(d, rn, add, rvol, c.rps)
                  : depth_d1<MAINTAIN, false>(d, rn, add, rvol, c.rps);
  }
  __syncthreads();

  /* flow pass on the tile and a 1-cell ring (region-1 coordinates) */
  for (int e = tid; e < FT_W1 * FT_H1; e += FT_NT)
  {
    const int ly = e / FT_W1, lx = e - ly * FT_W1;
    const int qy = ly + 1, qx = lx + 1; /* region-2 coordinates of the cell */
    float     fl = sm.fo[0][ly][lx], fr = sm.fo[1][ly][lx], ft = sm.fo[2][ly][lx], fb = sm.fo[3][ly][lx];
    const float zc = sm.z[qy][qx], dc = sm.d[qy][qx];
    const float zw = sm.z[qy][qx - 1], dw = sm.d[qy][qx - 1], ze = sm.z[qy][qx + 1], de = sm.d[qy][qx + 1];
    const float zs = sm.z[qy + 1][qx], ds = sm.d[qy + 1][qx], zn = sm.z[qy - 1][qx], dn = sm.d[qy - 1][qx];
    if (io.diffusion)
    {
      if (io.pl_one) flow_cell<true, true>(c, zc, dc, zw, dw, ze, de, zs, ds, zn, dn, fl, fr, ft, fb);
      else flow_cell<true, false>(c, zc, dc, zw, dw, ze, de, zs, ds, zn, dn, fl, fr, ft, fb);
    }
    else
    {
      if (io.pl_one) flow_cell<false, true>(c, zc, dc, zw, dw, ze, de, zs, ds, zn, dn, fl, fr, ft, fb);
      else flow_cell<false, false>(c, zc, dc, zw, dw, ze, de, zs, ds, zn, dn, fl, fr, ft, fb);
    }
    sm.fn[0][ly][lx] = fl;
    sm.fn[1][ly][lx] = fr;
    sm.fn[2][ly][lx] = ft;
    sm.fn[3][ly][lx] = fb;
    const int gx = x0 - 1 + lx, gy = y0 - 1 + ly;
    if (lx >= 1 && lx <= FT_TX && ly >= 1 && ly <= FT_TY && gx < nx && gy < ny)
    {
      const size_t k = (size_t)gy * nx + gx;
      io.out.fl[k] = fl;
      io.out.fr[k] = fr;
      io.out.ft[k] = ft;
      io.out.fb[k] = fb;
    }
  }
  __syncthreads();

  /* water and erosion on the tile: warp w takes rows w, w + 4, ...; a lane
   * is a column */
  double    part = 0.0;
  const int lane = tid & 31, w = tid >> 5;
  const int gx = x0 + lane;
  /* region-1 columns of the clamped x neighbours (new fluxes are derived:
   * outside the grid they are the edge cell's own values) */
  const int lxc = lane + 1;
  const int lxw = clampi(gx - 1, 0, nx - 1) - (x0 - 1);
  const int lxe = clampi(gx + 1, 0, nx - 1) - (x0 - 1);
  for (int ty = w; ty < FT_TY; ty += FT_NT / 32)
  {
    const int gy = y0 + ty;
    if (gx >= nx || gy >= ny) continue;
    const int ly = ty + 1;
    const int lyn = clampi(gy - 1, 0, ny - 1) - (y0 - 1);
    const int lys = clampi(gy + 1, 0, ny - 1) - (y0 - 1);
    const int qy = ty + 2, qx = lane + 2; /* region-2 coordinates */
    float     d2, u, v;
    const float d1c = sm.d[qy][qx];
    if (io.pl_one)
      water_cell<true>(c, d1c, sm.fn[0][ly][lxc], sm.fn[1][ly][lxc], sm.fn[2][ly][lxc], sm.fn[3][ly][lxc],
                       sm.fn[1][ly][lxw], sm.fn[0][ly][lxe], sm.fn[2][lyn][lxc], sm.fn[3][lys][lxc], d2, u, v);
    else
      water_cell<false>(c, d1c, sm.fn[0][ly][lxc], sm.fn[1][ly][lxc], sm.fn[2][ly][lxc], sm.fn[3][ly][lxc],
                        sm.fn[1][ly][lxw], sm.fn[0][ly][lxe], sm.fn[2][lyn][lxc], sm.fn[3][lys][lxc], d2, u, v);
    float zo, so;
    if (io.kexp_one)
      erosion_cell<true>(c, sm.z[qy][qx], sm.s[ly][lxc], sm.z[qy][qx - 1], sm.z[qy][qx + 1], sm.z[qy - 1][qx],
                         sm.z[qy + 1][qx], sm.s[ly][lxc - 1], sm.s[ly][lxc + 1], sm.s[ly - 1][lxc],
                         sm.s[ly + 1][lxc], d2, u, v, zo, so);
    else
      erosion_cell<false>(c, sm.z[qy][qx], sm.s[ly][lxc], sm.z[qy][qx - 1], sm.z[qy][qx + 1], sm.z[qy - 1][qx],
                          sm.z[qy + 1][qx], sm.s[ly][lxc - 1], sm.s[ly][lxc + 1], sm.s[ly - 1][lxc],
                          sm.s[ly + 1][lxc], d2, u, v, zo, so);
    const size_t k = (size_t)gy * nx + gx;
    const float  de = fmul(d2, c.keep);
    io.out.z[k] = zo;
    io.out.d[k] = de;
    io.s1[k] = so;
    io.u[k] = u;
    io.v[k] = v;
    if (io.u_out)
    {
      io.u_out[k] = u;
      io.v_out[k] = v;
    }
    part += (double)de;
  }

  if (MAINTAIN)
  {
    const float v0 = sc->v0;
    float      *outp = &sc->add[io.parity ^ 1];
    grid_sum_commit<FT_NT>(part, partials, &sc->ticket, (unsigned)(nbx * nby), (unsigned)(by * nbx + bx),
                           [&](double total) { *outp = fsub(v0, (float)total); });
  }
}

template <bool MAINTAIN>
__global__ void __launch_bounds__(FT_NT) k_vp_fwe(FweIo io, VpConst c, VpScalars *sc, double *partials)
{
  __shared__ FweSmem sm;
  fwe_tile<MAINTAIN>(io, c, sc, partials, blockIdx.x, blockIdx.y, gridDim.x, gridDim.y, sm);
}

/* advection of one cell: s_new = bilinear(s1, (i - dt u, j - dt v)) */
__device__ __forceinline__ float advect_cell(const float *__restrict__ s1, int i, int j, float u, float v,
                                             const VpConst &c)
{
  const float  x = fsub((float)i, fmul(c.dt, u));
  const float  y = fsub((float)j, fmul(c.dt, v));
  const Tap    t = linear_tap(x, y, c.nx, c.ny);
  const size_t r0 = (size_t)t.j0 * c.nx, r1 = (size_t)t.j1 * c.nx;
  return blend(t, __ldg(s1 + r0 + t.i0), __ldg(s1 + r0 + t.i1), __ldg(s1 + r1 + t.i0), __ldg(s1 + r1 + t.i1));
}

/* block x covers 256 columns of the rows blockIdx.y, blockIdx.y + gridDim.y, ... */
__global__ void __launch_bounds__(256) k_vp_advect(const float *__restrict__ s1,
                                                    const float *__restrict__ u,
                                                    const float *__restrict__ v,
                                                    float *__restrict__ s_out,
                                                    VpConst c)
{
  const int i = blockIdx.x * 256 + threadIdx.x;
  if (i >= c.nx) return;
  for (int j = blockIdx.y; j < c.ny; j += gridDim.y)
  {
    const size_t k = (size_t)j * c.nx + i;
    s_out[k] = advect_cell(s1, i, j, __ldg(u + k), __ldg(v + k), c);
  }
}

} // namespace hm

#endif
