/*
 * hm_vpipes_fused.cuh - one virtual-pipes step per launch.
 *
 * The four passes of HighMap/src/gpu_opencl/kernels/hydraulic_vpipes.cl
 * (flow :5-69, water :71-116, erosion :118-184, advection :186-211) and the
 * evaporation / volume-sum host step (hydraulic_vpipes_gpu.cpp:163-169)
 * fused into a single streaming kernel:
 *
 *   * a CTA owns a strip of W = TPB - 2 * XH output columns (one thread per
 *     column of the strip plus XH = R + 2 halo columns each side) and a
 *     chunk of H output rows, and streams down the rows;
 *   * iteration r loads row r of the old state (z, d, s, fl, fr, ft, fb)
 *     into shared-memory row rings with cp.async, turns row r-1's depth
 *     into the step's start depth d1, runs the flow pass on row r-3, the
 *     water + erosion passes on row r-5 and the advection pass on row
 *     r-6-R, then meets one __syncthreads: every stage reads rows finished
 *     in earlier iterations only;
 *   * the advection samples the eroded sediment s1 from the ring when the
 *     bilinear footprint lies within R columns and rows of the cell; a
 *     footprint outside it (fast water) is recomputed exactly from the old
 *     state in global memory (`s1_at`), which no CTA writes during the
 *     launch: every field is ping-ponged between launches.
 *
 * Reads are clamped to the grid as the reference's CLK_ADDRESS_CLAMP_TO_EDGE
 * sampler clamps coordinates (a neighbour outside the grid is the edge
 * cell's own value of the same quantity).
 *
 * HBM traffic per cell and step: the 7 state fields read once and written
 * once (56 B); halo columns and the pipeline's warm-up rows are re-read by
 * neighbouring CTAs through L2.
 */
#ifndef HM_VPIPES_FUSED_CUH
#define HM_VPIPES_FUSED_CUH

#include "hm_reduce.cuh"
#include "hm_vpipes_math.cuh"

namespace hm
{

/* one copy of the solver state (SoA grids) */
struct VpFields
{
  float *z, *d, *s, *fl, *fr, *ft, *fb;
};

struct VpState
{
  const float *z, *d, *s, *fl, *fr, *ft, *fb;
};

struct VpStateOut
{
  float *z, *d, *s, *fl, *fr, *ft, *fb;
  float *u, *v; /* written only when non-null (last step) */
};

struct VpScalars
{
  float    v0;     /* initial water volume (fp32 of the fp64 sum)         */
  float    rvol;   /* rain map volume                                     */
  float    add[2]; /* V0 - sum(d) of the previous step, ping-pong         */
  unsigned ticket;
  unsigned slow;   /* advection samples taken by the global slow path      */
  unsigned defer_count[2]; /* deferred cells of the step, one per parity   */
  unsigned error;  /* bit 0: a tile's TMA loads timed out (tile skipped)   */
};

struct VpStep
{
  VpState      in;
  VpStateOut   out;
  const float *rain; /* nullable */
  int          parity;  /* step parity: which top-up slot is read         */
  int          dparity; /* deferred-list slot this step appends to         */
  int          H;    /* output rows per CTA */
  int          maintain, diffusion, pl_one, kexp_one;
};

__device__ __forceinline__ void cp_async4(float *smem, const float *gmem)
{
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* ---- exact recomputation from the old state (slow path) -------------- */

struct Glob
{
  VpStep  st;
  VpConst c;
  float   add, rvol;
  __device__ float at(const float *f, int i, int j) const
  {
    return __ldg(f + (size_t)clampi(j, 0, c.ny - 1) * c.nx + clampi(i, 0, c.nx - 1));
  }
  __device__ float d1(int i, int j) const
  {
    i = clampi(i, 0, c.nx - 1);
    j = clampi(j, 0, c.ny - 1);
    size_t k = (size_t)j * c.nx + i;
    float  r = st.rain ? __ldg(st.rain + k) : 1.f;
    float  d = __ldg(st.in.d + k);
    float  dc = st.maintain ? fadd(d, fdiv(fmul(add, r), rvol)) : d;
    return c.rps != 0.f ? fadd(dc, fmul(c.rps, r)) : dc;
  }
  /* new fluxes of cell (i, j), i and j inside the grid */
  __device__ void flux(int i, int j, float &fl, float &fr, float &ft, float &fb) const
  {
    const float *z = st.in.z;
    size_t       k = (size_t)j * c.nx + i;
    fl = __ldg(st.in.fl + k);
    fr = __ldg(st.in.fr + k);
    ft = __ldg(st.in.ft + k);
    fb = __ldg(st.in.fb + k);
    if (st.diffusion)
    {
      if (st.pl_one)
        flow_cell<true, true>(c, at(z, i, j), d1(i, j), at(z, i - 1, j), d1(i - 1, j), at(z, i + 1, j), d1(i + 1, j),
                              at(z, i, j + 1), d1(i, j + 1), at(z, i, j - 1), d1(i, j - 1), fl, fr, ft, fb);
      else
        flow_cell<true, false>(c, at(z, i, j), d1(i, j), at(z, i - 1, j), d1(i - 1, j), at(z, i + 1, j), d1(i + 1, j),
                               at(z, i, j + 1), d1(i, j + 1), at(z, i, j - 1), d1(i, j - 1), fl, fr, ft, fb);
    }
    else
    {
      if (st.pl_one)
        flow_cell<false, true>(c, at(z, i, j), d1(i, j), at(z, i - 1, j), d1(i - 1, j), at(z, i + 1, j), d1(i + 1, j),
                               at(z, i, j + 1), d1(i, j + 1), at(z, i, j - 1), d1(i, j - 1), fl, fr, ft, fb);
      else
        flow_cell<false, false>(c, at(z, i, j), d1(i, j), at(z, i - 1, j), d1(i - 1, j), at(z, i + 1, j),
                                d1(i + 1, j), at(z, i, j + 1), d1(i, j + 1), at(z, i, j - 1), d1(i, j - 1), fl, fr, ft,
                                fb);
    }
  }
  /* eroded sediment s1 of cell (i, j), i and j inside the grid */
  __device__ __noinline__ float s1_at(int i, int j) const
  {
    float fl, fr, ft, fb, t0, t1, t2, t3;
    flux(i, j, fl, fr, ft, fb);
    float frw, fle, ftn, fbs;
    flux(clampi(i - 1, 0, c.nx - 1), j, t0, frw, t1, t2);
    flux(clampi(i + 1, 0, c.nx - 1), j, fle, t0, t1, t2);
    flux(i, clampi(j - 1, 0, c.ny - 1), t0, t1, ftn, t2);
    flux(i, clampi(j + 1, 0, c.ny - 1), t0, t1, t2, fbs);
    (void)t3;
    float d2, u, v;
    if (st.pl_one) water_cell<true>(c, d1(i, j), fl, fr, ft, fb, frw, fle, ftn, fbs, d2, u, v);
    else water_cell<false>(c, d1(i, j), fl, fr, ft, fb, frw, fle, ftn, fbs, d2, u, v);
    const float *z = st.in.z, *s = st.in.s;
    float        zo, so;
    if (st.kexp_one)
      erosion_cell<true>(c, at(z, i, j), at(s, i, j), at(z, i - 1, j), at(z, i + 1, j), at(z, i, j - 1),
                         at(z, i, j + 1), at(s, i - 1, j), at(s, i + 1, j), at(s, i, j - 1), at(s, i, j + 1), d2, u, v,
                         zo, so);
    else
      erosion_cell<false>(c, at(z, i, j), at(s, i, j), at(z, i - 1, j), at(z, i + 1, j), at(z, i, j - 1),
                          at(z, i, j + 1), at(s, i - 1, j), at(s, i + 1, j), at(s, i, j - 1), at(s, i, j + 1), d2, u,
                          v, zo, so);
    return so;
  }
};

/* ---- the fused step kernel ------------------------------------------- */

template <int TPB, int R>
struct FusedLayout
{
  static constexpr int XH = R + 2;          /* halo columns each side        */
  static constexpr int W = TPB - 2 * XH;    /* output columns per CTA        */
  static constexpr int DZ = 8;              /* rings of z, d (-> d1), s      */
  static constexpr int DF = 4;              /* rings of old and new fluxes   */
  static constexpr int DS1 = (2 * R + 2 <= 8) ? 8 : 16;
  static constexpr int DUV = (R + 2 <= 4) ? 4 : 8;
  static constexpr int ROWS = 3 * DZ + 8 * DF + DS1 + 2 * DUV;
  static constexpr size_t SMEM = (size_t)ROWS * TPB * sizeof(float);
  static_assert(W > 0, "strip too narrow for the halo");
};

/* A cell whose advection footprint leaves the staged window: its index and
 * velocity, resolved after the step by k_vp_fixup. */
struct Deferred
{
  unsigned job; /* index into the batch's job table (0 for a single solve) */
  unsigned k;
  float    u, v;
};

struct VpDefer
{
  Deferred *list;
  unsigned *count; /* [2], one per step parity */
  unsigned  cap;
};

/* s_new of one cell from the old state in global memory */
__device__ __forceinline__ float advect_global(const Glob &g, int gi, int gj, float u, float v)
{
  const float x = fsub((float)gi, fmul(g.c.dt, u));
  const float y = fsub((float)gj, fmul(g.c.dt, v));
  const Tap   t = linear_tap(x, y, g.c.nx, g.c.ny);
  return blend(t, g.s1_at(t.i0, t.j0), g.s1_at(t.i1, t.j0), g.s1_at(t.i0, t.j1), g.s1_at(t.i1, t.j1));
}

/* One tile (strip bx, chunk by of an nbx x nby decomposition) of one step;
 * the body of k_vp_fused and of the batched round kernel.  `smem` holds
 * FusedLayout<TPB, R>::SMEM bytes.  Every thread of the CTA calls it. */
template <int TPB, int R, bool MAINTAIN>
__device__ __forceinline__ void vp_tile(const VpStep &st,
                                        const VpConst &c,
                                        VpScalars *sc,
                                        double *partials,
                                        const VpDefer &df,
                                        unsigned job,
                                        int bx,
                                        int by,
                                        int nbx,
                                        int nby,
                                        float *smem)
{
  using L = FusedLayout<TPB, R>;
  float(*sZ)[TPB] = (float(*)[TPB])smem;
  float(*sD)[TPB] = sZ + L::DZ;
  float(*sS)[TPB] = sD + L::DZ;
  float(*sFo)[TPB] = sS + L::DZ;      /* [4 * DF]: field k, row slot q at k * DF + q */
  float(*sFn)[TPB] = sFo + 4 * L::DF; /* same                                       */
  float(*sS1)[TPB] = sFn + 4 * L::DF;
  float(*sU)[TPB] = sS1 + L::DS1;
  float(*sV)[TPB] = sU + L::DUV;

  const int  tid = threadIdx.x;
  const int  nx = c.nx, ny = c.ny;
  const int  x0 = bx * L::W;                  /* first output column         */
  const int  xs = x0 - L::XH;                 /* global column of thread 0    */
  const int  gi = xs + tid;                   /* this thread's column         */
  const bool in_grid = gi >= 0 && gi < nx;
  const int  y0 = by * st.H;                  /* first output row             */
  const int  y1 = min(ny, y0 + st.H);         /* one past the last output row  */
  const bool out_col = tid >= L::XH && tid < L::XH + L::W && gi < nx;

  const float add = MAINTAIN ? sc->add[st.parity] : 0.f;
  const float rvol = MAINTAIN ? sc->rvol : 1.f;
  const bool  rain_step = c.rps != 0.f;

  /* Local columns of the clamped neighbours, themselves clamped into the
   * strip: for every column whose results are used they equal the
   * reference's clamp-to-edge neighbour; elsewhere they only keep the
   * shared-memory reads in bounds. */
  auto loc = [&](int g) { return clampi(clampi(g, 0, nx - 1) - xs, 0, TPB - 1); };
  const int lw = loc(gi - 1), le = loc(gi + 1);
  const int gic = clampi(gi, 0, nx - 1);

  /* rows each stage has to cover for this chunk */
  const int load_lo = max(0, y0 - R - 2), load_hi = min(ny - 1, y1 + R + 1);
  const int f_lo = max(0, y0 - R - 1), f_hi = min(ny - 1, y1 + R);
  const int e_lo = max(0, y0 - R), e_hi = min(ny - 1, y1 - 1 + R);
  const int clo = max(x0 - R, 0), chi = min(x0 + L::W + R, nx) - 1;

  double part = 0.0;

  for (int r = y0 - R - 2; r <= y1 + R + 5; ++r)
  {
    /* L: row r of the old state into the rings (own column) */
    if (r >= load_lo && r <= load_hi && in_grid)
    {
      const size_t k = (size_t)r * nx + gi;
      const int    q = r & (L::DZ - 1), qf = r & (L::DF - 1);
      cp_async4(&sZ[q][tid], st.in.z + k);
      cp_async4(&sD[q][tid], st.in.d + k);
      cp_async4(&sS[q][tid], st.in.s + k);
      cp_async4(&sFo[0 * L::DF + qf][tid], st.in.fl + k);
      cp_async4(&sFo[1 * L::DF + qf][tid], st.in.fr + k);
      cp_async4(&sFo[2 * L::DF + qf][tid], st.in.ft + k);
      cp_async4(&sFo[3 * L::DF + qf][tid], st.in.fb + k);
    }
    cp_async_commit();
    cp_async_wait<1>();

    /* row r-1: stored depth -> depth at the start of the step.  The row
     * ranges of this and the following stages are the same for the whole
     * CTA, so their tests never split a warp. */
    if (r - 1 >= load_lo && r - 1 <= load_hi)
    {
      const int   j = r - 1;
      float      &d = sD[j & (L::DZ - 1)][tid];
      const float rn = st.rain ? __ldg(st.rain + (size_t)clampi(j, 0, ny - 1) * nx + gic) : 1.f;
      d = rain_step ? depth_d1<MAINTAIN, true>(d, rn, add, rvol, c.rps)
                    : depth_d1<MAINTAIN, false>(d, rn, add, rvol, c.rps);
    }

    /* F: flow pass on row r-3 */
    if (r - 3 >= f_lo && r - 3 <= f_hi)
    {
      const int j = r - 3;
      const int q = j & (L::DZ - 1), qn = max(j - 1, 0) & (L::DZ - 1), qs = min(j + 1, ny - 1) & (L::DZ - 1);
      const int qf = j & (L::DF - 1);
      float     fl = sFo[0 * L::DF + qf][tid], fr = sFo[1 * L::DF + qf][tid];
      float     ft = sFo[2 * L::DF + qf][tid], fb = sFo[3 * L::DF + qf][tid];
      const float zc = sZ[q][tid], d1c = sD[q][tid];
      if (st.diffusion)
      {
        if (st.pl_one)
          flow_cell<true, true>(c, zc, d1c, sZ[q][lw], sD[q][lw], sZ[q][le], sD[q][le], sZ[qs][tid], sD[qs][tid],
                                sZ[qn][tid], sD[qn][tid], fl, fr, ft, fb);
        else
          flow_cell<true, false>(c, zc, d1c, sZ[q][lw], sD[q][lw], sZ[q][le], sD[q][le], sZ[qs][tid], sD[qs][tid],
                                 sZ[qn][tid], sD[qn][tid], fl, fr, ft, fb);
      }
      else
      {
        if (st.pl_one)
          flow_cell<false, true>(c, zc, d1c, sZ[q][lw], sD[q][lw], sZ[q][le], sD[q][le], sZ[qs][tid], sD[qs][tid],
                                 sZ[qn][tid], sD[qn][tid], fl, fr, ft, fb);
        else
          flow_cell<false, false>(c, zc, d1c, sZ[q][lw], sD[q][lw], sZ[q][le], sD[q][le], sZ[qs][tid], sD[qs][tid],
                                  sZ[qn][tid], sD[qn][tid], fl, fr, ft, fb);
      }
      sFn[0 * L::DF + qf][tid] = fl;
      sFn[1 * L::DF + qf][tid] = fr;
      sFn[2 * L::DF + qf][tid] = ft;
      sFn[3 * L::DF + qf][tid] = fb;
      if (out_col && j >= y0 && j < y1)
      {
        const size_t k = (size_t)j * nx + gi;
        st.out.fl[k] = fl;
        st.out.fr[k] = fr;
        st.out.ft[k] = ft;
        st.out.fb[k] = fb;
      }
    }

    /* E: water + erosion passes on row r-5 */
    if (r - 5 >= e_lo && r - 5 <= e_hi)
    {
      const int j = r - 5;
      const int q = j & (L::DZ - 1), qn = max(j - 1, 0) & (L::DZ - 1), qs = min(j + 1, ny - 1) & (L::DZ - 1);
      const int qf = j & (L::DF - 1), qfn = max(j - 1, 0) & (L::DF - 1), qfs = min(j + 1, ny - 1) & (L::DF - 1);
      float     d2, u, v;
      const float d1c = sD[q][tid];
      if (st.pl_one)
        water_cell<true>(c, d1c, sFn[0 * L::DF + qf][tid], sFn[1 * L::DF + qf][tid], sFn[2 * L::DF + qf][tid],
                         sFn[3 * L::DF + qf][tid], sFn[1 * L::DF + qf][lw], sFn[0 * L::DF + qf][le],
                         sFn[2 * L::DF + qfn][tid], sFn[3 * L::DF + qfs][tid], d2, u, v);
      else
        water_cell<false>(c, d1c, sFn[0 * L::DF + qf][tid], sFn[1 * L::DF + qf][tid], sFn[2 * L::DF + qf][tid],
                          sFn[3 * L::DF + qf][tid], sFn[1 * L::DF + qf][lw], sFn[0 * L::DF + qf][le],
                          sFn[2 * L::DF + qfn][tid], sFn[3 * L::DF + qfs][tid], d2, u, v);
      float zo, so;
      if (st.kexp_one)
        erosion_cell<true>(c, sZ[q][tid], sS[q][tid], sZ[q][lw], sZ[q][le], sZ[qn][tid], sZ[qs][tid], sS[q][lw],
                           sS[q][le], sS[qn][tid], sS[qs][tid], d2, u, v, zo, so);
      else
        erosion_cell<false>(c, sZ[q][tid], sS[q][tid], sZ[q][lw], sZ[q][le], sZ[qn][tid], sZ[qs][tid], sS[q][lw],
                            sS[q][le], sS[qn][tid], sS[qs][tid], d2, u, v, zo, so);
      sS1[j & (L::DS1 - 1)][tid] = so;
      sU[j & (L::DUV - 1)][tid] = u;
      sV[j & (L::DUV - 1)][tid] = v;
      if (out_col && j >= y0 && j < y1)
      {
        const size_t k = (size_t)j * nx + gi;
        const float  de = fmul(d2, c.keep);
        st.out.z[k] = zo;
        st.out.d[k] = de;
        if (st.out.u)
        {
          st.out.u[k] = u;
          st.out.v[k] = v;
        }
        part += (double)de;
      }
    }

    /* A: advection on row r-6-R */
    if (r - 6 - R >= y0 && r - 6 - R < y1)
    {
      const int   j = r - 6 - R;
      const bool  valid = out_col;
      const float u = sU[j & (L::DUV - 1)][tid], v = sV[j & (L::DUV - 1)][tid];
      const float x = fsub((float)gi, fmul(c.dt, u));
      const float y = fsub((float)j, fmul(c.dt, v));
      const Tap   t = linear_tap(x, y, nx, ny);
      const bool  inside = t.j0 >= max(j - R, e_lo) && t.j1 <= min(j + R, e_hi) && t.i0 >= clo && t.i1 <= chi;
      const int   a0 = t.j0 & (L::DS1 - 1), a1 = t.j1 & (L::DS1 - 1);
      const int   c0 = clampi(t.i0 - xs, 0, TPB - 1), c1 = clampi(t.i1 - xs, 0, TPB - 1);
      const float sn = blend(t, sS1[a0][c0], sS1[a0][c1], sS1[a1][c0], sS1[a1][c1]);
      if (valid)
      {
        const size_t k = (size_t)j * nx + gi;
        if (inside)
          st.out.s[k] = sn;
        else
        {
          const unsigned slot = atomicAdd(&df.count[st.dparity], 1u);
          if (slot < df.cap)
            df.list[slot] = Deferred{job, (unsigned)k, u, v};
          else
          {
            const Glob g{st, c, add, rvol};
            st.out.s[k] = advect_global(g, gi, j, u, v);
          }
          atomicAdd(&sc->slow, 1u);
        }
      }
    }
    __syncthreads();
  }
  cp_async_wait<0>();

  if (MAINTAIN)
  {
    const unsigned nb = (unsigned)(nbx * nby);
    const unsigned bid = (unsigned)(by * nbx + bx);
    const float    v0 = sc->v0;
    float         *outp = &sc->add[st.parity ^ 1];
    grid_sum_commit<TPB>(part, partials, &sc->ticket, nb, bid,
                         [&](double total) { *outp = fsub(v0, (float)total); });
  }
}

template <int TPB, int R, bool MAINTAIN>
__global__ void __launch_bounds__(TPB) k_vp_fused(VpStep st, VpConst c, VpScalars *sc, double *partials, VpDefer df)
{
  extern __shared__ float smem[];
  vp_tile<TPB, R, MAINTAIN>(st, c, sc, partials, df, 0u, blockIdx.x, blockIdx.y, gridDim.x, gridDim.y, smem);
}

/* Resolves the cells k_vp_fused deferred in the same step: their sediment
 * sample recomputed exactly from the old state (still intact: the step
 * wrote only the other copy).  Re-arms the other parity's counter for the
 * next step. */
template <int NT>
__global__ void __launch_bounds__(NT) k_vp_fixup(VpStep st, VpConst c, VpScalars *sc, VpDefer df)
{
  const float    add = st.maintain ? sc->add[st.parity] : 0.f;
  const float    rvol = st.maintain ? sc->rvol : 1.f;
  const unsigned n = min(df.count[st.dparity], df.cap);
  if (blockIdx.x == 0 && threadIdx.x == 0) df.count[st.dparity ^ 1] = 0u;
  for (unsigned e = blockIdx.x * NT + threadIdx.x; e < n; e += gridDim.x * NT)
  {
    const Deferred d = df.list[e];
    const Glob     g{st, c, add, rvol};
    const int      gj = (int)(d.k / (unsigned)c.nx), gi = (int)(d.k - (unsigned)gj * (unsigned)c.nx);
    st.out.s[d.k] = advect_global(g, gi, gj, d.u, d.v);
  }
}

} // namespace hm

#endif
