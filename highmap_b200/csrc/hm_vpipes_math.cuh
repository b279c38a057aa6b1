/*
 * hm_vpipes_math.cuh - per-cell arithmetic of the virtual-pipes passes,
 * rounded exactly as the reference's fp32 kernel text evaluates it.
 *
 * Reference: HighMap/src/gpu_opencl/kernels/hydraulic_vpipes.cl
 *   flow pass         :5-69     water pass  :71-116
 *   erosion pass      :118-184  advection   :186-211
 * and the host steps of HighMap/src/erosion/hydraulic_vpipes_gpu.cpp:36-55,
 * :163-169.
 *
 * Every operation is an explicitly rounded intrinsic, so no multiply is
 * contracted into an add and each result is the reference's
 * one-rounding-per-operation value.  hypot is evaluated as
 * sqrt(x*x + y*y) in fp64 (both squares exact, one rounding for the sum,
 * a correctly rounded square root, one rounding to fp32), which equals the
 * C library's correctly rounded hypotf used by the CPU oracle.  pow with
 * exponent 1 is the identity; other exponents go through fp64 pow.
 */
#ifndef HM_VPIPES_MATH_CUH
#define HM_VPIPES_MATH_CUH

namespace hm
{

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
/* a / b rounded as fdiv, for dividends that are often zero: +-0 / b for
 * b > 0 (+inf included) is a itself, so it is selected instead and the
 * division is given the dividend 1 there (a zero dividend sends the whole
 * warp down the division's special-operand path).  Any other b divides. */
__device__ __forceinline__ float fdiv_z(float a, float b)
{
  const bool z = a == 0.f && b > 0.f;
  return z ? a : __fdiv_rn(z ? 1.f : a, b);
}
/* the reference's max / min as the oracle spells them: a > b ? a : b */
__device__ __forceinline__ float rmax(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float rmin(float a, float b) { return a < b ? a : b; }
/* a > b ? x : y */
__device__ __forceinline__ float sel_gt(float a, float b, float x, float y) { return a > b ? x : y; }

__device__ __forceinline__ float hyp(float x, float y)
{
  /* x*x is exact in fp64, so the fma's one rounding is that of the sum */
  double dx = (double)x, dy = (double)y;
  return __double2float_rn(__dsqrt_rn(__fma_rn(dx, dx, __dmul_rn(dy, dy))));
}

template <class T> __device__ __forceinline__ T bc(float v);
template <> __device__ __forceinline__ float bc<float>(float v) { return v; }

__device__ __forceinline__ float powr(float b, float e) { return __double2float_rn(pow((double)b, (double)e)); }

/* Scalars of one vpipes call, prepared on the host with the same float
 * operations the reference performs. */
struct VpConst
{
  int   nx, ny;
  float dt;
  float dtga;        /* dt * (gravity * pipe_area)                    */
  float pl;          /* pipe length                                    */
  float pl2;         /* pipe length squared                            */
  float c0, c1;      /* flux diffusion weights (c1 = 1 - 4 c0)         */
  float vel_floor;   /* 0.001 * water_height / dt                      */
  float water_height;
  float ratio;       /* downcutting_max_depth_ratio                     */
  float k_capacity, k_erode, k_depose, k_exp;
  float keep;        /* 1 - dt * evap_rate                              */
  float rps;         /* rain per step                                   */
  float fnx;         /* (float)nx, the slope scale of :156              */
  float xhi, yhi;    /* nx - 0.5, ny - 0.5 (exact; 0 for grids too wide to
                      * hold them exactly): sample points in [0.5, xhi) x
                      * [0.5, yhi) need no mirror and no index clamps      */
};

/* Depth at the start of a step: the stored evaporated depth, plus the
 * volume top-up of the previous step ((add * rain) / R, :167-168), plus the
 * optional per-step rain. */
template <bool MAINTAIN, bool RAIN, class T>
__device__ __forceinline__ T depth_d1(T d, T rain, float add, float rvol, float rps)
{
  T dc = d;
  if (MAINTAIN) dc = fadd(d, fdiv(fmul(bc<T>(add), rain), bc<T>(rvol)));
  if (RAIN) dc = fadd(dc, fmul(bc<T>(rps), rain));
  return dc;
}

/* Flow pass for one cell; the height differences are formed
 * as the reference subtracts them: (h0 - z_n) - d1_n.  "s" is j + 1 (the
 * reference's "top"), "n" is j - 1. */
template <bool DIFFUSION, bool PL_ONE, class T>
__device__ __forceinline__ void flow_cell(const VpConst &c,
                                          T zc, T d1c,
                                          T zw, T d1w,
                                          T ze, T d1e,
                                          T zs, T d1s,
                                          T zn, T d1n,
                                          T &fl, T &fr, T &ft, T &fb)
{
  const T zero = bc<T>(0.f);
  T       h0 = fadd(zc, d1c);
  T       dhl = fsub(fsub(h0, zw), d1w);
  T       dhr = fsub(fsub(h0, ze), d1e);
  T       dht = fsub(fsub(h0, zs), d1s);
  T       dhb = fsub(fsub(h0, zn), d1n);
  const T dtga = bc<T>(c.dtga);
  T       ql = fmul(dtga, dhl), qr = fmul(dtga, dhr), qt = fmul(dtga, dht), qb = fmul(dtga, dhb);
  if (!PL_ONE)
  {
    const T pl = bc<T>(c.pl);
    ql = fdiv(ql, pl);
    qr = fdiv(qr, pl);
    qt = fdiv(qt, pl);
    qb = fdiv(qb, pl);
  }
  T nl = rmax(zero, fadd(fl, ql));
  T nr = rmax(zero, fadd(fr, qr));
  T nt = rmax(zero, fadd(ft, qt));
  T nb = rmax(zero, fadd(fb, qb));
  if (DIFFUSION)
  {
    const T c1 = bc<T>(c.c1);
    T       f_diff = fmul(bc<T>(c.c0), fadd(fadd(fadd(nl, nr), nt), nb));
    nl = fadd(fmul(c1, nl), f_diff);
    nr = fadd(fmul(c1, nr), f_diff);
    nt = fadd(fmul(c1, nt), f_diff);
    nb = fadd(fmul(c1, nb), f_diff);
  }
  T sum = fadd(fadd(fadd(nl, nr), nt), nb);
  /* k = sum > 1e-5 ? d1 * l * l / (sum * dt) : 0, clamped to [0, 1]; with
   * l = 1 the two products are d1 itself (x * 1 is exact for every x) */
  const T num = PL_ONE ? d1c : fmul(fmul(d1c, bc<T>(c.pl)), bc<T>(c.pl));
  /* where the quotient is discarded (sum <= 1e-5 or NaN: pits have
   * sum = 0, and d1 / 0 takes the division's special-operand path) the
   * divisor is 1 */
  const bool wet = sum > bc<T>(1e-5f);
  T          kq = fdiv(num, wet ? fmul(sum, bc<T>(c.dt)) : bc<T>(1.f));
  T          k = wet ? kq : zero;
  k = rmin(rmax(k, zero), bc<T>(1.f));
  fl = fmul(nl, k);
  fr = fmul(nr, k);
  ft = fmul(nt, k);
  fb = fmul(nb, k);
}

/* Water pass for one cell: new depth d2 and velocity (u, v).
 * frw = fr(i-1, j), fle = fl(i+1, j), ftn = ft(i, j-1), fbs = fb(i, j+1). */
template <bool PL_ONE, class T>
__device__ __forceinline__ void water_cell(const VpConst &c,
                                           T d1c,
                                           T flc, T frc, T ftc, T fbc,
                                           T frw, T fle, T ftn, T fbs,
                                           T &d2, T &u, T &v)
{
  T dv = fmul(bc<T>(c.dt), fsub(fsub(fsub(fsub(fadd(fadd(fadd(frw, ftn), fle), fbs), flc), frc), ftc), fbc));
  d2 = rmax(bc<T>(0.f), fadd(d1c, PL_ONE ? dv : fdiv(dv, bc<T>(c.pl2))));
  T un = fmul(bc<T>(0.5f), fsub(fadd(fsub(frw, flc), frc), fle));
  T vn = fmul(bc<T>(0.5f), fsub(fadd(fsub(ftn, fbc), ftc), fbs));
  T dmean = rmax(bc<T>(c.vel_floor), d2);
  u = fdiv(un, dmean);
  v = fdiv(vn, dmean);
}

/* Erosion / deposition for one cell from the old z and s around it; both
 * branches of :170-183 are formed and one is selected. */
template <bool KEXP_ONE, class T>
__device__ __forceinline__ void erosion_cell(const VpConst &c,
                                             T zc, T sc,
                                             T zw, T ze, T zn, T zs,
                                             T sw, T se, T sn, T ss,
                                             T d2, T u, T v,
                                             T &z_out, T &s_out)
{
  const T half = bc<T>(0.5f);
  T       dzx = fmul(half, fsub(fadd(fsub(ze, zw), se), sw));
  T       dzy = fmul(half, fsub(fadd(fsub(zs, zn), ss), sn));
  T       talus = hyp(dzx, dzy);
  T       dzn = rmax(bc<T>(1e-3f), fmul(bc<T>(c.fnx), talus));
  T       salpha = rmax(bc<T>(0.01f), fdiv(dzn, hyp(bc<T>(1.f), dzn)));
  T       speed = hyp(u, v);
  /* d2 is zero on dry cells (about 6 % of the cells after a few hundred
   * steps of the 4096^2 benchmark, in over 90 % of the warps) */
  T       depth = rmin(fdiv_z(d2, bc<T>(c.water_height)), bc<T>(c.ratio));
  T       discharge = fmul(depth, speed);
  T       pw = KEXP_ONE ? discharge : powr(discharge, c.k_exp);
  T       capa = fmul(fmul(bc<T>(c.k_capacity), pw), salpha);
  T       ero = fmul(bc<T>(c.k_erode), fsub(capa, sc));
  T       dep = fmul(bc<T>(c.k_depose), fsub(sc, capa));
  z_out = sel_gt(capa, sc, fsub(zc, ero), fadd(zc, dep));
  s_out = sel_gt(capa, sc, fadd(sc, ero), fsub(sc, dep));
}

/* Mirror an unnormalised coordinate with period 2 * n (texel units):
 * |x - 2n * rint(x / 2n)|.  For |x| <= n the quotient rounds to at most
 * 1/2 in magnitude and rint gives +-0, so the result is |x| exactly; the
 * division is skipped there. */
__device__ __forceinline__ float mirror_coord(float x, int n)
{
  const float ax = fabsf(x);
  if (ax <= (float)n) return ax;
  float period = (float)(2 * n);
  float r = rintf(fdiv(x, period));
  return fabsf(fsub(x, fmul(period, r)));
}

/* Bilinear sample weights and texel indices of the linear sampler at
 * (x, y): texel centres at k + 0.5, mirrored repeat, indices clamped. */
struct Tap
{
  int   i0, i1, j0, j1;
  float a, b;
};

__device__ __forceinline__ Tap linear_tap(float x, float y, int nx, int ny)
{
  float xm = fsub(mirror_coord(x, nx), 0.5f);
  float ym = fsub(mirror_coord(y, ny), 0.5f);
  float fx = floorf(xm), fy = floorf(ym);
  Tap   t;
  t.a = fsub(xm, fx);
  t.b = fsub(ym, fy);
  /* after mirroring fx lies in [-1, nx - 1]; the clamp only matters for
   * coordinates too large to mirror exactly and keeps the taps in the grid */
  t.i0 = (int)fminf(fmaxf(fx, -1.f), (float)(nx - 1));
  t.j0 = (int)fminf(fmaxf(fy, -1.f), (float)(ny - 1));
  t.i1 = t.i0 + 1;
  t.j1 = t.j0 + 1;
  t.i0 = t.i0 < 0 ? 0 : t.i0;
  t.j0 = t.j0 < 0 ? 0 : t.j0;
  t.i1 = t.i1 > nx - 1 ? nx - 1 : t.i1;
  t.j1 = t.j1 > ny - 1 ? ny - 1 : t.j1;
  return t;
}

__device__ __forceinline__ float blend(const Tap &t, float s00, float s10, float s01, float s11)
{
  float oma = fsub(1.f, t.a), omb = fsub(1.f, t.b);
  float r = fmul(fmul(oma, omb), s00);
  r = fadd(r, fmul(fmul(t.a, omb), s10));
  r = fadd(r, fmul(fmul(oma, t.b), s01));
  r = fadd(r, fmul(fmul(t.a, t.b), s11));
  return r;
}

} // namespace hm

#endif
