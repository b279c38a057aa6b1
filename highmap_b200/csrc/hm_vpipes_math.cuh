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
/* the reference's max / min as the oracle spells them: a > b ? a : b */
__device__ __forceinline__ float rmax(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float rmin(float a, float b) { return a < b ? a : b; }

__device__ __forceinline__ float hyp(float x, float y)
{
  double dx = (double)x, dy = (double)y;
  return __double2float_rn(__dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy))));
}

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
};

/* Depth at the start of a step: the stored evaporated depth, plus the
 * volume top-up of the previous step ((add * rain) / R, :167-168), plus the
 * optional per-step rain. */
template <bool MAINTAIN, bool RAIN>
__device__ __forceinline__ float depth_d1(float d, float rain, float add, float rvol, float rps)
{
  float dc = MAINTAIN ? fadd(d, fdiv(fmul(add, rain), rvol)) : d;
  if (RAIN) dc = fadd(dc, fmul(rps, rain));
  return dc;
}

/* Flow pass for one cell; h* are z + d1 neighbours' terms split as the
 * reference subtracts them ((h0 - z_n) - d1_n). */
template <bool DIFFUSION, bool PL_ONE>
__device__ __forceinline__ void flow_cell(const VpConst &c,
                                          float zc, float d1c,
                                          float zw, float d1w,
                                          float ze, float d1e,
                                          float zs, float d1s,
                                          float zn, float d1n,
                                          float &fl, float &fr, float &ft, float &fb)
{
  float h0 = fadd(zc, d1c);
  float dhl = fsub(fsub(h0, zw), d1w);
  float dhr = fsub(fsub(h0, ze), d1e);
  float dht = fsub(fsub(h0, zs), d1s); /* "top" is j + 1 */
  float dhb = fsub(fsub(h0, zn), d1n);
  float ql = fmul(c.dtga, dhl), qr = fmul(c.dtga, dhr), qt = fmul(c.dtga, dht), qb = fmul(c.dtga, dhb);
  if (!PL_ONE)
  {
    ql = fdiv(ql, c.pl);
    qr = fdiv(qr, c.pl);
    qt = fdiv(qt, c.pl);
    qb = fdiv(qb, c.pl);
  }
  float nl = rmax(0.f, fadd(fl, ql));
  float nr = rmax(0.f, fadd(fr, qr));
  float nt = rmax(0.f, fadd(ft, qt));
  float nb = rmax(0.f, fadd(fb, qb));
  if (DIFFUSION)
  {
    float f_diff = fmul(c.c0, fadd(fadd(fadd(nl, nr), nt), nb));
    nl = fadd(fmul(c.c1, nl), f_diff);
    nr = fadd(fmul(c.c1, nr), f_diff);
    nt = fadd(fmul(c.c1, nt), f_diff);
    nb = fadd(fmul(c.c1, nb), f_diff);
  }
  float sum = fadd(fadd(fadd(nl, nr), nt), nb);
  float k = 0.f;
  if (sum > 1e-5f) k = fdiv(fmul(fmul(d1c, c.pl), c.pl), fmul(sum, c.dt));
  k = rmin(rmax(k, 0.f), 1.f);
  fl = fmul(nl, k);
  fr = fmul(nr, k);
  ft = fmul(nt, k);
  fb = fmul(nb, k);
}

/* Water pass for one cell: new depth d2 and velocity (u, v).
 * frw = fr(i-1, j), fle = fl(i+1, j), ftn = ft(i, j-1), fbs = fb(i, j+1). */
template <bool PL_ONE>
__device__ __forceinline__ void water_cell(const VpConst &c,
                                           float d1c,
                                           float flc, float frc, float ftc, float fbc,
                                           float frw, float fle, float ftn, float fbs,
                                           float &d2, float &u, float &v)
{
  float dv = fmul(c.dt, fsub(fsub(fsub(fsub(fadd(fadd(fadd(frw, ftn), fle), fbs), flc), frc), ftc), fbc));
  d2 = rmax(0.f, fadd(d1c, PL_ONE ? dv : fdiv(dv, c.pl2)));
  float un = fmul(0.5f, fsub(fadd(fsub(frw, flc), frc), fle));
  float vn = fmul(0.5f, fsub(fadd(fsub(ftn, fbc), ftc), fbs));
  float dmean = rmax(c.vel_floor, d2);
  u = fdiv(un, dmean);
  v = fdiv(vn, dmean);
}

/* Erosion / deposition for one cell from the old z and s around it. */
template <bool KEXP_ONE>
__device__ __forceinline__ void erosion_cell(const VpConst &c,
                                             float zc, float sc,
                                             float zw, float ze, float zn, float zs,
                                             float sw, float se, float sn, float ss,
                                             float d2, float u, float v,
                                             float &z_out, float &s_out)
{
  float dzx = fmul(0.5f, fsub(fadd(fsub(ze, zw), se), sw));
  float dzy = fmul(0.5f, fsub(fadd(fsub(zs, zn), ss), sn));
  float talus = hyp(dzx, dzy);
  float dzn = rmax(1e-3f, fmul(c.fnx, talus));
  float salpha = rmax(0.01f, fdiv(dzn, hyp(1.f, dzn)));
  float speed = hyp(u, v);
  float depth = rmin(fdiv(d2, c.water_height), c.ratio);
  float discharge = fmul(depth, speed);
  float pw = KEXP_ONE ? discharge : __double2float_rn(pow((double)discharge, (double)c.k_exp));
  float capa = fmul(fmul(c.k_capacity, pw), salpha);
  if (capa > sc)
  {
    float amount = fmul(c.k_erode, fsub(capa, sc));
    z_out = fsub(zc, amount);
    s_out = fadd(sc, amount);
  }
  else
  {
    float amount = fmul(c.k_depose, fsub(sc, capa));
    z_out = fadd(zc, amount);
    s_out = fsub(sc, amount);
  }
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
