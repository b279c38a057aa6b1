/*
 * hm_vpipes.cu - virtual-pipes hydraulic erosion on sm_100a.
 *
 * Replaces HighMap/src/erosion/hydraulic_vpipes_gpu.cpp:15-178 and the
 * OpenCL kernels of HighMap/src/gpu_opencl/kernels/hydraulic_vpipes.cl.
 * The reference uploads and downloads every field around each of its four
 * passes (about 40 host<->device image copies per iteration) and runs the
 * evaporation and volume top-up on the host; here all state stays in HBM
 * for the whole call and every step is device work only.
 *
 * State in HBM (fp32, nx*ny each, SoA): z (ping-pong with one workspace
 * grid), d (evaporated depth, before the volume top-up), s (sediment),
 * fl, fr, ft, fb (outflow fluxes), u, v (velocities), and s1 (sediment
 * after erosion, before advection).  The volume top-up (V0 - sum d) * rain
 * / R is applied lazily: the step that follows reads the stored depth plus
 * the top-up, and the grid-wide sum is a deterministic fp64 reduction
 * finished by the last block of the water/erosion kernel.
 *
 * Kernels per step
 *   k_vp_flow          flow pass (:5-69); reads z, d (radius 1), f;
 *                      writes f in place.
 *   k_vp_water_erosion water pass (:71-116) and erosion pass (:118-184);
 *                      reads f (radius 1), d, z, s (radius 1); writes z',
 *                      s1, u, v, d.
 *   k_vp_transport     advection (:186-211): s = bilinear(s1, x - dt u).
 */
#include <cuda_runtime.h>

#include <cstdint>

#include "hm_internal.h"
#include "hm_reduce.cuh"
#include "hm_vpipes.h"
#include "hm_vpipes_math.cuh"

namespace hm
{

struct VpScalars
{
  float    v0;     /* initial water volume (float of the fp64 sum)  */
  float    rvol;   /* rain map volume                               */
  float    add[2]; /* V0 - sum(d) of the previous step, ping-pong   */
  unsigned ticket;
  unsigned pad[3];
};

constexpr int VP_BX = 64;
constexpr int VP_BY = 4;
constexpr int VP_NT = VP_BX * VP_BY;

struct VpFields
{
  float *z, *zn, *d, *s, *s1, *fl, *fr, *ft, *fb, *u, *v;
  const float *rain; /* nullable */
};

/* ---- init --------------------------------------------------------- */

__global__ void __launch_bounds__(VP_NT)
    k_vp_init(VpFields f, size_t n, float init_depth, VpScalars *sc, double *partials)
{
  const unsigned bid = blockIdx.x;
  double         sd = 0.0, sr = 0.0;
  for (size_t k = bid * (size_t)VP_NT + threadIdx.x; k < n; k += (size_t)gridDim.x * VP_NT)
  {
    float r = f.rain ? f.rain[k] : 1.f;
    float d = fmul(init_depth, r);
    f.d[k] = d;
    f.s[k] = 0.f;
    f.fl[k] = 0.f;
    f.fr[k] = 0.f;
    f.ft[k] = 0.f;
    f.fb[k] = 0.f;
    f.u[k] = 0.f;
    f.v[k] = 0.f;
    sd += (double)d;
    sr += (double)r;
  }
  /* two sums: partials[0 .. G) for d, partials[G .. 2G) for rain */
  __shared__ double sm[VP_NT / 32];
  double            bd = block_sum<VP_NT>(sd, sm);
  double            br = block_sum<VP_NT>(sr, sm);
  if (threadIdx.x == 0)
  {
    partials[bid] = bd;
    partials[gridDim.x + bid] = br;
  }
}

__global__ void __launch_bounds__(VP_NT) k_vp_init_finish(VpScalars *sc, const double *partials, unsigned g)
{
  __shared__ double sm[VP_NT / 32];
  double            ad = 0.0, ar = 0.0;
  for (unsigned k = threadIdx.x; k < g; k += VP_NT)
  {
    ad += partials[k];
    ar += partials[g + k];
  }
  double td = block_sum<VP_NT>(ad, sm);
  double tr = block_sum<VP_NT>(ar, sm);
  if (threadIdx.x == 0)
  {
    sc->v0 = (float)td;
    sc->rvol = (float)tr;
    sc->add[0] = 0.f;
    sc->add[1] = 0.f;
    sc->ticket = 0u;
  }
}

/* ---- flow pass ------------------------------------------------------ */

template <bool MAINTAIN, bool DIFFUSION, bool PL_ONE>
__global__ void __launch_bounds__(VP_NT)
    k_vp_flow(VpFields f, VpConst c, const VpScalars *__restrict__ sc, int parity)
{
  const int i = blockIdx.x * VP_BX + threadIdx.x;
  const int j = blockIdx.y * VP_BY + threadIdx.y;
  if (i >= c.nx || j >= c.ny) return;
  const int   nx = c.nx;
  const int   im = i > 0 ? i - 1 : 0, ip = i < nx - 1 ? i + 1 : nx - 1;
  const int   jm = j > 0 ? j - 1 : 0, jp = j < c.ny - 1 ? j + 1 : c.ny - 1;
  const float add = MAINTAIN ? sc->add[parity] : 0.f;
  const float rvol = MAINTAIN ? sc->rvol : 1.f;
  const bool  rain_step = c.rps != 0.f;

  auto d1 = [&](int ii, int jj) -> float
  {
    size_t k = (size_t)jj * nx + ii;
    float  r = f.rain ? __ldg(f.rain + k) : 1.f;
    float  dd = __ldg(f.d + k);
    return rain_step ? depth_d1<MAINTAIN, true>(dd, r, add, rvol, c.rps)
                     : depth_d1<MAINTAIN, false>(dd, r, add, rvol, c.rps);
  };
  auto zz = [&](int ii, int jj) -> float { return __ldg(f.z + (size_t)jj * nx + ii); };

  const size_t k = (size_t)j * nx + i;
  float        fl = f.fl[k], fr = f.fr[k], ft = f.ft[k], fb = f.fb[k];
  flow_cell<DIFFUSION, PL_ONE>(c, zz(i, j), d1(i, j), zz(im, j), d1(im, j), zz(ip, j), d1(ip, j),
                               zz(i, jp), d1(i, jp), zz(i, jm), d1(i, jm), fl, fr, ft, fb);
  f.fl[k] = fl;
  f.fr[k] = fr;
  f.ft[k] = ft;
  f.fb[k] = fb;
}

/* ---- water + erosion ------------------------------------------------ */

template <bool MAINTAIN, bool PL_ONE, bool KEXP_ONE>
__global__ void __launch_bounds__(VP_NT)
    k_vp_water_erosion(VpFields f, VpConst c, VpScalars *sc, int parity, double *partials)
{
  const int i = blockIdx.x * VP_BX + threadIdx.x;
  const int j = blockIdx.y * VP_BY + threadIdx.y;
  const int nx = c.nx;
  double    part = 0.0;
  if (i < nx && j < c.ny)
  {
    const int    im = i > 0 ? i - 1 : 0, ip = i < nx - 1 ? i + 1 : nx - 1;
    const int    jm = j > 0 ? j - 1 : 0, jp = j < c.ny - 1 ? j + 1 : c.ny - 1;
    const size_t k = (size_t)j * nx + i;
    const float  add = MAINTAIN ? sc->add[parity] : 0.f;
    const float  rvol = MAINTAIN ? sc->rvol : 1.f;
    const float  r = f.rain ? __ldg(f.rain + k) : 1.f;
    const float  d1c = c.rps != 0.f ? depth_d1<MAINTAIN, true>(__ldg(f.d + k), r, add, rvol, c.rps)
                                    : depth_d1<MAINTAIN, false>(__ldg(f.d + k), r, add, rvol, c.rps);
    float d2, u, v;
    water_cell<PL_ONE>(c, d1c, __ldg(f.fl + k), __ldg(f.fr + k), __ldg(f.ft + k), __ldg(f.fb + k),
                       __ldg(f.fr + (size_t)j * nx + im), __ldg(f.fl + (size_t)j * nx + ip),
                       __ldg(f.ft + (size_t)jm * nx + i), __ldg(f.fb + (size_t)jp * nx + i), d2, u, v);
    const float *z = f.z, *s = f.s;
    float        zo, so;
    erosion_cell<KEXP_ONE>(c, __ldg(z + k), __ldg(s + k), __ldg(z + (size_t)j * nx + im),
                           __ldg(z + (size_t)j * nx + ip), __ldg(z + (size_t)jm * nx + i),
                           __ldg(z + (size_t)jp * nx + i), __ldg(s + (size_t)j * nx + im),
                           __ldg(s + (size_t)j * nx + ip), __ldg(s + (size_t)jm * nx + i),
                           __ldg(s + (size_t)jp * nx + i), d2, u, v, zo, so);
    const float de = fmul(d2, c.keep);
    f.zn[k] = zo;
    f.s1[k] = so;
    f.u[k] = u;
    f.v[k] = v;
    f.d[k] = de;
    part = (double)de;
  }
  if (MAINTAIN)
  {
    const unsigned nb = gridDim.x * gridDim.y;
    const unsigned bid = blockIdx.y * gridDim.x + blockIdx.x;
    const float    v0 = sc->v0;
    float         *out = &sc->add[parity ^ 1];
    grid_sum_commit<VP_NT>(part, partials, &sc->ticket, nb, bid,
                           [&](double total) { *out = fsub(v0, (float)total); });
  }
}

/* ---- advection ------------------------------------------------------ */

__global__ void __launch_bounds__(VP_NT) k_vp_transport(VpFields f, VpConst c)
{
  const int i = blockIdx.x * VP_BX + threadIdx.x;
  const int j = blockIdx.y * VP_BY + threadIdx.y;
  if (i >= c.nx || j >= c.ny) return;
  const size_t k = (size_t)j * c.nx + i;
  const float  x = fsub((float)i, fmul(c.dt, __ldg(f.u + k)));
  const float  y = fsub((float)j, fmul(c.dt, __ldg(f.v + k)));
  const Tap    t = linear_tap(x, y, c.nx, c.ny);
  const float *s1 = f.s1;
  const size_t r0 = (size_t)t.j0 * c.nx, r1 = (size_t)t.j1 * c.nx;
  f.s[k] = blend(t, __ldg(s1 + r0 + t.i0), __ldg(s1 + r0 + t.i1), __ldg(s1 + r1 + t.i0), __ldg(s1 + r1 + t.i1));
}

/* ---- outputs -------------------------------------------------------- */

template <bool MAINTAIN>
__global__ void k_vp_final_depth(const float *__restrict__ d,
                                 const float *__restrict__ rain,
                                 const VpScalars *__restrict__ sc,
                                 int parity,
                                 float *__restrict__ out,
                                 size_t n)
{
  const float add = MAINTAIN ? sc->add[parity] : 0.f;
  const float rvol = MAINTAIN ? sc->rvol : 1.f;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
  {
    float r = rain ? rain[k] : 1.f;
    out[k] = depth_d1<MAINTAIN, false>(d[k], r, add, rvol, 0.f);
  }
}

/* ------------------------------------------------------------------ */
/* host side                                                          */
/* ------------------------------------------------------------------ */

int vpipes_check_args(const float *z, int nx, int ny, const hm_vpipes_params *p)
{
  if (!z) return fail(HM_ERR_INVALID_ARGUMENT, "vpipes: z is NULL");
  if (nx < 1 || ny < 1) return fail(HM_ERR_INVALID_ARGUMENT, "vpipes: nx and ny must be >= 1");
  if ((long long)nx * (long long)ny > (1ll << 32))
    return fail(HM_ERR_INVALID_ARGUMENT, "vpipes: grid larger than 2^32 cells");
  if (p->iterations < 0) return fail(HM_ERR_INVALID_ARGUMENT, "vpipes: iterations < 0");
  if (!(p->dt != 0.f)) return fail(HM_ERR_INVALID_ARGUMENT, "vpipes: dt must be non-zero");
  if (!(p->pipe_length != 0.f)) return fail(HM_ERR_INVALID_ARGUMENT, "vpipes: pipe_length must be non-zero");
  return HM_OK;
}

constexpr unsigned VP_INIT_BLOCKS = 296;

/* fp64 partial sums: one per block of the step grid, and two per block of
 * the init grid */
static size_t partials_bytes(int nx, int ny)
{
  size_t grid_blocks = (size_t)((nx + VP_BX - 1) / VP_BX) * ((ny + VP_BY - 1) / VP_BY);
  if (grid_blocks < 2 * VP_INIT_BLOCKS) grid_blocks = 2 * VP_INIT_BLOCKS;
  return align_up(grid_blocks * sizeof(double), 256);
}

size_t vpipes_scratch_bytes(int nx, int ny)
{
  const size_t n = align_up((size_t)nx * ny, 64);
  return n * sizeof(float) * 10 + partials_bytes(nx, ny) + align_up(sizeof(VpScalars), 256);
}

VpConst vpipes_consts(int nx, int ny, const hm_vpipes_params &p)
{
  VpConst c;
  c.nx = nx;
  c.ny = ny;
  c.dt = p.dt;
  const float ga = p.gravity * p.pipe_area;
  c.dtga = p.dt * ga;
  c.pl = p.pipe_length;
  c.pl2 = p.pipe_length * p.pipe_length;
  c.c0 = p.flux_diffusion_strength;
  c.c1 = 1.f - 4.f * p.flux_diffusion_strength;
  c.vel_floor = 0.001f * p.water_height / p.dt;
  c.water_height = p.water_height;
  c.ratio = p.downcutting_max_depth_ratio;
  c.k_capacity = p.k_capacity;
  c.k_erode = p.k_erode;
  c.k_depose = p.k_depose;
  c.k_exp = p.k_discharge_exp;
  c.keep = 1.f - p.dt * p.evap_rate;
  c.rps = p.rain_per_step;
  c.fnx = (float)nx;
  return c;
}

template <bool M>
static void launch_flow(const VpFields &f, const VpConst &c, const VpScalars *sc, int parity, bool diff,
                        bool pl1, dim3 g, dim3 b, cudaStream_t s)
{
  if (diff)
  {
    if (pl1) k_vp_flow<M, true, true><<<g, b, 0, s>>>(f, c, sc, parity);
    else k_vp_flow<M, true, false><<<g, b, 0, s>>>(f, c, sc, parity);
  }
  else
  {
    if (pl1) k_vp_flow<M, false, true><<<g, b, 0, s>>>(f, c, sc, parity);
    else k_vp_flow<M, false, false><<<g, b, 0, s>>>(f, c, sc, parity);
  }
}

template <bool M>
static void launch_we(const VpFields &f, const VpConst &c, VpScalars *sc, int parity, double *partials, bool pl1,
                      bool k1, dim3 g, dim3 b, cudaStream_t s)
{
  if (pl1)
  {
    if (k1) k_vp_water_erosion<M, true, true><<<g, b, 0, s>>>(f, c, sc, parity, partials);
    else k_vp_water_erosion<M, true, false><<<g, b, 0, s>>>(f, c, sc, parity, partials);
  }
  else
  {
    if (k1) k_vp_water_erosion<M, false, true><<<g, b, 0, s>>>(f, c, sc, parity, partials);
    else k_vp_water_erosion<M, false, false><<<g, b, 0, s>>>(f, c, sc, parity, partials);
  }
}

int vpipes_core(float *z,
                int nx,
                int ny,
                const hm_vpipes_params &p,
                const float *rain,
                float *water_depth,
                float *sediment,
                float *vel_u,
                float *vel_v,
                void *scratch_buf,
                cudaStream_t s)
{
  const size_t n = (size_t)nx * ny;
  const size_t na = align_up(n, 64);
  float       *base = (float *)scratch_buf;
  VpFields     f;
  f.z = z;
  f.zn = base + 0 * na;
  f.d = base + 1 * na;
  f.s = base + 2 * na;
  f.s1 = base + 3 * na;
  f.fl = base + 4 * na;
  f.fr = base + 5 * na;
  f.ft = base + 6 * na;
  f.fb = base + 7 * na;
  f.u = base + 8 * na;
  f.v = base + 9 * na;
  f.rain = rain;
  double      *partials = (double *)(base + 10 * na);
  VpScalars   *sc = (VpScalars *)((char *)partials + partials_bytes(nx, ny));

  const VpConst c = vpipes_consts(nx, ny, p);
  const float   init_depth = p.initial_water < 0.f ? p.water_height : p.initial_water;

  /* init: fields and the two volumes (deterministic: fixed grid) */
  const unsigned gi = VP_INIT_BLOCKS;
  k_vp_init<<<gi, VP_NT, 0, s>>>(f, n, init_depth, sc, partials);
  HM_LAUNCH_CHECK("k_vp_init");
  k_vp_init_finish<<<1, VP_NT, 0, s>>>(sc, partials, gi);
  HM_LAUNCH_CHECK("k_vp_init_finish");

  const dim3 b(VP_BX, VP_BY);
  const dim3 g((nx + VP_BX - 1) / VP_BX, (ny + VP_BY - 1) / VP_BY);
  const bool maintain = p.maintain_water_volume != 0;
  const bool diff = p.flux_diffusion != 0;
  const bool pl1 = p.pipe_length == 1.f;
  const bool k1 = p.k_discharge_exp == 1.f;
  int        parity = 0;
  for (int it = 0; it < p.iterations; it++)
  {
    if (maintain) launch_flow<true>(f, c, sc, parity, diff, pl1, g, b, s);
    else launch_flow<false>(f, c, sc, parity, diff, pl1, g, b, s);
    HM_LAUNCH_CHECK("k_vp_flow");
    if (maintain) launch_we<true>(f, c, sc, parity, partials, pl1, k1, g, b, s);
    else launch_we<false>(f, c, sc, parity, partials, pl1, k1, g, b, s);
    HM_LAUNCH_CHECK("k_vp_water_erosion");
    k_vp_transport<<<g, b, 0, s>>>(f, c);
    HM_LAUNCH_CHECK("k_vp_transport");
    float *t = f.z;
    f.z = f.zn;
    f.zn = t;
    parity ^= 1;
  }
  if (f.z != z) HM_CUDA_TRY(cudaMemcpyAsync(z, f.z, n * sizeof(float), cudaMemcpyDeviceToDevice, s));

  if (water_depth)
  {
    if (maintain) k_vp_final_depth<true><<<592, 256, 0, s>>>(f.d, rain, sc, parity, water_depth, n);
    else k_vp_final_depth<false><<<592, 256, 0, s>>>(f.d, rain, sc, parity, water_depth, n);
    HM_LAUNCH_CHECK("k_vp_final_depth");
  }
  if (sediment) HM_CUDA_TRY(cudaMemcpyAsync(sediment, f.s, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
  if (vel_u) HM_CUDA_TRY(cudaMemcpyAsync(vel_u, f.u, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
  if (vel_v) HM_CUDA_TRY(cudaMemcpyAsync(vel_v, f.v, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
  return HM_OK;
}

} // namespace hm

extern "C" void hm_vpipes_default_params(hm_vpipes_params *p)
{
  if (!p) return;
  /* defaults of HighMap/include/highmap/erosion.hpp:1206-1223 */
  p->water_height = 1e-2f;
  p->maintain_water_volume = 1;
  p->evap_rate = 0.1f;
  p->iterations = 50;
  p->dt = 0.5f;
  p->k_capacity = 0.5f;
  p->k_erode = 0.001f;
  p->k_depose = 0.01f;
  p->k_discharge_exp = 1.f;
  p->downcutting_max_depth_ratio = 10.f;
  p->flux_diffusion = 1;
  p->flux_diffusion_strength = 0.01f;
  p->gravity = 1.f;
  p->pipe_length = 1.f;
  p->pipe_area = 1.f;
  p->rain_per_step = 0.f;
  p->initial_water = -1.f;
}
