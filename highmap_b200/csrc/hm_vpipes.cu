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
 * State in HBM (fp32, nx*ny each, SoA), two copies that alternate between
 * steps: z, d (evaporated depth, before the volume top-up), s (sediment)
 * and fl, fr, ft, fb (outflow fluxes); copy A's z is the caller's z.  The
 * volume top-up (V0 - sum d) * rain / R is applied lazily: the step that
 * follows reads the stored depth plus the top-up, and the grid-wide sum is
 * a deterministic fp64 reduction finished by the last block of the step.
 *
 * Kernels
 *   k_vp_init          initial depth, zero sediment and fluxes, V0 and R.
 *   k_vp_fwe(_tma), k_vp_advect   one step as two kernels over 2-D tiles
 *                      (hm_vpipes_tiled.cuh), the default.
 *   k_vp_fused         one whole step streaming down column strips
 *                      (hm_vpipes_fused.cuh).
 *   k_vp_final_depth   water-depth output with the last top-up applied.
 */
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "hm_internal.h"
#include "hm_reduce.cuh"
#include "hm_tune.h"
#include "hm_vpipes.h"
#include "hm_vpipes_fused.cuh"
#include "hm_vpipes_tiled.cuh"
#include "hm_vpipes_math.cuh"

namespace hm
{

constexpr int VP_NT = 256;
constexpr unsigned VP_INIT_BLOCKS = 296;

/* ---- init --------------------------------------------------------- */

/* d = initial depth * rain, s = f = 0; fp64 partial sums of d and rain
 * (hydraulic_vpipes_gpu.cpp:36-55). */
__global__ void __launch_bounds__(VP_NT)
    k_vp_init(VpFields f, const float *rain, size_t n, float init_depth, double *partials)
{
  const unsigned bid = blockIdx.x;
  double         sd = 0.0, sr = 0.0;
  for (size_t k = bid * (size_t)VP_NT + threadIdx.x; k < n; k += (size_t)gridDim.x * VP_NT)
  {
    float r = rain ? rain[k] : 1.f;
    float d = fmul(init_depth, r);
    f.d[k] = d;
    f.s[k] = 0.f;
    f.fl[k] = 0.f;
    f.fr[k] = 0.f;
    f.ft[k] = 0.f;
    f.fb[k] = 0.f;
    sd += (double)d;
    sr += (double)r;
  }
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
    sc->slow = 0u;
    sc->defer_count[0] = 0u;
    sc->defer_count[1] = 0u;
    sc->error = 0u;
  }
}

/* ---- outputs -------------------------------------------------------- */

/* water depth output: the stored depth plus the last step's top-up */
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

int vpipes_init(const VpFields &A, const float *rain, size_t n, float init_depth, VpScalars *sc, double *partials,
                cudaStream_t s)
{
  k_vp_init<<<VP_INIT_BLOCKS, VP_NT, 0, s>>>(A, rain, n, init_depth, partials);
  HM_LAUNCH_CHECK("k_vp_init");
  k_vp_init_finish<<<1, VP_NT, 0, s>>>(sc, partials, VP_INIT_BLOCKS);
  HM_LAUNCH_CHECK("k_vp_init_finish");
  return HM_OK;
}

int vpipes_final_depth(const float *d, const float *rain, const VpScalars *sc, int parity, bool maintain,
                       float *out, size_t n, cudaStream_t s)
{
  if (maintain) k_vp_final_depth<true><<<592, 256, 0, s>>>(d, rain, sc, parity, out, n);
  else k_vp_final_depth<false><<<592, 256, 0, s>>>(d, rain, sc, parity, out, n);
  HM_LAUNCH_CHECK("k_vp_final_depth");
  return HM_OK;
}

size_t vpipes_init_partials() { return 2 * VP_INIT_BLOCKS; }

/* launch shapes of the fused step kernel (threads per CTA = strip width
 * including the halo, sampler radius R) */
struct FusedCfg
{
  int tpb, r, h;
};

static FusedCfg g_cfg_override = {0, 0, 0};
/* step kernels: 0 = tiled (k_vp_fwe + k_vp_advect), 1 = streaming (k_vp_fused) */
static int g_algo_override = -1;
/* bytes a TMA tile's barrier expects beyond its boxes (hm_debug_tma_expect_extra) */
static unsigned g_tma_extra_tx = 0;

FusedCfg vpipes_pick_config(int nx, int ny)
{
  if (g_cfg_override.tpb) return g_cfg_override;
  TuneEntry e;
  if (tuned_vpipes(nx, ny, &e) && e.tpb) return FusedCfg{e.tpb, e.radius, e.rows};
  return FusedCfg{128, 2, 64};
}

int vpipes_pick_algo(int nx, int ny)
{
  if (g_algo_override >= 0) return g_algo_override;
  if (g_cfg_override.tpb) return 1;
  TuneEntry e;
  if (tuned_vpipes(nx, ny, &e)) return e.tpb ? 1 : (e.block == 2 ? 3 : 0);
  return 0;
}

static int fused_w(const FusedCfg &c) { return c.tpb - 2 * (c.r + 2); }

static dim3 fused_grid(const FusedCfg &c, int nx, int ny)
{
  const int w = fused_w(c);
  return dim3((nx + w - 1) / w, (ny + c.h - 1) / c.h);
}

static size_t partials_bytes(int nx, int ny)
{
  /* one slot per block of the step grid: the tiled kernel's 32 x 16 tiles
   * outnumber the streaming kernel's strips and chunks */
  size_t blocks = (size_t)((nx + FT_TX - 1) / FT_TX) * ((ny + FT_TY - 1) / FT_TY);
  const size_t streaming = (size_t)((nx + 63) / 64 + 1) * ((ny + 31) / 32 + 1);
  if (blocks < streaming) blocks = streaming;
  if (blocks < 2 * VP_INIT_BLOCKS) blocks = 2 * VP_INIT_BLOCKS;
  return align_up(blocks * sizeof(double), 256);
}

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

/* capacity of the deferred-advection list (cells per step); a step that
 * defers more cells resolves the excess inline */
static size_t defer_cap(int nx, int ny)
{
  size_t cap = (size_t)nx * ny / 32;
  return cap < 4096 ? 4096 : cap;
}

/* grids of the scratch: state copy B (7), state A's d, s and fluxes (6),
 * two copies of u, v and s1 (6: a folded step reads the previous step's
 * and writes its own) */
constexpr size_t VP_GRIDS = 19;

size_t vpipes_scratch_bytes(int nx, int ny)
{
  const size_t n = align_up((size_t)nx * ny, 64);
  /* the grids, fp64 partials, the scalar block, the deferred list */
  return n * sizeof(float) * VP_GRIDS + partials_bytes(nx, ny) + align_up(sizeof(VpScalars), 256) +
         align_up(defer_cap(nx, ny) * sizeof(Deferred), 256);
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
  /* nx - 0.5 is a float exactly while nx < 2^23 */
  c.xhi = nx < (1 << 22) ? (float)nx - 0.5f : 0.f;
  c.yhi = ny < (1 << 22) ? (float)ny - 0.5f : 0.f;
  return c;
}

template <int TPB, int R>
static int launch_fused(const VpStep &st, const VpConst &c, VpScalars *sc, double *partials, const VpDefer &df,
                        dim3 grid, cudaStream_t s)
{
  using L = FusedLayout<TPB, R>;
  static bool attr_set[64] = {};
  int         dev = 0;
  HM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64 || !attr_set[dev])
  {
    HM_CUDA_TRY(cudaFuncSetAttribute(k_vp_fused<TPB, R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)L::SMEM));
    HM_CUDA_TRY(cudaFuncSetAttribute(k_vp_fused<TPB, R, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)L::SMEM));
    if (dev >= 0 && dev < 64) attr_set[dev] = true;
  }
  if (st.maintain) k_vp_fused<TPB, R, true><<<grid, TPB, L::SMEM, s>>>(st, c, sc, partials, df);
  else k_vp_fused<TPB, R, false><<<grid, TPB, L::SMEM, s>>>(st, c, sc, partials, df);
  HM_LAUNCH_CHECK("k_vp_fused");
  k_vp_fixup<128><<<2 * 148, 128, 0, s>>>(st, c, sc, df);
  HM_LAUNCH_CHECK("k_vp_fixup");
  return HM_OK;
}

static int launch_step(const FusedCfg &cfg, const VpStep &st, const VpConst &c, VpScalars *sc, double *partials,
                       const VpDefer &df, cudaStream_t s)
{
  const dim3 grid = fused_grid(cfg, c.nx, c.ny);
  if (cfg.tpb == 128 && cfg.r == 2) return launch_fused<128, 2>(st, c, sc, partials, df, grid, s);
  if (cfg.tpb == 256 && cfg.r == 2) return launch_fused<256, 2>(st, c, sc, partials, df, grid, s);
  if (cfg.tpb == 128 && cfg.r == 3) return launch_fused<128, 3>(st, c, sc, partials, df, grid, s);
  if (cfg.tpb == 256 && cfg.r == 3) return launch_fused<256, 3>(st, c, sc, partials, df, grid, s);
  return fail(HM_ERR_INVALID_ARGUMENT, "vpipes: unsupported fused configuration");
}

/* the steps of vpipes_core with the tiled kernels (k_vp_fwe, k_vp_advect) */
/* ---- TMA tensor maps ---------------------------------------------- */

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
  static PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
    void                           *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
    {
      cudaGetLastError();
      return nullptr;
    }
    return (PFN_cuTensorMapEncodeTiled_v12000)p;
  }();
  return fn;
}

/* map of an nx x ny fp32 grid read in boxes of 40 x box_rows, zeros outside */
static bool encode_grid_map(CUtensorMap *m, const float *base, int nx, int ny, int box_rows)
{
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  cuuint64_t dims[2] = {(cuuint64_t)nx, (cuuint64_t)ny};
  cuuint64_t strides[1] = {(cuuint64_t)nx * sizeof(float)};
  cuuint32_t box[2] = {40u, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1u, 1u};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(base), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

bool adv_maps(const float *u, const float *v, const float *s1, int nx, int ny, AdvMaps *m)
{
  if (nx % 4 != 0 || nx < 40 || ny < FS_H) return false;
  if (!aligned16(u) || !aligned16(v) || !aligned16(s1)) return false;
  return encode_grid_map(&m->u, u, nx, ny, FT_H1) && encode_grid_map(&m->v, v, nx, ny, FT_H1) &&
         encode_grid_map(&m->s1, s1, nx, ny, FS_H);
}

/* tensor maps of one state copy; false if the grid or buffers do not meet
 * the TMA rules (row pitch and bases 16-byte aligned, boxes no larger than
 * the grid) */
bool fwe_maps(const VpFields &f, int nx, int ny, FweMaps *m)
{
  if (nx % 4 != 0 || nx < 40 || ny < FT_H2) return false;
  const float *all[7] = {f.z, f.d, f.s, f.fl, f.fr, f.ft, f.fb};
  for (const float *q : all)
    if (!aligned16(q)) return false;
  return encode_grid_map(&m->z, f.z, nx, ny, FT_H2) && encode_grid_map(&m->d, f.d, nx, ny, FT_H2) &&
         encode_grid_map(&m->s, f.s, nx, ny, FT_H1) && encode_grid_map(&m->fl, f.fl, nx, ny, FT_H1) &&
         encode_grid_map(&m->fr, f.fr, nx, ny, FT_H1) && encode_grid_map(&m->ft, f.ft, nx, ny, FT_H1) &&
         encode_grid_map(&m->fb, f.fb, nx, ny, FT_H1);
}

/* The steps of vpipes_core with the tiled kernels.  The first step is
 * k_vp_fwe(_tma); every later step is k_vp_step(_tma), which advects the
 * previous step's sediment inside its own tile: u, v and s1 alternate
 * between two copies (step k writes copy k % 2 and reads copy (k - 1) % 2),
 * and the last step's advection runs as k_vp_advect after the loop.  Tiles
 * are fetched by TMA where the grid and buffers allow it and allow_tma is
 * set, else by cp.async.  time_block 2: without the volume top-up, steps
 * after the first go in pairs through k_vp_tb2, which writes the pair's
 * s1, u, v into the copy its first step would have written (the copy of
 * the step before the pair is still being read), so the copies alternate
 * once per pair; a step left over at the end runs alone. */
static int vpipes_tiled_steps(float *z, int nx, int ny, const hm_vpipes_params &p, const VpConst &c, VpFields &A,
                              VpFields &B, float *const u_buf[2], float *const v_buf[2], float *const s1_buf[2],
                              const float *rain, float *water_depth, float *sediment, float *vel_u, float *vel_v,
                              VpScalars *sc, double *partials, bool allow_tma, int time_block, cudaStream_t s)
{
  const size_t n = (size_t)nx * ny;
  FweMaps      maps[2];
  AdvMaps      am[2];
  const bool   tma = allow_tma && fwe_maps(A, nx, ny, &maps[0]) && fwe_maps(B, nx, ny, &maps[1]);
  const bool   step_tma = tma && adv_maps(u_buf[0], v_buf[0], s1_buf[0], nx, ny, &am[0]) &&
                        adv_maps(u_buf[1], v_buf[1], s1_buf[1], nx, ny, &am[1]);
  FweIo        io;
  memset(&io, 0, sizeof io);
  io.rain = rain;
  io.maintain = p.maintain_water_volume != 0;
  io.diffusion = p.flux_diffusion != 0;
  io.pl_one = p.pipe_length == 1.f;
  io.kexp_one = p.k_discharge_exp == 1.f;
  io.tma_extra_tx = g_tma_extra_tx;
  {
    /* pair stores: an even row length and 8-byte aligned outputs */
    auto al8 = [](const void *q) { return ((uintptr_t)q & 7u) == 0; };
    const void *outs[] = {A.z,      A.d,      A.fl,     A.fr,     A.ft,      A.fb,      B.z,   B.d,   B.fl, B.fr,
                          B.ft,     B.fb,     s1_buf[0], s1_buf[1], u_buf[0], u_buf[1], v_buf[0], v_buf[1], vel_u,
                          vel_v};
    bool        ok = nx % 2 == 0;
    for (const void *q : outs) ok = ok && al8(q);
    io.vec = ok ? 1 : 0;
    /* 16-byte staging copies: a row length that is a multiple of 4 and
     * 16-byte aligned inputs */
    auto al16 = [](const void *q) { return ((uintptr_t)q & 15u) == 0; };
    const void *ins[] = {A.z, A.d, A.fl, A.fr, A.ft, A.fb, B.z,      B.d,      B.fl,     B.fr,
                         B.ft, B.fb, s1_buf[0], s1_buf[1], u_buf[0], u_buf[1], v_buf[0], v_buf[1]};
    bool        ok16 = nx % 4 == 0;
    for (const void *q : ins) ok16 = ok16 && al16(q);
    io.stage16 = ok16 ? 1 : 0;
  }
  const dim3 g1((nx + FT_TX - 1) / FT_TX, (ny + FT_TY - 1) / FT_TY);
  const int  row_groups = (ny + ADV_R - 1) / ADV_R;
  const dim3 g2((nx + 255) / 256, row_groups < 65535 ? row_groups : 65535);
  VpFields  *cur = &A, *nxt = &B;
  int        parity = 0;
  int        buf = 0; /* copy of u, v, s1 the current step writes */
  for (int it = 0; it < p.iterations; it++)
  {
    if (time_block == 2 && !io.maintain && it > 0 && it + 1 < p.iterations)
    {
      const bool last = it + 2 == p.iterations;
      TbIo       tb;
      tb.in = VpState{cur->z, cur->d, cur->s, cur->fl, cur->fr, cur->ft, cur->fb};
      tb.s1_prev = s1_buf[buf ^ 1];
      tb.u_prev = u_buf[buf ^ 1];
      tb.v_prev = v_buf[buf ^ 1];
      tb.rain = rain;
      tb.out = VpStateOut{nxt->z, nxt->d, nxt->s, nxt->fl, nxt->fr, nxt->ft, nxt->fb, nullptr, nullptr};
      tb.s1 = s1_buf[buf];
      tb.u = u_buf[buf];
      tb.v = v_buf[buf];
      tb.u_out = last ? vel_u : nullptr;
      tb.v_out = last ? vel_v : nullptr;
      tb.diffusion = io.diffusion;
      tb.pl_one = io.pl_one;
      tb.kexp_one = io.kexp_one;
      int rc = launch_vp_tb2(tb, c, s);
      if (rc) return rc;
      if (last)
      {
        k_vp_advect<ADV_R><<<g2, 256, 0, s>>>(tb.s1, tb.u, tb.v, nxt->s, c);
        HM_LAUNCH_CHECK("k_vp_advect");
      }
      VpFields *t = cur;
      cur = nxt;
      nxt = t;
      buf ^= 1;
      it++;
      continue;
    }
    const bool last = it == p.iterations - 1;
    io.in = VpState{cur->z, cur->d, cur->s, cur->fl, cur->fr, cur->ft, cur->fb};
    io.out = VpStateOut{nxt->z, nxt->d, nxt->s, nxt->fl, nxt->fr, nxt->ft, nxt->fb, nullptr, nullptr};
    io.s1 = s1_buf[buf];
    io.u = u_buf[buf];
    io.v = v_buf[buf];
    io.s1_prev = s1_buf[buf ^ 1];
    io.u_out = last ? vel_u : nullptr;
    io.v_out = last ? vel_v : nullptr;
    if (io.u_out && !io.v_out) io.v_out = io.v;
    if (io.v_out && !io.u_out) io.u_out = io.u;
    io.parity = parity;
    const FweMaps &mp = maps[cur == &A ? 0 : 1];
    int            rc;
    if (it > 0)
      rc = step_tma ? launch_step_tma(io, mp, am[buf ^ 1], c, sc, partials, g1, s)
                    : launch_step_cp_async(io, u_buf[buf ^ 1], v_buf[buf ^ 1], c, sc, partials, g1, s);
    else rc = tma ? launch_fwe_tma(io, mp, c, sc, partials, g1, s) : launch_fwe_cp_async(io, c, sc, partials, g1, s);
    if (rc) return rc;
    /* the advection of this step is folded into the next step's tiles; the
     * last step's runs here */
    if (last)
    {
      k_vp_advect<ADV_R><<<g2, 256, 0, s>>>(io.s1, io.u, io.v, nxt->s, c);
      HM_LAUNCH_CHECK("k_vp_advect");
    }
    VpFields *t = cur;
    cur = nxt;
    nxt = t;
    parity ^= 1;
    buf ^= 1;
  }
  if (cur->z != z) HM_CUDA_TRY(cudaMemcpyAsync(z, cur->z, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
  if (water_depth)
  {
    int rc = vpipes_final_depth(cur->d, rain, sc, parity, p.maintain_water_volume != 0, water_depth, n, s);
    if (rc) return rc;
  }
  if (sediment) HM_CUDA_TRY(cudaMemcpyAsync(sediment, cur->s, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
  if (p.iterations == 0)
  {
    if (vel_u) HM_CUDA_TRY(cudaMemsetAsync(vel_u, 0, n * sizeof(float), s));
    if (vel_v) HM_CUDA_TRY(cudaMemsetAsync(vel_v, 0, n * sizeof(float), s));
  }
  return HM_OK;
}

const unsigned *vpipes_error_word(const void *scratch_buf, int nx, int ny)
{
  const size_t na = align_up((size_t)nx * ny, 64);
  const char  *partials = (const char *)scratch_buf + VP_GRIDS * na * sizeof(float);
  return &((const VpScalars *)(partials + partials_bytes(nx, ny)))->error;
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
  VpFields     A, B;
  A.z = z;
  A.d = base + 0 * na;
  A.s = base + 1 * na;
  A.fl = base + 2 * na;
  A.fr = base + 3 * na;
  A.ft = base + 4 * na;
  A.fb = base + 5 * na;
  B.z = base + 6 * na;
  B.d = base + 7 * na;
  B.s = base + 8 * na;
  B.fl = base + 9 * na;
  B.fr = base + 10 * na;
  B.ft = base + 11 * na;
  B.fb = base + 12 * na;
  float *const u2[2] = {base + 13 * na, base + 16 * na};
  float *const v2[2] = {base + 14 * na, base + 17 * na};
  float *const s12[2] = {base + 15 * na, base + 18 * na};
  float       *u_buf = u2[0], *v_buf = v2[0];
  double      *partials = (double *)(base + VP_GRIDS * na);
  VpScalars *sc = (VpScalars *)((char *)partials + partials_bytes(nx, ny));
  VpDefer    df;
  df.list = (Deferred *)((char *)sc + align_up(sizeof(VpScalars), 256));
  df.count = sc->defer_count;
  df.cap = (unsigned)defer_cap(nx, ny);

  const VpConst c = vpipes_consts(nx, ny, p);
  const float   init_depth = p.initial_water < 0.f ? p.water_height : p.initial_water;

  {
    int rc = vpipes_init(A, rain, n, init_depth, sc, partials, s);
    if (rc) return rc;
  }

  const FusedCfg cfg = vpipes_pick_config(nx, ny);
  const int      algo = vpipes_pick_algo(nx, ny);
  if (algo == 0 || algo == 2 || algo == 3)
    return vpipes_tiled_steps(z, nx, ny, p, c, A, B, u2, v2, s12, rain, water_depth, sediment, vel_u, vel_v, sc,
                              partials, algo != 2, algo == 3 ? 2 : 1, s);
  VpStep         st;
  st.rain = rain;
  st.H = cfg.h;
  st.maintain = p.maintain_water_volume != 0;
  st.diffusion = p.flux_diffusion != 0;
  st.pl_one = p.pipe_length == 1.f;
  st.kexp_one = p.k_discharge_exp == 1.f;
  VpFields *cur = &A, *nxt = &B;
  int       parity = 0;
  for (int it = 0; it < p.iterations; it++)
  {
    const bool last = it == p.iterations - 1;
    st.in = VpState{cur->z, cur->d, cur->s, cur->fl, cur->fr, cur->ft, cur->fb};
    st.out = VpStateOut{nxt->z, nxt->d, nxt->s, nxt->fl, nxt->fr, nxt->ft, nxt->fb, nullptr, nullptr};
    if (last && (vel_u || vel_v))
    {
      st.out.u = vel_u ? vel_u : u_buf;
      st.out.v = vel_v ? vel_v : v_buf;
    }
    st.parity = parity;
    st.dparity = parity;
    int rc = launch_step(cfg, st, c, sc, partials, df, s);
    if (rc) return rc;
    VpFields *t = cur;
    cur = nxt;
    nxt = t;
    parity ^= 1;
  }
  if (cur->z != z) HM_CUDA_TRY(cudaMemcpyAsync(z, cur->z, n * sizeof(float), cudaMemcpyDeviceToDevice, s));

  if (water_depth)
  {
    int rc = vpipes_final_depth(cur->d, rain, sc, parity, p.maintain_water_volume != 0, water_depth, n, s);
    if (rc) return rc;
  }
  if (sediment) HM_CUDA_TRY(cudaMemcpyAsync(sediment, cur->s, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
  if (p.iterations == 0)
  {
    if (vel_u) HM_CUDA_TRY(cudaMemsetAsync(vel_u, 0, n * sizeof(float), s));
    if (vel_v) HM_CUDA_TRY(cudaMemsetAsync(vel_v, 0, n * sizeof(float), s));
  }
  return HM_OK;
}

} // namespace hm

extern "C" int hm_vpipes_set_algorithm(int algo)
{
  hm::clear_error();
  if (algo < -1 || algo > 3) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_vpipes_set_algorithm: unknown algorithm");
  hm::g_algo_override = algo;
  return HM_OK;
}

extern "C" int hm_debug_tma_expect_extra(unsigned bytes)
{
  hm::clear_error();
  if (bytes % 16u != 0u || bytes > 4096u)
    return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_debug_tma_expect_extra: bytes must be a multiple of 16, at most 4096");
  hm::g_tma_extra_tx = bytes;
  return HM_OK;
}

extern "C" int hm_vpipes_set_launch(int tpb, int radius, int rows)
{
  hm::clear_error();
  if (tpb == 0)
  {
    hm::g_cfg_override = hm::FusedCfg{0, 0, 0};
    return HM_OK;
  }
  /* rows >= 32 keeps the grid within the partial-sum buffer (partials_bytes) */
  if (!((tpb == 128 || tpb == 256) && (radius == 2 || radius == 3) && rows >= 32 && rows <= 4096))
    return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_vpipes_set_launch: unsupported launch shape");
  hm::g_cfg_override = hm::FusedCfg{tpb, radius, rows};
  return HM_OK;
}

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
