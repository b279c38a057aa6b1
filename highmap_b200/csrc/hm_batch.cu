/*
 * hm_batch.cu - many heightmaps of uneven sizes and iteration counts advanced
 * together.
 *
 * The reference solves one heightmap per call (hmap::gpu::thermal,
 * hmap::gpu::hydraulic_vpipes); a node-graph editor evaluating many
 * erosion nodes calls them one after another.  Small grids cannot fill a
 * B200 on their own, so here every admitted job's grid is cut into tiles
 * and the tiles of all jobs form one packed list:
 *   vpipes tiles  : strips of 120 output columns x 64 rows (the fused step
 *                   of hm_vpipes_fused.cuh, one tile per CTA pass);
 *   thermal tiles : strips of 128 columns x 32 rows (one Jacobi step).
 * A round advances every active job by one step: one persistent launch
 * whose CTAs (as many as fit on the device) take tiles from an atomic
 * counter, vpipes tiles first, then a fix-up launch for deferred advection
 * samples.  Jobs are listed by remaining steps, longest first, so the
 * active tiles of every round are a prefix of each list.  A job's step s
 * reads state copy s & 1 and writes the other; per-job volume sums use the
 * deterministic last-tile finish of hm_reduce.cuh.  hm_batch_run captures
 * all rounds of a batch into one CUDA graph.
 *
 * Results are bit-identical to solving each job alone (the same per-cell
 * code, the same Jacobi steps).
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "hm_internal.h"
#include "hm_thermal.h"
#include "hm_thermal_math.cuh"
#include "hm_vpipes.h"
#include "hm_vpipes_fused.cuh"

namespace hm
{

constexpr int BT = 128;  /* threads per CTA                          */
constexpr int BR = 2;    /* staged advection radius of vpipes tiles   */
constexpr int VP_H = 64; /* output rows of a vpipes tile              */
constexpr int TH_H = 32; /* rows of a thermal tile                    */
constexpr int VP_W = FusedLayout<BT, BR>::W;
constexpr int TH_W = BT;

/* device-side description of one job */
struct BJob
{
  int       kind, nx, ny, iters;
  long long start; /* global round of the job's first step */
  int       nbx, nby;
  /* thermal: tz[s & 1] holds step s */
  float       *tz[2];
  const float *talus;
  float        tv;
  const float *bed;
  int          bed_mode;
  /* vpipes: cp[s & 1] holds step s */
  VpFields     cp[2];
  VpConst      c;
  int          maintain, diffusion, pl_one, kexp_one;
  const float *rain;
  float       *u_out, *v_out;
  VpScalars   *sc;
  double      *partials;
};

/* ---- kernels ------------------------------------------------------- */

template <bool TMAP, int BED>
__device__ __forceinline__ void thermal_tile(const BJob &J, int par, int bx, int by)
{
  const int    nx = J.nx, ny = J.ny;
  const int    i = bx * TH_W + threadIdx.x;
  const int    y0 = by * TH_H, y1 = min(ny, y0 + TH_H);
  const float *__restrict__ a = J.tz[par];
  float *__restrict__ b = J.tz[par ^ 1];
  const float *__restrict__ talus = J.talus;
  const float *__restrict__ bed = J.bed;
  const float  tv = J.tv;
  if (i >= nx) return;
  for (int j = y0; j < y1; j++)
  {
    const size_t idx = (size_t)j * nx + i;
    /* apply_boundaries, _common_index.cl:106-132 */
    if (i == 0) { b[idx] = __ldg(a + idx + 1); continue; }
    if (i == nx - 1) { b[idx] = __ldg(a + idx - 1); continue; }
    if (j == 0) { b[idx] = __ldg(a + idx + nx); continue; }
    if (j == ny - 1) { b[idx] = __ldg(a + idx - nx); continue; }
    const float *up = a + idx - nx, *mid = a + idx, *dn = a + idx + nx;
    const float  t = TMAP ? __ldg(talus + idx) : tv;
    const float  zb = BED != BED_NONE ? __ldg(bed + idx) : 0.f;
    b[idx] = thermal_cell<BED>(__ldg(mid), __ldg(mid - 1), __ldg(dn), __ldg(up), __ldg(mid + 1), __ldg(up - 1),
                               __ldg(dn - 1), __ldg(up + 1), __ldg(dn + 1), t, zb);
  }
}

__device__ __forceinline__ VpStep job_step(const BJob &J, int par, int step, long long round)
{
  VpStep st;
  const VpFields &in = J.cp[par], &out = J.cp[par ^ 1];
  st.in = VpState{in.z, in.d, in.s, in.fl, in.fr, in.ft, in.fb};
  const bool last = step == J.iters - 1;
  st.out = VpStateOut{out.z, out.d, out.s, out.fl, out.fr, out.ft, out.fb, last ? J.u_out : nullptr,
                      last ? J.v_out : nullptr};
  st.rain = J.rain;
  st.parity = par;
  st.dparity = (int)(round & 1);
  st.H = VP_H;
  st.maintain = J.maintain;
  st.diffusion = J.diffusion;
  st.pl_one = J.pl_one;
  st.kexp_one = J.kexp_one;
  return st;
}

/* One round: every active tile of the packed lists, taken by persistent
 * CTAs from an atomic counter. */
__global__ void __launch_bounds__(BT)
    k_batch_round(const BJob *__restrict__ jobs,
                  const int4 *__restrict__ vt,
                  int nv,
                  const int4 *__restrict__ tt,
                  int nt,
                  long long round,
                  unsigned *counter,
                  VpDefer df)
{
  extern __shared__ float smem[];
  __shared__ int     s_tile;
  /* the current vpipes tile's job descriptor, staged in shared memory once
   * per tile (kept in a local struct, it lands on the stack and every use
   * in the row loop becomes a local-memory load) */
  __shared__ VpStep  s_st;
  __shared__ VpConst s_c;
  for (;;)
  {
    if (threadIdx.x == 0) s_tile = (int)atomicAdd(counter, 1u);
    __syncthreads();
    const int t = s_tile;
    if (t < nv && threadIdx.x == 0)
    {
      const BJob &J = jobs[vt[t].x];
      const int   step = (int)(round - J.start);
      s_st = job_step(J, step & 1, step, round);
      s_c = J.c;
    }
    __syncthreads();
    if (t >= nv + nt) return;
    if (t < nv)
    {
      const int4  tl = vt[t];
      const BJob &J = jobs[tl.x];
      VpScalars  *sc = J.sc;
      double     *partials = J.partials;
      const int   nbx = J.nbx, nby = J.nby;
      if (s_st.maintain) vp_tile<BT, BR, true>(s_st, s_c, sc, partials, df, (unsigned)tl.x, tl.y, tl.z, nbx, nby, smem);
      else vp_tile<BT, BR, false>(s_st, s_c, sc, partials, df, (unsigned)tl.x, tl.y, tl.z, nbx, nby, smem);
    }
    else
    {
      const int4  tl = tt[t - nv];
      const BJob &J = jobs[tl.x];
      const int   par = (int)((round - J.start) & 1);
      const int   mode = J.bed ? (J.bed_mode == HM_BEDROCK_LITERAL ? BED_LITERAL : BED_INTENDED) : BED_NONE;
      if (J.talus)
      {
        if (mode == BED_NONE) thermal_tile<true, BED_NONE>(J, par, tl.y, tl.z);
        else if (mode == BED_INTENDED) thermal_tile<true, BED_INTENDED>(J, par, tl.y, tl.z);
        else thermal_tile<true, BED_LITERAL>(J, par, tl.y, tl.z);
      }
      else
      {
        if (mode == BED_NONE) thermal_tile<false, BED_NONE>(J, par, tl.y, tl.z);
        else if (mode == BED_INTENDED) thermal_tile<false, BED_INTENDED>(J, par, tl.y, tl.z);
        else thermal_tile<false, BED_LITERAL>(J, par, tl.y, tl.z);
      }
    }
  }
}

/* Deferred advection samples of the round, any job; re-arms the other
 * round parity's counter. */
__global__ void __launch_bounds__(128) k_batch_fixup(const BJob *__restrict__ jobs, long long round, VpDefer df)
{
  const int      dpar = (int)(round & 1);
  const unsigned n = min(df.count[dpar], df.cap);
  if (blockIdx.x == 0 && threadIdx.x == 0) df.count[dpar ^ 1] = 0u;
  for (unsigned e = blockIdx.x * 128 + threadIdx.x; e < n; e += gridDim.x * 128)
  {
    const Deferred d = df.list[e];
    const BJob    &J = jobs[d.job];
    const int      step = (int)(round - J.start);
    const int      par = step & 1;
    const VpStep   st = job_step(J, par, step, round);
    const float    add = J.maintain ? J.sc->add[par] : 0.f;
    const float    rvol = J.maintain ? J.sc->rvol : 1.f;
    const Glob     g{st, J.c, add, rvol};
    const int      gj = (int)(d.k / (unsigned)J.nx), gi = (int)(d.k - (unsigned)gj * (unsigned)J.nx);
    st.out.s[d.k] = advect_global(g, gi, gj, d.u, d.v);
  }
}

} // namespace hm

/* ---- host side ---------------------------------------------------------- */

namespace
{

using hm::align_up;

struct HJob
{
  hm_job    desc;
  hm::BJob  dev;
  void     *mem = nullptr; /* device state, one allocation */
  size_t    bytes = 0;
  int       steps = 0;
  bool      live = false;     /* admitted and not released */
  bool      finished = false; /* outputs written            */
  float    *z0 = nullptr;     /* thermal input copy for the deposition map */
};

size_t job_bytes(const hm_job &j)
{
  const size_t n = align_up((size_t)j.nx * j.ny, 64) * sizeof(float);
  if (j.kind == HM_JOB_THERMAL) return n * (1 + (j.deposition_map ? 1 : 0));
  const size_t tiles = (size_t)((j.nx + hm::VP_W - 1) / hm::VP_W) * ((j.ny + hm::VP_H - 1) / hm::VP_H);
  const size_t parts = std::max(tiles, hm::vpipes_init_partials());
  return n * 13 + align_up(parts * sizeof(double), 256) + align_up(sizeof(hm::VpScalars), 256);
}

int check_job(const hm_job &j)
{
  if (j.kind != HM_JOB_THERMAL && j.kind != HM_JOB_VPIPES)
    return hm::fail(HM_ERR_INVALID_ARGUMENT, "batch: unknown job kind");
  if (!j.z) return hm::fail(HM_ERR_INVALID_ARGUMENT, "batch: job z is NULL");
  if (j.iterations < 0) return hm::fail(HM_ERR_INVALID_ARGUMENT, "batch: iterations < 0");
  if (j.kind == HM_JOB_THERMAL)
  {
    hm_thermal_options o;
    hm_thermal_default_options(&o);
    o.bedrock_mode = j.bedrock_mode;
    return hm::thermal_check_args(j.z, j.nx, j.ny, j.iterations, &o);
  }
  hm_vpipes_params p = j.vpipes;
  p.iterations = j.iterations;
  return hm::vpipes_check_args(j.z, j.nx, j.ny, &p);
}

} // namespace

struct hm_batch
{
  hm_context       *ctx = nullptr;
  int               device = 0;
  cudaStream_t      stream = nullptr;
  std::vector<HJob> jobs;
  long long         round = 0;
  int               grid_cap = 0; /* persistent CTAs */
  size_t            smem = 0;
  /* device tables */
  hm::BJob         *d_jobs = nullptr;
  size_t            d_jobs_cap = 0;
  int4             *d_tiles = nullptr;
  size_t            d_tiles_cap = 0;
  unsigned         *d_counters = nullptr;
  size_t            counters_cap = 0;
  hm::Deferred     *d_defer = nullptr;
  unsigned         *d_defer_count = nullptr;
  unsigned          defer_cap = 0;
  bool              dirty = true;
};

namespace
{

template <class T>
int grow(T **p, size_t *cap, size_t want, cudaStream_t s)
{
  if (*cap >= want) return HM_OK;
  size_t n = std::max(want, *cap * 2);
  if (*p) HM_CUDA_TRY(cudaFreeAsync(*p, s));
  *p = nullptr;
  cudaError_t e = cudaMallocAsync((void **)p, n * sizeof(T), s);
  if (e != cudaSuccess)
  {
    cudaGetLastError();
    *cap = 0;
    return hm::cuda_fail(e, "batch table allocation");
  }
  *cap = n;
  return HM_OK;
}

int upload_jobs(hm_batch *b)
{
  if (!b->dirty) return HM_OK;
  std::vector<hm::BJob> host(b->jobs.size());
  for (size_t k = 0; k < b->jobs.size(); k++) host[k] = b->jobs[k].dev;
  int st = grow(&b->d_jobs, &b->d_jobs_cap, std::max<size_t>(host.size(), 1), b->stream);
  if (st) return st;
  if (!host.empty())
    HM_CUDA_TRY(cudaMemcpyAsync(b->d_jobs, host.data(), host.size() * sizeof(hm::BJob), cudaMemcpyHostToDevice,
                                b->stream));
  /* the pageable source must stay valid until the copy is done */
  HM_CUDA_TRY(cudaStreamSynchronize(b->stream));
  b->dirty = false;
  return HM_OK;
}

int finalize_job(hm_batch *b, HJob &h)
{
  const hm_job &j = h.desc;
  const size_t  n = (size_t)j.nx * j.ny;
  const int     par = j.iterations & 1;
  cudaStream_t  s = b->stream;
  if (j.kind == HM_JOB_THERMAL)
  {
    if (par) HM_CUDA_TRY(cudaMemcpyAsync(j.z, h.dev.tz[1], n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    int rc = hm::thermal_finish(b->device, j.z, j.nx, j.ny, h.z0, j.deposition_map, nullptr, s);
    if (rc) return rc;
  }
  else
  {
    const hm::VpFields &f = h.dev.cp[par];
    if (f.z != j.z) HM_CUDA_TRY(cudaMemcpyAsync(j.z, f.z, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    if (j.water_depth)
    {
      int rc = hm::vpipes_final_depth(f.d, j.rain_map, h.dev.sc, par, h.dev.maintain != 0, j.water_depth, n, s);
      if (rc) return rc;
    }
    if (j.sediment) HM_CUDA_TRY(cudaMemcpyAsync(j.sediment, f.s, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    if (j.iterations == 0)
    {
      if (j.vel_u) HM_CUDA_TRY(cudaMemsetAsync(j.vel_u, 0, n * sizeof(float), s));
      if (j.vel_v) HM_CUDA_TRY(cudaMemsetAsync(j.vel_v, 0, n * sizeof(float), s));
    }
  }
  h.finished = true;
  return HM_OK;
}

/* The rounds of one step call, in three phases so that hm_batch_run can
 * capture the device work of the middle one into a CUDA graph:
 *   plan   : tile lists by remaining steps, uploads (host side, not
 *            capturable: pageable copies and the job-table sync);
 *   launch : counters, round and fix-up kernels, finalisation of the jobs
 *            that complete (device work on b->stream only);
 *   commit : step counts. */
struct Plan
{
  std::vector<int>  act;
  std::vector<int>  vrem, trem;
  size_t            nv = 0, nt = 0;
  int               N = 0;
};

int plan_rounds(hm_batch *b, int rounds, Plan &pl)
{
  for (size_t k = 0; k < b->jobs.size(); k++)
    if (b->jobs[k].live && !b->jobs[k].finished) pl.act.push_back((int)k);
  auto remaining = [&](int k) { return b->jobs[k].desc.iterations - b->jobs[k].steps; };
  std::stable_sort(pl.act.begin(), pl.act.end(), [&](int x, int y) { return remaining(x) > remaining(y); });
  int maxrem = 0;
  for (int k : pl.act) maxrem = std::max(maxrem, remaining(k));
  pl.N = std::min(rounds, maxrem);

  /* packed tile lists: vpipes then thermal, each longest-remaining first */
  std::vector<int4> vt, tt;
  for (int k : pl.act)
  {
    const HJob &h = b->jobs[k];
    for (int by = 0; by < h.dev.nby; by++)
      for (int bx = 0; bx < h.dev.nbx; bx++)
      {
        if (h.desc.kind == HM_JOB_VPIPES)
        {
          vt.push_back(make_int4(k, bx, by, 0));
          pl.vrem.push_back(remaining(k));
        }
        else
        {
          tt.push_back(make_int4(k, bx, by, 0));
          pl.trem.push_back(remaining(k));
        }
      }
  }
  pl.nv = vt.size();
  pl.nt = tt.size();
  int st;
  if ((st = upload_jobs(b))) return st;
  if (pl.N == 0) return HM_OK;
  if ((st = grow(&b->d_tiles, &b->d_tiles_cap, std::max<size_t>(pl.nv + pl.nt, 1), b->stream))) return st;
  if ((st = grow(&b->d_counters, &b->counters_cap, (size_t)pl.N, b->stream))) return st;
  std::vector<int4> all(vt);
  all.insert(all.end(), tt.begin(), tt.end());
  /* pageable source: the call returns once the data is staged */
  if (!all.empty())
    HM_CUDA_TRY(cudaMemcpyAsync(b->d_tiles, all.data(), all.size() * sizeof(int4), cudaMemcpyHostToDevice, b->stream));
  return HM_OK;
}

int launch_rounds(hm_batch *b, const Plan &pl)
{
  if (pl.N > 0)
  {
    HM_CUDA_TRY(cudaMemsetAsync(b->d_counters, 0, (size_t)pl.N * sizeof(unsigned), b->stream));
    hm::VpDefer df{b->d_defer, b->d_defer_count, b->defer_cap};
    size_t      iv = pl.nv, it = pl.nt;
    for (int r = 0; r < pl.N; r++)
    {
      /* tiles whose job still has steps left at this round */
      while (iv > 0 && pl.vrem[iv - 1] <= r) iv--;
      while (it > 0 && pl.trem[it - 1] <= r) it--;
      const int total = (int)(iv + it);
      const int grid = std::max(1, std::min(b->grid_cap, total));
      hm::k_batch_round<<<grid, hm::BT, b->smem, b->stream>>>(b->d_jobs, b->d_tiles, (int)iv, b->d_tiles + pl.nv,
                                                              (int)it, b->round + r, b->d_counters + r, df);
      HM_LAUNCH_CHECK("k_batch_round");
      if (iv > 0)
      {
        hm::k_batch_fixup<<<2 * 148, 128, 0, b->stream>>>(b->d_jobs, b->round + r, df);
        HM_LAUNCH_CHECK("k_batch_fixup");
      }
    }
  }
  for (int k : pl.act)
  {
    HJob     &h = b->jobs[k];
    const int rem = h.desc.iterations - h.steps;
    if (rem <= pl.N)
    {
      int st = finalize_job(b, h);
      if (st) return st;
    }
  }
  return HM_OK;
}

void commit_rounds(hm_batch *b, const Plan &pl)
{
  b->round += pl.N;
  for (int k : pl.act)
  {
    HJob &h = b->jobs[k];
    h.steps += std::min(pl.N, h.desc.iterations - h.steps);
  }
}

int run_rounds(hm_batch *b, int rounds)
{
  Plan pl;
  int  st = plan_rounds(b, rounds, pl);
  if (!st) st = launch_rounds(b, pl);
  if (!st) commit_rounds(b, pl);
  return st;
}

} // namespace

extern "C" {

int hm_batch_create(hm_context *ctx, hm_batch **out)
{
  hm::clear_error();
  if (!ctx || !out) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_batch_create: NULL argument");
  *out = nullptr;
  int st = hm::use_device(ctx->device);
  if (st) return st;
  hm_batch *b = new (std::nothrow) hm_batch();
  if (!b) return hm::fail(HM_ERR_OUT_OF_MEMORY, "hm_batch_create: host allocation failed");
  b->ctx = ctx;
  b->device = ctx->device;
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess)
  {
    delete b;
    return hm::cuda_fail(e, "hm_batch_create: cudaStreamCreate");
  }
  b->smem = hm::FusedLayout<hm::BT, hm::BR>::SMEM;
  int per_sm = 0, sms = 0;
  HM_CUDA_TRY(cudaFuncSetAttribute(hm::k_batch_round, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem));
  HM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hm::k_batch_round, hm::BT, b->smem));
  HM_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
  b->grid_cap = std::max(1, per_sm) * std::max(1, sms);
  b->defer_cap = 1u << 16;
  HM_CUDA_TRY(cudaMallocAsync((void **)&b->d_defer, b->defer_cap * sizeof(hm::Deferred), b->stream));
  HM_CUDA_TRY(cudaMallocAsync((void **)&b->d_defer_count, 2 * sizeof(unsigned), b->stream));
  HM_CUDA_TRY(cudaMemsetAsync(b->d_defer_count, 0, 2 * sizeof(unsigned), b->stream));
  *out = b;
  return HM_OK;
}

size_t hm_batch_job_bytes(const hm_job *job) { return job ? job_bytes(*job) : 0; }

int hm_batch_add(hm_batch *b, const hm_job *job, int *job_id)
{
  hm::clear_error();
  if (!b || !job || !job_id) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_batch_add: NULL argument");
  int st = check_job(*job);
  if (st) return st;
  if ((st = hm::use_device(b->device))) return st;
  HJob h;
  h.desc = *job;
  h.bytes = job_bytes(*job);
  cudaError_t e = cudaMallocAsync(&h.mem, h.bytes, b->stream);
  if (e != cudaSuccess)
  {
    cudaGetLastError();
    return hm::cuda_fail(e, "hm_batch_add: job state allocation");
  }
  const size_t na = align_up((size_t)job->nx * job->ny, 64);
  float       *base = (float *)h.mem;
  hm::BJob    &d = h.dev;
  memset(&d, 0, sizeof(d));
  d.kind = job->kind;
  d.nx = job->nx;
  d.ny = job->ny;
  d.iters = job->iterations;
  d.start = b->round;
  if (job->kind == HM_JOB_THERMAL)
  {
    d.nbx = (job->nx + hm::TH_W - 1) / hm::TH_W;
    d.nby = (job->ny + hm::TH_H - 1) / hm::TH_H;
    d.tz[0] = job->z;
    d.tz[1] = base;
    d.talus = job->talus;
    d.tv = job->talus_value;
    d.bed = job->bedrock;
    d.bed_mode = job->bedrock_mode;
    if (job->deposition_map)
    {
      h.z0 = base + na;
      HM_CUDA_TRY(cudaMemcpyAsync(h.z0, job->z, (size_t)job->nx * job->ny * sizeof(float),
                                  cudaMemcpyDeviceToDevice, b->stream));
    }
  }
  else
  {
    hm_vpipes_params p = job->vpipes;
    p.iterations = job->iterations;
    d.nbx = (job->nx + hm::VP_W - 1) / hm::VP_W;
    d.nby = (job->ny + hm::VP_H - 1) / hm::VP_H;
    hm::VpFields A{job->z, base + 0 * na, base + 1 * na, base + 2 * na, base + 3 * na, base + 4 * na, base + 5 * na};
    hm::VpFields B{base + 6 * na, base + 7 * na, base + 8 * na, base + 9 * na, base + 10 * na, base + 11 * na,
                   base + 12 * na};
    d.cp[0] = A;
    d.cp[1] = B;
    d.c = hm::vpipes_consts(job->nx, job->ny, p);
    d.maintain = p.maintain_water_volume != 0;
    d.diffusion = p.flux_diffusion != 0;
    d.pl_one = p.pipe_length == 1.f;
    d.kexp_one = p.k_discharge_exp == 1.f;
    d.rain = job->rain_map;
    d.u_out = job->vel_u;
    d.v_out = job->vel_v;
    d.partials = (double *)(base + 13 * na);
    const size_t tiles = (size_t)d.nbx * d.nby;
    const size_t parts = std::max(tiles, hm::vpipes_init_partials());
    d.sc = (hm::VpScalars *)((char *)d.partials + align_up(parts * sizeof(double), 256));
    const float init_depth = p.initial_water < 0.f ? p.water_height : p.initial_water;
    if ((st = hm::vpipes_init(A, job->rain_map, (size_t)job->nx * job->ny, init_depth, d.sc, d.partials, b->stream)))
      return st;
  }
  h.live = true;
  b->jobs.push_back(h);
  b->dirty = true;
  /* deferred-advection list: room for 1/32 of the admitted vpipes cells
   * (the same share as a single solve); overflowing samples would be
   * resolved inline, stalling their CTA */
  if (job->kind == HM_JOB_VPIPES)
  {
    size_t cells = 0;
    for (const HJob &x : b->jobs)
      if (x.live && x.desc.kind == HM_JOB_VPIPES) cells += (size_t)x.desc.nx * x.desc.ny;
    const size_t want = std::max<size_t>(1u << 16, cells / 32);
    if (want > b->defer_cap)
    {
      /* the list is empty between rounds: reallocation only has to be
       * ordered after the work already queued */
      HM_CUDA_TRY(cudaFreeAsync(b->d_defer, b->stream));
      b->d_defer = nullptr;
      const size_t cap = want + want / 2;
      e = cudaMallocAsync((void **)&b->d_defer, cap * sizeof(hm::Deferred), b->stream);
      if (e != cudaSuccess)
      {
        cudaGetLastError();
        b->defer_cap = 0;
        return hm::cuda_fail(e, "hm_batch_add: deferred list allocation");
      }
      b->defer_cap = (unsigned)cap;
    }
  }
  *job_id = (int)b->jobs.size() - 1;
  if (job->iterations == 0) return finalize_job(b, b->jobs.back());
  return HM_OK;
}

int hm_batch_step(hm_batch *b, int rounds)
{
  hm::clear_error();
  if (!b || rounds < 0) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_batch_step: bad argument");
  int st = hm::use_device(b->device);
  if (st) return st;
  return run_rounds(b, rounds);
}

int hm_batch_synchronize(hm_batch *b)
{
  if (!b) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_batch_synchronize: NULL batch");
  HM_CUDA_TRY(cudaStreamSynchronize(b->stream));
  return HM_OK;
}

int hm_batch_job_status(hm_batch *b, int job_id, int *steps_done, int *finished)
{
  if (!b || job_id < 0 || job_id >= (int)b->jobs.size())
    return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_batch_job_status: unknown job");
  if (steps_done) *steps_done = b->jobs[job_id].steps;
  if (finished) *finished = b->jobs[job_id].finished ? 1 : 0;
  return HM_OK;
}

int hm_batch_release(hm_batch *b, int job_id)
{
  if (!b || job_id < 0 || job_id >= (int)b->jobs.size() || !b->jobs[job_id].live)
    return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_batch_release: unknown job");
  HJob &h = b->jobs[job_id];
  if (h.mem) HM_CUDA_TRY(cudaFreeAsync(h.mem, b->stream));
  h.mem = nullptr;
  h.live = false;
  h.finished = true;
  return HM_OK;
}

size_t hm_batch_bytes_in_use(const hm_batch *b)
{
  if (!b) return 0;
  size_t t = 0;
  for (const HJob &h : b->jobs)
    if (h.live) t += h.bytes;
  return t;
}

long long hm_batch_round(const hm_batch *b) { return b ? b->round : -1; }

int hm_batch_destroy(hm_batch *b)
{
  if (!b) return HM_OK;
  hm::use_device(b->device);
  for (HJob &h : b->jobs)
    if (h.mem) cudaFreeAsync(h.mem, b->stream);
  if (b->d_jobs) cudaFreeAsync(b->d_jobs, b->stream);
  if (b->d_tiles) cudaFreeAsync(b->d_tiles, b->stream);
  if (b->d_counters) cudaFreeAsync(b->d_counters, b->stream);
  if (b->d_defer) cudaFreeAsync(b->d_defer, b->stream);
  if (b->d_defer_count) cudaFreeAsync(b->d_defer_count, b->stream);
  cudaStreamSynchronize(b->stream);
  cudaStreamDestroy(b->stream);
  delete b;
  return HM_OK;
}

int hm_batch_run(hm_context *ctx, const hm_job *jobs, int njobs, int use_graph)
{
  hm::clear_error();
  if (!ctx || (njobs > 0 && !jobs) || njobs < 0) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_batch_run: bad argument");
  hm_batch *b = nullptr;
  int       st = hm_batch_create(ctx, &b);
  if (st) return st;
  int maxit = 0;
  for (int k = 0; k < njobs && !st; k++)
  {
    int id;
    st = hm_batch_add(b, &jobs[k], &id);
    maxit = std::max(maxit, jobs[k].iterations);
  }
  if (!st) st = upload_jobs(b);
  if (!st && use_graph && maxit > 0)
  {
    /* every round of the batch in one graph; the host-side plan (tile
     * lists, uploads) is made before the capture */
    Plan            pl;
    cudaGraph_t     graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    st = plan_rounds(b, maxit, pl);
    if (!st) st = hm_batch_synchronize(b);
    cudaError_t e = cudaSuccess;
    if (!st)
    {
      e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) st = hm::cuda_fail(e, "hm_batch_run: cudaStreamBeginCapture");
    }
    if (!st)
    {
      int rc = launch_rounds(b, pl);
      e = cudaStreamEndCapture(b->stream, &graph);
      if (rc) st = rc;
      else if (e != cudaSuccess) st = hm::cuda_fail(e, "hm_batch_run: cudaStreamEndCapture");
      if (!st) commit_rounds(b, pl);
    }
    if (!st)
    {
      e = cudaGraphInstantiate(&exec, graph, 0);
      if (e != cudaSuccess) st = hm::cuda_fail(e, "hm_batch_run: cudaGraphInstantiate");
    }
    if (!st)
    {
      e = cudaGraphLaunch(exec, b->stream);
      if (e != cudaSuccess) st = hm::cuda_fail(e, "hm_batch_run: cudaGraphLaunch");
      hm::count_launch(0);
    }
    if (!st) st = hm_batch_synchronize(b);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
  else if (!st)
  {
    st = run_rounds(b, maxit);
    if (!st) st = hm_batch_synchronize(b);
  }
  int st2 = hm_batch_destroy(b);
  return st ? st : st2;
}

} // extern "C"
