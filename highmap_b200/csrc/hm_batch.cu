/*
 * hm_batch.cu - many heightmaps of uneven sizes and iteration counts advanced
 * together.
 *
 * The reference solves one heightmap per call (hmap::gpu::thermal,
 * hmap::gpu::hydraulic_vpipes); a node-graph editor evaluating many
 * erosion nodes calls them one after another.  Small grids cannot fill a
 * B200 on their own, so here every admitted job's grid is cut into tiles
 * and the tiles of all jobs form packed lists:
 *   vpipes tiles  : 32 x 16 tiles of a step (hm_vpipes_tiled.cuh,
 *                   cp.async staging, in 16-byte copies where the tile's
 *                   boxes lie inside an aligned grid): the first step's
 *                   flow / water / erosion, and for every later step the
 *                   previous step's advection folded into the same tile;
 *   thermal tiles : th_rows rows of 512 columns, a warp per 64 (column
 *                   pairs, for even rows on aligned grids) or of 256
 *                   columns, a warp per 32 (hm_thermal_sweep.cuh).
 * A round advances every active job by one step: ONE persistent launch
 * whose CTAs take vpipes and thermal tiles from an atomic counter.  A
 * vpipes job's last advection runs when the job finishes.  Jobs are
 * listed by remaining steps, longest first, so the active tiles of every
 * round are a prefix of each list.  A job's step s reads state copy s & 1
 * and writes the other, and writes copy s & 1 of its s1, u, v while its
 * tiles gather the previous step's from the other; per-job volume sums use
 * the deterministic last-tile finish of hm_reduce.cuh.  hm_batch_run
 * captures all rounds of a batch into one CUDA graph.  The persistent CTA
 * count and the thermal tile's rows come from the autotuner
 * (hm_autotune with HM_TUNE_BATCH) or a built-in choice.
 *
 * Results are bit-identical to solving each job alone (the same per-cell
 * code, the same Jacobi steps).
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "hm_internal.h"
#include "hm_thermal.h"
#include "hm_thermal_math.cuh"
#include "hm_thermal_sweep.cuh"
#include "hm_tune.h"
#include "hm_vpipes.h"
#include "hm_vpipes_tiled.cuh"

namespace hm
{

constexpr int BT = FT_NT;  /* threads per CTA (8 warps)                  */
constexpr int TH_W = 256;  /* thermal tile: a warp per 32 columns        */
/* Resident CTAs per SM the round kernel is compiled for, and the rows
 * whose loads a thermal tile's sweep keeps in flight (one column per lane,
 * column pairs).  The plain sweeps' 8 and 4 rows need 80 registers here,
 * three CTAs per SM; with 4 and 2 the kernel fits 64 registers (a few
 * words spill) and four CTAs, whose extra warps hide the latency instead:
 * 8 % less time for the round graphs of the 206 jobs under 1024^2 cells of
 * the batched benchmark's mix. */
constexpr int BATCH_CTAS_PER_SM = 4;
/* built-in launch of the rounds: one CTA per tile (true) or persistent
 * CTAs taking tiles from a counter (false) */
constexpr bool BATCH_ONE_TILE = false;
constexpr int BATCH_TH_ROWS_1 = 4, BATCH_TH_ROWS_2 = 2;

/* device-side description of one job */
struct BJob
{
  int       kind, nx, ny, iters;
  long long start; /* global round of the job's first step */
  int       nbx, nby;   /* vpipes step or thermal tiles */
  int       th_rows;    /* rows of a thermal tile */
  /* thermal: tz[s & 1] holds step s */
  float       *tz[2];
  const float *talus;
  float        tv;
  const float *bed;
  int          bed_mode;
  int          pairs; /* column-pair sweep (even nx, 8-byte aligned grids) */
  /* vpipes: cp[s & 1] holds step s; step s writes s1[s & 1], u[s & 1],
   * v[s & 1] (its eroded sediment and velocity), which step s + 1's tiles
   * advect */
  VpFields     cp[2];
  float       *s1[2], *u[2], *v[2];
  VpConst      c;
  int          maintain, diffusion, pl_one, kexp_one;
  int          vec; /* pair stores (even nx, 8-byte aligned outputs) */
  int          stage16; /* 16-byte staging copies (nx % 4 == 0, 16-byte aligned grids) */
  const float *rain;
  float       *u_out, *v_out;
  VpScalars   *sc;
  double      *partials;
};

/* ---- kernels ------------------------------------------------------- */

/* the fwe inputs of step `step` of vpipes job J */
__device__ __forceinline__ void job_io(const BJob &J, int step, FweIo &io)
{
  const int       par = step & 1;
  const VpFields &in = J.cp[par], &out = J.cp[par ^ 1];
  io.in = VpState{in.z, in.d, in.s, in.fl, in.fr, in.ft, in.fb};
  io.out = VpStateOut{out.z, out.d, out.s, out.fl, out.fr, out.ft, out.fb, nullptr, nullptr};
  io.s1 = J.s1[par];
  io.u = J.u[par];
  io.v = J.v[par];
  io.s1_prev = J.s1[par ^ 1];
  io.rain = J.rain;
  io.parity = par;
  io.maintain = J.maintain;
  io.diffusion = J.diffusion;
  io.pl_one = J.pl_one;
  io.kexp_one = J.kexp_one;
  const bool last = step == J.iters - 1;
  io.u_out = last ? J.u_out : nullptr;
  io.v_out = last ? J.v_out : nullptr;
  if (io.u_out && !io.v_out) io.v_out = io.v;
  if (io.v_out && !io.u_out) io.u_out = io.u;
  io.vec = J.vec;
  io.stage16 = J.stage16;
  io.flow_only = 0;
}

template <bool TMAP, int BED>
__device__ __forceinline__ void thermal_tile(const BJob &J, int par, int bx, int by)
{
  const int y0 = by * J.th_rows, y1 = min(J.ny, y0 + J.th_rows);
  if (J.pairs)
  {
    const int wx = bx * 2 * TH_W + (threadIdx.x >> 5) * 64;
    if (wx < J.nx) /* whole warp */
      thermal_sweep2_warp<TMAP, TalusExchange<BED>, BATCH_TH_ROWS_2>(
          J.tz[par], J.tz[par ^ 1], J.nx, J.ny, J.talus, J.tv, J.bed, 0, wx, y0, y1);
    return;
  }
  const int wx = bx * TH_W + (threadIdx.x >> 5) * 32;
  if (wx < J.nx) /* whole warp */
    thermal_sweep_warp<TMAP, TalusExchange<BED>, BATCH_TH_ROWS_1>(
        J.tz[par], J.tz[par ^ 1], J.nx, J.ny, J.talus, J.tv, J.bed, 0, wx, y0, y1);
}

/* One round: every active vpipes tile and thermal tile, taken by
 * persistent CTAs from an atomic counter.  A vpipes tile of a job's first
 * step stages the job's sediment; later steps advect the previous step's
 * eroded sediment into the tile (fwe_stage_cp_async_step, advect_region1).
 * F: FWE_RTOPTS when every active vpipes job has pipe length 1 and
 * discharge exponent 1 (the lean form without fp64 pow), else FWE_GENERIC;
 * both compiled for BATCH_CTAS_PER_SM CTAs per SM.  PERSIST: thread 0
 * takes the CTA's next tile index while the current tile is computed, so
 * the atomic's latency is hidden.  Without it the grid has one CTA per
 * tile of the round and CTA b takes tile b (counter unused): the block
 * scheduler starts a tile whenever a CTA slot frees, and a tile's staging
 * wait overlaps the other resident CTAs' tiles, as in the plain step
 * kernels. */
template <int F, bool PERSIST>
__global__ void __launch_bounds__(BT, BATCH_CTAS_PER_SM)
    k_batch_round(const BJob *__restrict__ jobs,
                  const int4 *__restrict__ vt,
                  int nv,
                  const int4 *__restrict__ tt,
                  int nt,
                  long long round,
                  unsigned *counter)
{
  __shared__ FweSmem sm;
  __shared__ int            s_tile;
  /* the current vpipes tile's step description, staged once per tile */
  __shared__ FweIo   s_io;
  __shared__ VpConst s_c;
  __shared__ int     s_step;
  int                next = PERSIST ? (threadIdx.x == 0 ? (int)atomicAdd(counter, 1u) : 0) : (int)blockIdx.x;
  for (;;)
  {
    __syncthreads(); /* the previous tile is done with the shared state */
    if (threadIdx.x == 0)
    {
      const int t = next;
      s_tile = t;
      if (!PERSIST) next = nv + nt; /* one tile: the next iteration returns */
      else if (t < nv + nt) next = (int)atomicAdd(counter, 1u); /* used by the next iteration */
      if (t < nv)
      {
        const BJob &J = jobs[vt[t].x];
        s_step = (int)(round - J.start);
        job_io(J, s_step, s_io);
        s_c = J.c;
      }
    }
    __syncthreads();
    const int t = s_tile;
    if (t >= nv + nt) return;
    if (t < nv)
    {
      const int4  tl = vt[t];
      const BJob &J = jobs[tl.x];
      const int   x0 = tl.y * FT_TX, y0 = tl.z * FT_TY;
      const int   step = s_step;
      if (step == 0)
        fwe_stage_cp_async(s_io, J.nx, J.ny, x0, y0, sm);
      else if (stage16_tile(s_io, J.nx, J.ny, x0, y0))
        fwe_stage_cp_async16_step(s_io, J.u[(step & 1) ^ 1], J.v[(step & 1) ^ 1], J.nx, x0, y0, sm);
      else
        fwe_stage_cp_async_step(s_io, J.u[(step & 1) ^ 1], J.v[(step & 1) ^ 1], J.nx, J.ny, x0, y0, sm);
      __syncthreads();
      if (step > 0) advect_region1<false>(s_c, s_io.s1_prev, x0, y0, sm);
      if (J.maintain)
        fwe_compute<true, F>(s_io, s_c, J.sc, J.partials, tl.y, tl.z, J.nbx, J.nby, sm);
      else
        fwe_compute<false, F>(s_io, s_c, J.sc, J.partials, tl.y, tl.z, J.nbx, J.nby, sm);
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
  bool      evicted = false;  /* state held by the caller (hm_batch_evict) */
  uintptr_t dev_block = 0;    /* device address of the state block the descriptor points into */
  float    *z0 = nullptr;     /* thermal input copy for the deposition map */
};

/* a vpipes job's grids allow 16-byte staging copies (rows a multiple of 4
 * floats, every staged grid 16-byte aligned) */
int stage16_ok(const hm::BJob &d)
{
  auto al16 = [](const void *q) { return ((uintptr_t)q & 15u) == 0; };
  if (d.nx % 4 != 0) return 0;
  for (const hm::VpFields &f : d.cp)
    for (const void *q : {(const void *)f.z, (const void *)f.d, (const void *)f.fl, (const void *)f.fr,
                          (const void *)f.ft, (const void *)f.fb})
      if (!al16(q)) return 0;
  for (int k = 0; k < 2; k++)
    if (!al16(d.s1[k]) || !al16(d.u[k]) || !al16(d.v[k])) return 0;
  return 1;
}

/* the pointer p moved with its block from old_base to new_base, if it
 * points into the bytes-long block */
template <class T>
void rebase(T *&p, uintptr_t old_base, size_t bytes, char *new_base)
{
  const uintptr_t q = (uintptr_t)p;
  if (p && q >= old_base && q < old_base + bytes) p = (T *)(new_base + (q - old_base));
}

/* every pointer of a job's descriptor into its state block, moved to the
 * block's new address */
void rebase_job(HJob &h, uintptr_t old_base, char *new_base)
{
  const size_t n = h.bytes;
  hm::BJob    &d = h.dev;
  for (auto &t : d.tz) rebase(t, old_base, n, new_base);
  for (auto &f : d.cp)
  {
    rebase(f.z, old_base, n, new_base);
    rebase(f.d, old_base, n, new_base);
    rebase(f.s, old_base, n, new_base);
    rebase(f.fl, old_base, n, new_base);
    rebase(f.fr, old_base, n, new_base);
    rebase(f.ft, old_base, n, new_base);
    rebase(f.fb, old_base, n, new_base);
  }
  for (int k = 0; k < 2; k++)
  {
    rebase(d.s1[k], old_base, n, new_base);
    rebase(d.u[k], old_base, n, new_base);
    rebase(d.v[k], old_base, n, new_base);
  }
  rebase(d.partials, old_base, n, new_base);
  rebase(d.sc, old_base, n, new_base);
  rebase(h.z0, old_base, n, new_base);
  if (h.desc.kind == HM_JOB_VPIPES) d.stage16 = stage16_ok(d);
}

size_t job_bytes(const hm_job &j)
{
  const size_t n = align_up((size_t)j.nx * j.ny, 64) * sizeof(float);
  if (j.kind == HM_JOB_THERMAL) return n * (1 + (j.deposition_map ? 1 : 0));
  const size_t tiles = (size_t)((j.nx + hm::FT_TX - 1) / hm::FT_TX) * ((j.ny + hm::FT_TY - 1) / hm::FT_TY);
  const size_t parts = std::max(tiles, hm::vpipes_init_partials());
  /* state copies A (but z) and B, two copies of s1, u, v */
  return n * 19 + align_up(parts * sizeof(double), 256) + align_up(sizeof(hm::VpScalars), 256);
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

namespace
{
struct TileLists;
}

struct hm_batch
{
  hm_context       *ctx = nullptr;
  int               device = 0;
  cudaStream_t      stream = nullptr;
  std::vector<HJob> jobs;
  long long         round = 0;
  int               grid_cap = 0; /* persistent CTAs of k_batch_round<FWE_RTOPTS>  */
  int               grid_cap_gen = 0; /* persistent CTAs of k_batch_round<FWE_GENERIC> */
  int               th_rows = 16; /* rows of a thermal tile            */
  bool              one_tile = hm::BATCH_ONE_TILE; /* one CTA per tile instead of persistent CTAs */
  /* device tables */
  hm::BJob         *d_jobs = nullptr;
  size_t            d_jobs_cap = 0;
  int4             *d_tiles = nullptr;
  size_t            d_tiles_cap = 0;
  unsigned         *d_counters = nullptr;
  size_t            counters_cap = 0;
  bool              dirty = true;       /* job table needs an upload       */
  bool              tiles_dirty = true; /* tile lists need a rebuild        */
  TileLists        *lists = nullptr;
  cudaMemPool_t     pool = nullptr;     /* job state; keeps freed memory    */
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
    if (j.iterations > 0)
    {
      /* the last step's advection (every earlier one ran in the next step's
       * tiles): s of the final state from that step's s1, u, v */
      const int  lb = (j.iterations - 1) & 1;
      const int  row_groups = (j.ny + hm::ADV_R - 1) / hm::ADV_R;
      const dim3 g2((j.nx + 255) / 256, row_groups < 65535 ? row_groups : 65535);
      hm::k_vp_advect<hm::ADV_R><<<g2, 256, 0, s>>>(h.dev.s1[lb], h.dev.u[lb], h.dev.v[lb], f.s, h.dev.c);
      HM_LAUNCH_CHECK("k_vp_advect");
    }
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
  b->tiles_dirty = true;
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
  std::vector<int> act; /* active jobs, longest remaining first           */
  std::vector<int> rem; /* their remaining steps                          */
  int              N = 0;
};

/* Packed tile lists of the active jobs (cached in the batch, rebuilt and
 * uploaded only when a job is admitted or finishes): vpipes step tiles and
 * thermal tiles, each in the order of act; cum*[m]
 * counts the tiles of the first m jobs, so the tiles of the jobs that still
 * have steps left at a round are a prefix of each list. */
struct TileLists
{
  std::vector<int>    act;
  std::vector<size_t> vcum, tcum;
  bool                generic = false; /* an active vpipes job has pipe length or exponent != 1 */
};

int plan_rounds(hm_batch *b, int rounds, Plan &pl)
{
  auto remaining = [&](int k) { return b->jobs[k].desc.iterations - b->jobs[k].steps; };
  int  st;
  if (b->tiles_dirty)
  {
    TileLists &tl = *b->lists;
    tl.act.clear();
    for (size_t k = 0; k < b->jobs.size(); k++)
      if (b->jobs[k].live && !b->jobs[k].finished && !b->jobs[k].evicted) tl.act.push_back((int)k);
    /* every active job advances by the same number of steps per round, so
     * this order holds until the set of jobs changes */
    std::stable_sort(tl.act.begin(), tl.act.end(), [&](int x, int y) { return remaining(x) > remaining(y); });
    std::vector<int4> vt, tt;
    tl.vcum.assign(1, 0);
    tl.tcum.assign(1, 0);
    tl.generic = false;
    for (int k : tl.act)
    {
      const HJob &h = b->jobs[k];
      if (h.desc.kind == HM_JOB_VPIPES && !(h.dev.pl_one && h.dev.kexp_one)) tl.generic = true;
      for (int by = 0; by < h.dev.nby; by++)
        for (int bx = 0; bx < h.dev.nbx; bx++)
          (h.desc.kind == HM_JOB_VPIPES ? vt : tt).push_back(make_int4(k, bx, by, 0));
      tl.vcum.push_back(vt.size());
      tl.tcum.push_back(tt.size());
    }
    std::vector<int4> all(vt);
    all.insert(all.end(), tt.begin(), tt.end());
    if ((st = grow(&b->d_tiles, &b->d_tiles_cap, std::max<size_t>(all.size(), 1), b->stream))) return st;
    /* pageable source: the call returns once the data is staged */
    if (!all.empty())
      HM_CUDA_TRY(
          cudaMemcpyAsync(b->d_tiles, all.data(), all.size() * sizeof(int4), cudaMemcpyHostToDevice, b->stream));
    b->tiles_dirty = false;
  }
  pl.act = b->lists->act;
  int maxrem = 0;
  for (int k : pl.act)
  {
    pl.rem.push_back(std::max(0, remaining(k)));
    maxrem = std::max(maxrem, pl.rem.back());
  }
  pl.N = std::min(rounds, maxrem);
  if ((st = upload_jobs(b))) return st;
  if (pl.N == 0) return HM_OK;
  if ((st = grow(&b->d_counters, &b->counters_cap, (size_t)pl.N, b->stream))) return st;
  return HM_OK;
}

int launch_rounds(hm_batch *b, const Plan &pl)
{
  if (pl.N > 0)
  {
    HM_CUDA_TRY(cudaMemsetAsync(b->d_counters, 0, (size_t)pl.N * sizeof(unsigned), b->stream));
    const TileLists &tl = *b->lists;
    const size_t     nv = tl.vcum.back();
    size_t           m = pl.act.size();
    for (int r = 0; r < pl.N; r++)
    {
      /* the jobs (a prefix of act) that still have steps left at this round */
      while (m > 0 && pl.rem[m - 1] <= r) m--;
      const size_t iv = tl.vcum[m], it = tl.tcum[m];
      const int total = (int)(iv + it);
      if (b->one_tile)
      {
        const int grid = std::max(1, total);
        if (tl.generic)
          hm::k_batch_round<hm::FWE_GENERIC, false><<<grid, hm::BT, 0, b->stream>>>(
              b->d_jobs, b->d_tiles, (int)iv, b->d_tiles + nv, (int)it, b->round + r, nullptr);
        else
          hm::k_batch_round<hm::FWE_RTOPTS, false><<<grid, hm::BT, 0, b->stream>>>(
              b->d_jobs, b->d_tiles, (int)iv, b->d_tiles + nv, (int)it, b->round + r, nullptr);
        HM_LAUNCH_CHECK("k_batch_round");
        continue;
      }
      const int grid = std::max(1, std::min(tl.generic ? b->grid_cap_gen : b->grid_cap, total));
      if (tl.generic)
        hm::k_batch_round<hm::FWE_GENERIC, true><<<grid, hm::BT, 0, b->stream>>>(
            b->d_jobs, b->d_tiles, (int)iv, b->d_tiles + nv, (int)it, b->round + r, b->d_counters + r);
      else
        hm::k_batch_round<hm::FWE_RTOPTS, true><<<grid, hm::BT, 0, b->stream>>>(
            b->d_jobs, b->d_tiles, (int)iv, b->d_tiles + nv, (int)it, b->round + r, b->d_counters + r);
      HM_LAUNCH_CHECK("k_batch_round");
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
  /* the highest stream priority: a batch of small jobs runs beside plain
   * solves of large grids (the served form) and its rounds go first */
  int lo_prio = 0, hi_prio = 0;
  cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio);
  cudaError_t e = cudaStreamCreateWithPriority(&b->stream, cudaStreamNonBlocking, hi_prio);
  if (e != cudaSuccess)
  {
    delete b;
    return hm::cuda_fail(e, "hm_batch_create: cudaStreamCreate");
  }
  b->lists = new (std::nothrow) TileLists();
  if (!b->lists)
  {
    cudaStreamDestroy(b->stream);
    delete b;
    return hm::fail(HM_ERR_OUT_OF_MEMORY, "hm_batch_create: host allocation failed");
  }
  /* job state comes from a pool of the batch's own that keeps freed memory
   * for the next admission (the served form admits and releases jobs all
   * the time; mapping fresh memory for each would cost milliseconds) */
  {
    cudaMemPoolProps props;
    memset(&props, 0, sizeof props);
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = b->device;
    e = cudaMemPoolCreate(&b->pool, &props);
    if (e != cudaSuccess)
    {
      delete b->lists;
      cudaStreamDestroy(b->stream);
      delete b;
      return hm::cuda_fail(e, "hm_batch_create: cudaMemPoolCreate");
    }
    cuuint64_t keep = ~(cuuint64_t)0;
    HM_CUDA_TRY(cudaMemPoolSetAttribute(b->pool, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  int per_sm = 0, per_sm_gen = 0, sms = 0;
  HM_CUDA_TRY(
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hm::k_batch_round<hm::FWE_RTOPTS, true>, hm::BT, 0));
  HM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_gen, hm::k_batch_round<hm::FWE_GENERIC, true>,
                                                            hm::BT, 0));
  HM_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
  /* persistent CTAs per SM (0: one CTA per tile) and thermal tile rows:
   * the tuned choice, or the built-in one and 16 rows */
  hm::TuneEntry te;
  if (hm::tuned_batch(&te))
  {
    b->one_tile = te.tpb == 0;
    if (te.tpb >= 1)
    {
      per_sm = std::min(per_sm, te.tpb);
      per_sm_gen = std::min(per_sm_gen, te.tpb);
    }
    if (te.rows >= 1) b->th_rows = te.rows;
  }
  b->grid_cap = std::max(1, per_sm) * std::max(1, sms);
  b->grid_cap_gen = std::max(1, per_sm_gen) * std::max(1, sms);
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
  cudaError_t e = cudaMallocFromPoolAsync(&h.mem, h.bytes, b->pool, b->stream);
  if (e != cudaSuccess)
  {
    cudaGetLastError();
    return hm::cuda_fail(e, "hm_batch_add: job state allocation");
  }
  h.dev_block = (uintptr_t)h.mem;
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
    d.tz[0] = job->z;
    d.tz[1] = base;
    d.talus = job->talus;
    d.tv = job->talus_value;
    d.bed = job->bedrock;
    d.bed_mode = job->bedrock_mode;
    auto al8 = [](const void *p) { return ((uintptr_t)p & 7u) == 0; };
    d.pairs = job->nx % 2 == 0 && al8(d.tz[0]) && al8(d.tz[1]) && (!d.talus || al8(d.talus)) && (!d.bed || al8(d.bed));
    const int tw = d.pairs ? 2 * hm::TH_W : hm::TH_W;
    d.th_rows = b->th_rows;
    d.nbx = (job->nx + tw - 1) / tw;
    d.nby = (job->ny + d.th_rows - 1) / d.th_rows;
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
    d.nbx = (job->nx + hm::FT_TX - 1) / hm::FT_TX;
    d.nby = (job->ny + hm::FT_TY - 1) / hm::FT_TY;
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
    d.s1[0] = base + 13 * na;
    d.u[0] = base + 14 * na;
    d.v[0] = base + 15 * na;
    d.s1[1] = base + 16 * na;
    d.u[1] = base + 17 * na;
    d.v[1] = base + 18 * na;
    d.vec = job->nx % 2 == 0 && ((uintptr_t)job->z & 7u) == 0 && ((uintptr_t)job->vel_u & 7u) == 0 &&
            ((uintptr_t)job->vel_v & 7u) == 0;
    d.stage16 = stage16_ok(d);
    d.partials = (double *)(base + 19 * na);
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
  b->tiles_dirty = true;
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
  /* a job released before it finished (cancelled) leaves the rounds: the
   * tile lists are rebuilt without it before the next round, which would
   * otherwise still hold tiles over the freed state */
  if (!h.finished) b->tiles_dirty = true;
  h.finished = true;
  return HM_OK;
}

size_t hm_batch_bytes_in_use(const hm_batch *b)
{
  if (!b) return 0;
  size_t t = 0;
  for (const HJob &h : b->jobs)
    if (h.live && !h.evicted) t += h.bytes;
  return t;
}

size_t hm_batch_snapshot_bytes(const hm_batch *b, int job_id)
{
  if (!b || job_id < 0 || job_id >= (int)b->jobs.size()) return 0;
  const HJob &h = b->jobs[job_id];
  return h.bytes + (size_t)h.desc.nx * h.desc.ny * sizeof(float);
}

int hm_batch_evict(hm_batch *b, int job_id, void *snapshot)
{
  hm::clear_error();
  if (!b || job_id < 0 || job_id >= (int)b->jobs.size() || !snapshot)
    return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_batch_evict: unknown job or NULL snapshot");
  HJob &h = b->jobs[job_id];
  if (!h.live || h.finished || h.evicted || !h.mem)
    return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_batch_evict: the job is not an unfinished, resident job");
  int st = hm::use_device(b->device);
  if (st) return st;
  /* the job's state block, then its heights (the caller's grid, which the
   * steps update in place) */
  char *dst = (char *)snapshot;
  HM_CUDA_TRY(cudaMemcpyAsync(dst, h.mem, h.bytes, cudaMemcpyDeviceToHost, b->stream));
  HM_CUDA_TRY(cudaMemcpyAsync(dst + h.bytes, h.desc.z, (size_t)h.desc.nx * h.desc.ny * sizeof(float),
                              cudaMemcpyDeviceToHost, b->stream));
  HM_CUDA_TRY(cudaStreamSynchronize(b->stream));
  HM_CUDA_TRY(cudaFreeAsync(h.mem, b->stream));
  h.mem = nullptr;
  h.evicted = true;
  b->tiles_dirty = true;
  return HM_OK;
}

int hm_batch_restore(hm_batch *b, int job_id, const void *snapshot)
{
  hm::clear_error();
  if (!b || job_id < 0 || job_id >= (int)b->jobs.size() || !snapshot)
    return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_batch_restore: unknown job or NULL snapshot");
  HJob &h = b->jobs[job_id];
  if (!h.live || !h.evicted) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_batch_restore: the job is not evicted");
  int st = hm::use_device(b->device);
  if (st) return st;
  void       *mem = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&mem, h.bytes, b->pool, b->stream);
  if (e != cudaSuccess)
  {
    cudaGetLastError();
    return hm::cuda_fail(e, "hm_batch_restore: job state allocation");
  }
  const char *src = (const char *)snapshot;
  HM_CUDA_TRY(cudaMemcpyAsync(mem, src, h.bytes, cudaMemcpyHostToDevice, b->stream));
  HM_CUDA_TRY(cudaMemcpyAsync(h.desc.z, src + h.bytes, (size_t)h.desc.nx * h.desc.ny * sizeof(float),
                              cudaMemcpyHostToDevice, b->stream));
  /* the pageable source must stay valid until the copies are done */
  HM_CUDA_TRY(cudaStreamSynchronize(b->stream));
  /* the state block moved: its pointers follow it.  The block held by the
   * snapshot's job was freed at eviction, so only its old address is used,
   * as a number. */
  rebase_job(h, h.dev_block, (char *)mem);
  h.mem = mem;
  h.dev_block = (uintptr_t)mem;
  /* the job goes on from the step it had reached: its next step is the
   * batch's next round */
  h.dev.start = b->round - h.steps;
  h.evicted = false;
  b->dirty = true;
  b->tiles_dirty = true;
  return HM_OK;
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
  cudaStreamSynchronize(b->stream);
  cudaStreamDestroy(b->stream);
  if (b->pool) cudaMemPoolDestroy(b->pool);
  delete b->lists;
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
  /* Jobs of at least HM_BATCH_LARGE_CELLS cells fill the GPU on their
   * own, and the plain step kernels (specialised on the step's
   * options, TMA staging, five CTAs per SM) run them faster than the
   * batch's generic tiles.  They go through the plain solvers on
   * HM_BATCH_LANES side streams, each lane's jobs one after another, the
   * lanes balanced by cell-updates (longest first onto the least loaded
   * lane), beside the rounds of the smaller jobs.  The lanes are launched
   * directly, before the rounds are captured, so they run while the graph
   * is built; the batch stream joins them at the end.  On the 256-job mix
   * of the batched benchmark, 2^20 cells and one lane ran 1.41x plain
   * per-job calls; 2^18 and three lanes 1.34x, 2^20 and three lanes 1.29x,
   * 2^18 and one lane 1.12x (bit-identical results in every case). */
  struct Lane
  {
    std::vector<int> jobs;
    size_t           bytes = 0;
    double           work = 0.0;
    void            *mem = nullptr;
    cudaStream_t     s = nullptr;
    cudaEvent_t      join = nullptr;
  };
  Lane             lanes[HM_BATCH_LANES];
  std::vector<int> large;
  int              maxit = 0;
  for (int k = 0; k < njobs && !st; k++)
  {
    const hm_job &j = jobs[k];
    if ((st = check_job(j))) break;
    if ((long long)j.nx * j.ny >= HM_BATCH_LARGE_CELLS && j.iterations > 0)
    {
      large.push_back(k);
      continue;
    }
    int id;
    st = hm_batch_add(b, &j, &id);
    maxit = std::max(maxit, j.iterations);
  }
  auto work = [&](int k) { return (double)jobs[k].nx * jobs[k].ny * jobs[k].iterations *
                                  (jobs[k].kind == HM_JOB_VPIPES ? 5.0 : 1.0); };
  std::stable_sort(large.begin(), large.end(), [&](int x, int y) { return work(x) > work(y); });
  for (int k : large)
  {
    Lane *l = &lanes[0];
    for (Lane &c : lanes)
      if (c.work < l->work) l = &c;
    const hm_job &j = jobs[k];
    l->jobs.push_back(k);
    l->work += work(k);
    l->bytes = std::max(l->bytes, j.kind == HM_JOB_THERMAL
                                      ? hm::thermal_scratch_floats(j.nx, j.ny, j.deposition_map != nullptr) * sizeof(float)
                                      : hm::vpipes_scratch_bytes(j.nx, j.ny));
  }
  cudaEvent_t fork = nullptr;
  if (!st && !large.empty())
  {
    cudaError_t e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
    for (Lane &l : lanes)
    {
      if (l.jobs.empty() || e != cudaSuccess) continue;
      e = cudaMallocFromPoolAsync(&l.mem, l.bytes, b->pool, b->stream);
      if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&l.s, cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&l.join, cudaEventDisableTiming);
    }
    if (e != cudaSuccess)
    {
      cudaGetLastError();
      st = hm::cuda_fail(e, "hm_batch_run: large-job lane set-up");
    }
  }
  if (!st) st = upload_jobs(b);
  /* the large jobs' plain solves, each lane forked from and joined to the
   * batch stream */
  auto launch_large = [&]() -> int {
    if (large.empty()) return HM_OK;
    HM_CUDA_TRY(cudaEventRecord(fork, b->stream));
    for (Lane &l : lanes)
    {
      if (l.jobs.empty()) continue;
      HM_CUDA_TRY(cudaStreamWaitEvent(l.s, fork, 0));
      for (int k : l.jobs)
      {
        const hm_job &j = jobs[k];
        int           rc;
        if (j.kind == HM_JOB_THERMAL)
        {
          hm_thermal_options o;
          hm_thermal_default_options(&o);
          o.bedrock_mode = j.bedrock_mode;
          rc = hm::thermal_core(b->device, j.z, j.nx, j.ny, j.talus, j.talus_value, j.iterations, j.bedrock,
                                j.deposition_map, nullptr, &o, (float *)l.mem, l.s);
        }
        else
        {
          hm_vpipes_params p = j.vpipes;
          p.iterations = j.iterations;
          rc = hm::vpipes_core(j.z, j.nx, j.ny, p, j.rain_map, j.water_depth, j.sediment, j.vel_u, j.vel_v, l.mem,
                               l.s);
        }
        if (rc) return rc;
      }
      HM_CUDA_TRY(cudaEventRecord(l.join, l.s));
    }
    return HM_OK;
  };
  auto join_large = [&]() -> int {
    for (Lane &l : lanes)
      if (!l.jobs.empty()) HM_CUDA_TRY(cudaStreamWaitEvent(b->stream, l.join, 0));
    return HM_OK;
  };
  if (!st && use_graph && maxit > 0)
  {
    /* every round of the batch in one graph; the host-side plan (tile
     * lists, uploads) is made before the capture */
    Plan            pl;
    cudaGraph_t     graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    st = plan_rounds(b, maxit, pl);
    if (!st) st = hm_batch_synchronize(b);
    if (!st) st = launch_large();
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
    if (!st) st = join_large();
    if (!st) st = hm_batch_synchronize(b);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
  else if (!st)
  {
    st = launch_large();
    if (!st) st = run_rounds(b, maxit);
    if (!st) st = join_large();
    if (!st) st = hm_batch_synchronize(b);
  }
  /* the lanes are done (joined, or synchronised here on an error path)
   * before their memory goes back to the pool */
  for (Lane &l : lanes)
    if (l.s) cudaStreamSynchronize(l.s);
  for (Lane &l : lanes)
    if (l.mem) cudaFreeAsync(l.mem, b->stream);
  cudaStreamSynchronize(b->stream);
  for (Lane &l : lanes)
  {
    if (l.join) cudaEventDestroy(l.join);
    if (l.s) cudaStreamDestroy(l.s);
  }
  if (fork) cudaEventDestroy(fork);
  int st2 = hm_batch_destroy(b);
  return st ? st : st2;
}

} // extern "C"
