/*
 * hm_tune.cu - the launch-shape autotuner.
 *
 * For one solver and grid size it times every candidate launch shape on a
 * synthetic terrain of that size (generated on the device: a sum of
 * sinusoids with the value range of a remapped fBm field) and keeps the
 * fastest per size class (nx and ny rounded up to powers of two):
 *   vpipes  : the tiled step kernels at one or two steps per launch
 *             (temporal-block depth 1, 2), and the streaming kernel's
 *             threads per CTA (strip width) x staged advection radius x
 *             output rows per CTA (the occupancy / halo / warm-up trade);
 *   thermal : steps per launch (temporal-block depth 1, 2, 4, 8) x rows
 *             per CTA of the blocked kernel;
 *   batch   : persistent CTAs per SM (occupancy; 0 = one CTA per tile of
 *             the round) x rows of a thermal tile
 *             of the batched form's round kernel, on a synthetic mixed
 *             batch (one entry for the process).
 * The solvers consult the table whenever the caller leaves the choice to
 * the library (time_block 0, no hm_vpipes_set_launch override).  Results
 * never depend on the shape; only the speed does.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "hm_internal.h"
#include "hm_thermal.h"
#include "hm_tune.h"
#include "hm_vpipes.h"

namespace hm
{

namespace
{

std::mutex                                   g_mu;
std::map<std::pair<int, int>, TuneEntry>     g_vp, g_th; /* size class -> shape */
TuneEntry                                    g_batch;
bool                                         g_batch_set = false;

int pow2_class(int v)
{
  int c = 0;
  while ((1 << c) < v && c < 30) c++;
  return c;
}

std::pair<int, int> size_class(int nx, int ny) { return {pow2_class(nx), pow2_class(ny)}; }

__global__ void k_synthetic_terrain(float *z, int nx, int ny)
{
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < (size_t)nx * ny;
       k += (size_t)gridDim.x * blockDim.x)
  {
    const float x = (float)(k % nx) / nx, y = (float)(k / nx) / ny;
    float       v = 0.f, a = 0.5f, f = 4.f;
    for (int o = 0; o < 6; o++)
    {
      v += a * __sinf(6.2831853f * f * x + 1.7f * o) * __cosf(6.2831853f * f * y + 0.9f * o);
      a *= 0.5f;
      f *= 2.f;
    }
    z[k] = 0.5f + 0.5f * v;
  }
}

} // namespace

bool tuned_vpipes(int nx, int ny, TuneEntry *out)
{
  std::lock_guard<std::mutex> lk(g_mu);
  auto                        it = g_vp.find(size_class(nx, ny));
  if (it == g_vp.end()) return false;
  *out = it->second;
  return true;
}

bool tuned_batch(TuneEntry *out)
{
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_batch_set) return false;
  *out = g_batch;
  return true;
}

bool tuned_thermal(int nx, int ny, TuneEntry *out)
{
  std::lock_guard<std::mutex> lk(g_mu);
  auto                        it = g_th.find(size_class(nx, ny));
  if (it == g_th.end()) return false;
  *out = it->second;
  return true;
}

} // namespace hm

namespace hm
{
namespace
{

/* Tunes the batched form: each candidate (CTAs per SM, thermal tile rows)
 * runs 3 warm-up and `steps` timed rounds of the same synthetic batch. */
int autotune_batch(hm_context *ctx, int side_max, int steps, hm_tune_result *result)
{
  cudaStream_t         s = ctx->stream;
  const int            sides[8] = {128, 192, 256, 384, 512, 768, 1024, 1536};
  std::vector<hm_job>  jobs;
  std::vector<float *> bufs;
  int                  st = HM_OK;
  for (int k = 0; k < 16 && !st; k++)
  {
    const int side = std::min(sides[k % 8], std::max(side_max, 128));
    hm_job    j;
    memset(&j, 0, sizeof j);
    j.kind = (k & 1) ? HM_JOB_VPIPES : HM_JOB_THERMAL;
    j.nx = side;
    j.ny = side - (k & 2 ? 64 : 0);
    j.iterations = steps + 3;
    float      *z = nullptr;
    cudaError_t e = cudaMallocAsync((void **)&z, (size_t)j.nx * j.ny * sizeof(float), s);
    if (e != cudaSuccess)
    {
      cudaGetLastError();
      st = cuda_fail(e, "hm_autotune: batch job allocation");
      break;
    }
    bufs.push_back(z);
    j.z = z;
    j.talus_value = 1.f / (float)j.nx;
    hm_vpipes_default_params(&j.vpipes);
    j.vpipes.maintain_water_volume = 0;
    j.vpipes.flux_diffusion = 0;
    j.vpipes.dt = 0.1f;
    j.vpipes.gravity = 9.81f;
    j.vpipes.rain_per_step = 1e-4f;
    j.vpipes.initial_water = 0.f;
    jobs.push_back(j);
  }
  std::vector<TuneEntry> cands;
  /* per_sm 0: one CTA per tile of the round instead of persistent CTAs */
  for (int per_sm = 0; per_sm <= 4; per_sm++)
    for (int rows : {8, 16, 32}) cands.push_back(TuneEntry{per_sm, 0, rows, 0, 0.f});
  int   best = -1;
  float best_ms = 0.f;
  for (size_t c = 0; c < cands.size() && !st; c++)
  {
    {
      std::lock_guard<std::mutex> lk(g_mu);
      g_batch = cands[c];
      g_batch_set = true;
    }
    for (size_t k = 0; k < jobs.size(); k++) k_synthetic_terrain<<<592, 256, 0, s>>>(bufs[k], jobs[k].nx, jobs[k].ny);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
    {
      st = cuda_fail(e, "hm_autotune: synthetic terrain");
      break;
    }
    hm_batch *b = nullptr;
    if ((st = hm_batch_create(ctx, &b))) break;
    for (size_t k = 0; k < jobs.size() && !st; k++)
    {
      int id;
      st = hm_batch_add(b, &jobs[k], &id);
    }
    float ms = 0.f;
    if (!st) st = hm_batch_step(b, 3);
    if (!st) st = hm_batch_synchronize(b);
    if (!st)
    {
      const auto t0 = std::chrono::steady_clock::now();
      st = hm_batch_step(b, steps);
      if (!st) st = hm_batch_synchronize(b);
      ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    hm_batch_destroy(b);
    cands[c].ms_per_step = ms / steps;
    if (!st && (best < 0 || ms < best_ms))
    {
      best = (int)c;
      best_ms = ms;
    }
  }
  for (float *z : bufs) cudaFreeAsync(z, s);
  cudaStreamSynchronize(s);
  std::lock_guard<std::mutex> lk(g_mu);
  if (st || best < 0)
  {
    g_batch_set = false;
    return st ? st : fail(HM_ERR_CUDA, "hm_autotune: no batch candidate ran");
  }
  g_batch = cands[best];
  g_batch_set = true;
  if (result)
  {
    memset(result, 0, sizeof *result);
    result->tpb = g_batch.tpb;
    result->rows = g_batch.rows;
    result->ms_per_step = g_batch.ms_per_step;
    result->candidates = (int)cands.size();
  }
  return HM_OK;
}

} // namespace
} // namespace hm

extern "C" {

int hm_autotune(hm_context *ctx, int kind, int nx, int ny, int steps, hm_tune_result *result)
{
  hm::clear_error();
  if (!ctx || (kind != HM_JOB_THERMAL && kind != HM_JOB_VPIPES && kind != HM_TUNE_BATCH) || nx < 3 || ny < 3 ||
      steps < 1)
    return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_autotune: bad argument");
  if (kind == HM_TUNE_BATCH)
  {
    int st = hm::use_device(ctx->device);
    if (st) return st;
    return hm::autotune_batch(ctx, nx > ny ? nx : ny, steps, result);
  }
  int st = hm::use_device(ctx->device);
  if (st) return st;
  cudaStream_t s = ctx->stream;
  const size_t n = (size_t)nx * ny;
  float       *z = nullptr, *z0 = nullptr;
  HM_CUDA_TRY(cudaMallocAsync((void **)&z, n * sizeof(float), s));
  HM_CUDA_TRY(cudaMallocAsync((void **)&z0, n * sizeof(float), s));
  hm::k_synthetic_terrain<<<592, 256, 0, s>>>(z0, nx, ny);
  HM_LAUNCH_CHECK("k_synthetic_terrain");
  cudaEvent_t e0, e1;
  HM_CUDA_TRY(cudaEventCreate(&e0));
  HM_CUDA_TRY(cudaEventCreate(&e1));

  std::vector<hm::TuneEntry> cands;
  if (kind == HM_JOB_VPIPES)
  {
    /* {0, 0, 0}: the tiled step kernels; the others: the streaming kernel */
    const int shapes[][3] = {{0, 0, 0},     {128, 2, 32}, {128, 2, 64}, {128, 2, 128},
                             {256, 2, 64},  {128, 3, 32}, {128, 3, 64}, {256, 3, 64}};
    for (auto &c : shapes) cands.push_back(hm::TuneEntry{c[0], c[1], c[2], 0, 0.f});
    /* the tiled kernels with two steps per launch (time_block 2) */
    cands.push_back(hm::TuneEntry{0, 0, 0, 2, 0.f});
  }
  else
  {
    const int shapes[][2] = {{1, 0}, {2, 64}, {4, 64}, {4, 128}, {8, 64}, {8, 128}};
    for (auto &c : shapes) cands.push_back(hm::TuneEntry{0, 0, c[1], c[0], 0.f});
  }

  /* the benchmark configuration's parameters: rain per step, gravity 9.81 */
  hm_vpipes_params vp;
  hm_vpipes_default_params(&vp);
  vp.maintain_water_volume = 0;
  vp.flux_diffusion = 0;
  vp.dt = 0.1f;
  vp.k_capacity = 0.05f;
  vp.k_erode = vp.k_depose = 0.01f;
  vp.evap_rate = 0.01f;
  vp.gravity = 9.81f;
  vp.rain_per_step = 1e-4f;
  vp.initial_water = 0.f;
  vp.iterations = steps;

  int       best = -1;
  float     best_ms = 0.f;
  /* one warm-up run, then the best of three timed runs: at small sizes a
   * run lasts a few hundred microseconds and one timing alone can pick a
   * slower candidate */
  const int warm = 1, timed = 3;
  for (size_t k = 0; k < cands.size() && !st; k++)
  {
    const hm::TuneEntry &c = cands[k];
    float                ms = 0.f;
    for (int rep = 0; rep < warm + timed && !st; rep++)
    {
      HM_CUDA_TRY(cudaMemcpyAsync(z, z0, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
      HM_CUDA_TRY(cudaEventRecord(e0, s));
      if (kind == HM_JOB_VPIPES)
      {
        if (c.tpb == 0) st = hm_vpipes_set_algorithm(c.block == 2 ? HM_VPIPES_TILED_TB2 : HM_VPIPES_TILED);
        else if (!(st = hm_vpipes_set_algorithm(HM_VPIPES_STREAMING))) st = hm_vpipes_set_launch(c.tpb, c.radius, c.rows);
        if (st) break;
        st = hm_vpipes_device(ctx, z, nx, ny, &vp, nullptr, nullptr, nullptr, nullptr, nullptr, s);
      }
      else
      {
        hm_thermal_options o;
        hm_thermal_default_options(&o);
        o.time_block = c.block;
        if ((st = hm_thermal_set_launch(c.rows))) break;
        st = hm_thermal_device(ctx, z, nx, ny, nullptr, 1.f / nx, steps, nullptr, nullptr, nullptr, &o, s);
      }
      HM_CUDA_TRY(cudaEventRecord(e1, s));
      HM_CUDA_TRY(cudaEventSynchronize(e1));
      float t = 0.f;
      HM_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
      if (rep == warm || (rep > warm && t < ms)) ms = t;
    }
    cands[k].ms_per_step = ms / steps;
    if (!st && (best < 0 || ms < best_ms))
    {
      best = (int)k;
      best_ms = ms;
    }
  }
  if (kind == HM_JOB_VPIPES)
  {
    hm_vpipes_set_launch(0, 0, 0);
    hm_vpipes_set_algorithm(HM_VPIPES_AUTO);
  }
  else
    hm_thermal_set_launch(0);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(z, s);
  cudaFreeAsync(z0, s);
  cudaStreamSynchronize(s);
  if (st) return st;

  {
    std::lock_guard<std::mutex> lk(hm::g_mu);
    (kind == HM_JOB_VPIPES ? hm::g_vp : hm::g_th)[hm::size_class(nx, ny)] = cands[best];
  }
  if (result)
  {
    result->tpb = cands[best].tpb;
    result->radius = cands[best].radius;
    result->rows = cands[best].rows;
    result->time_block = cands[best].block;
    result->ms_per_step = cands[best].ms_per_step;
    result->candidates = (int)cands.size();
  }
  return HM_OK;
}

int hm_autotune_save(const char *path)
{
  if (!path) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_autotune_save: NULL path");
  FILE *f = fopen(path, "w");
  if (!f) return hm::fail(HM_ERR_INVALID_ARGUMENT, std::string("hm_autotune_save: cannot open ") + path);
  std::lock_guard<std::mutex> lk(hm::g_mu);
  fprintf(f, "# highmap_b200 launch shapes: kind log2nx log2ny tpb radius rows time_block ms_per_step\n");
  for (auto &kv : hm::g_vp)
    fprintf(f, "vpipes %d %d %d %d %d %d %.6f\n", kv.first.first, kv.first.second, kv.second.tpb, kv.second.radius,
            kv.second.rows, kv.second.block, kv.second.ms_per_step);
  for (auto &kv : hm::g_th)
    fprintf(f, "thermal %d %d %d %d %d %d %.6f\n", kv.first.first, kv.first.second, kv.second.tpb,
            kv.second.radius, kv.second.rows, kv.second.block, kv.second.ms_per_step);
  if (hm::g_batch_set)
    fprintf(f, "batch 0 0 %d 0 %d 0 %.6f\n", hm::g_batch.tpb, hm::g_batch.rows, hm::g_batch.ms_per_step);
  fclose(f);
  return HM_OK;
}

int hm_autotune_load(const char *path, int *loaded_out)
{
  if (loaded_out) *loaded_out = 0;
  if (!path) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_autotune_load: NULL path");
  FILE *f = fopen(path, "r");
  if (!f) return hm::fail(HM_ERR_INVALID_ARGUMENT, std::string("hm_autotune_load: cannot open ") + path);
  char line[256];
  int  loaded = 0;
  while (fgets(line, sizeof line, f))
  {
    char          kind[16];
    int           cx, cy;
    hm::TuneEntry e{};
    if (line[0] == '#') continue;
    if (sscanf(line, "%15s %d %d %d %d %d %d %f", kind, &cx, &cy, &e.tpb, &e.radius, &e.rows, &e.block,
               &e.ms_per_step) != 8)
      continue;
    std::string k(kind);
    /* keep only shapes the kernels accept */
    if (k == "vpipes" && ((e.tpb == 0 && e.block >= 0 && e.block <= 2) ||
                          (e.tpb != 0 && hm_vpipes_set_launch(e.tpb, e.radius, e.rows) == HM_OK)))
    {
      std::lock_guard<std::mutex> lk(hm::g_mu);
      hm::g_vp[{cx, cy}] = e;
      loaded++;
    }
    else if (k == "thermal" && e.block >= 1 && e.block <= 8 && (e.rows == 0 || (e.rows >= 8 && e.rows <= 4096)))
    {
      std::lock_guard<std::mutex> lk(hm::g_mu);
      hm::g_th[{cx, cy}] = e;
      loaded++;
    }
    else if (k == "batch" && e.tpb >= 0 && e.tpb <= 4 && (e.rows == 8 || e.rows == 16 || e.rows == 32))
    {
      std::lock_guard<std::mutex> lk(hm::g_mu);
      hm::g_batch = e;
      hm::g_batch_set = true;
      loaded++;
    }
  }
  hm_vpipes_set_launch(0, 0, 0);
  fclose(f);
  if (loaded_out) *loaded_out = loaded;
  return HM_OK;
}

void hm_autotune_clear(void)
{
  std::lock_guard<std::mutex> lk(hm::g_mu);
  hm::g_vp.clear();
  hm::g_th.clear();
  hm::g_batch_set = false;
}

} // extern "C"
