/*
 * hm_api.cpp - the C-ABI entry points of include/hm_erosion.h.
 *
 * Host-pointer calls reproduce the reference drivers' boundary
 * (HighMap/src/erosion/thermal_gpu.cpp:30-46 uploads z, talus and bedrock,
 * runs the steps, reads z back): one upload of each input, the whole solve
 * on the device, one download of each output, all ordered on the context's
 * stream and finished before the call returns.
 */
#include <cstring>

#include "hm_internal.h"
#include "hm_thermal.h"
#include "hm_vpipes.h"

namespace
{

using hm::align_up;

struct Slab
{
  char  *base;
  size_t off = 0;
  float *take(size_t nfloats) { return (float *)take_bytes(nfloats * sizeof(float)); }
  void  *take_bytes(size_t bytes)
  {
    void *p = base + off;
    off += align_up(bytes, 256);
    return p;
  }
};

int thermal_host(hm_context *ctx, float *z, int nx, int ny, const float *talus, float talus_value,
                 int iterations, const float *bedrock, float *depo, const float *mask,
                 const hm_thermal_options *opts, bool auto_bed = false)
{
  hm::clear_error();
  if (!ctx) return hm::fail(HM_ERR_INVALID_ARGUMENT, "thermal: ctx is NULL");
  int st = hm::thermal_check_args(z, nx, ny, iterations, opts);
  if (st) return st;
  if ((st = hm::use_device(ctx->device))) return st;
  const size_t n = (size_t)nx * ny;
  const size_t nbytes = n * sizeof(float);
  const bool   need_z0 = depo || mask || auto_bed;
  size_t       fields = 1 + (talus ? 1 : 0) + (bedrock ? 1 : 0) + (depo ? 1 : 0) + (mask ? 1 : 0);
  size_t total = fields * align_up(nbytes, 256) + align_up(hm::thermal_scratch_floats(nx, ny, need_z0) * 4, 256);
  void  *ws = nullptr;
  if ((st = hm::workspace(ctx, total, &ws))) return st;
  Slab         sl{(char *)ws};
  float       *dz = sl.take(n);
  float       *dt = talus ? sl.take(n) : nullptr;
  float       *db = bedrock ? sl.take(n) : nullptr;
  float       *dd = depo ? sl.take(n) : nullptr;
  float       *dm = mask ? sl.take(n) : nullptr;
  float       *scr = sl.take(hm::thermal_scratch_floats(nx, ny, need_z0));
  cudaStream_t s = ctx->stream;
  HM_CUDA_TRY(cudaMemcpyAsync(dz, z, nbytes, cudaMemcpyHostToDevice, s));
  if (dt) HM_CUDA_TRY(cudaMemcpyAsync(dt, talus, nbytes, cudaMemcpyHostToDevice, s));
  if (db) HM_CUDA_TRY(cudaMemcpyAsync(db, bedrock, nbytes, cudaMemcpyHostToDevice, s));
  if (dm) HM_CUDA_TRY(cudaMemcpyAsync(dm, mask, nbytes, cudaMemcpyHostToDevice, s));
  st = hm::thermal_core(ctx->device, dz, nx, ny, dt, talus_value, iterations, db, dd, dm, opts, scr, s, auto_bed);
  if (st)
  {
    cudaStreamSynchronize(s);
    return st;
  }
  HM_CUDA_TRY(cudaMemcpyAsync(z, dz, nbytes, cudaMemcpyDeviceToHost, s));
  if (dd) HM_CUDA_TRY(cudaMemcpyAsync(depo, dd, nbytes, cudaMemcpyDeviceToHost, s));
  HM_CUDA_TRY(cudaStreamSynchronize(s));
  return HM_OK;
}

} // namespace

extern "C" {

int hm_thermal(hm_context *ctx, float *z, int nx, int ny, const float *talus, int iterations,
               const float *bedrock, float *deposition_map, const hm_thermal_options *opts)
{
  if (!talus) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_thermal: talus is NULL");
  return thermal_host(ctx, z, nx, ny, talus, 0.f, iterations, bedrock, deposition_map, nullptr, opts);
}

int hm_thermal_scalar(hm_context *ctx, float *z, int nx, int ny, float talus, int iterations,
                      const float *bedrock, float *deposition_map, const hm_thermal_options *opts)
{
  return thermal_host(ctx, z, nx, ny, nullptr, talus, iterations, bedrock, deposition_map, nullptr, opts);
}

int hm_thermal_masked(hm_context *ctx, float *z, int nx, int ny, const float *mask, const float *talus,
                      int iterations, const float *bedrock, float *deposition_map,
                      const hm_thermal_options *opts)
{
  if (!talus) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_thermal_masked: talus is NULL");
  return thermal_host(ctx, z, nx, ny, talus, 0.f, iterations, bedrock, deposition_map, mask, opts);
}

int hm_thermal_device(hm_context *ctx, float *z, int nx, int ny, const float *talus, float talus_value,
                      int iterations, const float *bedrock, float *deposition_map, const float *mask,
                      const hm_thermal_options *opts, void *stream)
{
  hm::clear_error();
  if (!ctx) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_thermal_device: ctx is NULL");
  int st = hm::thermal_check_args(z, nx, ny, iterations, opts);
  if (st) return st;
  if ((st = hm::use_device(ctx->device))) return st;
  const bool need_z0 = deposition_map || mask;
  void      *ws = nullptr;
  if ((st = hm::workspace(ctx, hm::thermal_scratch_floats(nx, ny, need_z0) * sizeof(float), &ws))) return st;
  return hm::thermal_core(ctx->device, z, nx, ny, talus, talus_value, iterations, bedrock, deposition_map, mask,
                          opts, (float *)ws, (cudaStream_t)stream);
}

int hm_thermal_auto_bedrock(hm_context *ctx, float *z, int nx, int ny, const float *talus, int iterations,
                            float *deposition_map, const hm_thermal_options *opts)
{
  if (!talus) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_thermal_auto_bedrock: talus is NULL");
  return thermal_host(ctx, z, nx, ny, talus, 0.f, iterations, nullptr, deposition_map, nullptr, opts, true);
}

int hm_thermal_auto_bedrock_scalar(hm_context *ctx, float *z, int nx, int ny, float talus, int iterations,
                                   float *deposition_map, const hm_thermal_options *opts)
{
  return thermal_host(ctx, z, nx, ny, nullptr, talus, iterations, nullptr, deposition_map, nullptr, opts, true);
}

int hm_thermal_auto_bedrock_masked(hm_context *ctx, float *z, int nx, int ny, const float *mask,
                                   const float *talus, int iterations, float *deposition_map,
                                   const hm_thermal_options *opts)
{
  if (!talus) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_thermal_auto_bedrock_masked: talus is NULL");
  return thermal_host(ctx, z, nx, ny, talus, 0.f, iterations, nullptr, deposition_map, mask, opts, true);
}

int hm_thermal_auto_bedrock_device(hm_context *ctx, float *z, int nx, int ny, const float *talus,
                                   float talus_value, int iterations, float *deposition_map, const float *mask,
                                   const hm_thermal_options *opts, void *stream)
{
  hm::clear_error();
  if (!ctx) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_thermal_auto_bedrock_device: ctx is NULL");
  int st = hm::thermal_check_args(z, nx, ny, iterations, opts);
  if (st) return st;
  if ((st = hm::use_device(ctx->device))) return st;
  void *ws = nullptr;
  if ((st = hm::workspace(ctx, hm::thermal_scratch_floats(nx, ny, true) * sizeof(float), &ws))) return st;
  return hm::thermal_core(ctx->device, z, nx, ny, talus, talus_value, iterations, nullptr, deposition_map, mask,
                          opts, (float *)ws, (cudaStream_t)stream, true);
}

namespace
{
int sibling_host(hm_context *ctx, int rule, float *z, int nx, int ny, const float *talus, const float *zmax,
                 float intensity, int iterations, float *depo, const float *mask, float p1 = 0.f)
{
  hm::clear_error();
  if (!ctx) return hm::fail(HM_ERR_INVALID_ARGUMENT, "thermal stencil: ctx is NULL");
  int st = hm::sibling_check_args(rule, z, nx, ny, talus, zmax, iterations);
  if (st) return st;
  if ((st = hm::use_device(ctx->device))) return st;
  const size_t n = (size_t)nx * ny;
  const size_t nbytes = n * sizeof(float);
  size_t       fields = 1 + (talus ? 1 : 0) + (zmax ? 1 : 0) + (depo ? 1 : 0) + (mask ? 1 : 0);
  size_t total = fields * align_up(nbytes, 256) + align_up(hm::thermal_scratch_floats(nx, ny, true) * 4, 256);
  void  *ws = nullptr;
  if ((st = hm::workspace(ctx, total, &ws))) return st;
  Slab         sl{(char *)ws};
  float       *dz = sl.take(n);
  float       *dt = talus ? sl.take(n) : nullptr;
  float       *dzm = zmax ? sl.take(n) : nullptr;
  float       *dd = depo ? sl.take(n) : nullptr;
  float       *dm = mask ? sl.take(n) : nullptr;
  float       *scr = sl.take(hm::thermal_scratch_floats(nx, ny, true));
  cudaStream_t s = ctx->stream;
  HM_CUDA_TRY(cudaMemcpyAsync(dz, z, nbytes, cudaMemcpyHostToDevice, s));
  if (dt) HM_CUDA_TRY(cudaMemcpyAsync(dt, talus, nbytes, cudaMemcpyHostToDevice, s));
  if (dzm) HM_CUDA_TRY(cudaMemcpyAsync(dzm, zmax, nbytes, cudaMemcpyHostToDevice, s));
  if (dm) HM_CUDA_TRY(cudaMemcpyAsync(dm, mask, nbytes, cudaMemcpyHostToDevice, s));
  st = hm::sibling_core(ctx->device, rule, dz, nx, ny, dt, dzm, intensity, iterations, dd, dm, scr, s, p1);
  if (st)
  {
    cudaStreamSynchronize(s);
    return st;
  }
  HM_CUDA_TRY(cudaMemcpyAsync(z, dz, nbytes, cudaMemcpyDeviceToHost, s));
  if (dd) HM_CUDA_TRY(cudaMemcpyAsync(depo, dd, nbytes, cudaMemcpyDeviceToHost, s));
  HM_CUDA_TRY(cudaStreamSynchronize(s));
  return HM_OK;
}
} // namespace

namespace
{
int deposition_check(hm_context *ctx, const float *z, int nx, int ny, const float *talus, int iterations,
                     int thermal_subiterations)
{
  if (!ctx) return hm::fail(HM_ERR_INVALID_ARGUMENT, "sediment_deposition: ctx is NULL");
  if (!talus) return hm::fail(HM_ERR_INVALID_ARGUMENT, "sediment_deposition: talus is NULL");
  if (iterations < 0 || thermal_subiterations < 0)
    return hm::fail(HM_ERR_INVALID_ARGUMENT, "sediment_deposition: negative iteration count");
  return hm::thermal_check_args(z, nx, ny, thermal_subiterations, nullptr);
}
} // namespace

int hm_sediment_deposition(hm_context *ctx, float *z, int nx, int ny, const float *talus, float max_deposition,
                           int iterations, int thermal_subiterations, float *deposition_map, const float *mask)
{
  hm::clear_error();
  int st = deposition_check(ctx, z, nx, ny, talus, iterations, thermal_subiterations);
  if (st) return st;
  if ((st = hm::use_device(ctx->device))) return st;
  const size_t n = (size_t)nx * ny;
  const size_t nbytes = n * sizeof(float);
  const size_t fields = 2 + (deposition_map ? 1 : 0) + (mask ? 1 : 0);
  const size_t total = fields * align_up(nbytes, 256) + align_up(hm::deposition_scratch_floats(nx, ny) * 4, 256);
  void        *ws = nullptr;
  if ((st = hm::workspace(ctx, total, &ws))) return st;
  Slab         sl{(char *)ws};
  float       *dz = sl.take(n);
  float       *dt = sl.take(n);
  float       *dd = deposition_map ? sl.take(n) : nullptr;
  float       *dm = mask ? sl.take(n) : nullptr;
  float       *scr = sl.take(hm::deposition_scratch_floats(nx, ny));
  cudaStream_t s = ctx->stream;
  HM_CUDA_TRY(cudaMemcpyAsync(dz, z, nbytes, cudaMemcpyHostToDevice, s));
  HM_CUDA_TRY(cudaMemcpyAsync(dt, talus, nbytes, cudaMemcpyHostToDevice, s));
  if (dm) HM_CUDA_TRY(cudaMemcpyAsync(dm, mask, nbytes, cudaMemcpyHostToDevice, s));
  st = hm::deposition_core(ctx->device, dz, nx, ny, dt, max_deposition, iterations, thermal_subiterations, dd, dm,
                           scr, s);
  if (st)
  {
    cudaStreamSynchronize(s);
    return st;
  }
  HM_CUDA_TRY(cudaMemcpyAsync(z, dz, nbytes, cudaMemcpyDeviceToHost, s));
  if (dd) HM_CUDA_TRY(cudaMemcpyAsync(deposition_map, dd, nbytes, cudaMemcpyDeviceToHost, s));
  HM_CUDA_TRY(cudaStreamSynchronize(s));
  return HM_OK;
}

int hm_sediment_deposition_device(hm_context *ctx, float *z, int nx, int ny, const float *talus,
                                  float max_deposition, int iterations, int thermal_subiterations,
                                  float *deposition_map, const float *mask, void *stream)
{
  hm::clear_error();
  int st = deposition_check(ctx, z, nx, ny, talus, iterations, thermal_subiterations);
  if (st) return st;
  if ((st = hm::use_device(ctx->device))) return st;
  void *ws = nullptr;
  if ((st = hm::workspace(ctx, hm::deposition_scratch_floats(nx, ny) * sizeof(float), &ws))) return st;
  return hm::deposition_core(ctx->device, z, nx, ny, talus, max_deposition, iterations, thermal_subiterations,
                             deposition_map, mask, (float *)ws, (cudaStream_t)stream);
}

namespace
{
int layer_check(hm_context *ctx, const float *z, int nx, int ny, const float *talus_layer,
                const float *talus_upper_limit, int iterations)
{
  if (!ctx) return hm::fail(HM_ERR_INVALID_ARGUMENT, "sediment_layer: ctx is NULL");
  if (!talus_layer || !talus_upper_limit)
    return hm::fail(HM_ERR_INVALID_ARGUMENT, "sediment_layer: talus_layer or talus_upper_limit is NULL");
  return hm::thermal_check_args(z, nx, ny, iterations, nullptr);
}
} // namespace

int hm_sediment_layer(hm_context *ctx, float *z, int nx, int ny, const float *talus_layer,
                      const float *talus_upper_limit, int iterations, int apply_post_filter, float *deposition_map)
{
  hm::clear_error();
  int st = layer_check(ctx, z, nx, ny, talus_layer, talus_upper_limit, iterations);
  if (st) return st;
  if ((st = hm::use_device(ctx->device))) return st;
  const size_t n = (size_t)nx * ny;
  const size_t nbytes = n * sizeof(float);
  const size_t fields = 3 + (deposition_map ? 1 : 0);
  const size_t total = fields * align_up(nbytes, 256) + align_up(hm::layer_scratch_floats(nx, ny) * 4, 256);
  void        *ws = nullptr;
  if ((st = hm::workspace(ctx, total, &ws))) return st;
  Slab         sl{(char *)ws};
  float       *dz = sl.take(n);
  float       *dl = sl.take(n);
  float       *du = sl.take(n);
  float       *dd = deposition_map ? sl.take(n) : nullptr;
  float       *scr = sl.take(hm::layer_scratch_floats(nx, ny));
  cudaStream_t s = ctx->stream;
  HM_CUDA_TRY(cudaMemcpyAsync(dz, z, nbytes, cudaMemcpyHostToDevice, s));
  HM_CUDA_TRY(cudaMemcpyAsync(dl, talus_layer, nbytes, cudaMemcpyHostToDevice, s));
  HM_CUDA_TRY(cudaMemcpyAsync(du, talus_upper_limit, nbytes, cudaMemcpyHostToDevice, s));
  st = hm::layer_core(ctx->device, dz, nx, ny, dl, du, iterations, apply_post_filter != 0, dd, scr, s);
  if (st)
  {
    cudaStreamSynchronize(s);
    return st;
  }
  HM_CUDA_TRY(cudaMemcpyAsync(z, dz, nbytes, cudaMemcpyDeviceToHost, s));
  if (dd) HM_CUDA_TRY(cudaMemcpyAsync(deposition_map, dd, nbytes, cudaMemcpyDeviceToHost, s));
  HM_CUDA_TRY(cudaStreamSynchronize(s));
  return HM_OK;
}

int hm_sediment_layer_device(hm_context *ctx, float *z, int nx, int ny, const float *talus_layer,
                             const float *talus_upper_limit, int iterations, int apply_post_filter,
                             float *deposition_map, void *stream)
{
  hm::clear_error();
  int st = layer_check(ctx, z, nx, ny, talus_layer, talus_upper_limit, iterations);
  if (st) return st;
  if ((st = hm::use_device(ctx->device))) return st;
  void *ws = nullptr;
  if ((st = hm::workspace(ctx, hm::layer_scratch_floats(nx, ny) * sizeof(float), &ws))) return st;
  return hm::layer_core(ctx->device, z, nx, ny, talus_layer, talus_upper_limit, iterations, apply_post_filter != 0,
                        deposition_map, (float *)ws, (cudaStream_t)stream);
}

namespace
{
int snow_check(hm_context *ctx, const float *z, const float *s, int nx, int ny, int iterations)
{
  if (!ctx) return hm::fail(HM_ERR_INVALID_ARGUMENT, "snow_post_filter: ctx is NULL");
  if (!s) return hm::fail(HM_ERR_INVALID_ARGUMENT, "snow_post_filter: s is NULL");
  return hm::thermal_check_args(z, nx, ny, iterations, nullptr);
}
} // namespace

int hm_snow_post_filter(hm_context *ctx, const float *z, float *s, int nx, int ny, float snow_depth, int iterations,
                        float thermal_talus_ratio)
{
  hm::clear_error();
  int st = snow_check(ctx, z, s, nx, ny, iterations);
  if (st) return st;
  if ((st = hm::use_device(ctx->device))) return st;
  const size_t n = (size_t)nx * ny;
  const size_t nbytes = n * sizeof(float);
  const size_t total = 2 * align_up(nbytes, 256) + align_up(hm::snow_scratch_floats(nx, ny) * 4, 256);
  void        *ws = nullptr;
  if ((st = hm::workspace(ctx, total, &ws))) return st;
  Slab         sl{(char *)ws};
  float       *dz = sl.take(n);
  float       *ds = sl.take(n);
  float       *scr = sl.take(hm::snow_scratch_floats(nx, ny));
  cudaStream_t cs = ctx->stream;
  HM_CUDA_TRY(cudaMemcpyAsync(dz, z, nbytes, cudaMemcpyHostToDevice, cs));
  HM_CUDA_TRY(cudaMemcpyAsync(ds, s, nbytes, cudaMemcpyHostToDevice, cs));
  st = hm::snow_post_filter_core(ctx->device, dz, ds, nx, ny, snow_depth, iterations, thermal_talus_ratio, scr, cs);
  if (st)
  {
    cudaStreamSynchronize(cs);
    return st;
  }
  HM_CUDA_TRY(cudaMemcpyAsync(s, ds, nbytes, cudaMemcpyDeviceToHost, cs));
  HM_CUDA_TRY(cudaStreamSynchronize(cs));
  return HM_OK;
}

int hm_snow_post_filter_device(hm_context *ctx, const float *z, float *s, int nx, int ny, float snow_depth,
                               int iterations, float thermal_talus_ratio, void *stream)
{
  hm::clear_error();
  int st = snow_check(ctx, z, s, nx, ny, iterations);
  if (st) return st;
  if ((st = hm::use_device(ctx->device))) return st;
  void *ws = nullptr;
  if ((st = hm::workspace(ctx, hm::snow_scratch_floats(nx, ny) * sizeof(float), &ws))) return st;
  return hm::snow_post_filter_core(ctx->device, z, s, nx, ny, snow_depth, iterations, thermal_talus_ratio,
                                   (float *)ws, (cudaStream_t)stream);
}

int hm_thermal_ridge(hm_context *ctx, float *z, int nx, int ny, const float *talus, int iterations,
                     float *deposition_map, const float *mask)
{
  return sibling_host(ctx, HM_RIDGE, z, nx, ny, talus, nullptr, 0.f, iterations, deposition_map, mask);
}

int hm_thermal_scree(hm_context *ctx, float *z, int nx, int ny, const float *talus, const float *zmax,
                     int iterations, float *deposition_map, const float *mask)
{
  return sibling_host(ctx, HM_SCREE, z, nx, ny, talus, zmax, 0.f, iterations, deposition_map, mask);
}

int hm_thermal_schott(hm_context *ctx, float *z, int nx, int ny, const float *talus, int iterations,
                      float intensity, float *deposition_map, const float *mask)
{
  return sibling_host(ctx, HM_SCHOTT, z, nx, ny, talus, nullptr, intensity, iterations, deposition_map, mask);
}

int hm_thermal_olsen(hm_context *ctx, float *z, int nx, int ny, const float *talus, int iterations,
                     const float *mask)
{
  return sibling_host(ctx, HM_OLSEN, z, nx, ny, talus, nullptr, 0.f, iterations, nullptr, mask);
}

int hm_thermal_stencil_device(hm_context *ctx, int rule, float *z, int nx, int ny, const float *talus,
                              const float *zmax, float intensity, int iterations, float *deposition_map,
                              const float *mask, void *stream)
{
  hm::clear_error();
  if (!ctx) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_thermal_stencil_device: ctx is NULL");
  if (rule > HM_OLSEN)
    return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_thermal_stencil_device: rules above HM_OLSEN go through "
                                             "hm_thermal_relief_device");
  int st = hm::sibling_check_args(rule, z, nx, ny, talus, zmax, iterations);
  if (st) return st;
  if ((st = hm::use_device(ctx->device))) return st;
  void *ws = nullptr;
  if ((st = hm::workspace(ctx, hm::thermal_scratch_floats(nx, ny, true) * sizeof(float), &ws))) return st;
  return hm::sibling_core(ctx->device, rule, z, nx, ny, talus, zmax, intensity, iterations, deposition_map, mask,
                          (float *)ws, (cudaStream_t)stream);
}

int hm_flow_simulation(hm_context *ctx, const float *z, int nx, int ny, float water_height, const float *depth_map,
                       int iterations, float dt, int flux_diffusion, float flux_diffusion_strength,
                       float dry_out_ratio, float *water_depth)
{
  hm::clear_error();
  if (!ctx) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_flow_simulation: ctx is NULL");
  int st = hm::flow_check_args(z, depth_map, water_depth, nx, ny, iterations, dt);
  if (st) return st;
  if ((st = hm::use_device(ctx->device))) return st;
  const size_t n = (size_t)nx * ny;
  const size_t nbytes = n * sizeof(float);
  const size_t total = 3 * align_up(nbytes, 256) + align_up(hm::flow_scratch_bytes(nx, ny), 256);
  void        *ws = nullptr;
  if ((st = hm::workspace(ctx, total, &ws))) return st;
  Slab         sl{(char *)ws};
  float       *dz = sl.take(n);
  float       *dm = sl.take(n);
  float       *dd = sl.take(n);
  void        *scr = sl.take_bytes(hm::flow_scratch_bytes(nx, ny));
  cudaStream_t s = ctx->stream;
  HM_CUDA_TRY(cudaMemcpyAsync(dz, z, nbytes, cudaMemcpyHostToDevice, s));
  HM_CUDA_TRY(cudaMemcpyAsync(dm, depth_map, nbytes, cudaMemcpyHostToDevice, s));
  st = hm::flow_simulation_core(dz, nx, ny, water_height, dm, iterations, dt, flux_diffusion, flux_diffusion_strength,
                                dry_out_ratio, dd, scr, s);
  if (st)
  {
    cudaStreamSynchronize(s);
    return st;
  }
  HM_CUDA_TRY(cudaMemcpyAsync(water_depth, dd, nbytes, cudaMemcpyDeviceToHost, s));
  unsigned dev_error = 0;
  HM_CUDA_TRY(
      cudaMemcpyAsync(&dev_error, hm::flow_error_word(scr, nx, ny), sizeof dev_error, cudaMemcpyDeviceToHost, s));
  HM_CUDA_TRY(cudaStreamSynchronize(s));
  if (dev_error) return hm::fail(HM_ERR_TIMEOUT, "hm_flow_simulation: tile loads timed out on the device");
  return HM_OK;
}

int hm_flow_simulation_device(hm_context *ctx, const float *z, int nx, int ny, float water_height,
                              const float *depth_map, int iterations, float dt, int flux_diffusion,
                              float flux_diffusion_strength, float dry_out_ratio, float *water_depth, void *stream)
{
  hm::clear_error();
  if (!ctx) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_flow_simulation_device: ctx is NULL");
  int st = hm::flow_check_args(z, depth_map, water_depth, nx, ny, iterations, dt);
  if (st) return st;
  if ((st = hm::use_device(ctx->device))) return st;
  void *ws = nullptr;
  if ((st = hm::workspace(ctx, hm::flow_scratch_bytes(nx, ny), &ws))) return st;
  return hm::flow_simulation_core(z, nx, ny, water_height, depth_map, iterations, dt, flux_diffusion,
                                  flux_diffusion_strength, dry_out_ratio, water_depth, ws, (cudaStream_t)stream);
}

int hm_flow_simulation_viscous(hm_context *ctx, const float *z, int nx, int ny, float water_height,
                               const float *depth_map, int iterations, float dt, float dry_out_ratio,
                               float viscosity, float power, float *water_depth)
{
  hm::clear_error();
  if (!ctx) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_flow_simulation_viscous: ctx is NULL");
  int st = hm::vflow_check_args(z, depth_map, water_depth, nx, ny, iterations);
  if (st) return st;
  if ((st = hm::use_device(ctx->device))) return st;
  const size_t n = (size_t)nx * ny;
  const size_t nbytes = n * sizeof(float);
  const size_t total = 3 * align_up(nbytes, 256) + align_up(hm::vflow_scratch_bytes(nx, ny), 256);
  void        *ws = nullptr;
  if ((st = hm::workspace(ctx, total, &ws))) return st;
  Slab         sl{(char *)ws};
  float       *dz = sl.take(n);
  float       *ddm = sl.take(n);
  float       *dout = sl.take(n);
  void        *scr = sl.take_bytes(hm::vflow_scratch_bytes(nx, ny));
  cudaStream_t s = ctx->stream;
  HM_CUDA_TRY(cudaMemcpyAsync(dz, z, nbytes, cudaMemcpyHostToDevice, s));
  HM_CUDA_TRY(cudaMemcpyAsync(ddm, depth_map, nbytes, cudaMemcpyHostToDevice, s));
  st = hm::vflow_core(dz, nx, ny, water_height, ddm, iterations, dt, dry_out_ratio, viscosity, power, dout, scr, s);
  if (st)
  {
    cudaStreamSynchronize(s);
    return st;
  }
  HM_CUDA_TRY(cudaMemcpyAsync(water_depth, dout, nbytes, cudaMemcpyDeviceToHost, s));
  HM_CUDA_TRY(cudaStreamSynchronize(s));
  return HM_OK;
}

int hm_flow_simulation_viscous_device(hm_context *ctx, const float *z, int nx, int ny, float water_height,
                                      const float *depth_map, int iterations, float dt, float dry_out_ratio,
                                      float viscosity, float power, float *water_depth, void *stream)
{
  hm::clear_error();
  if (!ctx) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_flow_simulation_viscous_device: ctx is NULL");
  int st = hm::vflow_check_args(z, depth_map, water_depth, nx, ny, iterations);
  if (st) return st;
  if ((st = hm::use_device(ctx->device))) return st;
  void *ws = nullptr;
  if ((st = hm::workspace(ctx, hm::vflow_scratch_bytes(nx, ny), &ws))) return st;
  return hm::vflow_core(z, nx, ny, water_height, depth_map, iterations, dt, dry_out_ratio, viscosity, power,
                        water_depth, ws, (cudaStream_t)stream);
}

int hm_vpipes(hm_context *ctx, float *z, int nx, int ny, const hm_vpipes_params *params, const float *rain_map,
              float *water_depth, float *sediment, float *vel_u, float *vel_v)
{
  hm::clear_error();
  if (!ctx) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_vpipes: ctx is NULL");
  hm_vpipes_params p;
  hm_vpipes_default_params(&p);
  if (params) p = *params;
  int st = hm::vpipes_check_args(z, nx, ny, &p);
  if (st) return st;
  if ((st = hm::use_device(ctx->device))) return st;
  const size_t n = (size_t)nx * ny;
  const size_t nbytes = n * sizeof(float);
  size_t       fields = 1 + (rain_map ? 1 : 0) + (water_depth ? 1 : 0) + (sediment ? 1 : 0) + (vel_u ? 1 : 0) +
                  (vel_v ? 1 : 0);
  size_t total = fields * align_up(nbytes, 256) + align_up(hm::vpipes_scratch_bytes(nx, ny), 256);
  void  *ws = nullptr;
  if ((st = hm::workspace(ctx, total, &ws))) return st;
  Slab         sl{(char *)ws};
  float       *dz = sl.take(n);
  float       *dr = rain_map ? sl.take(n) : nullptr;
  float       *dd = water_depth ? sl.take(n) : nullptr;
  float       *ds = sediment ? sl.take(n) : nullptr;
  float       *du = vel_u ? sl.take(n) : nullptr;
  float       *dv = vel_v ? sl.take(n) : nullptr;
  void        *scr = sl.take_bytes(hm::vpipes_scratch_bytes(nx, ny));
  cudaStream_t s = ctx->stream;
  HM_CUDA_TRY(cudaMemcpyAsync(dz, z, nbytes, cudaMemcpyHostToDevice, s));
  if (dr) HM_CUDA_TRY(cudaMemcpyAsync(dr, rain_map, nbytes, cudaMemcpyHostToDevice, s));
  st = hm::vpipes_core(dz, nx, ny, p, dr, dd, ds, du, dv, scr, s);
  if (st)
  {
    cudaStreamSynchronize(s);
    return st;
  }
  /* a tile whose loads timed out wrote nothing: report it before the
   * results reach the caller's buffers, which then keep their contents */
  unsigned dev_error = 0;
  HM_CUDA_TRY(cudaMemcpyAsync(&dev_error, hm::vpipes_error_word(scr, nx, ny), sizeof dev_error,
                              cudaMemcpyDeviceToHost, s));
  HM_CUDA_TRY(cudaStreamSynchronize(s));
  if (dev_error) return hm::fail(HM_ERR_TIMEOUT, "hm_vpipes: tile loads timed out on the device");
  HM_CUDA_TRY(cudaMemcpyAsync(z, dz, nbytes, cudaMemcpyDeviceToHost, s));
  if (dd) HM_CUDA_TRY(cudaMemcpyAsync(water_depth, dd, nbytes, cudaMemcpyDeviceToHost, s));
  if (ds) HM_CUDA_TRY(cudaMemcpyAsync(sediment, ds, nbytes, cudaMemcpyDeviceToHost, s));
  if (du) HM_CUDA_TRY(cudaMemcpyAsync(vel_u, du, nbytes, cudaMemcpyDeviceToHost, s));
  if (dv) HM_CUDA_TRY(cudaMemcpyAsync(vel_v, dv, nbytes, cudaMemcpyDeviceToHost, s));
  HM_CUDA_TRY(cudaStreamSynchronize(s));
  return HM_OK;
}

int hm_vpipes_device(hm_context *ctx, float *z, int nx, int ny, const hm_vpipes_params *params,
                     const float *rain_map, float *water_depth, float *sediment, float *vel_u, float *vel_v,
                     void *stream)
{
  hm::clear_error();
  if (!ctx) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_vpipes_device: ctx is NULL");
  hm_vpipes_params p;
  hm_vpipes_default_params(&p);
  if (params) p = *params;
  int st = hm::vpipes_check_args(z, nx, ny, &p);
  if (st) return st;
  if ((st = hm::use_device(ctx->device))) return st;
  void *ws = nullptr;
  if ((st = hm::workspace(ctx, hm::vpipes_scratch_bytes(nx, ny), &ws))) return st;
  return hm::vpipes_core(z, nx, ny, p, rain_map, water_depth, sediment, vel_u, vel_v, ws, (cudaStream_t)stream);
}


int hm_thermal_flatten(hm_context *ctx, float *z, int nx, int ny, const float *talus, int iterations,
                       float sigma_inf, float sigma_sup, const float *mask)
{
  return sibling_host(ctx, HM_FLATTEN, z, nx, ny, talus, nullptr, sigma_inf, iterations, nullptr, mask, sigma_sup);
}

int hm_thermal_inflate(hm_context *ctx, float *z, int nx, int ny, const float *talus, int iterations,
                       const float *mask)
{
  return sibling_host(ctx, HM_INFLATE, z, nx, ny, talus, nullptr, 0.f, iterations, nullptr, mask);
}

int hm_thermal_rib(hm_context *ctx, float *z, int nx, int ny, int iterations, const float *mask)
{
  return sibling_host(ctx, HM_RIB, z, nx, ny, nullptr, nullptr, 0.f, iterations, nullptr, mask);
}

int hm_thermal_relief_device(hm_context *ctx, int rule, float *z, int nx, int ny, const float *talus, float sigma_inf,
                             float sigma_sup, int iterations, const float *mask, void *stream)
{
  hm::clear_error();
  if (!ctx) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_thermal_relief_device: ctx is NULL");
  if (rule < HM_FLATTEN || rule > HM_RIB)
    return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_thermal_relief_device: rule must be HM_FLATTEN .. HM_RIB");
  const float *t = rule == HM_RIB ? nullptr : talus;
  int          st = hm::sibling_check_args(rule, z, nx, ny, t, nullptr, iterations);
  if (st) return st;
  if ((st = hm::use_device(ctx->device))) return st;
  void *ws = nullptr;
  if ((st = hm::workspace(ctx, hm::thermal_scratch_floats(nx, ny, true) * sizeof(float), &ws))) return st;
  return hm::sibling_core(ctx->device, rule, z, nx, ny, t, nullptr, sigma_inf, iterations, nullptr, mask,
                          (float *)ws, (cudaStream_t)stream, sigma_sup);
}

} // extern "C"
