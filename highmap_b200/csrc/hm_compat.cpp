/*
 * hm_compat.cpp - hmap::gpu::thermal / hydraulic_vpipes / init_opencl over
 * the C-ABI (include/highmap_b200/hmap_gpu.hpp).
 *
 * Mirrors the reference drivers' interface and error behaviour:
 *   thermal          HighMap/src/erosion/thermal_gpu.cpp:17-96
 *   thermal_auto_bedrock  HighMap/src/erosion/thermal_gpu.cpp:98-152
 *   hydraulic_vpipes HighMap/src/erosion/hydraulic_vpipes_gpu.cpp:15-178
 *   flow_simulation  HighMap/src/hydrology/flow_simulation.cpp:26-110
 *   thermal_olsen / _ridge / _schott / _scree  HighMap/src/erosion/thermal_gpu.cpp:221-396
 *   sediment_deposition  HighMap/src/erosion/deposition.cpp:19-66
 *   sediment_layer       HighMap/src/erosion/deposition.cpp:68-113
 *   thermal_flatten, thermal_inflate, thermal_rib  thermal_gpu.cpp:154-219,249-272
 *   flow_simulation_viscous  HighMap/src/hydrology/flow_simulation.cpp:112-157
 *   init_opencl      HighMap/src/gpu_opencl/gpu_opencl.cpp:32-134
 * The reference functions return void and report problems only through
 * their logger; here a failed call leaves z untouched, prints the status
 * to stderr and records it for hmap::gpu::last_error().  Optional outputs
 * are resized to z's shape and overwritten, as `*p = d` does in the
 * reference.  Each thread uses its own context on device 0.
 */
#include <algorithm>
#include <cstdio>
#include <memory>
#include <string>

#include "highmap_b200/hmap_gpu.hpp"
#include "hm_erosion.h"

namespace hmap
{
namespace gpu
{

namespace
{

thread_local std::string g_err;

struct CtxHolder
{
  hm_context *ctx = nullptr;
  ~CtxHolder()
  {
    if (ctx) hm_context_destroy(ctx);
  }
};

hm_context *context()
{
  thread_local CtxHolder h;
  if (!h.ctx)
  {
    if (hm_context_create(&h.ctx, 0) != HM_OK) h.ctx = nullptr;
  }
  return h.ctx;
}

bool report(int st, const char *fn)
{
  if (st == HM_OK)
  {
    g_err.clear();
    return true;
  }
  g_err = std::string(fn) + ": " + hm_status_string(st) + ": " + hm_last_error();
  std::fprintf(stderr, "[highmap_b200] %s\n", g_err.c_str());
  return false;
}

void shape_like(Array *p, const Array &z)
{
  if (!p) return;
  p->shape = z.shape;
  p->vector.resize((size_t)z.shape.x * (size_t)z.shape.y);
}

bool same_shape(const Array *a, const Array &z)
{
  return !a || (a->shape.x == z.shape.x && a->shape.y == z.shape.y &&
                a->vector.size() == (size_t)z.shape.x * (size_t)z.shape.y);
}

void thermal_impl(Array &z, const Array *p_mask, const Array *talus, float talus_value, int iterations,
                  Array *p_bedrock, Array *p_deposition_map, bool auto_bed = false)
{
  const char *fn = auto_bed ? "hmap::gpu::thermal_auto_bedrock" : "hmap::gpu::thermal";
  if (!same_shape(talus, z) || !same_shape(p_mask, z) || !same_shape(p_bedrock, z) ||
      z.vector.size() != (size_t)z.shape.x * (size_t)z.shape.y)
  {
    report(HM_ERR_INVALID_ARGUMENT, fn);
    g_err += "arrays of different shapes";
    return;
  }
  hm_context *ctx = context();
  if (!ctx)
  {
    report(HM_ERR_NO_DEVICE, fn);
    return;
  }
  std::vector<float> depo;
  if (p_deposition_map) depo.resize(z.vector.size());
  std::vector<float> zw(z.vector);
  float             *dp = p_deposition_map ? depo.data() : nullptr;
  const float       *bp = p_bedrock ? p_bedrock->vector.data() : nullptr;
  int                st;
  if (auto_bed)
  {
    if (p_mask)
      st = hm_thermal_auto_bedrock_masked(ctx, zw.data(), z.shape.x, z.shape.y, p_mask->vector.data(),
                                          talus->vector.data(), iterations, dp, nullptr);
    else if (talus)
      st = hm_thermal_auto_bedrock(ctx, zw.data(), z.shape.x, z.shape.y, talus->vector.data(), iterations, dp,
                                   nullptr);
    else
      st = hm_thermal_auto_bedrock_scalar(ctx, zw.data(), z.shape.x, z.shape.y, talus_value, iterations, dp,
                                          nullptr);
  }
  else if (p_mask)
    st = hm_thermal_masked(ctx, zw.data(), z.shape.x, z.shape.y, p_mask->vector.data(), talus->vector.data(),
                           iterations, bp, dp, nullptr);
  else if (talus)
    st = hm_thermal(ctx, zw.data(), z.shape.x, z.shape.y, talus->vector.data(), iterations, bp, dp, nullptr);
  else
    st = hm_thermal_scalar(ctx, zw.data(), z.shape.x, z.shape.y, talus_value, iterations, bp, dp, nullptr);
  if (!report(st, fn)) return;
  z.vector.swap(zw);
  if (p_deposition_map)
  {
    shape_like(p_deposition_map, z);
    p_deposition_map->vector.swap(depo);
  }
}

} // namespace

bool init_opencl() { return hm_init() == HM_OK; }

std::string last_error() { return g_err; }

void thermal(Array &z, const Array &talus, int iterations, Array *p_bedrock, Array *p_deposition_map)
{
  thermal_impl(z, nullptr, &talus, 0.f, iterations, p_bedrock, p_deposition_map);
}

void thermal(Array &z, const Array *p_mask, const Array &talus, int iterations, Array *p_bedrock,
             Array *p_deposition_map)
{
  thermal_impl(z, p_mask, &talus, 0.f, iterations, p_bedrock, p_deposition_map);
}

void thermal(Array &z, float talus, int iterations, Array *p_bedrock, Array *p_deposition_map)
{
  thermal_impl(z, nullptr, nullptr, talus, iterations, p_bedrock, p_deposition_map);
}

void thermal_auto_bedrock(Array &z, const Array &talus, int iterations, Array *p_deposition_map)
{
  thermal_impl(z, nullptr, &talus, 0.f, iterations, nullptr, p_deposition_map, true);
}

void thermal_auto_bedrock(Array &z, const Array *p_mask, const Array &talus, int iterations,
                          Array *p_deposition_map)
{
  thermal_impl(z, p_mask, &talus, 0.f, iterations, nullptr, p_deposition_map, true);
}

void thermal_auto_bedrock(Array &z, float talus, int iterations, Array *p_deposition_map)
{
  thermal_impl(z, nullptr, nullptr, talus, iterations, nullptr, p_deposition_map, true);
}

namespace
{
void sibling_impl(int rule, const char *fn, Array &z, const Array *p_mask, const Array &talus, const Array *zmax,
                  float intensity, int iterations, Array *p_deposition_map)
{
  if (!same_shape(&talus, z) || !same_shape(p_mask, z) || !same_shape(zmax, z) ||
      z.vector.size() != (size_t)z.shape.x * (size_t)z.shape.y)
  {
    report(HM_ERR_INVALID_ARGUMENT, fn);
    g_err += "arrays of different shapes";
    return;
  }
  hm_context *ctx = context();
  if (!ctx)
  {
    report(HM_ERR_NO_DEVICE, fn);
    return;
  }
  std::vector<float> depo;
  if (p_deposition_map) depo.resize(z.vector.size());
  std::vector<float> zw(z.vector);
  float             *dp = p_deposition_map ? depo.data() : nullptr;
  const float       *mp = p_mask ? p_mask->vector.data() : nullptr;
  int                st;
  switch (rule)
  {
  case HM_RIDGE: st = hm_thermal_ridge(ctx, zw.data(), z.shape.x, z.shape.y, talus.vector.data(), iterations, dp, mp); break;
  case HM_SCREE:
    st = hm_thermal_scree(ctx, zw.data(), z.shape.x, z.shape.y, talus.vector.data(), zmax->vector.data(), iterations,
                          dp, mp);
    break;
  case HM_SCHOTT:
    st = hm_thermal_schott(ctx, zw.data(), z.shape.x, z.shape.y, talus.vector.data(), iterations, intensity, dp, mp);
    break;
  default: st = hm_thermal_olsen(ctx, zw.data(), z.shape.x, z.shape.y, talus.vector.data(), iterations, mp);
  }
  if (!report(st, fn)) return;
  z.vector.swap(zw);
  if (p_deposition_map)
  {
    shape_like(p_deposition_map, z);
    p_deposition_map->vector.swap(depo);
  }
}
} // namespace

void sediment_deposition(Array &z, Array *p_mask, const Array &talus, Array *p_deposition_map, float max_deposition,
                         int iterations, int thermal_subiterations)
{
  const char *fn = "hmap::gpu::sediment_deposition";
  if (!same_shape(&talus, z) || !same_shape(p_mask, z) || z.vector.size() != (size_t)z.shape.x * (size_t)z.shape.y)
  {
    report(HM_ERR_INVALID_ARGUMENT, fn);
    g_err += "arrays of different shapes";
    return;
  }
  hm_context *ctx = context();
  if (!ctx)
  {
    report(HM_ERR_NO_DEVICE, fn);
    return;
  }
  std::vector<float> zw(z.vector), depo(p_deposition_map ? z.vector.size() : 0);
  int st = hm_sediment_deposition(ctx, zw.data(), z.shape.x, z.shape.y, talus.vector.data(), max_deposition,
                                  iterations, thermal_subiterations, p_deposition_map ? depo.data() : nullptr,
                                  p_mask ? p_mask->vector.data() : nullptr);
  if (!report(st, fn)) return;
  z.vector.swap(zw);
  if (p_deposition_map)
  {
    shape_like(p_deposition_map, z);
    p_deposition_map->vector.swap(depo);
  }
}

void sediment_deposition(Array &z, const Array &talus, Array *p_deposition_map, float max_deposition,
                         int iterations, int thermal_subiterations)
{
  sediment_deposition(z, nullptr, talus, p_deposition_map, max_deposition, iterations, thermal_subiterations);
}

void sediment_layer(Array &z, const Array &talus_layer, const Array &talus_upper_limit, int iterations,
                    bool apply_post_filter, Array *p_deposition_map)
{
  const char *fn = "hmap::gpu::sediment_layer";
  if (!same_shape(&talus_layer, z) || !same_shape(&talus_upper_limit, z) ||
      z.vector.size() != (size_t)z.shape.x * (size_t)z.shape.y)
  {
    report(HM_ERR_INVALID_ARGUMENT, fn);
    g_err += "arrays of different shapes";
    return;
  }
  hm_context *ctx = context();
  if (!ctx)
  {
    report(HM_ERR_NO_DEVICE, fn);
    return;
  }
  std::vector<float> zw(z.vector), depo(p_deposition_map ? z.vector.size() : 0);
  int st = hm_sediment_layer(ctx, zw.data(), z.shape.x, z.shape.y, talus_layer.vector.data(),
                             talus_upper_limit.vector.data(), iterations, apply_post_filter ? 1 : 0,
                             p_deposition_map ? depo.data() : nullptr);
  if (!report(st, fn)) return;
  z.vector.swap(zw);
  if (p_deposition_map)
  {
    shape_like(p_deposition_map, z);
    p_deposition_map->vector.swap(depo);
  }
}

/* thermal_flatten / thermal_inflate / thermal_rib (thermal_gpu.cpp:154-219,
 * 249-272): talus NULL for rib */
void relief_impl(int rule, const char *fn, Array &z, const Array *p_mask, const Array *talus, float sigma_inf,
                 float sigma_sup, int iterations)
{
  if (!same_shape(talus, z) || !same_shape(p_mask, z) || z.vector.size() != (size_t)z.shape.x * (size_t)z.shape.y)
  {
    report(HM_ERR_INVALID_ARGUMENT, fn);
    g_err += "arrays of different shapes";
    return;
  }
  hm_context *ctx = context();
  if (!ctx)
  {
    report(HM_ERR_NO_DEVICE, fn);
    return;
  }
  std::vector<float> zw(z.vector);
  const float       *mp = p_mask ? p_mask->vector.data() : nullptr;
  int                st;
  if (rule == HM_FLATTEN)
    st = hm_thermal_flatten(ctx, zw.data(), z.shape.x, z.shape.y, talus->vector.data(), iterations, sigma_inf,
                            sigma_sup, mp);
  else if (rule == HM_INFLATE)
    st = hm_thermal_inflate(ctx, zw.data(), z.shape.x, z.shape.y, talus->vector.data(), iterations, mp);
  else
    st = hm_thermal_rib(ctx, zw.data(), z.shape.x, z.shape.y, iterations, mp);
  if (!report(st, fn)) return;
  z.vector.swap(zw);
}

void thermal_flatten(Array &z, const Array &talus, int iterations, float sigma_inf, float sigma_sup)
{
  relief_impl(HM_FLATTEN, "hmap::gpu::thermal_flatten", z, nullptr, &talus, sigma_inf, sigma_sup, iterations);
}

void thermal_flatten(Array &z, const Array *p_mask, const Array &talus, int iterations, float sigma_inf,
                     float sigma_sup)
{
  relief_impl(HM_FLATTEN, "hmap::gpu::thermal_flatten", z, p_mask, &talus, sigma_inf, sigma_sup, iterations);
}

void thermal_inflate(Array &z, const Array &talus, int iterations)
{
  relief_impl(HM_INFLATE, "hmap::gpu::thermal_inflate", z, nullptr, &talus, 0.f, 0.f, iterations);
}

void thermal_inflate(Array &z, const Array *p_mask, const Array &talus, int iterations)
{
  relief_impl(HM_INFLATE, "hmap::gpu::thermal_inflate", z, p_mask, &talus, 0.f, 0.f, iterations);
}

void thermal_rib(Array &z, int iterations)
{
  relief_impl(HM_RIB, "hmap::gpu::thermal_rib", z, nullptr, nullptr, 0.f, 0.f, iterations);
}

void thermal_rib(Array &z, const Array *p_mask, int iterations)
{
  relief_impl(HM_RIB, "hmap::gpu::thermal_rib", z, p_mask, nullptr, 0.f, 0.f, iterations);
}

void thermal_olsen(Array &z, const Array &talus, int iterations)
{
  sibling_impl(HM_OLSEN, "hmap::gpu::thermal_olsen", z, nullptr, talus, nullptr, 0.f, iterations, nullptr);
}

void thermal_olsen(Array &z, const Array *p_mask, const Array &talus, int iterations)
{
  sibling_impl(HM_OLSEN, "hmap::gpu::thermal_olsen", z, p_mask, talus, nullptr, 0.f, iterations, nullptr);
}

void thermal_ridge(Array &z, const Array &talus, int iterations, Array *p_deposition_map)
{
  sibling_impl(HM_RIDGE, "hmap::gpu::thermal_ridge", z, nullptr, talus, nullptr, 0.f, iterations, p_deposition_map);
}

void thermal_ridge(Array &z, const Array *p_mask, const Array &talus, int iterations, Array *p_deposition_map)
{
  sibling_impl(HM_RIDGE, "hmap::gpu::thermal_ridge", z, p_mask, talus, nullptr, 0.f, iterations, p_deposition_map);
}

void thermal_schott(Array &z, const Array &talus, int iterations, float intensity, Array *p_deposition_map)
{
  sibling_impl(HM_SCHOTT, "hmap::gpu::thermal_schott", z, nullptr, talus, nullptr, intensity, iterations,
               p_deposition_map);
}

void thermal_schott(Array &z, const Array *p_mask, const Array &talus, int iterations, float intensity,
                    Array *p_deposition_map)
{
  sibling_impl(HM_SCHOTT, "hmap::gpu::thermal_schott", z, p_mask, talus, nullptr, intensity, iterations,
               p_deposition_map);
}

void thermal_scree(Array &z, const Array &talus, const Array &zmax, int iterations, Array *p_deposition_map)
{
  sibling_impl(HM_SCREE, "hmap::gpu::thermal_scree", z, nullptr, talus, &zmax, 0.f, iterations, p_deposition_map);
}

void thermal_scree(Array &z, const Array *p_mask, const Array &talus, const Array &zmax, int iterations,
                   Array *p_deposition_map)
{
  sibling_impl(HM_SCREE, "hmap::gpu::thermal_scree", z, p_mask, talus, &zmax, 0.f, iterations, p_deposition_map);
}

Array flow_simulation(const Array &z, float water_height, const Array &depth_map, int iterations, float dt,
                      bool flux_diffusion, float flux_diffusion_strength, float dry_out_ratio)
{
  const char *fn = "hmap::gpu::flow_simulation";
  Array       out;
  shape_like(&out, z);
  std::fill(out.vector.begin(), out.vector.end(), 0.f);
  if (!same_shape(&depth_map, z) || z.vector.size() != (size_t)z.shape.x * (size_t)z.shape.y)
  {
    report(HM_ERR_INVALID_ARGUMENT, fn);
    g_err += "arrays of different shapes";
    return out;
  }
  hm_context *ctx = context();
  if (!ctx)
  {
    report(HM_ERR_NO_DEVICE, fn);
    return out;
  }
  std::vector<float> d(z.vector.size());
  int st = hm_flow_simulation(ctx, z.vector.data(), z.shape.x, z.shape.y, water_height, depth_map.vector.data(),
                              iterations, dt, flux_diffusion ? 1 : 0, flux_diffusion_strength, dry_out_ratio,
                              d.data());
  if (report(st, fn)) out.vector.swap(d);
  return out;
}

Array flow_simulation_viscous(const Array &z, float water_depth, const Array &depth_map, int iterations, float dt,
                              float dry_out_ratio, float viscosity, float power)
{
  const char *fn = "hmap::gpu::flow_simulation_viscous";
  Array       out;
  shape_like(&out, z);
  std::fill(out.vector.begin(), out.vector.end(), 0.f);
  if (!same_shape(&depth_map, z) || z.vector.size() != (size_t)z.shape.x * (size_t)z.shape.y)
  {
    report(HM_ERR_INVALID_ARGUMENT, fn);
    g_err += "arrays of different shapes";
    return out;
  }
  hm_context *ctx = context();
  if (!ctx)
  {
    report(HM_ERR_NO_DEVICE, fn);
    return out;
  }
  std::vector<float> d(z.vector.size());
  int st = hm_flow_simulation_viscous(ctx, z.vector.data(), z.shape.x, z.shape.y, water_depth,
                                      depth_map.vector.data(), iterations, dt, dry_out_ratio, viscosity, power,
                                      d.data());
  if (report(st, fn)) out.vector.swap(d);
  return out;
}

void hydraulic_vpipes(Array &z, float water_height, bool maintain_water_volume, float evap_rate, int iterations,
                      float dt, float k_capacity, float k_erode, float k_depose, float k_discharge_exp,
                      float downcutting_max_depth_ratio, bool flux_diffusion, float flux_diffusion_strength,
                      Array *p_rain_map, Array *p_water_depth, Array *p_sediment, Array *p_vel_u, Array *p_vel_v)
{
  const char *fn = "hmap::gpu::hydraulic_vpipes";
  if (!same_shape(p_rain_map, z) || z.vector.size() != (size_t)z.shape.x * (size_t)z.shape.y)
  {
    report(HM_ERR_INVALID_ARGUMENT, fn);
    g_err += "arrays of different shapes";
    return;
  }
  hm_context *ctx = context();
  if (!ctx)
  {
    report(HM_ERR_NO_DEVICE, fn);
    return;
  }
  hm_vpipes_params p;
  hm_vpipes_default_params(&p);
  p.water_height = water_height;
  p.maintain_water_volume = maintain_water_volume ? 1 : 0;
  p.evap_rate = evap_rate;
  p.iterations = iterations;
  p.dt = dt;
  p.k_capacity = k_capacity;
  p.k_erode = k_erode;
  p.k_depose = k_depose;
  p.k_discharge_exp = k_discharge_exp;
  p.downcutting_max_depth_ratio = downcutting_max_depth_ratio;
  p.flux_diffusion = flux_diffusion ? 1 : 0;
  p.flux_diffusion_strength = flux_diffusion_strength;
  const size_t       n = z.vector.size();
  std::vector<float> zw(z.vector), d, s, u, v;
  if (p_water_depth) d.resize(n);
  if (p_sediment) s.resize(n);
  if (p_vel_u) u.resize(n);
  if (p_vel_v) v.resize(n);
  int st = hm_vpipes(ctx, zw.data(), z.shape.x, z.shape.y, &p, p_rain_map ? p_rain_map->vector.data() : nullptr,
                     p_water_depth ? d.data() : nullptr, p_sediment ? s.data() : nullptr,
                     p_vel_u ? u.data() : nullptr, p_vel_v ? v.data() : nullptr);
  if (!report(st, fn)) return;
  z.vector.swap(zw);
  Array *outs[4] = {p_water_depth, p_sediment, p_vel_u, p_vel_v};
  std::vector<float> *vals[4] = {&d, &s, &u, &v};
  for (int k = 0; k < 4; k++)
    if (outs[k])
    {
      shape_like(outs[k], z);
      outs[k]->vector.swap(*vals[k]);
    }
}

} // namespace gpu
} // namespace hmap
