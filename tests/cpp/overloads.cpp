/*
 * overloads.cpp - takes the address of every hmap::gpu function that
 * include/highmap_b200/hmap_gpu.hpp declares, each with its exact
 * signature, so that linking this file against libhm_erosion.so proves every
 * declared overload is defined (built and linked by tests/test_lib.py; it is
 * not run).
 */
#include <cstdio>

#include "highmap_b200/hmap_gpu.hpp"

using hmap::Array;

int main()
{
  const void *fns[] = {
      (void *)static_cast<bool (*)()>(&hmap::gpu::init_opencl),
      (void *)static_cast<void (*)(Array &, const Array &, int, Array *, Array *)>(&hmap::gpu::thermal),
      (void *)static_cast<void (*)(Array &, const Array *, const Array &, int, Array *, Array *)>(&hmap::gpu::thermal),
      (void *)static_cast<void (*)(Array &, float, int, Array *, Array *)>(&hmap::gpu::thermal),
      (void *)static_cast<void (*)(Array &, const Array &, int, Array *)>(&hmap::gpu::thermal_auto_bedrock),
      (void *)static_cast<void (*)(Array &, const Array *, const Array &, int, Array *)>(
          &hmap::gpu::thermal_auto_bedrock),
      (void *)static_cast<void (*)(Array &, float, int, Array *)>(&hmap::gpu::thermal_auto_bedrock),
      (void *)static_cast<void (*)(Array &, Array *, const Array &, Array *, float, int, int)>(
          &hmap::gpu::sediment_deposition),
      (void *)static_cast<void (*)(Array &, const Array &, Array *, float, int, int)>(&hmap::gpu::sediment_deposition),
      (void *)static_cast<void (*)(Array &, const Array &, const Array &, int, bool, Array *)>(
          &hmap::gpu::sediment_layer),
      (void *)static_cast<void (*)(Array &, const Array &, int, float, float)>(&hmap::gpu::thermal_flatten),
      (void *)static_cast<void (*)(Array &, const Array *, const Array &, int, float, float)>(
          &hmap::gpu::thermal_flatten),
      (void *)static_cast<void (*)(Array &, const Array &, int)>(&hmap::gpu::thermal_inflate),
      (void *)static_cast<void (*)(Array &, const Array *, const Array &, int)>(&hmap::gpu::thermal_inflate),
      (void *)static_cast<void (*)(Array &, int)>(&hmap::gpu::thermal_rib),
      (void *)static_cast<void (*)(Array &, const Array *, int)>(&hmap::gpu::thermal_rib),
      (void *)static_cast<void (*)(Array &, const Array &, int)>(&hmap::gpu::thermal_olsen),
      (void *)static_cast<void (*)(Array &, const Array *, const Array &, int)>(&hmap::gpu::thermal_olsen),
      (void *)static_cast<void (*)(Array &, const Array &, int, Array *)>(&hmap::gpu::thermal_ridge),
      (void *)static_cast<void (*)(Array &, const Array *, const Array &, int, Array *)>(&hmap::gpu::thermal_ridge),
      (void *)static_cast<void (*)(Array &, const Array &, int, float, Array *)>(&hmap::gpu::thermal_schott),
      (void *)static_cast<void (*)(Array &, const Array *, const Array &, int, float, Array *)>(
          &hmap::gpu::thermal_schott),
      (void *)static_cast<void (*)(Array &, const Array &, const Array &, int, Array *)>(&hmap::gpu::thermal_scree),
      (void *)static_cast<void (*)(Array &, const Array *, const Array &, const Array &, int, Array *)>(
          &hmap::gpu::thermal_scree),
      (void *)static_cast<Array (*)(const Array &, float, const Array &, int, float, bool, float, float)>(
          &hmap::gpu::flow_simulation),
      (void *)static_cast<Array (*)(const Array &, float, const Array &, int, float, float, float, float)>(
          &hmap::gpu::flow_simulation_viscous),
      (void *)static_cast<void (*)(Array &, float, bool, float, int, float, float, float, float, float, float, bool,
                                   float, Array *, Array *, Array *, Array *, Array *)>(&hmap::gpu::hydraulic_vpipes),
      (void *)static_cast<std::string (*)()>(&hmap::gpu::last_error),
  };
  int n = 0;
  for (const void *f : fns) n += f != nullptr;
  std::printf("%d\n", n);
  return n == (int)(sizeof(fns) / sizeof(fns[0])) ? 0 : 1;
}
