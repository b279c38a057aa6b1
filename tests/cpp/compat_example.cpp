/*
 * compat_example.cpp - a caller written against HighMap's hmap::gpu API,
 * in the style of the reference's examples (examples/ex_thermal/ex_thermal.cpp,
 * examples/ex_hydraulic_vpipes_gpu/ex_hydraulic_vpipes_gpu.cpp), linked
 * against libhm_erosion.so.  Reads a raw float32 heightmap, runs the
 * requested solver, writes the results as raw float32 for the test to
 * compare with the oracle.
 *
 * usage: compat_example <thermal|config1|thermal_scalar|thermal_mask|auto_bedrock|auto_bedrock_mask|vpipes|flow|ridge|scree|schott|olsen|deposition|layer|flatten|inflate|rib|viscous>
 *        nx ny in.f32 out_prefix
 */
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "highmap_b200/hmap_gpu.hpp"

static bool read_raw(const char *path, hmap::Array &a)
{
  FILE *f = std::fopen(path, "rb");
  if (!f) return false;
  size_t n = std::fread(a.vector.data(), sizeof(float), a.vector.size(), f);
  std::fclose(f);
  return n == a.vector.size();
}

static void write_raw(const std::string &path, const hmap::Array &a)
{
  FILE *f = std::fopen(path.c_str(), "wb");
  std::fwrite(a.vector.data(), sizeof(float), a.vector.size(), f);
  std::fclose(f);
}

int main(int argc, char **argv)
{
  if (argc != 6) return 2;
  if (!hmap::gpu::init_opencl()) return 3;
  std::string mode = argv[1];
  glm::ivec2  shape(std::atoi(argv[2]), std::atoi(argv[3]));
  hmap::Array z(shape);
  if (!read_raw(argv[4], z)) return 4;
  std::string out = argv[5];

  if (mode == "thermal" || mode == "thermal_mask")
  {
    hmap::Array talus(shape, 1.f / shape.x);
    hmap::Array bedrock(shape);
    for (size_t k = 0; k < z.vector.size(); k++) bedrock.vector[k] = 0.3f * z.vector[k];
    hmap::Array depo;
    if (mode == "thermal")
      hmap::gpu::thermal(z, talus, 50, &bedrock, &depo);
    else
    {
      hmap::Array mask(shape, 0.25f);
      hmap::gpu::thermal(z, &mask, talus, 50, nullptr, &depo);
    }
    write_raw(out + "_z.f32", z);
    write_raw(out + "_depo.f32", depo);
  }
  else if (mode == "config1")
  {
    /* the thermal benchmark configuration: uniform talus 1/256, no bedrock,
     * 100 iterations, deposition map */
    hmap::Array depo;
    hmap::gpu::thermal(z, 1.f / 256.f, 100, nullptr, &depo);
    write_raw(out + "_z.f32", z);
    write_raw(out + "_depo.f32", depo);
  }
  else if (mode == "thermal_scalar")
  {
    hmap::gpu::thermal(z, 0.1f / shape.x, 60);
    write_raw(out + "_z.f32", z);
  }
  else if (mode == "auto_bedrock" || mode == "auto_bedrock_mask")
  {
    hmap::Array depo;
    if (mode == "auto_bedrock")
      hmap::gpu::thermal_auto_bedrock(z, 0.5f / shape.x, 40, &depo);
    else
    {
      hmap::Array talus(shape, 0.5f / shape.x);
      hmap::Array mask(shape, 0.75f);
      hmap::gpu::thermal_auto_bedrock(z, &mask, talus, 40, &depo);
    }
    write_raw(out + "_z.f32", z);
    write_raw(out + "_depo.f32", depo);
  }
  else if (mode == "flow")
  {
    hmap::Array depth_map(shape, 0.f);
    for (size_t k = 0; k < z.vector.size(); k++) depth_map.vector[k] = 1.f - z.vector[k];
    hmap::Array w = hmap::gpu::flow_simulation(z, 0.01f, depth_map, 50, 0.5f, true, 0.01f, 0.05f);
    write_raw(out + "_water.f32", w);
  }
  else if (mode == "ridge" || mode == "scree" || mode == "schott" || mode == "olsen")
  {
    hmap::Array talus(shape, 0.5f / shape.x), zmax(shape), mask(shape, 0.6f), depo;
    for (size_t k = 0; k < z.vector.size(); k++) zmax.vector[k] = z.vector[k] + 0.2f;
    if (mode == "ridge") hmap::gpu::thermal_ridge(z, talus, 20, &depo);
    else if (mode == "scree") hmap::gpu::thermal_scree(z, &mask, talus, zmax, 20, &depo);
    else if (mode == "schott") hmap::gpu::thermal_schott(z, talus, 20, 0.2f, &depo);
    else hmap::gpu::thermal_olsen(z, &mask, talus, 20);
    write_raw(out + "_z.f32", z);
    if (mode != "olsen") write_raw(out + "_depo.f32", depo);
  }
  else if (mode == "deposition")
  {
    hmap::Array talus(shape, 0.5f / shape.x), depo;
    hmap::gpu::sediment_deposition(z, talus, &depo, 0.02f, 4, 8);
    write_raw(out + "_z.f32", z);
    write_raw(out + "_depo.f32", depo);
  }
  else if (mode == "flatten" || mode == "inflate" || mode == "rib")
  {
    hmap::Array talus(shape, 0.6f / shape.x), mask(shape, 0.5f);
    if (mode == "flatten") hmap::gpu::thermal_flatten(z, talus, 12, 0.5f, 0.2f);
    else if (mode == "inflate") hmap::gpu::thermal_inflate(z, &mask, talus, 12);
    else hmap::gpu::thermal_rib(z, 6);
    write_raw(out + "_z.f32", z);
  }
  else if (mode == "viscous")
  {
    hmap::Array dm(shape, 1.f);
    hmap::Array d = hmap::gpu::flow_simulation_viscous(z, 0.05f, dm, 40);
    write_raw(out + "_d.f32", d);
  }
  else if (mode == "layer")
  {
    hmap::Array tl(shape, 0.5f / shape.x), tu(shape, 4.f / shape.x), depo;
    hmap::gpu::sediment_layer(z, tl, tu, 20, true, &depo);
    write_raw(out + "_z.f32", z);
    write_raw(out + "_depo.f32", depo);
  }
  else if (mode == "vpipes")
  {
    hmap::Array water, sediment, u, v;
    hmap::gpu::hydraulic_vpipes(z, 1e-2f, true, 0.1f, 25, 0.5f, 0.5f, 0.001f, 0.01f, 1.f, 10.f, false, 0.01f,
                                nullptr, &water, &sediment, &u, &v);
    write_raw(out + "_z.f32", z);
    write_raw(out + "_water.f32", water);
    write_raw(out + "_sediment.f32", sediment);
  }
  else
    return 5;
  return hmap::gpu::last_error().empty() ? 0 : 6;
}
