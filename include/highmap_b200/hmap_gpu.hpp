/*
 * hmap_gpu.hpp - HighMap's hmap::gpu erosion API, served by libhm_erosion.so.
 *
 * Source-compatible with the declarations of
 * HighMap/include/highmap/erosion.hpp:1206-1223 (hydraulic_vpipes),
 * :1784-1801 (thermal, three overloads), :1824-1838 (thermal_auto_bedrock, three
 * overloads), :1887-2028 (thermal_olsen, _ridge, _schott, _scree, two overloads each)
 * HighMap/include/highmap/hydrology/hydrology.hpp:875-882 (flow_simulation)
 * and HighMap/include/highmap/opencl/gpu_opencl.hpp:30 (init_opencl).
 * To use HighMap's own hmap::Array, include "highmap/array.hpp" first and
 * define HMAP_B200_EXTERNAL_ARRAY; otherwise this header brings in the
 * layout-identical minimal one (highmap_b200/hmap_array.hpp).
 *
 * Error behaviour follows the reference: the functions return void and do
 * not throw.  On failure z is left as it was, the C-ABI status message is
 * printed to stderr and kept in hmap::gpu::last_error().
 */
#ifndef HMAP_B200_GPU_HPP
#define HMAP_B200_GPU_HPP

#include <string>

#ifndef HMAP_B200_EXTERNAL_ARRAY
#include "highmap_b200/hmap_array.hpp"
#endif

namespace hmap
{
namespace gpu
{

bool init_opencl();

void thermal(Array       &z,
             const Array &talus,
             int          iterations = 10,
             Array       *p_bedrock = nullptr,
             Array       *p_deposition_map = nullptr);

void thermal(Array       &z,
             const Array *p_mask,
             const Array &talus,
             int          iterations = 10,
             Array       *p_bedrock = nullptr,
             Array       *p_deposition_map = nullptr);

void thermal(Array &z,
             float  talus,
             int    iterations = 10,
             Array *p_bedrock = nullptr,
             Array *p_deposition_map = nullptr);

void thermal_auto_bedrock(Array       &z,
                          const Array &talus,
                          int          iterations = 10,
                          Array       *p_deposition_map = nullptr);

void thermal_auto_bedrock(Array       &z,
                          const Array *p_mask,
                          const Array &talus,
                          int          iterations = 10,
                          Array       *p_deposition_map = nullptr);

void thermal_auto_bedrock(Array &z,
                          float  talus,
                          int    iterations = 10,
                          Array *p_deposition_map = nullptr);

/* HighMap/include/highmap/erosion.hpp:1366-1379 */
void sediment_deposition(Array       &z,
                         Array       *p_mask,
                         const Array &talus,
                         Array       *p_deposition_map = nullptr,
                         float        max_deposition = 0.01,
                         int          iterations = 5,
                         int          thermal_subiterations = 10);

void sediment_deposition(Array       &z,
                         const Array &talus,
                         Array       *p_deposition_map = nullptr,
                         float        max_deposition = 0.01,
                         int          iterations = 5,
                         int          thermal_subiterations = 10);

/* HighMap/include/highmap/erosion.hpp:1402-1407 */
void sediment_layer(Array       &z,
                    const Array &talus_layer,
                    const Array &talus_upper_limit,
                    int          iterations,
                    bool         apply_post_filter = true,
                    Array       *p_deposition_map = nullptr);

/* HighMap/include/highmap/erosion.hpp:1855-1866, 1911-1916, 1930-1932 */
void thermal_flatten(Array       &z,
                     const Array &talus,
                     int          iterations,
                     float        sigma_inf = 0.5f,
                     float        sigma_sup = 0.f);
void thermal_flatten(Array       &z,
                     const Array *p_mask,
                     const Array &talus,
                     int          iterations,
                     float        sigma_inf = 0.5f,
                     float        sigma_sup = 0.f);
void thermal_inflate(Array &z, const Array &talus, int iterations = 10);
void thermal_inflate(Array &z, const Array *p_mask, const Array &talus, int iterations = 10);
void thermal_rib(Array &z, int iterations);
void thermal_rib(Array &z, const Array *p_mask, int iterations);

/* sibling talus stencils, HighMap/include/highmap/erosion.hpp:1887-2028 */
void thermal_olsen(Array &z, const Array &talus, int iterations);

void thermal_olsen(Array &z, const Array *p_mask, const Array &talus, int iterations);

void thermal_ridge(Array       &z,
                   const Array &talus,
                   int          iterations = 10,
                   Array       *p_deposition_map = nullptr);

void thermal_ridge(Array       &z,
                   const Array *p_mask,
                   const Array &talus,
                   int          iterations = 10,
                   Array       *p_deposition_map = nullptr);

void thermal_schott(Array       &z,
                    const Array &talus,
                    int          iterations = 10,
                    float        intensity = 0.2f,
                    Array       *p_deposition_map = nullptr);

void thermal_schott(Array       &z,
                    const Array *p_mask,
                    const Array &talus,
                    int          iterations = 10,
                    float        intensity = 0.2f,
                    Array       *p_deposition_map = nullptr);

void thermal_scree(Array       &z,
                   const Array &talus,
                   const Array &zmax,
                   int          iterations = 10,
                   Array       *p_deposition_map = nullptr);

void thermal_scree(Array       &z,
                   const Array *p_mask,
                   const Array &talus,
                   const Array &zmax,
                   int          iterations = 10,
                   Array       *p_deposition_map = nullptr);

/* HighMap/include/highmap/hydrology/hydrology.hpp:875-882; returns the
 * water depth (an array of zeros of z's shape if the call fails) */
Array flow_simulation(const Array &z,
                      float        water_height,
                      const Array &depth_map,
                      int          iterations,
                      float        dt = 0.5f,
                      bool         flux_diffusion = true,
                      float        flux_diffusion_strength = 0.01f,
                      float        dry_out_ratio = 0.f);

/* HighMap/include/highmap/hydrology/hydrology.hpp:884-891 */
Array flow_simulation_viscous(const Array &z,
                              float        water_depth,
                              const Array &depth_map,
                              int          iterations,
                              float        dt = 0.5f,
                              float        dry_out_ratio = 0.f,
                              float        viscosity = 1.f,
                              float        power = 2.5f);

void hydraulic_vpipes(Array &z,
                      float  water_height = 1e-2f,
                      bool   maintain_water_volume = true,
                      float  evap_rate = 0.1f,
                      int    iterations = 50,
                      float  dt = 0.5f,
                      float  k_capacity = 0.5f,
                      float  k_erode = 0.001f,
                      float  k_depose = 0.01f,
                      float  k_discharge_exp = 1.f,
                      float  downcutting_max_depth_ratio = 10.f,
                      bool   flux_diffusion = true,
                      float  flux_diffusion_strength = 0.01f,
                      Array *p_rain_map = nullptr,
                      Array *p_water_depth = nullptr,
                      Array *p_sediment = nullptr,
                      Array *p_vel_u = nullptr,
                      Array *p_vel_v = nullptr);

/* message of the last failure of a call above on this thread ("" if none) */
std::string last_error();

} // namespace gpu
} // namespace hmap

#endif
