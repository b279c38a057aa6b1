/* hm_thermal.h - internal entry points of hm_thermal.cu */
#ifndef HM_THERMAL_H
#define HM_THERMAL_H

#include <cuda_runtime.h>

#include "hm_erosion.h"

namespace hm
{
int    thermal_check_args(const float *z, int nx, int ny, int iterations, const hm_thermal_options *o);
/* floats of workspace thermal_core needs (one grid, two with a z0 copy) */
size_t thermal_scratch_floats(int nx, int ny, bool need_z0);
/* Device pointers; ordered on s.  talus NULL selects talus_value.
 * auto_bed: thermal_auto_bedrock (bedrock must be NULL; needs the z0 copy). */
int    thermal_core(int device, float *z, int nx, int ny, const float *talus, float talus_value, int iterations,
                    const float *bedrock, float *depo, const float *mask, const hm_thermal_options *opts,
                    float *scratch_buf, cudaStream_t s, bool auto_bed = false);
/* border extrapolation, deposition map and mask blend after the steps */
int    thermal_finish(int device, float *z, int nx, int ny, const float *z0, float *depo, const float *mask,
                      cudaStream_t s, bool depo_abs = false, int nbuffer = 1);
/* sediment_deposition (hm_deposition.cu): device pointers, ordered on s */
size_t deposition_scratch_floats(int nx, int ny);
int    deposition_core(int device, float *z, int nx, int ny, const float *talus, float max_deposition,
                       int iterations, int thermal_subiterations, float *depo, const float *mask, float *scratch,
                       cudaStream_t s);
/* sediment_layer (hm_layer.cu): device pointers, ordered on s; depo
 * nullable; scratch of layer_scratch_floats(nx, ny) floats */
size_t layer_scratch_floats(int nx, int ny);
int    layer_core(int device, float *z, int nx, int ny, const float *talus_layer, const float *talus_upper_limit,
                  int iterations, bool post_filter, float *depo, float *scratch, cudaStream_t s);
/* snow_simulation's post-filter (hm_snow.cu): device pointers, ordered on
 * s; scratch of snow_scratch_floats(nx, ny) floats */
size_t snow_scratch_floats(int nx, int ny);
int    snow_post_filter_core(int device, const float *z, float *s, int nx, int ny, float snow_depth, int iterations,
                             float ratio, float *scratch, cudaStream_t st);
/* sibling talus stencils (hm_sibling.cu): rule HM_RIDGE .. HM_RIB; zmax
 * for scree, intensity for schott, intensity and p1 (sigma_inf, sigma_sup)
 * for flatten; talus NULL for rib; scratch of thermal_scratch_floats(nx,
 * ny, true) floats */
int    sibling_check_args(int rule, const float *z, int nx, int ny, const float *talus, const float *zmax,
                          int iterations);
int    sibling_core(int device, int rule, float *z, int nx, int ny, const float *talus, const float *zmax,
                    float intensity, int iterations, float *depo, const float *mask, float *scratch_buf,
                    cudaStream_t s, float p1 = 0.f);
} // namespace hm

#endif
