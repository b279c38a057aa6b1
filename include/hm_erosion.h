/*
 * hm_erosion.h - C-ABI of the B200 erosion solvers (libhm_erosion.so).
 *
 * Drop-in replacement for HighMap's GPU thermal and virtual-pipes erosion:
 * every entry point below replaces one reference interface, cited beside
 * it.  Grids are float32, element (i, j) at [j * nx + i] (x fastest), the
 * layout of hmap::Array (HighMap/include/highmap/array.hpp:236-252).
 *
 * Semantics of the reference that are decided here:
 *  - Thermal steps are Jacobi: step t+1 is computed from the whole step-t
 *    field.  The reference kernel updates z in place from racing
 *    work-items (HighMap/src/gpu_opencl/kernels/thermal.cl:26-58), which
 *    is not reproducible; Jacobi is its deterministic form.
 *  - Bedrock: HM_BEDROCK_INTENDED (default) applies the talus update and
 *    then clamps to bedrock; HM_BEDROCK_LITERAL reproduces thermal.cl:96-99,
 *    where the update is overwritten by max(z_before, bedrock).
 *  - The advection pass samples sediment with OpenCL's linear filter and
 *    mirrored-repeat addressing at unnormalised coordinates
 *    (hydraulic_vpipes.cl:201-208), defined here as the specification's
 *    normalised rule in texel units, fp32 weights.
 *
 * Every function returns an hm_status (0 = success).  On failure the
 * output buffers are left unmodified where the failure is detected before
 * any device work (argument checks), and hm_last_error() describes it.
 * Contexts are not shared between threads; one context serialises its own
 * calls on its stream.  The device-pointer calls (hm_*_device) run on the
 * caller's stream but use their context's workspace, so two of them on one
 * context must be ordered (the same stream, or an event between streams);
 * a context per stream lets them overlap.
 */
#ifndef HM_EROSION_H
#define HM_EROSION_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define HM_OK 0
#define HM_ERR_INVALID_ARGUMENT 1
#define HM_ERR_NO_DEVICE 2
#define HM_ERR_OUT_OF_MEMORY 3
#define HM_ERR_CUDA 4
#define HM_ERR_TIMEOUT 5
#define HM_ERR_BUSY 6

/* bedrock handling of the thermal step */
#define HM_BEDROCK_INTENDED 0
#define HM_BEDROCK_LITERAL 1

typedef struct hm_context hm_context;

/* Replaces hmap::gpu::init_opencl() (HighMap/include/highmap/opencl/
 * gpu_opencl.hpp:166, HighMap/src/gpu_opencl/gpu_opencl.cpp:32-134):
 * returns HM_OK when device 0 is of compute capability 10.0 (the library
 * holds sm_100a code only, which runs on no other capability) and a
 * context can be made on it. */
int hm_init(void);

/* Context: a CUDA stream for the host-pointer calls and a grow-only device
 * workspace.  Replaces the OpenCL device/queue singleton that the reference
 * keeps inside CLWrapper (gpu_opencl.cpp:34). */
int hm_context_create(hm_context **ctx, int device);
int hm_context_destroy(hm_context *ctx);
/* Release the workspace (it grows again on demand). */
int hm_context_trim(hm_context *ctx);

const char *hm_status_string(int status);
/* Message of the last failure on the calling thread ("" if none). */
const char *hm_last_error(void);

typedef struct hm_thermal_options
{
  int bedrock_mode; /* HM_BEDROCK_INTENDED or HM_BEDROCK_LITERAL */
  int time_block;   /* steps advanced per sweep: 0 = tuned default, 1 = one launch per step */
} hm_thermal_options;

void hm_thermal_default_options(hm_thermal_options *opts);

/* ---- thermal, host buffers ------------------------------------------- */

/* Replaces hmap::gpu::thermal(Array &z, const Array &talus, int iterations,
 * Array *p_bedrock, Array *p_deposition_map)
 * (HighMap/include/highmap/erosion.hpp:1784-1788,
 *  HighMap/src/erosion/thermal_gpu.cpp:17-72).
 * z: nx*ny, in/out.  talus: nx*ny.  bedrock, deposition_map: nullable.
 * After the iterations the outer ring is linearly extrapolated
 * (extrapolate_borders, HighMap/src/boundary/boundary.cpp:19-41) and the
 * deposition map is max(z_out - z_in, 0).  opts may be NULL.
 * nx, ny >= 3, iterations >= 0. */
int hm_thermal(hm_context               *ctx,
               float                    *z,
               int                       nx,
               int                       ny,
               const float              *talus,
               int                       iterations,
               const float              *bedrock,
               float                    *deposition_map,
               const hm_thermal_options *opts);

/* Replaces hmap::gpu::thermal(Array &z, float talus, int iterations,
 * Array *p_bedrock, Array *p_deposition_map) (erosion.hpp:1797-1801,
 * thermal_gpu.cpp:88-96).  The uniform talus is passed to the kernel as a
 * scalar instead of being expanded into a map. */
int hm_thermal_scalar(hm_context               *ctx,
                      float                    *z,
                      int                       nx,
                      int                       ny,
                      float                     talus,
                      int                       iterations,
                      const float              *bedrock,
                      float                    *deposition_map,
                      const hm_thermal_options *opts);

/* Replaces hmap::gpu::thermal(Array &z, const Array *p_mask,
 * const Array &talus, int iterations, Array *p_bedrock,
 * Array *p_deposition_map) (erosion.hpp:1790-1795, thermal_gpu.cpp:74-86):
 * z = lerp(z, thermal(z), mask) (operator.hpp:405-418).  mask NULL means no
 * mask. */
int hm_thermal_masked(hm_context               *ctx,
                      float                    *z,
                      int                       nx,
                      int                       ny,
                      const float              *mask,
                      const float              *talus,
                      int                       iterations,
                      const float              *bedrock,
                      float                    *deposition_map,
                      const hm_thermal_options *opts);

/* ---- thermal, device-resident buffers --------------------------------- */

/* All pointers are device pointers; the call is ordered on `stream`
 * (a cudaStream_t, NULL = legacy default stream) and returns without
 * synchronising.  talus NULL selects the scalar talus_value.  mask,
 * bedrock and deposition_map are nullable. */
int hm_thermal_device(hm_context               *ctx,
                      float                    *z,
                      int                       nx,
                      int                       ny,
                      const float              *talus,
                      float                     talus_value,
                      int                       iterations,
                      const float              *bedrock,
                      float                    *deposition_map,
                      const float              *mask,
                      const hm_thermal_options *opts,
                      void                     *stream);

/* ---- thermal with an automatic bedrock -------------------------------- */

/* Replaces hmap::gpu::thermal_auto_bedrock(Array &z, const Array &talus,
 * int iterations, Array *p_deposition_map)
 * (HighMap/include/highmap/erosion.hpp:1824-1827,
 *  HighMap/src/erosion/thermal_gpu.cpp:98-130, kernel thermal_auto_bedrock
 *  in HighMap/src/gpu_opencl/kernels/thermal.cl:102-145).  The talus
 * exchange of hm_thermal with the reference's self-built bedrock: a cell
 * never drops below its input height nor below its previous value, so the
 * solve only deposits.  Then the border extrapolation and the deposition
 * map, as hm_thermal.  opts: only time_block is used (NULL = defaults). */
int hm_thermal_auto_bedrock(hm_context               *ctx,
                            float                    *z,
                            int                       nx,
                            int                       ny,
                            const float              *talus,
                            int                       iterations,
                            float                    *deposition_map,
                            const hm_thermal_options *opts);

/* Replaces hmap::gpu::thermal_auto_bedrock(Array &z, float talus,
 * int iterations, Array *p_deposition_map) (erosion.hpp:1835-1838,
 * thermal_gpu.cpp:132-139); the talus is a kernel scalar. */
int hm_thermal_auto_bedrock_scalar(hm_context               *ctx,
                                   float                    *z,
                                   int                       nx,
                                   int                       ny,
                                   float                     talus,
                                   int                       iterations,
                                   float                    *deposition_map,
                                   const hm_thermal_options *opts);

/* Replaces hmap::gpu::thermal_auto_bedrock(Array &z, const Array *p_mask,
 * const Array &talus, int iterations, Array *p_deposition_map)
 * (erosion.hpp:1829-1833, thermal_gpu.cpp:141-152): z = lerp(z, solve(z),
 * mask).  mask NULL means no mask. */
int hm_thermal_auto_bedrock_masked(hm_context               *ctx,
                                   float                    *z,
                                   int                       nx,
                                   int                       ny,
                                   const float              *mask,
                                   const float              *talus,
                                   int                       iterations,
                                   float                    *deposition_map,
                                   const hm_thermal_options *opts);

/* Device-pointer form of the three above, ordered on `stream`; talus NULL
 * selects talus_value; deposition_map and mask are nullable. */
int hm_thermal_auto_bedrock_device(hm_context               *ctx,
                                   float                    *z,
                                   int                       nx,
                                   int                       ny,
                                   const float              *talus,
                                   float                     talus_value,
                                   int                       iterations,
                                   float                    *deposition_map,
                                   const float              *mask,
                                   const hm_thermal_options *opts,
                                   void                     *stream);

/* ---- sediment deposition ------------------------------------------------- */

/* Replaces hmap::gpu::sediment_deposition(Array &z, const Array &talus,
 * Array *p_deposition_map, float max_deposition, int iterations,
 * int thermal_subiterations) and the masked overload
 * (HighMap/include/highmap/erosion.hpp:1366-1379,
 *  HighMap/src/erosion/deposition.cpp:19-66): max_deposition laid down in
 * `iterations` layers, each settled by thermal_subiterations thermal steps
 * (talus map); z += sediment (blended with the input by mask when given);
 * deposition_map receives the sediment.  mask and deposition_map nullable. */
int hm_sediment_deposition(hm_context  *ctx,
                           float       *z,
                           int          nx,
                           int          ny,
                           const float *talus,
                           float        max_deposition,
                           int          iterations,
                           int          thermal_subiterations,
                           float       *deposition_map,
                           const float *mask);

/* The same on device buffers, ordered on `stream`. */
int hm_sediment_deposition_device(hm_context  *ctx,
                                  float       *z,
                                  int          nx,
                                  int          ny,
                                  const float *talus,
                                  float        max_deposition,
                                  int          iterations,
                                  int          thermal_subiterations,
                                  float       *deposition_map,
                                  const float *mask,
                                  void        *stream);

/* Replaces hmap::gpu::sediment_layer(Array &z, const Array &talus_layer,
 * const Array &talus_upper_limit, int iterations, bool apply_post_filter,
 * Array *p_deposition_map) (HighMap/include/highmap/erosion.hpp:1402-1407,
 *  HighMap/src/erosion/deposition.cpp:68-113): talus from the terrain's
 * gradient_talus (gradient.cpp:217-243), steepened to
 * 4 (g - limit) + limit where g exceeds talus_upper_limit; `iterations`
 * thermal steps with that talus map; with apply_post_filter (non-zero),
 * z = z_in + deposition, smoothed by hmap::laplace (sigma 0.125, 3 steps)
 * where the smoothed mask of the unclamped cells allows.  deposition_map
 * (nullable) receives max(z_thermal - z_in, 0). */
int hm_sediment_layer(hm_context  *ctx,
                      float       *z,
                      int          nx,
                      int          ny,
                      const float *talus_layer,
                      const float *talus_upper_limit,
                      int          iterations,
                      int          apply_post_filter,
                      float       *deposition_map);

/* The same on device buffers, ordered on `stream`. */
int hm_sediment_layer_device(hm_context  *ctx,
                             float       *z,
                             int          nx,
                             int          ny,
                             const float *talus_layer,
                             const float *talus_upper_limit,
                             int          iterations,
                             int          apply_post_filter,
                             float       *deposition_map,
                             void        *stream);

/* Replaces the post-filter of hmap::gpu::snow_simulation
 * (HighMap/src/hydrology/snow_simulation.cpp:140-152, with the
 * clamp_min(s, 0) that follows it), for a caller that runs the snow
 * kernel itself: on terrain z and snow depth s (updated in place),
 * mask = clamp_max_smooth(s / snow_depth, 1), z_w = z + s, `iterations`
 * thermal steps of z_w with talus thermal_talus_ratio * gradient_norm(z_w)
 * blended in by the mask, then s = max(z_w - z, 0). */
int hm_snow_post_filter(hm_context  *ctx,
                        const float *z,
                        float       *s,
                        int          nx,
                        int          ny,
                        float        snow_depth,
                        int          iterations,
                        float        thermal_talus_ratio);

/* The same on device buffers, ordered on `stream`. */
int hm_snow_post_filter_device(hm_context  *ctx,
                               const float *z,
                               float       *s,
                               int          nx,
                               int          ny,
                               float        snow_depth,
                               int          iterations,
                               float        thermal_talus_ratio,
                               void        *stream);

/* ---- sibling talus stencils ---------------------------------------------- */

/* Rules of hm_thermal_stencil_device (ridge .. olsen) and
 * hm_thermal_relief_device (flatten .. rib). */
#define HM_RIDGE 0
#define HM_SCREE 1
#define HM_SCHOTT 2
#define HM_OLSEN 3
#define HM_FLATTEN 4
#define HM_INFLATE 5
#define HM_RIB 6

/* Replaces hmap::gpu::thermal_ridge(Array &z, const Array &talus,
 * int iterations, Array *p_deposition_map) and its masked overload
 * (HighMap/include/highmap/erosion.hpp:1953-1962,
 *  HighMap/src/erosion/thermal_gpu.cpp:274-311, kernel thermal_ridge.cl).
 * Then extrapolate_borders, deposition map |z_out - z_in|, and with a mask
 * z = lerp(z, result, mask).  mask and deposition_map are nullable. */
int hm_thermal_ridge(hm_context  *ctx,
                     float       *z,
                     int          nx,
                     int          ny,
                     const float *talus,
                     int          iterations,
                     float       *deposition_map,
                     const float *mask);

/* Replaces hmap::gpu::thermal_scree(Array &z, const Array &talus,
 * const Array &zmax, int iterations, Array *p_deposition_map) and its
 * masked overload (erosion.hpp:2017-2028, thermal_gpu.cpp:355-396, kernel
 * thermal_scree.cl).  Deposition map max(z_out - z_in, 0). */
int hm_thermal_scree(hm_context  *ctx,
                     float       *z,
                     int          nx,
                     int          ny,
                     const float *talus,
                     const float *zmax,
                     int          iterations,
                     float       *deposition_map,
                     const float *mask);

/* Replaces hmap::gpu::thermal_schott(Array &z, const Array &talus,
 * int iterations, float intensity, Array *p_deposition_map) and its masked
 * overload (erosion.hpp:1985-1996, thermal_gpu.cpp:313-353, kernel
 * thermal_schott.cl).  Deposition map |z_out - z_in|. */
int hm_thermal_schott(hm_context  *ctx,
                      float       *z,
                      int          nx,
                      int          ny,
                      const float *talus,
                      int          iterations,
                      float        intensity,
                      float       *deposition_map,
                      const float *mask);

/* Replaces hmap::gpu::thermal_olsen(Array &z, const Array &talus,
 * int iterations) and its masked overload (erosion.hpp:1887-1892,
 * thermal_gpu.cpp:221-247, kernel thermal_olsen.cl).  nx, ny >= 7. */
int hm_thermal_olsen(hm_context  *ctx,
                     float       *z,
                     int          nx,
                     int          ny,
                     const float *talus,
                     int          iterations,
                     const float *mask);

/* The four on device buffers, ordered on `stream`: rule HM_RIDGE ..
 * HM_OLSEN; zmax (scree) and intensity (schott) as above; deposition_map
 * (not written for olsen) and mask nullable. */
int hm_thermal_stencil_device(hm_context  *ctx,
                              int          rule,
                              float       *z,
                              int          nx,
                              int          ny,
                              const float *talus,
                              const float *zmax,
                              float        intensity,
                              int          iterations,
                              float       *deposition_map,
                              const float *mask,
                              void        *stream);

/* Replaces hmap::gpu::thermal_flatten(Array &z, const Array &talus,
 * int iterations, float sigma_inf, float sigma_sup) and its masked overload
 * (HighMap/include/highmap/erosion.hpp:1855-1866,
 *  HighMap/src/erosion/thermal_gpu.cpp:154-190, kernel thermal_flatten.cl):
 * a cell loses sigma_inf (slope below its talus) or sigma_sup (above)
 * times its steepest descent and gains half of each neighbour's steepest
 * descent that points at it; border cells within 2 of the edge copy the
 * nearest interior cell; then extrapolate_borders; with a mask
 * z = lerp(z, result, mask).  nx, ny >= 5; mask nullable.  The reference's
 * defaults are sigma_inf 0.5, sigma_sup 0. */
int hm_thermal_flatten(hm_context  *ctx,
                       float       *z,
                       int          nx,
                       int          ny,
                       const float *talus,
                       int          iterations,
                       float        sigma_inf,
                       float        sigma_sup,
                       const float *mask);

/* Replaces hmap::gpu::thermal_inflate(Array &z, const Array &talus,
 * int iterations) and its masked overload (erosion.hpp:1911-1916,
 * thermal_gpu.cpp:192-219, kernel thermal_inflate.cl), then
 * extrapolate_borders and the mask blend.  mask nullable. */
int hm_thermal_inflate(hm_context  *ctx,
                       float       *z,
                       int          nx,
                       int          ny,
                       const float *talus,
                       int          iterations,
                       const float *mask);

/* Replaces hmap::gpu::thermal_rib(Array &z, int iterations) and its masked
 * overload (erosion.hpp:1930-1932, thermal_gpu.cpp:249-272, kernel
 * thermal_rib.cl): each cell drops by its least |slope| to a neighbour;
 * then extrapolate_borders(z, 3) and the mask blend.  nx, ny >= 5; mask
 * nullable. */
int hm_thermal_rib(hm_context *ctx, float *z, int nx, int ny, int iterations, const float *mask);

/* The three on device buffers, ordered on `stream`: rule HM_FLATTEN,
 * HM_INFLATE or HM_RIB; talus unused (may be NULL) for rib; sigma_inf and
 * sigma_sup used by flatten only; mask nullable. */
int hm_thermal_relief_device(hm_context  *ctx,
                             int          rule,
                             float       *z,
                             int          nx,
                             int          ny,
                             const float *talus,
                             float        sigma_inf,
                             float        sigma_sup,
                             int          iterations,
                             const float *mask,
                             void        *stream);

/* ---- flow simulation ---------------------------------------------------- */

/* Replaces hmap::gpu::flow_simulation(const Array &z, float water_height,
 * const Array &depth_map, int iterations, float dt, bool flux_diffusion,
 * float flux_diffusion_strength, float dry_out_ratio)
 * (HighMap/include/highmap/hydrology/hydrology.hpp:875-882,
 *  HighMap/src/hydrology/flow_simulation.cpp:26-110): the flow and water
 * passes of the pipe model (hydraulic_vpipes.cl:5-116) on the fixed terrain
 * z, water starting at water_height * depth_map, `iterations` steps, then,
 * if dry_out_ratio != 0, depth = max(0, depth - dry_out_ratio * max(depth))
 * (water_depth.cpp:40-66).  z and depth_map: nx*ny in; water_depth: nx*ny
 * out.  dt != 0, iterations >= 0. */
int hm_flow_simulation(hm_context  *ctx,
                       const float *z,
                       int          nx,
                       int          ny,
                       float        water_height,
                       const float *depth_map,
                       int          iterations,
                       float        dt,
                       int          flux_diffusion,
                       float        flux_diffusion_strength,
                       float        dry_out_ratio,
                       float       *water_depth);

/* The same on device buffers, ordered on `stream` (a cudaStream_t, NULL =
 * legacy default stream); returns without synchronising. */
int hm_flow_simulation_device(hm_context  *ctx,
                              const float *z,
                              int          nx,
                              int          ny,
                              float        water_height,
                              const float *depth_map,
                              int          iterations,
                              float        dt,
                              int          flux_diffusion,
                              float        flux_diffusion_strength,
                              float        dry_out_ratio,
                              float       *water_depth,
                              void        *stream);

/* Replaces hmap::gpu::flow_simulation_viscous(const Array &z,
 * float water_depth, const Array &depth_map, int iterations, float dt,
 * float dry_out_ratio, float viscosity, float power)
 * (HighMap/include/highmap/hydrology/hydrology.hpp:884-891,
 *  HighMap/src/hydrology/flow_simulation.cpp:112-157, kernel
 *  shallow_viscous_flow.cl): water_height * depth_map spread as a viscous
 * film over the fixed terrain z for `iterations` steps, the time step
 * re-derived from the deepest water every 10 steps (so `dt` matters only
 * for iterations == 0), then the dry-out.  water_depth receives the depth.
 * The reference's defaults: dt 0.5, dry_out_ratio 0, viscosity 1, power
 * 2.5. */
int hm_flow_simulation_viscous(hm_context  *ctx,
                               const float *z,
                               int          nx,
                               int          ny,
                               float        water_height,
                               const float *depth_map,
                               int          iterations,
                               float        dt,
                               float        dry_out_ratio,
                               float        viscosity,
                               float        power,
                               float       *water_depth);

/* The same on device buffers, ordered on `stream`. */
int hm_flow_simulation_viscous_device(hm_context  *ctx,
                                      const float *z,
                                      int          nx,
                                      int          ny,
                                      float        water_height,
                                      const float *depth_map,
                                      int          iterations,
                                      float        dt,
                                      float        dry_out_ratio,
                                      float        viscosity,
                                      float        power,
                                      float       *water_depth,
                                      void        *stream);

/* No counterpart in the reference (which allocates its OpenCL buffers on
 * every call).  Thermal erosion on device buffers for callers that cannot
 * allocate device memory when they run it (an application whose own pool
 * allocator owns the device memory, or a loop that must not stall on
 * cudaMalloc/cudaFree): the same solve as hm_thermal_device without the
 * deposition map and mask, with the Jacobi scratch grid taken from a
 * statically reserved device array of HM_NOALLOC_MAX_CELLS floats (16 MiB).
 * No allocation, no context.  Grids larger than HM_NOALLOC_MAX_CELLS cells
 * are refused with HM_ERR_INVALID_ARGUMENT.  Runs on the calling thread's
 * current device and looks up the array's address there on every call.
 * With CUDA's lazy module loading (the default) the array is placed on a
 * GPU by the first call on that device and held until exit: make that
 * first call before an application pool claims the free device memory
 * (or set CUDA_MODULE_LOADING=EAGER) and before any stream capture.  All
 * calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller.  talus NULL selects talus_value; bedrock is
 * nullable. */
#define HM_NOALLOC_MAX_CELLS (1 << 22)
int hm_thermal_device_noalloc(float       *z,
                              int          nx,
                              int          ny,
                              const float *talus,
                              float        talus_value,
                              int          iterations,
                              const float *bedrock,
                              int          bedrock_mode,
                              void        *stream);

/* ---- virtual pipes ----------------------------------------------------- */

typedef struct hm_vpipes_params
{
  /* the reference's parameters, erosion.hpp:1206-1223 (same defaults) */
  float water_height;
  int   maintain_water_volume;
  float evap_rate;
  int   iterations;
  float dt;
  float k_capacity;
  float k_erode;
  float k_depose;
  float k_discharge_exp;
  float downcutting_max_depth_ratio;
  int   flux_diffusion;
  float flux_diffusion_strength;
  /* extensions; the defaults 1, 1, 1, 0, -1 reproduce the reference */
  float gravity;       /* hydraulic_vpipes.cl:31 hard-codes 1                  */
  float pipe_length;   /* hydraulic_vpipes.cl:30 hard-codes 1                  */
  float pipe_area;     /* pipe cross-section, scales the flux update            */
  float rain_per_step; /* depth added (times rain map) before every flow pass  */
  float initial_water; /* < 0: water_height (reference); else initial depth     */
} hm_vpipes_params;

void hm_vpipes_default_params(hm_vpipes_params *p);

/* Replaces hmap::gpu::hydraulic_vpipes(Array &z, float water_height,
 * bool maintain_water_volume, float evap_rate, int iterations, float dt,
 * float k_capacity, float k_erode, float k_depose, float k_discharge_exp,
 * float downcutting_max_depth_ratio, bool flux_diffusion,
 * float flux_diffusion_strength, Array *p_rain_map, Array *p_water_depth,
 * Array *p_sediment, Array *p_vel_u, Array *p_vel_v)
 * (erosion.hpp:1206-1223, HighMap/src/erosion/hydraulic_vpipes_gpu.cpp:15-178).
 * Host buffers; rain_map and the four outputs are nullable.  params NULL
 * means the reference defaults. */
int hm_vpipes(hm_context             *ctx,
              float                  *z,
              int                     nx,
              int                     ny,
              const hm_vpipes_params *params,
              const float            *rain_map,
              float                  *water_depth,
              float                  *sediment,
              float                  *vel_u,
              float                  *vel_v);

/* Device-pointer form of hm_vpipes, ordered on `stream`. */
int hm_vpipes_device(hm_context             *ctx,
                     float                  *z,
                     int                     nx,
                     int                     ny,
                     const hm_vpipes_params *params,
                     const float            *rain_map,
                     float                  *water_depth,
                     float                  *sediment,
                     float                  *vel_u,
                     float                  *vel_v,
                     void                   *stream);

/* Launch shape of the fused vpipes step kernel, process-wide: threads per
 * CTA (128 or 256, the strip width including its halo), advection radius
 * staged in shared memory (2 or 3 cells; samples beyond it are recomputed
 * exactly from global memory), output rows per CTA (32..4096).  tpb = 0
 * restores the built-in choice.  Results do not depend on the shape. */
int hm_vpipes_set_launch(int tpb, int radius, int rows);

/* Step kernels of the vpipes solver, process-wide: HM_VPIPES_TILED (flow,
 * water and erosion in one kernel over 32 x 16 tiles, then an advection
 * gather; the tiles are fetched by TMA when nx is a multiple of 4, nx >= 40,
 * ny >= 20 and the state buffers are 16-byte aligned, else by cp.async),
 * HM_VPIPES_TILED_CP_ASYNC (the same, always cp.async),
 * HM_VPIPES_STREAMING (all four passes in one kernel streaming down column
 * strips, shaped by hm_vpipes_set_launch), HM_VPIPES_TILED_TB2 (temporal
 * blocking: without the water-volume top-up, every pair of steps after the
 * first in one launch over 32 x 16 tiles, 16 x 8 on small grids, that
 * compute the pair's first step on a 4-cell halo; with the top-up, as
 * HM_VPIPES_TILED), or HM_VPIPES_AUTO (-1: the tuned or built-in choice).
 * Results do not depend on it. */
#define HM_VPIPES_AUTO (-1)
#define HM_VPIPES_TILED 0
#define HM_VPIPES_STREAMING 1
#define HM_VPIPES_TILED_CP_ASYNC 2
#define HM_VPIPES_TILED_TB2 3
int hm_vpipes_set_algorithm(int algo);

/* Fault injection for tests of the device-side timeout (no counterpart in
 * the reference, whose OpenCL path has no device-side wait), process-wide:
 * every TMA-staged vpipes tile arms its barrier with `bytes` more than its
 * boxes deliver.  Every box still lands, but the barrier's phase cannot
 * complete, so each tile's bounded wait runs out (about two seconds), the
 * tile records the timeout and returns, and hm_vpipes reports
 * HM_ERR_TIMEOUT with the caller's buffers untouched (hm_vpipes_device, being
 * asynchronous, does not wait to read the error).  bytes must be a multiple
 * of 16 and at most 4096; 0 (the default) turns it off. */
int hm_debug_tma_expect_extra(unsigned bytes);

/* Output rows per CTA of the temporally blocked thermal kernel,
 * process-wide (8..4096; 0 restores the built-in choice).  Results do not
 * depend on it. */
int hm_thermal_set_launch(int rows);

/* ---- batched and served forms ------------------------------------------ */

/* No counterpart in the reference, which solves one heightmap per call.
 * A batch holds many device-resident solves of uneven sizes and iteration
 * counts and advances them together: every job's grid is cut into tiles,
 * the tiles of all jobs form one packed list, and each round (one step of
 * every active job) is one persistent kernel over that list.  Results are
 * bit-identical to solving each job alone with hm_thermal_device /
 * hm_vpipes_device. */

#define HM_JOB_THERMAL 1
#define HM_JOB_VPIPES 2

typedef struct hm_job
{
  int    kind; /* HM_JOB_THERMAL or HM_JOB_VPIPES */
  int    nx, ny;
  int    iterations;
  float *z; /* device grid, in/out; must stay valid until the job is released */
  /* thermal (hm_thermal_device's arguments; mask unsupported) */
  const float *talus; /* NULL selects talus_value */
  float        talus_value;
  const float *bedrock;
  int          bedrock_mode;
  float       *deposition_map;
  /* vpipes (hm_vpipes_device's arguments; vpipes.iterations is ignored) */
  hm_vpipes_params vpipes;
  const float     *rain_map;
  float           *water_depth, *sediment, *vel_u, *vel_v;
} hm_job;

typedef struct hm_batch hm_batch;

/* A batch on ctx's device with its own CUDA stream. */
int       hm_batch_create(hm_context *ctx, hm_batch **batch);
int       hm_batch_destroy(hm_batch *batch);
/* Device bytes a job holds from hm_batch_add to hm_batch_release. */
size_t    hm_batch_job_bytes(const hm_job *job);
/* Admits a job: allocates its state (stream-ordered) and initialises it.
 * The job's first step is the batch's next round. */
int       hm_batch_add(hm_batch *batch, const hm_job *job, int *job_id);
/* Advances every admitted, unfinished job by up to `rounds` steps (queued
 * on the batch stream); jobs that reach their iteration count get their
 * outputs written (borders, deposition map, water depth ...). */
int       hm_batch_step(hm_batch *batch, int rounds);
int       hm_batch_synchronize(hm_batch *batch);
int       hm_batch_job_status(hm_batch *batch, int job_id, int *steps_done, int *finished);
/* Frees a job's device state (after its outputs are read).  A job released
 * before it finished is cancelled: it leaves the rounds, its outputs are not
 * written, and the other jobs go on unaffected. */
int       hm_batch_release(hm_batch *batch, int job_id);
size_t    hm_batch_bytes_in_use(const hm_batch *batch);
/* Eviction under an HBM budget (no counterpart in the reference).
 * hm_batch_evict copies an unfinished job's device state (its state block,
 * then its heights) into `snapshot`, hm_batch_snapshot_bytes bytes of host
 * memory, and frees the block: the job leaves the rounds and stops counting
 * in hm_batch_bytes_in_use.  Its z grid stays the caller's.
 * hm_batch_restore admits it again from the snapshot (z must still be
 * valid).  The job goes on from the step it had reached with the batch's
 * next round, and its results are the same as if it had never left. */
size_t    hm_batch_snapshot_bytes(const hm_batch *batch, int job_id);
int       hm_batch_evict(hm_batch *batch, int job_id, void *snapshot);
int       hm_batch_restore(hm_batch *batch, int job_id, const void *snapshot);
long long hm_batch_round(const hm_batch *batch);
/* All jobs to completion in one call; use_graph != 0 captures every round
 * into one CUDA graph.  Returns after the results are written.  Jobs of at
 * least HM_BATCH_LARGE_CELLS cells, which fill the GPU on their own, are
 * solved by the plain step kernels on HM_BATCH_LANES side streams (balanced
 * by cell-updates) beside the rounds of the smaller jobs, launched while the
 * rounds' graph is built; results are the same either way. */
#define HM_BATCH_LARGE_CELLS (1 << 20)
#define HM_BATCH_LANES 1
int       hm_batch_run(hm_context *ctx, const hm_job *jobs, int njobs, int use_graph);

/* ---- autotuner ----------------------------------------------------------- */

/* No counterpart in the reference.  Times every candidate launch shape of
 * one solver on a synthetic terrain of nx x ny (steps steps each) and keeps
 * the fastest for grids of that size class (nx, ny rounded up to powers of
 * two); solves that leave the choice to the library (time_block 0, no
 * hm_vpipes_set_launch override) then use it.  Process-wide; do not run
 * while other threads solve.  kind: HM_JOB_THERMAL or HM_JOB_VPIPES, or
 * HM_TUNE_BATCH: the batched form's round launch (persistent CTAs per SM,
 * 1..4, or 0: one CTA per tile of the round) and thermal tile rows (8, 16,
 * 32), timed over `steps` rounds of a synthetic batch of 16 jobs, half
 * thermal and half vpipes, with sides from 128 up to max(nx, ny); batches
 * created afterwards use the fastest (result: tpb = CTAs per SM or 0,
 * rows = thermal tile rows, ms_per_step = per round).  The time_block field
 * of the result holds the steps per launch of the vpipes tiled kernels for
 * HM_JOB_VPIPES and of the thermal kernel for HM_JOB_THERMAL. */
#define HM_TUNE_BATCH 3
typedef struct hm_tune_result
{
  int   tpb, radius, rows; /* vpipes launch shape (rows: also thermal's blocked kernel) */
  int   time_block;        /* steps per launch: thermal, or vpipes' tiled kernels (0, 1: one; 2: two) */
  float ms_per_step;
  int   candidates;
} hm_tune_result;

int  hm_autotune(hm_context *ctx, int kind, int nx, int ny, int steps, hm_tune_result *result);
/* the tuned table as text, and back (unknown or invalid lines skipped) */
int  hm_autotune_save(const char *path);
int  hm_autotune_load(const char *path, int *loaded);
void hm_autotune_clear(void);

/* ---- instrumentation --------------------------------------------------- */

/* Number of kernel launches issued by this library on the calling thread
 * since the last reset (counted on the host at each launch). */
unsigned long long hm_launch_count(void);
void               hm_launch_count_reset(void);

#ifdef __cplusplus
}
#endif

#endif
