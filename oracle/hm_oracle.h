/*
 * hm_oracle.h - CPU restatement of HighMap's thermal and virtual-pipes
 * erosion solvers.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity oracle: the test
 * suite, the smoke check and the CPU-baseline leg of the benchmark call it
 * as the checker.  The product (libhm_erosion.so) never links or calls it.
 *
 * The reference has no CPU implementation of either solver (both live only
 * in namespace hmap::gpu as OpenCL kernels plus host drivers), so this is a
 * restatement of the kernel arithmetic and the host-driver steps:
 *   thermal : HighMap/src/gpu_opencl/kernels/thermal.cl:5-100,
 *             HighMap/src/gpu_opencl/kernels/_common_index.cl:106-132,
 *             HighMap/src/erosion/thermal_gpu.cpp:17-96,
 *             HighMap/src/boundary/boundary.cpp:19-41,
 *             HighMap/src/range/range.cpp:253-262,
 *             HighMap/include/highmap/operator.hpp:405-418
 *   vpipes  : HighMap/src/gpu_opencl/kernels/hydraulic_vpipes.cl:5-211,
 *             HighMap/src/erosion/hydraulic_vpipes_gpu.cpp:15-178
 * and the callers and relatives of the two (each declaration below cites
 * its lines): thermal_auto_bedrock, flow_simulation and
 * flow_simulation_viscous, sediment_deposition and sediment_layer (with
 * gradient_talus and laplace), the post-filter of snow_simulation, and the
 * talus stencils ridge, scree, schott, olsen, flatten, inflate and rib.
 * The host loops of those callers are evaluated in their source order, one
 * rounding per operation.
 *
 * Parity pin: the restatement is checked against the reference's own kernel
 * text compiled for the CPU (oracle/ref_harness.cpp, built into oracle/_ref/
 * by oracle/build_oracle.py) and against the fixtures in tests/golden/ that
 * the same harness generated.
 *
 * Execution semantics: Jacobi (every cell of step t+1 is computed from the
 * complete step-t field).  The reference updates z in place from racing
 * work-items, which is not reproducible; Jacobi is its deterministic form.
 *
 * Layout: element (i, j) of an nx x ny grid is at [j * nx + i] (x fastest),
 * as hmap::Array (HighMap/include/highmap/array.hpp:236-252).
 */
#ifndef HM_ORACLE_H
#define HM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Bedrock handling of the thermal step.
 * HMO_BEDROCK_INTENDED : z = max(z + amount, bedrock) for cells at or above
 *                        bedrock (the evident intent; the same form as
 *                        thermal.cl:142 in thermal_auto_bedrock).
 * HMO_BEDROCK_LITERAL  : z = max(z_before_update, bedrock), which is what
 *                        thermal.cl:96-99 computes (the update of :96 is
 *                        overwritten by :99). */
#define HMO_BEDROCK_INTENDED 0
#define HMO_BEDROCK_LITERAL 1

typedef struct hmo_vpipes_params
{
  /* reference parameters, erosion.hpp:1206-1223 */
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
  /* extensions; the values 1, 1, 1, 0, -1 reproduce the reference */
  float gravity;       /* hydraulic_vpipes.cl:31 hard-codes 1          */
  float pipe_length;   /* hydraulic_vpipes.cl:30 hard-codes 1          */
  float pipe_area;     /* cross-section, multiplies the flux update     */
  float rain_per_step; /* depth added (x rain map) before each flow pass */
  float initial_water; /* < 0: water_height (reference), else this depth */
} hmo_vpipes_params;

void hmo_vpipes_default_params(hmo_vpipes_params *p);

/* Thermal erosion; z is nx*ny and updated in place.  talus is nx*ny.
 * bedrock, deposition map and mask may be NULL.  Returns 0 on success. */
int hmo_thermal_f32(float       *z,
                    int          nx,
                    int          ny,
                    const float *talus,
                    int          iterations,
                    const float *bedrock,
                    float       *deposition_map,
                    const float *mask,
                    int          bedrock_mode);
int hmo_thermal_f64(double       *z,
                    int           nx,
                    int           ny,
                    const double *talus,
                    int           iterations,
                    const double *bedrock,
                    double       *deposition_map,
                    const double *mask,
                    int           bedrock_mode);

/* thermal_auto_bedrock (thermal_gpu.cpp:98-130, thermal.cl:102-145). */
int hmo_thermal_auto_bedrock_f32(float       *z,
                                 int          nx,
                                 int          ny,
                                 const float *talus,
                                 int          iterations,
                                 float       *deposition_map);

/* Virtual-pipes hydraulic erosion; z is nx*ny and updated in place.
 * rain_map and the four outputs may be NULL. */
int hmo_vpipes_f32(float                   *z,
                   int                      nx,
                   int                      ny,
                   const hmo_vpipes_params *p,
                   const float             *rain_map,
                   float                   *water_depth,
                   float                   *sediment,
                   float                   *vel_u,
                   float                   *vel_v);
int hmo_vpipes_f64(double                  *z,
                   int                      nx,
                   int                      ny,
                   const hmo_vpipes_params *p,
                   const double            *rain_map,
                   double                  *water_depth,
                   double                  *sediment,
                   double                  *vel_u,
                   double                  *vel_v);

/* sediment_deposition (HighMap/src/erosion/deposition.cpp:19-66) and its
 * masked overload; deposition_map and mask nullable. */
int hmo_sediment_deposition_f32(float       *z,
                                int          nx,
                                int          ny,
                                const float *talus,
                                float        max_deposition,
                                int          iterations,
                                int          thermal_subiterations,
                                float       *deposition_map,
                                const float *mask);
int hmo_sediment_deposition_f64(double       *z,
                                int           nx,
                                int           ny,
                                const double *talus,
                                double        max_deposition,
                                int           iterations,
                                int           thermal_subiterations,
                                double       *deposition_map,
                                const double *mask);

/* sediment_layer (HighMap/src/erosion/deposition.cpp:68-113):
 * apply_post_filter 0/1; deposition_map nullable. */
int hmo_sediment_layer_f32(float       *z,
                           int          nx,
                           int          ny,
                           const float *talus_layer,
                           const float *talus_upper_limit,
                           int          iterations,
                           int          apply_post_filter,
                           float       *deposition_map);
int hmo_sediment_layer_f64(double       *z,
                           int           nx,
                           int           ny,
                           const double *talus_layer,
                           const double *talus_upper_limit,
                           int           iterations,
                           int           apply_post_filter,
                           double       *deposition_map);

/* thermal_flatten (rule 4; sigma_inf, sigma_sup), thermal_inflate (rule 5)
 * and thermal_rib (rule 6; talus unused, may be NULL),
 * HighMap/src/erosion/thermal_gpu.cpp:154-219,249-272, Jacobi form; mask:
 * apply_with_mask blend, nullable.  No deposition maps (the reference
 * functions have none). */
int hmo_thermal_relief_f32(int          rule,
                           float       *z,
                           int          nx,
                           int          ny,
                           const float *talus,
                           float        sigma_inf,
                           float        sigma_sup,
                           int          iterations,
                           const float *mask);
int hmo_thermal_relief_f64(int           rule,
                           double       *z,
                           int           nx,
                           int           ny,
                           const double *talus,
                           double        sigma_inf,
                           double        sigma_sup,
                           int           iterations,
                           const double *mask);

/* flow_simulation_viscous (HighMap/src/hydrology/flow_simulation.cpp:112-157,
 * kernel shallow_viscous_flow.cl): returns the water depth in water_depth. */
int hmo_flow_simulation_viscous_f32(const float *z,
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
int hmo_flow_simulation_viscous_f64(const double *z,
                                    int           nx,
                                    int           ny,
                                    double        water_height,
                                    const double *depth_map,
                                    int           iterations,
                                    double        dt,
                                    double        dry_out_ratio,
                                    double        viscosity,
                                    double        power,
                                    double       *water_depth);

/* snow_simulation's post-filter (HighMap/src/hydrology/snow_simulation.cpp:
 * 140-152, then its clamp_min(s, 0)): z the terrain, s the snow depth,
 * updated in place. */
int hmo_snow_post_filter_f32(const float *z,
                             float       *s,
                             int          nx,
                             int          ny,
                             float        snow_depth,
                             int          iterations,
                             float        thermal_talus_ratio);
int hmo_snow_post_filter_f64(const double *z,
                             double       *s,
                             int           nx,
                             int           ny,
                             double        snow_depth,
                             int           iterations,
                             double        thermal_talus_ratio);

/* Sibling talus stencils (thermal_gpu.cpp:221-396; kernels thermal_ridge.cl,
 * thermal_scree.cl, thermal_schott.cl, thermal_olsen.cl), Jacobi form.
 * zmax: scree only; intensity: schott only; deposition_map: |z - z0| for
 * ridge and schott, max(z - z0, 0) for scree, not written for olsen;
 * mask: apply_with_mask blend, nullable. */
#define HMO_RIDGE 0
#define HMO_SCREE 1
#define HMO_SCHOTT 2
#define HMO_OLSEN 3
int hmo_thermal_sibling_f32(int          rule,
                            float       *z,
                            int          nx,
                            int          ny,
                            const float *talus,
                            const float *zmax,
                            float        intensity,
                            int          iterations,
                            float       *deposition_map,
                            const float *mask);
int hmo_thermal_sibling_f64(int           rule,
                            double       *z,
                            int           nx,
                            int           ny,
                            const double *talus,
                            const double *zmax,
                            double        intensity,
                            int           iterations,
                            double       *deposition_map,
                            const double *mask);

/* flow_simulation (HighMap/src/hydrology/flow_simulation.cpp:26-110):
 * water depth after `iterations` flow and water passes of the pipe model
 * (hydraulic_vpipes.cl:5-116, gravity, pipe area and length 1) on the fixed
 * terrain z, starting from water_height * depth_map, then the optional
 * dry-out (water_depth.cpp:40-66). */
int hmo_flow_simulation_f32(const float *z,
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
int hmo_flow_simulation_f64(const double *z,
                            int           nx,
                            int           ny,
                            double        water_height,
                            const double *depth_map,
                            int           iterations,
                            double        dt,
                            int           flux_diffusion,
                            double        flux_diffusion_strength,
                            double        dry_out_ratio,
                            double       *water_depth);

/* OpenCL linear sampler with mirrored-repeat addressing, evaluated on an
 * nx x ny texel grid at unnormalised coordinate (x, y) (texel centres at
 * k + 0.5).  Exposed for the tests of the advection pass. */
float hmo_sample_linear_mirror_f32(const float *s, int nx, int ny, float x, float y);

int hmo_num_threads(void);

#ifdef __cplusplus
}
#endif

#endif
