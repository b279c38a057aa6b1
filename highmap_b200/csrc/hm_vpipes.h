/* hm_vpipes.h - internal entry points of hm_vpipes.cu */
#ifndef HM_VPIPES_H
#define HM_VPIPES_H

#include <cuda_runtime.h>

#include "hm_erosion.h"

namespace hm
{
int    vpipes_check_args(const float *z, int nx, int ny, const hm_vpipes_params *p);
size_t vpipes_scratch_bytes(int nx, int ny);
/* Device pointers; ordered on s.  rain and the outputs are nullable. */
int    vpipes_core(float *z, int nx, int ny, const hm_vpipes_params &p, const float *rain, float *water_depth,
                   float *sediment, float *vel_u, float *vel_v, void *scratch_buf, cudaStream_t s);
struct VpFields;
struct VpScalars;
struct VpConst;
VpConst vpipes_consts(int nx, int ny, const hm_vpipes_params &p);
/* initial state of copy A (depth, zero sediment and fluxes) and V0, R */
int     vpipes_init(const VpFields &A, const float *rain, size_t n, float init_depth, VpScalars *sc,
                    double *partials, cudaStream_t s);
/* device address of the solve's error word (bit 0: a tile's TMA loads
 * timed out and the tile was skipped) inside the scratch of vpipes_core */
const unsigned *vpipes_error_word(const void *scratch_buf, int nx, int ny);
/* flow_simulation (hm_flow.cu): device pointers, ordered on s; scratch of
 * flow_scratch_bytes; water_depth receives the final depth */
int             flow_check_args(const float *z, const float *depth_map, const float *out, int nx, int ny,
                                int iterations, float dt);
size_t          flow_scratch_bytes(int nx, int ny);
int             flow_simulation_core(const float *z, int nx, int ny, float water_height, const float *depth_map,
                                     int iterations, float dt, int flux_diffusion, float flux_diffusion_strength,
                                     float dry_out_ratio, float *water_depth, void *scratch, cudaStream_t s);
const unsigned *flow_error_word(const void *scratch, int nx, int ny);
/* flow_simulation_viscous (hm_vflow.cu): device pointers, ordered on s;
 * scratch of vflow_scratch_bytes; water_depth receives the final depth */
int             vflow_check_args(const float *z, const float *depth_map, const float *out, int nx, int ny,
                                 int iterations);
size_t          vflow_scratch_bytes(int nx, int ny);
int             vflow_core(const float *z, int nx, int ny, float water_height, const float *depth_map, int iterations,
                           float dt, float dry_out_ratio, float viscosity, float power, float *water_depth,
                           void *scratch, cudaStream_t s);
/* fp64 partial-sum slots vpipes_init needs */
size_t  vpipes_init_partials();
/* water-depth output: stored depth plus the top-up of the last step */
int     vpipes_final_depth(const float *d, const float *rain, const VpScalars *sc, int parity, bool maintain,
                           float *out, size_t n, cudaStream_t s);
} // namespace hm

#endif
