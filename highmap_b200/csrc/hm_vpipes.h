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
} // namespace hm

#endif
