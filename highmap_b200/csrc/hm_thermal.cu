/*
 * hm_thermal.cu - talus thermal erosion on sm_100a.
 *
 * Replaces the host loop of HighMap/src/erosion/thermal_gpu.cpp:17-96 and
 * the OpenCL kernels thermal / thermal_with_bedrock
 * (HighMap/src/gpu_opencl/kernels/thermal.cl:26-100).
 *
 * Device data: z, talus and bedrock stay in HBM for the whole call; steps
 * ping-pong between z and one workspace grid (Jacobi).  After the steps:
 * extrapolate_borders (HighMap/src/boundary/boundary.cpp:19-41) on the
 * outer ring, then, when asked, the deposition map max(z - z0, 0)
 * (HighMap/src/range/range.cpp:253-262) and the mask blend
 * lerp(z0, z, mask) (HighMap/include/highmap/operator.hpp:405-418).
 *
 * Kernels
 *   k_thermal_step    one step per launch, one cell per thread; HBM bound:
 *                     reads z (9-point, reuse through L1/L2), talus and
 *                     bedrock, writes z: 12 B/cell (16 B with bedrock).
 *   k_thermal_tb      several steps per launch (temporal blocking): a
 *                     strip of columns streams down the grid; each time
 *                     level keeps a 4-row ring in shared memory.
 *   k_extrapolate     the outer ring, one block.
 *   k_thermal_final   deposition map and mask blend, elementwise.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "hm_internal.h"
#include "hm_thermal.h"
#include "hm_thermal_math.cuh"

namespace hm
{

/* ------------------------------------------------------------------ */
/* one step per launch                                                */
/* ------------------------------------------------------------------ */

constexpr int STEP_BX = 64;
constexpr int STEP_BY = 4;

template <bool TMAP, int BED>
__global__ void __launch_bounds__(STEP_BX *STEP_BY)
    k_thermal_step(const float *__restrict__ a,
                   float *__restrict__ b,
                   int nx,
                   int ny,
                   const float *__restrict__ talus,
                   float talus_value,
                   const float *__restrict__ bedrock)
{
  const int i = blockIdx.x * STEP_BX + threadIdx.x;
  const int j = blockIdx.y * STEP_BY + threadIdx.y;
  if (i >= nx || j >= ny) return;
  const size_t idx = (size_t)j * nx + i;
  /* apply_boundaries, _common_index.cl:106-132 */
  if (i == 0) { b[idx] = __ldg(a + idx + 1); return; }
  if (i == nx - 1) { b[idx] = __ldg(a + idx - 1); return; }
  if (j == 0) { b[idx] = __ldg(a + idx + nx); return; }
  if (j == ny - 1) { b[idx] = __ldg(a + idx - nx); return; }

  const float *up = a + idx - nx;
  const float *mid = a + idx;
  const float *dn = a + idx + nx;
  const float  t = TMAP ? __ldg(talus + idx) : talus_value;
  const float  zb = BED != BED_NONE ? __ldg(bedrock + idx) : 0.f;
  b[idx] = thermal_cell<BED>(__ldg(mid), __ldg(mid - 1), __ldg(dn), __ldg(up), __ldg(mid + 1),
                             __ldg(up - 1), __ldg(dn - 1), __ldg(up + 1), __ldg(dn + 1), t, zb);
}

/* ------------------------------------------------------------------ */
/* borders and finalisation                                           */
/* ------------------------------------------------------------------ */

/* extrapolate_borders(z, 1, 0): columns first, then rows, as the loops of
 * boundary.cpp:26-40 order them (the row pass reads the column pass's
 * corner values). */
__global__ void __launch_bounds__(1024) k_extrapolate(float *z, int nx, int ny)
{
  for (int j = threadIdx.x; j < ny; j += blockDim.x)
  {
    float *r = z + (size_t)j * nx;
    r[0] = __fsub_rn(__fmul_rn(2.f, r[1]), r[2]);
    r[nx - 1] = __fsub_rn(__fmul_rn(2.f, r[nx - 2]), r[nx - 3]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nx; i += blockDim.x)
  {
    z[i] = __fsub_rn(__fmul_rn(2.f, z[(size_t)nx + i]), z[(size_t)2 * nx + i]);
    size_t l = (size_t)(ny - 1) * nx + i;
    z[l] = __fsub_rn(__fmul_rn(2.f, z[l - nx]), z[l - 2 * (size_t)nx]);
  }
}

__global__ void k_thermal_final(float *__restrict__ z,
                                const float *__restrict__ z0,
                                float *__restrict__ depo,
                                const float *__restrict__ mask,
                                size_t n)
{
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
  {
    float r = z[k];
    float o = z0[k];
    if (depo)
    {
      float dz = __fsub_rn(r, o);
      depo[k] = dz > 0.f ? dz : 0.f;
    }
    if (mask)
    {
      float m = mask[k];
      z[k] = __fadd_rn(__fmul_rn(o, __fsub_rn(1.f, m)), __fmul_rn(r, m));
    }
  }
}

/* ------------------------------------------------------------------ */
/* host side                                                          */
/* ------------------------------------------------------------------ */

static int num_sms(int device)
{
  static int cached[64] = {0};
  if (device >= 0 && device < 64 && cached[device]) return cached[device];
  int n = 0;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
  if (n <= 0) n = 148;
  if (device >= 0 && device < 64) cached[device] = n;
  return n;
}

template <bool TMAP, int BED>
static void launch_step(const float *a, float *b, int nx, int ny, const float *talus, float tv,
                        const float *bed, cudaStream_t s)
{
  dim3 block(STEP_BX, STEP_BY);
  dim3 grid((nx + STEP_BX - 1) / STEP_BX, (ny + STEP_BY - 1) / STEP_BY);
  k_thermal_step<TMAP, BED><<<grid, block, 0, s>>>(a, b, nx, ny, talus, tv, bed);
}

static void step_dispatch(const float *a, float *b, int nx, int ny, const float *talus, float tv,
                          const float *bed, int bed_mode, cudaStream_t s)
{
  const int mode = bed ? (bed_mode == HM_BEDROCK_LITERAL ? BED_LITERAL : BED_INTENDED) : BED_NONE;
  if (talus)
  {
    if (mode == BED_NONE) launch_step<true, BED_NONE>(a, b, nx, ny, talus, tv, bed, s);
    else if (mode == BED_INTENDED) launch_step<true, BED_INTENDED>(a, b, nx, ny, talus, tv, bed, s);
    else launch_step<true, BED_LITERAL>(a, b, nx, ny, talus, tv, bed, s);
  }
  else
  {
    if (mode == BED_NONE) launch_step<false, BED_NONE>(a, b, nx, ny, talus, tv, bed, s);
    else if (mode == BED_INTENDED) launch_step<false, BED_INTENDED>(a, b, nx, ny, talus, tv, bed, s);
    else launch_step<false, BED_LITERAL>(a, b, nx, ny, talus, tv, bed, s);
  }
}

int thermal_check_args(const float *z, int nx, int ny, int iterations, const hm_thermal_options *o)
{
  if (!z) return fail(HM_ERR_INVALID_ARGUMENT, "thermal: z is NULL");
  if (nx < 3 || ny < 3) return fail(HM_ERR_INVALID_ARGUMENT, "thermal: nx and ny must be >= 3");
  if ((long long)nx * (long long)ny > (1ll << 34))
    return fail(HM_ERR_INVALID_ARGUMENT, "thermal: grid larger than 2^34 cells");
  if (iterations < 0) return fail(HM_ERR_INVALID_ARGUMENT, "thermal: iterations < 0");
  if (o && o->bedrock_mode != HM_BEDROCK_INTENDED && o->bedrock_mode != HM_BEDROCK_LITERAL)
    return fail(HM_ERR_INVALID_ARGUMENT, "thermal: unknown bedrock_mode");
  if (o && o->time_block < 0) return fail(HM_ERR_INVALID_ARGUMENT, "thermal: time_block < 0");
  return HM_OK;
}

size_t thermal_scratch_floats(int nx, int ny, bool need_z0)
{
  size_t n = align_up((size_t)nx * ny, 64);
  return n * (need_z0 ? 2 : 1);
}

int thermal_core(int device,
                 float *z,
                 int nx,
                 int ny,
                 const float *talus,
                 float talus_value,
                 int iterations,
                 const float *bedrock,
                 float *depo,
                 const float *mask,
                 const hm_thermal_options *opts,
                 float *scratch_buf,
                 cudaStream_t s)
{
  hm_thermal_options o;
  hm_thermal_default_options(&o);
  if (opts) o = *opts;
  const size_t n = (size_t)nx * ny;
  const bool   need_z0 = depo || mask;
  float       *tmp = scratch_buf;
  float       *z0 = need_z0 ? scratch_buf + align_up(n, 64) : nullptr;
  (void)device;

  if (need_z0) HM_CUDA_TRY(cudaMemcpyAsync(z0, z, n * sizeof(float), cudaMemcpyDeviceToDevice, s));

  const float *src = z;
  float       *dst = tmp;
  for (int it = 0; it < iterations; it++)
  {
    step_dispatch(src, dst, nx, ny, talus, talus_value, bedrock, o.bedrock_mode, s);
    HM_LAUNCH_CHECK("k_thermal_step");
    const float *t = src;
    src = dst;
    dst = const_cast<float *>(t);
  }
  if (src != z) HM_CUDA_TRY(cudaMemcpyAsync(z, src, n * sizeof(float), cudaMemcpyDeviceToDevice, s));

  k_extrapolate<<<1, 1024, 0, s>>>(z, nx, ny);
  HM_LAUNCH_CHECK("k_extrapolate");

  if (need_z0)
  {
    int blocks = num_sms(device) * 8;
    k_thermal_final<<<blocks, 256, 0, s>>>(z, z0, depo, mask, n);
    HM_LAUNCH_CHECK("k_thermal_final");
  }
  return HM_OK;
}

} // namespace hm

extern "C" void hm_thermal_default_options(hm_thermal_options *opts)
{
  if (!opts) return;
  opts->bedrock_mode = HM_BEDROCK_INTENDED;
  opts->time_block = 0;
}
