/*
 * hm_noalloc.cu - thermal erosion on device buffers without allocating.
 *
 * Some callers cannot call cudaMalloc at the moment they run erosion:
 * applications that give all device memory to their own pool allocator at
 * start-up and run plug-ins inside that fixed budget, and interactive or
 * real-time loops that must not pay for driver allocations (cudaFree
 * synchronises the whole device, which stalls every other stream).  For
 * them, hm_thermal_device_noalloc keeps its one piece of scratch memory,
 * the Jacobi ping-pong grid, in a statically reserved device array of
 * HM_NOALLOC_MAX_CELLS floats (16 MiB).  The caller still passes z,
 * talus and bedrock; nothing here calls cudaMalloc, cudaFree or an
 * allocating library routine.
 *
 * When the memory is taken: with CUDA's lazy module loading (the default
 * since CUDA 12.2) the array, like the kernels' code, is placed on a GPU
 * when the first call on that device loads them, not when the library is
 * loaded; it is then held until the process exits.  An application that
 * hands all free device memory to its own pool at start-up must therefore
 * make its first call on each device before that (or run with
 * CUDA_MODULE_LOADING=EAGER, which loads everything when the context is
 * created).  Make that first call before any stream capture begins, too.
 *
 * Set-up: every call looks up the array's device address on the current
 * device (cudaGetSymbolAddress, a table lookup once the module is loaded),
 * so a context recreated after cudaDeviceReset gets the new address.  In
 * host code the array's name is only a host-side handle, never a device
 * address, so only the looked-up pointer is passed to the kernels.
 *
 * Sharing: every call on a device uses the same array, which keeps the
 * last call's contents.  The step kernel writes every cell of the grid it
 * produces before anything reads it, so nothing needs clearing between
 * calls.  Calls that overlap on the GPU (different streams, or different
 * host threads, on one device) race on the array and must be serialised
 * by the caller.
 */
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "hm_internal.h"
#include "hm_thermal.h"

namespace
{

static __device__ __align__(256) float hm_noalloc_scratch[HM_NOALLOC_MAX_CELLS];

std::mutex g_setup_mutex;

/* Device address of the scratch array on the current device, looked up
 * on every call (the first lookup on a device loads the module). */
int scratch_for_current_device(int *device, float **out)
{
  int         dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return hm::cuda_fail(e, "hm_thermal_device_noalloc: cudaGetDevice");
  float                      *ptr = nullptr;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  e = cudaGetSymbolAddress((void **)&ptr, hm_noalloc_scratch);
  if (e != cudaSuccess) return hm::cuda_fail(e, "hm_thermal_device_noalloc: cudaGetSymbolAddress");
  if (!ptr) return hm::fail(HM_ERR_CUDA, "hm_thermal_device_noalloc: scratch array has no device address");
  *device = dev;
  *out = ptr;
  return HM_OK;
}

} // namespace

extern "C" int hm_thermal_device_noalloc(float       *z,
                                         int          nx,
                                         int          ny,
                                         const float *talus,
                                         float        talus_value,
                                         int          iterations,
                                         const float *bedrock,
                                         int          bedrock_mode,
                                         void        *stream)
{
  hm::clear_error();
  hm_thermal_options o;
  hm_thermal_default_options(&o);
  o.bedrock_mode = bedrock_mode;
  int st = hm::thermal_check_args(z, nx, ny, iterations, &o);
  if (st) return st;
  const size_t cells = (size_t)nx * (size_t)ny;
  if (cells > (size_t)HM_NOALLOC_MAX_CELLS)
    return hm::fail(HM_ERR_INVALID_ARGUMENT,
                    "hm_thermal_device_noalloc: grid of " + std::to_string(cells) +
                        " cells exceeds the no-allocation limit of " + std::to_string(HM_NOALLOC_MAX_CELLS) +
                        " cells (HM_NOALLOC_MAX_CELLS); use hm_thermal_device");
  int    device = 0;
  float *scratch = nullptr;
  if ((st = scratch_for_current_device(&device, &scratch))) return st;
  return hm::thermal_core(device, z, nx, ny, talus, talus_value, iterations, bedrock, nullptr, nullptr, &o,
                          scratch, (cudaStream_t)stream);
}
