/*
 * hm_context.cpp - context, workspace, errors, hm_init.
 *
 * hm_init replaces hmap::gpu::init_opencl() (HighMap/src/gpu_opencl/
 * gpu_opencl.cpp:32-134), which builds every OpenCL kernel of the library
 * once; here the kernels are compiled ahead of time for sm_100a, so the
 * check is that such a device is present and a context can be made on it.
 */
#include <cstring>
#include <new>
#include <string>

#include "hm_internal.h"

namespace hm
{

static thread_local std::string        g_last_error;
static thread_local unsigned long long g_launches = 0;

void set_error(const std::string &msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }

int fail(int status, const std::string &msg)
{
  g_last_error = msg;
  return status;
}

int cuda_fail(cudaError_t e, const char *what)
{
  int status = HM_ERR_CUDA;
  if (e == cudaErrorMemoryAllocation) status = HM_ERR_OUT_OF_MEMORY;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) status = HM_ERR_NO_DEVICE;
  g_last_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  return status;
}

void count_launch(unsigned n) { g_launches += n; }

int use_device(int device)
{
  int cur = -1;
  if (cudaGetDevice(&cur) == cudaSuccess && cur == device) return HM_OK;
  HM_CUDA_TRY(cudaSetDevice(device));
  return HM_OK;
}

int workspace(hm_context *ctx, size_t bytes, void **out)
{
  bytes = align_up(bytes ? bytes : 256, 1 << 20);
  if (ctx->ws_bytes < bytes)
  {
    if (ctx->ws)
    {
      HM_CUDA_TRY(cudaDeviceSynchronize());
      HM_CUDA_TRY(cudaFree(ctx->ws));
      ctx->ws = nullptr;
      ctx->ws_bytes = 0;
    }
    cudaError_t e = cudaMalloc(&ctx->ws, bytes);
    if (e != cudaSuccess)
    {
      cudaGetLastError();
      ctx->ws = nullptr;
      return cuda_fail(e, "workspace cudaMalloc");
    }
    ctx->ws_bytes = bytes;
  }
  *out = ctx->ws;
  return HM_OK;
}

int scratch(hm_context *ctx, size_t bytes, void **out)
{
  bytes = align_up(bytes ? bytes : 256, 4096);
  if (ctx->scratch_bytes < bytes)
  {
    if (ctx->scratch)
    {
      HM_CUDA_TRY(cudaDeviceSynchronize());
      HM_CUDA_TRY(cudaFree(ctx->scratch));
      ctx->scratch = nullptr;
      ctx->scratch_bytes = 0;
    }
    cudaError_t e = cudaMalloc(&ctx->scratch, bytes);
    if (e != cudaSuccess)
    {
      cudaGetLastError();
      ctx->scratch = nullptr;
      return cuda_fail(e, "scratch cudaMalloc");
    }
    ctx->scratch_bytes = bytes;
  }
  *out = ctx->scratch;
  return HM_OK;
}

} // namespace hm

extern "C" {

int hm_init(void)
{
  hm::clear_error();
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
  {
    cudaGetLastError();
    return hm::fail(HM_ERR_NO_DEVICE, "no CUDA device is visible");
  }
  cudaDeviceProp prop;
  HM_CUDA_TRY(cudaGetDeviceProperties(&prop, 0));
  if (prop.major != 10 || prop.minor != 0)
    return hm::fail(HM_ERR_NO_DEVICE, std::string("device 0 is ") + prop.name + " (compute capability " +
                                          std::to_string(prop.major) + "." + std::to_string(prop.minor) +
                                          "), this library is built for sm_100a only");
  HM_CUDA_TRY(cudaFree(nullptr)); /* create the primary context */
  return HM_OK;
}

int hm_context_create(hm_context **ctx, int device)
{
  hm::clear_error();
  if (!ctx) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_context_create: ctx is NULL");
  *ctx = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
  {
    cudaGetLastError();
    return hm::fail(HM_ERR_NO_DEVICE, "no CUDA device is visible");
  }
  if (device < 0 || device >= n) return hm::fail(HM_ERR_INVALID_ARGUMENT, "device index out of range");
  int major = 0, minor = 0;
  HM_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
  HM_CUDA_TRY(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device));
  if (major != 10 || minor != 0)
    return hm::fail(HM_ERR_NO_DEVICE, "device " + std::to_string(device) + " has compute capability " +
                                          std::to_string(major) + "." + std::to_string(minor) +
                                          ", this library is built for sm_100a only");
  int st = hm::use_device(device);
  if (st) return st;
  hm_context *c = new (std::nothrow) hm_context();
  if (!c) return hm::fail(HM_ERR_OUT_OF_MEMORY, "host allocation of the context failed");
  c->device = device;
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess)
  {
    delete c;
    return hm::cuda_fail(e, "cudaStreamCreate");
  }
  *ctx = c;
  return HM_OK;
}

int hm_context_trim(hm_context *ctx)
{
  if (!ctx) return hm::fail(HM_ERR_INVALID_ARGUMENT, "hm_context_trim: ctx is NULL");
  int st = hm::use_device(ctx->device);
  if (st) return st;
  HM_CUDA_TRY(cudaDeviceSynchronize());
  if (ctx->ws) HM_CUDA_TRY(cudaFree(ctx->ws));
  ctx->ws = nullptr;
  ctx->ws_bytes = 0;
  return HM_OK;
}

int hm_context_destroy(hm_context *ctx)
{
  if (!ctx) return HM_OK;
  hm::use_device(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->ws) cudaFree(ctx->ws);
  if (ctx->scratch) cudaFree(ctx->scratch);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return HM_OK;
}

const char *hm_status_string(int status)
{
  switch (status)
  {
  case HM_OK: return "ok";
  case HM_ERR_INVALID_ARGUMENT: return "invalid argument";
  case HM_ERR_NO_DEVICE: return "no usable CUDA device";
  case HM_ERR_OUT_OF_MEMORY: return "out of device memory";
  case HM_ERR_CUDA: return "CUDA error";
  case HM_ERR_TIMEOUT: return "timed out";
  case HM_ERR_BUSY: return "busy";
  default: return "unknown status";
  }
}

const char *hm_last_error(void) { return hm::g_last_error.c_str(); }

unsigned long long hm_launch_count(void) { return hm::g_launches; }
void               hm_launch_count_reset(void) { hm::g_launches = 0; }

} // extern "C"
