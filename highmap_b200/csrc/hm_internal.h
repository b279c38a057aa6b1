/*
 * hm_internal.h - shared host-side plumbing of libhm_erosion.so: context,
 * workspace, error reporting and launch accounting.
 */
#ifndef HM_INTERNAL_H
#define HM_INTERNAL_H

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>

#include "hm_erosion.h"

struct hm_context
{
  int          device = 0;
  cudaStream_t stream = nullptr; /* stream of the host-pointer calls */
  void        *ws = nullptr;     /* grow-only device workspace       */
  size_t       ws_bytes = 0;
  /* small device area for reductions and per-call scalars */
  void        *scratch = nullptr;
  size_t       scratch_bytes = 0;
};

namespace hm
{

/* thread-local last error */
void        set_error(const std::string &msg);
void        clear_error();
int         fail(int status, const std::string &msg);
int         cuda_fail(cudaError_t e, const char *what);
void        count_launch(unsigned n = 1);

/* Make `device` current on the calling thread; HM_OK or an error status. */
int         use_device(int device);

/* Workspace of at least `bytes` (256-byte aligned), grown on demand.  The
 * previous contents are not preserved across growth.  Growth synchronises
 * the device so no in-flight kernel can still use the old block. */
int         workspace(hm_context *ctx, size_t bytes, void **out);
/* Scratch area for reductions (at least `bytes`). */
int         scratch(hm_context *ctx, size_t bytes, void **out);

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

} // namespace hm

#define HM_CUDA_TRY(expr)                                                                    \
  do                                                                                         \
  {                                                                                          \
    cudaError_t hm_e_ = (expr);                                                              \
    if (hm_e_ != cudaSuccess) return hm::cuda_fail(hm_e_, #expr);                            \
  } while (0)

#define HM_LAUNCH_CHECK(name)                                                                \
  do                                                                                         \
  {                                                                                          \
    hm::count_launch();                                                                      \
    cudaError_t hm_e_ = cudaGetLastError();                                                  \
    if (hm_e_ != cudaSuccess) return hm::cuda_fail(hm_e_, name);                             \
  } while (0)

#endif
