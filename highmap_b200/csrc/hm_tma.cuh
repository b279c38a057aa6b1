/*
 * hm_tma.cuh - tensor-memory-accelerator (TMA) tile loads and the shared
 * memory barrier that tracks them (sm_90+ PTX, used here on sm_100a).
 *
 * One elected thread arms a CTA-local mbarrier with the byte count of the
 * tiles and issues cp.async.bulk.tensor loads (no cluster multicast: every
 * CTA fetches its own tiles from this GPU's memory); the other threads wait
 * on the barrier's phase.  A waiting warp asks to be suspended until the
 * phase completes (mbarrier.try_wait with a suspend-time hint), so it
 * spends no issue slots polling while the boxes are in flight.  Waits are
 * bounded twice over: by HM_TMA_WAIT_NS of the global timer and by
 * HM_TMA_SPIN_LIMIT polls; the waiter then gives up and reports failure so
 * the kernel can record an error and return instead of hanging.
 *
 * Tensor-map rules the host side keeps (cuTensorMapEncodeTiled): 16-byte
 * aligned base, row pitch a multiple of 16 bytes, innermost box extent a
 * multiple of 16 bytes.  The device side keeps the innermost coordinate a
 * multiple of 4 floats (16 bytes); out-of-range elements of a box read as
 * zero.
 */
#ifndef HM_TMA_CUH
#define HM_TMA_CUH

#include <cuda.h>
#include <cstdint>

namespace hm
{

constexpr unsigned HM_TMA_SPIN_LIMIT = 1u << 22;
/* one wait window: a second of the global timer (the boxes of a tile land
 * within microseconds) */
constexpr unsigned long long HM_TMA_WAIT_NS = 1000000000ull;
/* longest a waiting warp asks to be suspended per poll (ns); it resumes as
 * soon as the phase completes.  0 selects the form without a hint. */
#ifndef HM_TMA_SUSPEND_NS
#define HM_TMA_SUSPEND_NS 20000u
#endif

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

/* make the initialised barrier visible to the async (TMA) proxy */
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
  unsigned ok;
  asm volatile("{\n"
               ".reg .pred p;\n"
               "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
               "selp.u32 %0, 1, 0, p;\n"
               "}\n"
               : "=r"(ok)
               : "r"(smem_u32(bar)), "r"(parity)
               : "memory");
  return ok != 0;
}

/* the same test, the warp suspended until the phase completes or
 * `hint_ns` nanoseconds have passed */
__device__ __forceinline__ bool mbar_try_wait_suspend(uint64_t *bar, unsigned parity, unsigned hint_ns)
{
  unsigned ok;
  asm volatile("{\n"
               ".reg .pred p;\n"
               "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
               "selp.u32 %0, 1, 0, p;\n"
               "}\n"
               : "=r"(ok)
               : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
               : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

/* bounded wait for the barrier phase `parity` to complete: true once it
 * has, false after HM_TMA_WAIT_NS or HM_TMA_SPIN_LIMIT polls */
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity)
{
  /* first poll (suspended up to the hint): the phase has usually completed
   * by its end, and the clock is not read */
  if (HM_TMA_SUSPEND_NS ? mbar_try_wait_suspend(bar, parity, HM_TMA_SUSPEND_NS) : mbar_try_wait(bar, parity))
    return true;
  const unsigned long long t0 = global_ns();
  for (unsigned i = 0; i < HM_TMA_SPIN_LIMIT; i++)
  {
    if (HM_TMA_SUSPEND_NS ? mbar_try_wait_suspend(bar, parity, HM_TMA_SUSPEND_NS) : mbar_try_wait(bar, parity))
      return true;
    if (global_ns() - t0 > HM_TMA_WAIT_NS) return false;
  }
  return false;
}

/* 2-D tile load: box of the tensor map at (x, y) into dst, completion
 * counted on bar.  x must be a multiple of 4 for 32-bit elements. */
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
  asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
               " [%0], [%1, {%2, %3}], [%4];\n" ::"r"(smem_u32(dst)),
               "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
               : "memory");
}

} // namespace hm

#endif
