/*
 * hm_reduce.cuh - deterministic grid-wide fp64 sum with a last-block
 * finish, used for the water volume of the virtual-pipes solver
 * (Array::sum, HighMap/src/array/methods.cpp:428-431, as called by
 * HighMap/src/erosion/hydraulic_vpipes_gpu.cpp:54-55,167).
 *
 * Each block writes its fp64 partial; the block that takes the last ticket
 * adds the partials in index order (fixed grid => fixed order => the same
 * bits on every run) and calls `finish(sum)` from thread 0, then re-arms
 * the ticket for the next launch.
 */
#ifndef HM_REDUCE_CUH
#define HM_REDUCE_CUH

namespace hm
{

template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sm /* >= NT/32 */)
{
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int tid = threadIdx.x + threadIdx.y * blockDim.x + threadIdx.z * blockDim.x * blockDim.y;
  if ((tid & 31) == 0) sm[tid >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (tid < 32)
  {
    r = tid < NT / 32 ? sm[tid] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  return r; /* valid in thread 0 */
}

/* Commit this block's partial; the last block finishes the sum.
 * nblocks = number of blocks in the grid, bid = this block's linear id. */
template <int NT, class Finish>
__device__ __forceinline__ void grid_sum_commit(double   partial,
                                                double  *partials,
                                                unsigned *ticket,
                                                unsigned nblocks,
                                                unsigned bid,
                                                Finish   finish)
{
  __shared__ double   sm[NT / 32];
  __shared__ unsigned s_last;
  const int           tid = threadIdx.x + threadIdx.y * blockDim.x + threadIdx.z * blockDim.x * blockDim.y;
  double              b = block_sum<NT>(partial, sm);
  if (tid == 0)
  {
    partials[bid] = b;
    __threadfence();
    unsigned t = atomicAdd(ticket, 1u);
    s_last = (t == nblocks - 1) ? 1u : 0u;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double acc = 0.0;
  for (unsigned k = tid; k < nblocks; k += NT) acc += __ldcg(partials + k);
  double total = block_sum<NT>(acc, sm);
  if (tid == 0)
  {
    finish(total);
    *ticket = 0u;
    __threadfence();
  }
}

} // namespace hm

#endif
