/*
 * hm_vflow.cu - flow_simulation_viscous on sm_100a: water spreading over a
 * fixed terrain as a viscous thin film.
 *
 * Replaces HighMap/src/hydrology/flow_simulation.cpp:112-157 and its
 * kernel shallow_viscous_flow.cl.  Per step (h_in -> h_out, clamp-to-edge
 * reads):
 *   M_face = ((h + h_n) / 2)^power / viscosity       for the four faces,
 *   q = -M (H_n - H_c), H = h + z,
 *   h' = max(0, h - dt ((q_e - q_w) + q_n - q_s)),
 * and every 10 steps, before the step, dt = 0.2 / max(hmax^power /
 * viscosity, 1e-6) (helper_vflow_compute_adaptive_dt, :16-24; the caller's
 * dt is replaced before the first step).  Afterwards the dry-out of
 * water_depth.cpp:40-66.
 *
 * The reference round-trips the depth to the host around every step and
 * takes hmax on the host; here the depth stays in HBM and dt is formed on
 * the device: a max reduction over order-preserving integer keys of the
 * depth (exact for negative values too), then one thread computes dt into
 * a device slot that the step kernels read.  pow is evaluated in fp64 and
 * rounded once to fp32, which equals the host's powf except where the
 * exact power lies within about 2^-52 of a float rounding boundary.
 */
#include <cuda_runtime.h>

#include "hm_internal.h"
#include "hm_vpipes.h"
#include "hm_vpipes_math.cuh"

namespace hm
{

namespace
{

constexpr int VF_NT = 256;
constexpr int VF_GRID = 148 * 8;

/* float -> unsigned key that orders like the values (negatives below
 * positives), and back */
__device__ __forceinline__ unsigned fkey(float v)
{
  const unsigned b = __float_as_uint(v);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float funkey(unsigned k)
{
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__global__ void __launch_bounds__(VF_NT) k_vflow_init(float *__restrict__ h, const float *__restrict__ depth_map,
                                                      float water_height, size_t n)
{
  for (size_t k = blockIdx.x * (size_t)VF_NT + threadIdx.x; k < n; k += (size_t)gridDim.x * VF_NT)
    h[k] = __fmul_rn(water_height, depth_map[k]);
}

/* clear the key slot; dt = the caller's (replaced before the first step) */
__global__ void k_vflow_reset(unsigned *slot, float *dtp, float dt)
{
  *slot = 0u;
  *dtp = dt;
}

/* slot = key of max(h); the slot must hold 0 (the least key) before */
__global__ void __launch_bounds__(VF_NT) k_vflow_max(const float *__restrict__ h, size_t n, unsigned *slot)
{
  unsigned m = 0u;
  for (size_t k = blockIdx.x * (size_t)VF_NT + threadIdx.x; k < n; k += (size_t)gridDim.x * VF_NT)
  {
    const unsigned c = fkey(h[k]);
    m = c > m ? c : m;
  }
  for (int o = 16; o > 0; o >>= 1)
  {
    const unsigned t = __shfl_xor_sync(0xffffffffu, m, o);
    m = t > m ? t : m;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(slot, m);
}

/* dt = 0.2 / fmax(hmax^power / viscosity, 1e-6); the key slot is cleared
 * for the next reduction */
__global__ void k_vflow_dt(unsigned *slot, float viscosity, float power, float *dt)
{
  const float hmax = funkey(*slot);
  const float mobility = fdiv(powr(hmax, power), viscosity);
  *dt = fdiv(0.2f, fmaxf(mobility, 1e-6f));
  *slot = 0u;
}

__device__ __forceinline__ float face_mobility(float h, float hn, float viscosity, float power)
{
  return fdiv(powr(fmul(0.5f, fadd(h, hn)), power), viscosity);
}

/* One step over a 32 x 8 tile.  Each face mobility is evaluated once, by
 * the thread of the cell west / south of it (plus the tile's west and
 * south edges), into shared memory; a face is the same value for the two
 * cells it separates (fadd is commutative), so this equals evaluating it
 * from both sides, at about half the pow calls.  Faces on the grid's edge
 * pair a cell with itself, as the clamped reads do. */
constexpr int VT_X = 32, VT_Y = 8;

__global__ void __launch_bounds__(VT_X *VT_Y) k_vflow_step(const float *__restrict__ z, const float *__restrict__ hin,
                                                          float *__restrict__ hout, int nx, int ny,
                                                          const float *__restrict__ dtp, float viscosity, float power)
{
  __shared__ float me[VT_Y][VT_X + 1]; /* me[ty][tx + 1]: east face of (tx, ty); [ty][0]: west edge  */
  __shared__ float mn[VT_Y + 1][VT_X]; /* mn[ty + 1][tx]: north face of (tx, ty); [0][tx]: south edge */
  const int  tx = threadIdx.x, ty = threadIdx.y;
  const int  i = blockIdx.x * VT_X + tx, j = blockIdx.y * VT_Y + ty;
  const bool in = i < nx && j < ny;
  const int  ic = in ? i : 0, jc = in ? j : 0;
  const size_t k = (size_t)jc * nx + ic;
  const size_t ke = ic < nx - 1 ? k + 1 : k, kw = ic > 0 ? k - 1 : k;
  const size_t kn = jc < ny - 1 ? k + nx : k, ks = jc > 0 ? k - nx : k; /* j + 1, j - 1 */
  const float  h = hin[k];
  const float  hxp = hin[ke], hxm = hin[kw], hyp = hin[kn], hym = hin[ks];
  if (in)
  {
    me[ty][tx + 1] = face_mobility(h, hxp, viscosity, power);
    mn[ty + 1][tx] = face_mobility(h, hyp, viscosity, power);
    if (tx == 0) me[ty][0] = face_mobility(h, hxm, viscosity, power);
    if (ty == 0) mn[0][tx] = face_mobility(h, hym, viscosity, power);
  }
  __syncthreads();
  if (!in) return;
  const float dt = *dtp;
  const float zc = z[k];
  const float Hc = fadd(h, zc);
  const float Hxp = fadd(hxp, z[ke]), Hxm = fadd(hxm, z[kw]), Hyp = fadd(hyp, z[kn]), Hym = fadd(hym, z[ks]);
  const float Mp = me[ty][tx + 1], Mm = me[ty][tx], Myp = mn[ty + 1][tx], Mym = mn[ty][tx];
  const float qxp = fmul(-Mp, fsub(Hxp, Hc));
  const float qxm = fmul(-Mm, fsub(Hc, Hxm));
  const float qyp = fmul(-Myp, fsub(Hyp, Hc));
  const float qym = fmul(-Mym, fsub(Hc, Hym));
  const float dhdt = -fsub(fadd(fsub(qxp, qxm), qyp), qym);
  hout[k] = fmaxf(0.f, fadd(h, fmul(dt, dhdt)));
}

/* water_depth_dry_out: h -= ratio * hmax, then max(0, h) */
__global__ void __launch_bounds__(VF_NT) k_vflow_dry_out(const float *__restrict__ h, const unsigned *slot,
                                                         float ratio, float *__restrict__ out, size_t n)
{
  const float drop = fmul(ratio, funkey(*slot));
  for (size_t k = blockIdx.x * (size_t)VF_NT + threadIdx.x; k < n; k += (size_t)gridDim.x * VF_NT)
  {
    const float w = fsub(h[k], drop);
    out[k] = 0.f < w ? w : 0.f;
  }
}

} // namespace

size_t vflow_scratch_bytes(int nx, int ny)
{
  /* two depth grids, then the key slot and dt */
  return 2 * align_up((size_t)nx * ny, 64) * sizeof(float) + 256;
}

int vflow_check_args(const float *z, const float *depth_map, const float *out, int nx, int ny, int iterations)
{
  if (!z || !depth_map || !out) return fail(HM_ERR_INVALID_ARGUMENT, "flow_simulation_viscous: NULL grid");
  if (nx < 1 || ny < 1) return fail(HM_ERR_INVALID_ARGUMENT, "flow_simulation_viscous: nx and ny must be >= 1");
  if ((long long)nx * (long long)ny > (1ll << 34))
    return fail(HM_ERR_INVALID_ARGUMENT, "flow_simulation_viscous: grid larger than 2^34 cells");
  if (iterations < 0) return fail(HM_ERR_INVALID_ARGUMENT, "flow_simulation_viscous: iterations < 0");
  if ((ny + VT_Y - 1) / VT_Y > 65535)
    return fail(HM_ERR_INVALID_ARGUMENT, "flow_simulation_viscous: ny larger than 524280 rows");
  return HM_OK;
}

int vflow_core(const float *z, int nx, int ny, float water_height, const float *depth_map, int iterations,
               float dt, float dry_out_ratio, float viscosity, float power, float *water_depth, void *scratch,
               cudaStream_t s)
{
  const size_t n = (size_t)nx * ny;
  const size_t na = align_up(n, 64);
  float       *hA = (float *)scratch, *hB = hA + na;
  unsigned    *slot = (unsigned *)(hB + na);
  float       *dtp = (float *)(slot + 1);
  k_vflow_reset<<<1, 1, 0, s>>>(slot, dtp, dt);
  HM_LAUNCH_CHECK("k_vflow_reset");
  k_vflow_init<<<VF_GRID, VF_NT, 0, s>>>(hA, depth_map, water_height, n);
  HM_LAUNCH_CHECK("k_vflow_init");
  const dim3 tiles((nx + VT_X - 1) / VT_X, (ny + VT_Y - 1) / VT_Y);
  float     *cur = hA, *nxt = hB;
  for (int it = 0; it < iterations; ++it)
  {
    if (it % 10 == 0)
    {
      k_vflow_max<<<VF_GRID, VF_NT, 0, s>>>(cur, n, slot);
      HM_LAUNCH_CHECK("k_vflow_max");
      k_vflow_dt<<<1, 1, 0, s>>>(slot, viscosity, power, dtp);
      HM_LAUNCH_CHECK("k_vflow_dt");
    }
    k_vflow_step<<<tiles, dim3(VT_X, VT_Y), 0, s>>>(z, cur, nxt, nx, ny, dtp, viscosity, power);
    HM_LAUNCH_CHECK("k_vflow_step");
    float *t = cur;
    cur = nxt;
    nxt = t;
  }
  if (dry_out_ratio != 0.f)
  {
    k_vflow_max<<<VF_GRID, VF_NT, 0, s>>>(cur, n, slot);
    HM_LAUNCH_CHECK("k_vflow_max");
    k_vflow_dry_out<<<VF_GRID, VF_NT, 0, s>>>(cur, slot, dry_out_ratio, water_depth, n);
    HM_LAUNCH_CHECK("k_vflow_dry_out");
  }
  else
    HM_CUDA_TRY(cudaMemcpyAsync(water_depth, cur, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
  return HM_OK;
}

} // namespace hm
