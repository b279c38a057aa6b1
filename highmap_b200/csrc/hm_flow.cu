/*
 * hm_flow.cu - flow_simulation on sm_100a: the water-only use of the
 * virtual-pipes model.
 *
 * Replaces HighMap/src/hydrology/flow_simulation.cpp:26-110, which runs
 * the flow and water passes of hydraulic_vpipes.cl (:5-116) on a fixed
 * terrain with host round trips around every pass, then the optional
 * dry-out of HighMap/src/hydrology/water_depth.cpp:40-66.  Here the steps
 * are the tiled vpipes kernels in their flow-only form (FWE_FLOWONLY:
 * flow, water, no erosion or advection, depth and fluxes written), the
 * state stays in HBM, and the dry-out is a max reduction plus one
 * elementwise pass.
 *
 * State: depth and the four fluxes in two copies (A, B), the terrain read
 * in place, a zero sediment grid (staged, unused).  Gravity, pipe area and
 * pipe length are 1, evaporation 0, as in the reference's kernels.
 */
#include <cuda_runtime.h>

#include <cstdint>

#include "hm_internal.h"
#include "hm_vpipes.h"
#include "hm_vpipes_tiled.cuh"

namespace hm
{

namespace
{

/* d = water_height * depth_map; fluxes of copy A and the sediment grid 0 */
__global__ void k_flow_init(float *__restrict__ d, const float *__restrict__ depth_map, float water_height,
                            float *__restrict__ fl, float *__restrict__ fr, float *__restrict__ ft,
                            float *__restrict__ fb, float *__restrict__ s0, size_t n)
{
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
  {
    d[k] = __fmul_rn(water_height, depth_map[k]);
    fl[k] = fr[k] = ft[k] = fb[k] = s0[k] = 0.f;
  }
}

/* max of the depth (Array::max); depths are >= 0 (or -0), so the bit
 * patterns of the non-negative values order like the values */
__global__ void k_flow_max(const float *__restrict__ d, size_t n, unsigned *__restrict__ out)
{
  unsigned m = 0u;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
  {
    const float v = d[k];
    const unsigned b = v > 0.f ? __float_as_uint(v) : 0u;
    m = b > m ? b : m;
  }
  for (int o = 16; o > 0; o >>= 1)
  {
    const unsigned t = __shfl_xor_sync(0xffffffffu, m, o);
    m = t > m ? t : m;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

/* water_depth_dry_out (water_depth.cpp:59-64): d = max(0, d - ratio * dmax),
 * written to the output */
__global__ void k_flow_dry_out(const float *__restrict__ d, const unsigned *__restrict__ dmax_bits, float ratio,
                               float *__restrict__ out, size_t n)
{
  const float drop = __fmul_rn(ratio, __uint_as_float(*dmax_bits));
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
  {
    const float w = __fsub_rn(d[k], drop);
    out[k] = 0.f < w ? w : 0.f;
  }
}

} // namespace

size_t flow_scratch_bytes(int nx, int ny)
{
  /* depth and fluxes of two copies, the zero sediment grid, a max slot,
   * the scalar block (its error word records TMA load timeouts) */
  return align_up((size_t)nx * ny, 64) * sizeof(float) * 11 + 256 + align_up(sizeof(VpScalars), 256);
}

int flow_check_args(const float *z, const float *depth_map, const float *out, int nx, int ny, int iterations,
                    float dt)
{
  if (!z || !depth_map || !out) return fail(HM_ERR_INVALID_ARGUMENT, "flow_simulation: NULL grid");
  if (nx < 1 || ny < 1) return fail(HM_ERR_INVALID_ARGUMENT, "flow_simulation: nx and ny must be >= 1");
  if ((long long)nx * (long long)ny > (1ll << 32))
    return fail(HM_ERR_INVALID_ARGUMENT, "flow_simulation: grid larger than 2^32 cells");
  if (iterations < 0) return fail(HM_ERR_INVALID_ARGUMENT, "flow_simulation: iterations < 0");
  if (!(dt != 0.f)) return fail(HM_ERR_INVALID_ARGUMENT, "flow_simulation: dt must be non-zero");
  return HM_OK;
}

int flow_simulation_core(const float *z, int nx, int ny, float water_height, const float *depth_map, int iterations,
                         float dt, int flux_diffusion, float flux_diffusion_strength, float dry_out_ratio,
                         float *water_depth, void *scratch, cudaStream_t s)
{
  const size_t n = (size_t)nx * ny;
  const size_t na = align_up(n, 64);
  float       *base = (float *)scratch;
  float       *dA = base, *dB = base + na, *s0 = base + 10 * na;
  unsigned    *dmax = (unsigned *)(base + 11 * na);
  VpScalars   *sc = (VpScalars *)((char *)(base + 11 * na) + 256);
  VpFields     A{const_cast<float *>(z), dA, s0, base + 2 * na, base + 3 * na, base + 4 * na, base + 5 * na};
  VpFields     B{const_cast<float *>(z), dB, s0, base + 6 * na, base + 7 * na, base + 8 * na, base + 9 * na};

  hm_vpipes_params p;
  hm_vpipes_default_params(&p);
  p.water_height = water_height;
  p.dt = dt;
  p.flux_diffusion = flux_diffusion != 0;
  p.flux_diffusion_strength = flux_diffusion_strength;
  p.evap_rate = 0.f;
  p.maintain_water_volume = 0;
  const VpConst c = vpipes_consts(nx, ny, p);

  HM_CUDA_TRY(cudaMemsetAsync(sc, 0, sizeof(VpScalars), s));
  k_flow_init<<<592, 256, 0, s>>>(dA, depth_map, water_height, A.fl, A.fr, A.ft, A.fb, s0, n);
  HM_LAUNCH_CHECK("k_flow_init");

  FweIo io;
  memset(&io, 0, sizeof io);
  io.diffusion = p.flux_diffusion;
  io.pl_one = 1;
  io.kexp_one = 1;
  io.flow_only = 1;
  {
    auto al8 = [](const void *q) { return ((uintptr_t)q & 7u) == 0; };
    const void *outs[] = {A.d, A.fl, A.fr, A.ft, A.fb, B.d, B.fl, B.fr, B.ft, B.fb};
    bool        ok = nx % 2 == 0;
    for (const void *q : outs) ok = ok && al8(q);
    io.vec = ok ? 1 : 0;
  }
  FweMaps    maps[2];
  const bool tma = fwe_maps(A, nx, ny, &maps[0]) && fwe_maps(B, nx, ny, &maps[1]);
  const dim3 g1((nx + FT_TX - 1) / FT_TX, (ny + FT_TY - 1) / FT_TY);
  VpFields  *cur = &A, *nxt = &B;
  for (int it = 0; it < iterations; it++)
  {
    io.in = VpState{cur->z, cur->d, cur->s, cur->fl, cur->fr, cur->ft, cur->fb};
    io.out = VpStateOut{nxt->z, nxt->d, nxt->s, nxt->fl, nxt->fr, nxt->ft, nxt->fb, nullptr, nullptr};
    io.parity = it & 1;
    const int rc = tma ? launch_fwe_tma(io, maps[cur == &A ? 0 : 1], c, sc, nullptr, g1, s)
                       : launch_fwe_cp_async(io, c, sc, nullptr, g1, s);
    if (rc) return rc;
    VpFields *t = cur;
    cur = nxt;
    nxt = t;
  }
  if (dry_out_ratio != 0.f)
  {
    HM_CUDA_TRY(cudaMemsetAsync(dmax, 0, sizeof(unsigned), s));
    k_flow_max<<<592, 256, 0, s>>>(cur->d, n, dmax);
    HM_LAUNCH_CHECK("k_flow_max");
    k_flow_dry_out<<<592, 256, 0, s>>>(cur->d, dmax, dry_out_ratio, water_depth, n);
    HM_LAUNCH_CHECK("k_flow_dry_out");
  }
  else
    HM_CUDA_TRY(cudaMemcpyAsync(water_depth, cur->d, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
  return HM_OK;
}

const unsigned *flow_error_word(const void *scratch, int nx, int ny)
{
  const size_t na = align_up((size_t)nx * ny, 64);
  return &((const VpScalars *)((const char *)((const float *)scratch + 11 * na) + 256))->error;
}

} // namespace hm
