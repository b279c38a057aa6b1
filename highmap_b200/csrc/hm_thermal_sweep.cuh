/*
 * hm_thermal_sweep.cuh - one Jacobi step of the talus exchange for the 32
 * columns of one warp, walking down a range of rows.  Used by the plain
 * one-step kernel (hm_thermal.cu) and by the thermal tiles of the batched
 * form (hm_batch.cu).
 *
 * Every row of z is loaded once per warp (lanes 0 and 31 also load the
 * column just outside the warp) and the west / east neighbours come from
 * warp shuffles, so a cell costs two coalesced loads per 32 cells instead
 * of nine loads.  The loads of P rows (z, talus, bedrock; a template
 * parameter) are issued before any of them is used, which keeps enough
 * bytes in flight to cover the HBM latency: the plain kernels take 8 (4
 * row pairs), the batched form's persistent kernel fewer, as its
 * occupancy hides the latency instead.  Cell rule and border copies as the reference kernel
 * (HighMap/src/gpu_opencl/kernels/thermal.cl:26-100, Jacobi form; border
 * copies _common_index.cl:106-132).
 */
#ifndef HM_THERMAL_SWEEP_CUH
#define HM_THERMAL_SWEEP_CUH

#include "hm_thermal_math.cuh"

namespace hm
{

constexpr int SW_P = 8; /* rows whose loads are issued together */

/* Cell rules of the sweeps: R::cell(c, w, s, n, e, nw, sw, ne, se, talus,
 * extra, first, param) is the new value of an interior cell from its 3 x 3
 * neighbourhood (named by position: w = (i-1, j), s = (i, j+1), n =
 * (i, j-1), ...), its talus, the value of the optional per-cell grid
 * `extra` (R::EXTRA), the first-step flag and a scalar parameter. */
template <int BED>
struct TalusExchange
{
  static constexpr bool EXTRA = BED != BED_NONE;
  __device__ static __forceinline__ float cell(float c, float w, float s, float n, float e, float nw, float sw,
                                               float ne, float se, float t, float x, bool first, float)
  {
    return thermal_cell<BED>(c, w, s, n, e, nw, sw, ne, se, t, x, first);
  }
};

/* Columns wx .. wx+31 (lane = column; columns past nx only feed the
 * shuffles), output rows y0 .. y1-1, the loads of P rows in flight
 * together.  The whole warp must call it. */
template <bool TMAP, class R, int P = SW_P>
__device__ __forceinline__ void thermal_sweep_warp(const float *__restrict__ a,
                                                   float *__restrict__ b,
                                                   int nx,
                                                   int ny,
                                                   const float *__restrict__ talus,
                                                   float talus_value,
                                                   const float *__restrict__ bedrock,
                                                   int first,
                                                   int wx,
                                                   int y0,
                                                   int y1,
                                                   float param = 0.f)
{
  const int  lane = threadIdx.x & 31;
  const int  gx = wx + lane;
  const bool live = gx < nx;
  const int  gxc = live ? gx : nx - 1;
  /* lanes 0 and 31 also load the column west / east of the warp */
  const int  hx = lane == 0 ? max(wx - 1, 0) : (lane == 31 ? min(wx + 32, nx - 1) : gxc);

  float vc[P + 2], vl[P + 2], vr[P + 2];
  {
    const float *r0 = a + (size_t)max(y0 - 1, 0) * nx, *r1 = a + (size_t)y0 * nx;
    vc[0] = __ldg(r0 + gxc);
    vl[0] = __ldg(r0 + hx);
    vc[1] = __ldg(r1 + gxc);
    vl[1] = __ldg(r1 + hx);
#pragma unroll
    for (int q = 0; q < 2; q++)
    {
      const float up = __shfl_up_sync(0xffffffffu, vc[q], 1), dn = __shfl_down_sync(0xffffffffu, vc[q], 1);
      vr[q] = lane == 31 ? vl[q] : dn;
      vl[q] = lane == 0 ? vl[q] : up;
    }
  }
  for (int j0 = y0; j0 < y1; j0 += P)
  {
    float tl[P], bd[P];
#pragma unroll
    for (int q = 0; q < P; q++)
    {
      const float *r = a + (size_t)min(j0 + 1 + q, ny - 1) * nx;
      vc[q + 2] = __ldg(r + gxc);
      vl[q + 2] = __ldg(r + hx); /* the halo value until the shuffles below */
      const size_t o = (size_t)min(j0 + q, ny - 1) * nx + gxc;
      tl[q] = TMAP ? __ldg(talus + o) : talus_value;
      bd[q] = R::EXTRA ? __ldg(bedrock + o) : 0.f;
    }
#pragma unroll
    for (int q = 2; q < P + 2; q++)
    {
      const float up = __shfl_up_sync(0xffffffffu, vc[q], 1), dn = __shfl_down_sync(0xffffffffu, vc[q], 1);
      vr[q] = lane == 31 ? vl[q] : dn;
      vl[q] = lane == 0 ? vl[q] : up;
    }
#pragma unroll
    for (int q = 0; q < P; q++)
    {
      const int j = j0 + q;
      if (!live || j >= y1) continue;
      float out;
      /* apply_boundaries, _common_index.cl:106-132 */
      if (gx == 0) out = vr[q + 1];
      else if (gx == nx - 1) out = vl[q + 1];
      else if (j == 0) out = vc[q + 2];
      else if (j == ny - 1) out = vc[q];
      else
        out = R::cell(vc[q + 1], vl[q + 1], vc[q + 2], vc[q], vr[q + 1], vl[q], vl[q + 2], vr[q], vr[q + 2], tl[q],
                      bd[q], first != 0, param);
      b[(size_t)j * nx + gx] = out;
    }
    vc[0] = vc[P];
    vl[0] = vl[P];
    vr[0] = vr[P];
    vc[1] = vc[P + 1];
    vl[1] = vl[P + 1];
    vr[1] = vr[P + 1];
  }
}


/* The same sweep with two adjacent columns per lane (a warp owns the 64
 * columns wx .. wx+63): z, talus and bedrock move as 8-byte pairs, and one
 * pair of shuffles per row serves both cells, which halves the per-cell
 * load, shuffle and address work.  Needs an even nx and 8-byte aligned
 * grids; identical bits to thermal_sweep_warp. */
constexpr int S2_P = 4; /* rows whose loads are issued together */

template <bool TMAP, class R, int P = S2_P>
__device__ __forceinline__ void thermal_sweep2_warp(const float *__restrict__ a,
                                                    float *__restrict__ b,
                                                    int nx,
                                                    int ny,
                                                    const float *__restrict__ talus,
                                                    float talus_value,
                                                    const float *__restrict__ bedrock,
                                                    int first,
                                                    int wx,
                                                    int y0,
                                                    int y1,
                                                    float param = 0.f)
{
  const int  lane = threadIdx.x & 31;
  const int  gx = wx + 2 * lane; /* first of the lane's two columns (nx is even) */
  const bool live = gx < nx;
  const int  gxc = live ? gx : nx - 2;
  /* lanes 0 and 31 also load the column west / east of the warp */
  const int  hx = lane == 0 ? max(wx - 1, 0) : (lane == 31 ? min(wx + 64, nx - 1) : gxc);

  /* per row: the pair (x, y), the west neighbour of x and the east one of y */
  float vx[P + 2], vy[P + 2], vw[P + 2], ve[P + 2];
  const bool halo_lane = lane == 0 || lane == 31;
  auto load = [&](int r, int q) {
    const float *row = a + (size_t)r * nx;
    const float2 t = __ldg(reinterpret_cast<const float2 *>(row + gxc));
    vx[q] = t.x;
    vy[q] = t.y;
    /* the halo value until the shuffles; only the edge lanes keep theirs */
    vw[q] = halo_lane ? __ldg(row + hx) : 0.f;
  };
  auto exchange = [&](int q) {
    const float up = __shfl_up_sync(0xffffffffu, vy[q], 1), dn = __shfl_down_sync(0xffffffffu, vx[q], 1);
    ve[q] = lane == 31 ? vw[q] : dn;
    vw[q] = lane == 0 ? vw[q] : up;
  };
  load(max(y0 - 1, 0), 0);
  load(y0, 1);
  exchange(0);
  exchange(1);
  for (int j0 = y0; j0 < y1; j0 += P)
  {
    float2 tl[P], bd[P];
#pragma unroll
    for (int q = 0; q < P; q++)
    {
      load(min(j0 + 1 + q, ny - 1), q + 2);
      const size_t o = (size_t)min(j0 + q, ny - 1) * nx + gxc;
      tl[q] = TMAP ? __ldg(reinterpret_cast<const float2 *>(talus + o)) : make_float2(talus_value, talus_value);
      bd[q] = R::EXTRA ? __ldg(reinterpret_cast<const float2 *>(bedrock + o)) : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int q = 2; q < P + 2; q++) exchange(q);
    /* a warp whose columns and rows are all interior: no border tests
     * (10 % of the step at 4096^2) */
    if (wx > 0 && wx + 64 < nx && j0 > 0 && j0 + P < ny - 1 && j0 + P <= y1)
    {
#pragma unroll
      for (int q = 0; q < P; q++)
      {
        float2 out;
        out.x = R::cell(vx[q + 1], vw[q + 1], vx[q + 2], vx[q], vy[q + 1], vw[q], vw[q + 2], vy[q], vy[q + 2],
                        tl[q].x, bd[q].x, first != 0, param);
        out.y = R::cell(vy[q + 1], vx[q + 1], vy[q + 2], vy[q], ve[q + 1], vx[q], vx[q + 2], ve[q], ve[q + 2],
                        tl[q].y, bd[q].y, first != 0, param);
        *reinterpret_cast<float2 *>(b + (size_t)(j0 + q) * nx + gx) = out;
      }
    }
    else
    {
#pragma unroll
      for (int q = 0; q < P; q++)
      {
        const int j = j0 + q;
        if (!live || j >= y1) continue;
        float2 out;
        /* apply_boundaries, _common_index.cl:106-132, for each of the two cells */
        if (gx == 0) out.x = vy[q + 1];
        else if (j == 0) out.x = vx[q + 2];
        else if (j == ny - 1) out.x = vx[q];
        else
          out.x = R::cell(vx[q + 1], vw[q + 1], vx[q + 2], vx[q], vy[q + 1], vw[q], vw[q + 2], vy[q], vy[q + 2],
                          tl[q].x, bd[q].x, first != 0, param);
        if (gx + 1 == nx - 1) out.y = vx[q + 1];
        else if (j == 0) out.y = vy[q + 2];
        else if (j == ny - 1) out.y = vy[q];
        else
          out.y = R::cell(vy[q + 1], vx[q + 1], vy[q + 2], vy[q], ve[q + 1], vx[q], vx[q + 2], ve[q], ve[q + 2],
                          tl[q].y, bd[q].y, first != 0, param);
        *reinterpret_cast<float2 *>(b + (size_t)j * nx + gx) = out;
      }
    }
    vx[0] = vx[P];
    vy[0] = vy[P];
    vw[0] = vw[P];
    ve[0] = ve[P];
    vx[1] = vx[P + 1];
    vy[1] = vy[P + 1];
    vw[1] = vw[P + 1];
    ve[1] = ve[P + 1];
  }
}

} // namespace hm

#endif
