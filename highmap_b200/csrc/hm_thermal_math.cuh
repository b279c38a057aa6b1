/*
 * hm_thermal_math.cuh - the talus exchange of one cell, bit-exact with the
 * reference's fp32 arithmetic.
 *
 * Reference: helper_thermal_exchange and the neighbour loop of
 * HighMap/src/gpu_opencl/kernels/thermal.cl:5-24,41-57 (neighbour order
 * HMAP_DI / HMAP_DJ, HighMap/include/highmap/erosion.hpp:21-22; distance
 * 1 for the four axial neighbours and 1.414 for the diagonals; rate 0.2).
 *
 * Every operation is an explicitly rounded intrinsic so the compiler cannot
 * contract a multiply into a following add: the result equals the
 * reference evaluated one rounding per operation.  The reference's
 * branches are folded:  with n = other - self,
 *     x = max(|n| - dist * talus, 0),   e = (0.2 * x) / dist,
 *     contribution = copysign(e, n),
 * which is the reference's value for every finite input (n = +0 gives
 * +e, as the reference's `else` branch does).
 *
 * Division by the diagonal distance 1.414f uses Markstein's correction of
 * the product by the correctly rounded reciprocal (P. Markstein, "Computation
 * of elementary functions on the IBM RISC System/6000 processor", IBM J.
 * Res. Dev. 34(1), 1990):  q = x * RN(1/b), r = fma(-q, b, x),
 * q' = fma(r, RN(1/b), q).  q' equals the correctly rounded x / 1.414f for
 * every normal x with a normal quotient (checked exhaustively over all
 * float mantissas; the identity is exponent independent).
 */
#ifndef HM_THERMAL_MATH_CUH
#define HM_THERMAL_MATH_CUH

#include <cfloat>

namespace hm
{

__device__ __forceinline__ float div_by_diag(float x)
{
  const float b = 1.414f;
  const float y = 0x1.6a17e6p-1f; /* RN(1 / 1.414f) */
  float       q = __fmul_rn(x, y);
  float       r = __fmaf_rn(-q, b, x);
  return __fmaf_rn(r, y, q);
}

__device__ __forceinline__ float exch_axial(float self, float other, float talus)
{
  float n = __fsub_rn(other, self);
  float x = fmaxf(__fsub_rn(fabsf(n), talus), 0.f);
  return copysignf(__fmul_rn(0.2f, x), n);
}

__device__ __forceinline__ float exch_diag(float self, float other, float max_dif_diag)
{
  float n = __fsub_rn(other, self);
  float x = fmaxf(__fsub_rn(fabsf(n), max_dif_diag), 0.f);
  return copysignf(div_by_diag(__fmul_rn(0.2f, x)), n);
}

/* Sum of the eight exchanges in reference order:
 * (-1,0) (0,+1) (0,-1) (+1,0) (-1,-1) (-1,+1) (+1,-1) (+1,+1)
 * with (di, dj) = (x offset, y offset).  Arguments are named by position:
 * w = (i-1, j), e = (i+1, j), n = (i, j-1), s = (i, j+1), nw = (i-1, j-1) ... */
__device__ __forceinline__ float thermal_amount(float c,
                                                float w,
                                                float s,
                                                float n,
                                                float e,
                                                float nw,
                                                float sw,
                                                float ne,
                                                float se,
                                                float talus)
{
  const float md = __fmul_rn(1.414f, talus);
  float       a = exch_axial(c, w, talus);
  a = __fadd_rn(a, exch_axial(c, s, talus));
  a = __fadd_rn(a, exch_axial(c, n, talus));
  a = __fadd_rn(a, exch_axial(c, e, talus));
  a = __fadd_rn(a, exch_diag(c, nw, md));
  a = __fadd_rn(a, exch_diag(c, sw, md));
  a = __fadd_rn(a, exch_diag(c, ne, md));
  a = __fadd_rn(a, exch_diag(c, se, md));
  return a;
}

/* Bedrock modes of the kernel templates */
enum BedMode
{
  BED_NONE = 0,
  BED_INTENDED = 1,
  BED_LITERAL = 2,
  BED_AUTO = 3
};

/* New value of an interior cell.  BED_INTENDED: max(val + amount, bedrock)
 * when val >= bedrock, else bedrock.  BED_LITERAL: max(val, bedrock), the
 * value thermal.cl:99 leaves.
 *
 * BED_AUTO is thermal_auto_bedrock (thermal.cl:102-145) with `bedrock` =
 * z0, the heights the solve started from, and `first` set on the first
 * step.  The reference keeps a bedrock grid: -FLT_MAX before the first
 * step, then max(z0, z_new) after every update, where
 * z_new = max(max(val + amount, z0), bedrock) is never below z0 (the
 * selects return z0 when val + amount is NaN).  So after a step the grid
 * holds exactly the new value, every later step finds bedrock == val and
 * passes the gate val >= bedrock, and the grid need not exist: the gate
 * becomes z0 >= -FLT_MAX (false only for cells that start NaN or -inf,
 * which then never change) and the last max takes -FLT_MAX on the first
 * step and val afterwards. */
template <int BED>
__device__ __forceinline__ float thermal_cell(float c,
                                              float w,
                                              float s,
                                              float n,
                                              float e,
                                              float nw,
                                              float sw,
                                              float ne,
                                              float se,
                                              float talus,
                                              float bedrock,
                                              bool  first = false)
{
  if (BED == BED_LITERAL) return c > bedrock ? c : bedrock;
  if (BED == BED_AUTO)
  {
    if (!(bedrock >= -FLT_MAX)) return c;
    const float x = __fadd_rn(c, thermal_amount(c, w, s, n, e, nw, sw, ne, se, talus));
    const float zn = x > bedrock ? x : bedrock;
    const float fl = first ? -FLT_MAX : c;
    return zn > fl ? zn : fl;
  }
  float out = c;
  if (BED == BED_NONE || c >= bedrock)
    out = __fadd_rn(c, thermal_amount(c, w, s, n, e, nw, sw, ne, se, talus));
  if (BED == BED_INTENDED) out = out > bedrock ? out : bedrock;
  return out;
}

} // namespace hm

#endif
