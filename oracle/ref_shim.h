/*
 * ref_shim.h - just enough OpenCL C for the reference's thermal and
 * virtual-pipes kernel text to compile as C++ on the host.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/build_oracle.py feeds the kernel files
 * (HighMap/src/gpu_opencl/kernels/_common_index.cl, thermal.cl,
 * hydraulic_vpipes.cl) straight from the reference tree through the
 * compiler with this header in front; the compiled object lands in
 * oracle/_ref/ and is used only to pin the oracle.
 *
 * Two mechanical source rewrites are applied on the way in (OpenCL vector
 * literals have no C++ spelling): "(int2)(" -> "HM_INT2(" and
 * "(float2)(" -> "HM_FLOAT2(".  The raw-string wrapper lines R""( and )""
 * are dropped.
 *
 * Image emulation: an image is a plain float grid.  The nearest sampler
 * clamps to the edge (CLK_ADDRESS_CLAMP_TO_EDGE | CLK_FILTER_NEAREST).  The
 * linear sampler with CLK_ADDRESS_MIRRORED_REPEAT on unnormalised
 * coordinates is implementation-defined in OpenCL; it is defined here, and
 * identically in the oracle, as the normalised-coordinate rule of the
 * OpenCL specification expressed in texel units (mirror with period
 * 2 * size, texel centres at k + 0.5, indices clamped), with full fp32
 * weights.
 */
#ifndef HM_REF_SHIM_H
#define HM_REF_SHIM_H

#include <cfloat>
#include <cmath>

#define kernel
#define global
#define read_only
#define write_only

#define CLK_NORMALIZED_COORDS_FALSE 0
#define CLK_ADDRESS_CLAMP_TO_EDGE 2
#define CLK_ADDRESS_MIRRORED_REPEAT 4
#define CLK_FILTER_NEAREST 0
#define CLK_FILTER_LINEAR 16

namespace hmref
{

struct int2
{
  int x, y;
};
struct float2
{
  float x, y;
};
struct float4
{
  float x, y, z, w;
};

inline int2   HM_INT2(int a, int b) { return int2{a, b}; }
inline float2 HM_FLOAT2(float a, float b) { return float2{a, b}; }

/* work-item id, set by the harness before each kernel call */
extern thread_local int g_gid0;
extern thread_local int g_gid1;
inline int get_global_id(int d) { return d == 0 ? g_gid0 : g_gid1; }

/* OpenCL built-ins used by the kernels */
inline float max(float a, float b) { return std::fmax(a, b); }
inline float min(float a, float b) { return std::fmin(a, b); }
inline int   max(int a, int b) { return a > b ? a : b; }
inline int   min(int a, int b) { return a < b ? a : b; }
inline float clamp(float x, float lo, float hi) { return std::fmin(std::fmax(x, lo), hi); }
inline int   clamp(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }
using std::fabs;
using std::floor;
using std::hypot;
using std::pow;

typedef int      sampler_t;
typedef unsigned uint;

struct hm_image
{
  float *data;
  int    w, h;
};
typedef hm_image *image2d_t;

inline float4 read_imagef(image2d_t img, sampler_t, int2 c)
{
  int i = clamp(c.x, 0, img->w - 1);
  int j = clamp(c.y, 0, img->h - 1);
  float v = img->data[(long)j * img->w + i];
  return float4{v, 0.f, 0.f, 1.f};
}

inline float hm_mirror(float x, int n)
{
  float period = (float)(2 * n);
  float r = std::rint(x / period);
  return std::fabs(x - period * r);
}

inline float4 read_imagef(image2d_t img, sampler_t, float2 c)
{
  const int nx = img->w, ny = img->h;
  float     xm = hm_mirror(c.x, nx) - 0.5f;
  float     ym = hm_mirror(c.y, ny) - 0.5f;
  float     fx = std::floor(xm), fy = std::floor(ym);
  float     a = xm - fx, b = ym - fy;
  float     fxc = std::fmin(std::fmax(fx, -1.f), (float)(nx - 1));
  float     fyc = std::fmin(std::fmax(fy, -1.f), (float)(ny - 1));
  int       i0 = (int)fxc, j0 = (int)fyc;
  int       i1 = i0 + 1, j1 = j0 + 1;
  i0 = i0 < 0 ? 0 : i0;
  j0 = j0 < 0 ? 0 : j0;
  i1 = i1 > nx - 1 ? nx - 1 : i1;
  j1 = j1 > ny - 1 ? ny - 1 : j1;
  const float *s = img->data;
  float v = (1.f - a) * (1.f - b) * s[(long)j0 * nx + i0] + a * (1.f - b) * s[(long)j0 * nx + i1] +
            (1.f - a) * b * s[(long)j1 * nx + i0] + a * b * s[(long)j1 * nx + i1];
  return float4{v, 0.f, 0.f, 1.f};
}

inline void write_imagef(image2d_t img, int2 c, float v) { img->data[(long)c.y * img->w + c.x] = v; }

} // namespace hmref

#endif
