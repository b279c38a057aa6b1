/*
 * hm_oracle.c - CPU oracle for the thermal and virtual-pipes erosion
 * solvers.  TEST INFRASTRUCTURE ONLY: see hm_oracle.h for the scope, the
 * reference lines each function restates and how the oracle is pinned.
 *
 * Built with -O2 -ffp-contract=off -fopenmp so that every float operation
 * rounds exactly once, as in the reference's kernel text.
 */
#include "hm_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* float instance */
#define REAL float
#define K(x) ((float)(x))
#define FN(name) name##_f32
#define HYPOT hypotf
#define POW powf
#define RINT rintf
#define FABS fabsf
#define SQRT sqrtf
#define FLOOR floorf
#define FMIN fminf
#define FMAX fmaxf
#include "hm_oracle_body.inc"
#undef REAL
#undef K
#undef FN
#undef HYPOT
#undef POW
#undef RINT
#undef FABS
#undef SQRT
#undef FLOOR
#undef FMIN
#undef FMAX

/* double instance: the same scheme in FP64 (the "FP64 CPU run") */
#define REAL double
#define K(x) ((double)(x))
#define FN(name) name##_f64
#define HYPOT hypot
#define POW pow
#define RINT rint
#define FABS fabs
#define SQRT sqrt
#define FLOOR floor
#define FMIN fmin
#define FMAX fmax
#include "hm_oracle_body.inc"
#undef REAL
#undef K
#undef FN
#undef HYPOT
#undef POW
#undef RINT
#undef FABS
#undef SQRT
#undef FLOOR
#undef FMIN
#undef FMAX

float hmo_sample_linear_mirror_f32(const float *s, int nx, int ny, float x, float y)
{
  return sample_linear_mirror_f32(s, nx, ny, x, y);
}

void hmo_vpipes_default_params(hmo_vpipes_params *p)
{
  /* defaults of erosion.hpp:1206-1223 */
  p->water_height = 1e-2f;
  p->maintain_water_volume = 1;
  p->evap_rate = 0.1f;
  p->iterations = 50;
  p->dt = 0.5f;
  p->k_capacity = 0.5f;
  p->k_erode = 0.001f;
  p->k_depose = 0.01f;
  p->k_discharge_exp = 1.f;
  p->downcutting_max_depth_ratio = 10.f;
  p->flux_diffusion = 1;
  p->flux_diffusion_strength = 0.01f;
  p->gravity = 1.f;
  p->pipe_length = 1.f;
  p->pipe_area = 1.f;
  p->rain_per_step = 0.f;
  p->initial_water = -1.f;
}

/* thermal_auto_bedrock, thermal.cl:102-145 driven as thermal_gpu.cpp:98-130
 * (Jacobi form).  The bedrock buffer starts at zero (Array(shape)) and the
 * kernel sets interior cells to -FLT_MAX on iteration 0. */
int hmo_thermal_auto_bedrock_f32(float       *z,
                                 int          nx,
                                 int          ny,
                                 const float *talus,
                                 int          iterations,
                                 float       *deposition_map)
{
  static const int di[8] = {-1, 0, 0, 1, -1, -1, 1, 1};
  static const int dj[8] = {0, 1, -1, 0, -1, 1, -1, 1};
  static const float c[8] = {1.f, 1.f, 1.f, 1.f, 1.414f, 1.414f, 1.414f, 1.414f};
  if (!z || !talus || nx < 3 || ny < 3 || iterations < 0) return 1;
  size_t n = (size_t)nx * (size_t)ny;
  float *z0 = (float *)malloc(n * sizeof(float));
  float *a = (float *)malloc(n * sizeof(float));
  float *b = (float *)malloc(n * sizeof(float));
  float *bed = (float *)calloc(n, sizeof(float));
  if (!z0 || !a || !b || !bed)
  {
    free(z0); free(a); free(b); free(bed);
    return 2;
  }
  memcpy(z0, z, n * sizeof(float));
  memcpy(a, z, n * sizeof(float));
  for (int it = 0; it < iterations; it++)
  {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
      {
        size_t idx = (size_t)j * nx + i;
        if (i == 0) { b[idx] = a[(size_t)j * nx + 1]; continue; }
        if (i == nx - 1) { b[idx] = a[(size_t)j * nx + nx - 2]; continue; }
        if (j == 0) { b[idx] = a[(size_t)1 * nx + i]; continue; }
        if (j == ny - 1) { b[idx] = a[(size_t)(ny - 2) * nx + i]; continue; }
        if (it == 0) bed[idx] = -FLT_MAX;
        float val = a[idx];
        float zb = bed[idx];
        b[idx] = val;
        if (val >= zb)
        {
          float z_init = z0[idx];
          float amount = 0.f;
          for (int k = 0; k < 8; k++)
            amount += thermal_exchange_f32(val, a[(size_t)(j + dj[k]) * nx + i + di[k]], c[k], talus[idx]);
          float zn = val + amount;
          zn = zn > z_init ? zn : z_init;
          zn = zn > zb ? zn : zb;
          b[idx] = zn;
          bed[idx] = z_init > zn ? z_init : zn;
        }
      }
    float *t = a;
    a = b;
    b = t;
  }
  extrapolate_borders_f32(a, nx, ny);
  if (deposition_map)
    for (size_t k = 0; k < n; k++)
    {
      float dz = a[k] - z0[k];
      deposition_map[k] = dz > 0.f ? dz : 0.f;
    }
  memcpy(z, a, n * sizeof(float));
  free(z0); free(a); free(b); free(bed);
  return 0;
}

int hmo_num_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
