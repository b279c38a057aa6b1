/*
 * abi_example.c - a plain C11 caller of include/hm_erosion.h: the C-ABI
 * compiles as C (no C++ in the header) and links against libhm_erosion.so
 * (built and linked by tests/test_lib.py; run, it needs a CUDA device).
 */
#include <stdio.h>
#include <stdlib.h>

#include "hm_erosion.h"

int main(void)
{
  const int nx = 64, ny = 48;
  float    *z = calloc((size_t)nx * ny, sizeof(float));
  float    *depo = calloc((size_t)nx * ny, sizeof(float));
  if (!z || !depo) return 2;
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) z[j * nx + i] = (float)((i * 7 + j * 13) % 17) / 17.f;
  if (hm_init() != HM_OK)
  {
    printf("no device: %s\n", hm_last_error());
    return 3;
  }
  hm_context *ctx = NULL;
  int         st = hm_context_create(&ctx, 0);
  if (!st) st = hm_thermal_scalar(ctx, z, nx, ny, 1.f / nx, 20, NULL, depo, NULL);
  hm_vpipes_params p;
  hm_vpipes_default_params(&p);
  p.iterations = 5;
  if (!st) st = hm_vpipes(ctx, z, nx, ny, &p, NULL, NULL, NULL, NULL, NULL);
  if (!st) st = hm_sediment_layer(ctx, z, nx, ny, depo, depo, 4, 1, NULL);
  if (!st) st = hm_thermal_rib(ctx, z, nx, ny, 2, NULL);
  printf("%s\n", st ? hm_status_string(st) : "ok");
  hm_context_destroy(ctx);
  free(z);
  free(depo);
  return st ? 1 : 0;
}
