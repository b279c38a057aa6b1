/*
 * ref_harness.cpp - host driver around the reference's own kernel text
 * compiled for the CPU (see ref_shim.h and build_oracle.py).
 *
 * TEST INFRASTRUCTURE ONLY: pins the oracle and serves as the timed CPU
 * baseline of the benchmark's reference arm.  Built into oracle/_ref/.
 *
 * The host drivers of the reference (thermal_gpu.cpp, hydraulic_vpipes_gpu.cpp)
 * need glm and the absent CLWrapper submodule, so their loops are restated
 * here around the compiled kernels:
 *   ref_thermal    : HighMap/src/erosion/thermal_gpu.cpp:17-96
 *   ref_thermal_auto_bedrock : thermal_gpu.cpp:98-130
 *   ref_vpipes     : HighMap/src/erosion/hydraulic_vpipes_gpu.cpp:15-178
 *   ref_flow_simulation : HighMap/src/hydrology/flow_simulation.cpp:26-110
 *   ref_thermal_sibling : HighMap/src/erosion/thermal_gpu.cpp:221-396
 *   ref_sediment_deposition : HighMap/src/erosion/deposition.cpp:19-66
 *   ref_sediment_layer : HighMap/src/erosion/deposition.cpp:68-113 (with
 *                        gradient.cpp:217-243 and filters.cpp:290-324)
 *   ref_snow_post_filter : HighMap/src/hydrology/snow_simulation.cpp:140-152
 *   ref_thermal_relief : HighMap/src/erosion/thermal_gpu.cpp:154-219,249-272
 *   ref_flow_simulation_viscous : HighMap/src/hydrology/flow_simulation.cpp:112-157
 *
 * Work-items run as a host loop (OpenMP over rows).  The in-place thermal
 * kernels are given a private copy of the three rows around the work-item,
 * restored after each call, so every work-item reads step t and the result
 * is the Jacobi (deterministic) form of the racing in-place update.
 */
#include <algorithm>
#include <cfloat>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "hm_oracle.h"
#include "ref_shim.h"

namespace hmref
{
thread_local int g_gid0 = 0;
thread_local int g_gid1 = 0;

/* compiled from the reference's kernel text (ref_kernels.o) */
void thermal(float *z, const float *talus, const int nx, const int ny, const int it);
void thermal_with_bedrock(float       *z,
                          const float *talus,
                          const float *bedrock,
                          const int    nx,
                          const int    ny,
                          const int    it);
void thermal_auto_bedrock(float       *z,
                          const float *talus,
                          float       *bedrock,
                          const float *z0,
                          const int    nx,
                          const int    ny,
                          const int    it);
void thermal_ridge(float *z, const float *talus, const int nx, const int ny);
void thermal_scree(float *z, const float *talus, const float *zmax, const int nx, const int ny);
void thermal_schott(float *z, const float *talus, const int nx, const int ny, const float intensity);
void thermal_olsen(float *z, const float *talus, const int nx, const int ny);
void thermal_flatten(float       *z,
                     const float *talus,
                     const int    nx,
                     const int    ny,
                     const float  sigma_inf,
                     const float  sigma_sup);
void thermal_inflate(float *z, const float *talus, const int nx, const int ny);
void thermal_rib(float *z, const int nx, const int ny);
void shallow_viscous_flow(image2d_t, image2d_t, image2d_t, int, int, float, float, float);
void hydraulic_vpipes_flow_pass(image2d_t, image2d_t, image2d_t, image2d_t, image2d_t, image2d_t,
                                image2d_t, image2d_t, image2d_t, image2d_t, const int, const int,
                                const float, const int, const float);
void hydraulic_vpipes_water_pass(image2d_t, image2d_t, image2d_t, image2d_t, image2d_t, image2d_t,
                                 image2d_t, image2d_t, image2d_t, const int, const int, const float,
                                 const float);
void hydraulic_vpipes_erosion_pass(image2d_t, image2d_t, image2d_t, image2d_t, image2d_t, image2d_t,
                                   image2d_t, const int, const int, const float, const float,
                                   const float, const float, const float, const float);
void hydraulic_vpipes_sediment_transport_pass(image2d_t, image2d_t, image2d_t, image2d_t, const int,
                                              const int, const float);
} // namespace hmref

namespace
{

/* extrapolate_borders(z, nbuffer=1, sigma=0), boundary.cpp:19-41 */
void extrapolate_borders(float *z, int ni, int nj)
{
  auto at = [&](int i, int j) -> float & { return z[(long)j * ni + i]; };
  for (int j = 0; j < nj; j++)
  {
    at(0, j) = 2.f * at(1, j) - at(2, j);
    at(ni - 1, j) = 2.f * at(ni - 2, j) - at(ni - 3, j);
  }
  for (int i = 0; i < ni; i++)
  {
    at(i, 0) = 2.f * at(i, 1) - at(i, 2);
    at(i, nj - 1) = 2.f * at(i, nj - 2) - at(i, nj - 3);
  }
}

/* extrapolate_borders(z, nbuffer, sigma = 0), boundary.cpp:19-41 */
void extrapolate_borders_n(float *z, int ni, int nj, int nb)
{
  auto at = [&](int i, int j) -> float & { return z[(long)j * ni + i]; };
  for (int j = 0; j < nj; j++)
    for (int k = nb - 1; k > -1; k--)
    {
      at(k, j) = 2.f * at(k + 1, j) - at(k + 2, j);
      at(ni - 1 - k, j) = 2.f * at(ni - 2 - k, j) - at(ni - 3 - k, j);
    }
  for (int i = 0; i < ni; i++)
    for (int k = nb - 1; k > -1; k--)
    {
      at(i, k) = 2.f * at(i, k + 1) - at(i, k + 2);
      at(i, nj - 1 - k) = 2.f * at(i, nj - 2 - k) - at(i, nj - 3 - k);
    }
}

/* One launch of an in-place thermal kernel over the nx x ny NDRange,
 * Jacobi form: a is step t, b receives step t+1.  `launch(zw)` runs the
 * kernel for the current work-item with zw addressing the row window. */
template <class Launch>
void run_inplace(const float *a, float *b, float *bed, int nx, int ny, Launch launch, int R = 1)
{
  (void)bed;
#pragma omp parallel
  {
    /* rows j-R .. j+R; R = 1 for the 3 x 3 kernels, 3 for thermal_olsen
     * (radius-2 reads, border cells copied from 3 rows in) */
    std::vector<float> win((size_t)(2 * R + 1) * nx, NAN);
#pragma omp for schedule(static)
    for (int j = 0; j < ny; j++)
    {
      for (int r = -R; r <= R; r++)
        if (j + r >= 0 && j + r < ny)
          std::memcpy(&win[(size_t)(r + R) * nx], a + (size_t)(j + r) * nx, sizeof(float) * nx);
        else
          std::fill(win.begin() + (size_t)(r + R) * nx, win.begin() + (size_t)(r + R + 1) * nx, NAN);
      /* zw[(j + r) * nx + i] == win[(r + R) * nx + i] */
      float *zw = win.data() - ((ptrdiff_t)j - R) * (ptrdiff_t)nx;
      hmref::g_gid1 = j;
      for (int i = 0; i < nx; i++)
      {
        hmref::g_gid0 = i;
        launch(zw);
        b[(size_t)j * nx + i] = win[(size_t)R * nx + i];
        win[(size_t)R * nx + i] = a[(size_t)j * nx + i];
      }
    }
  }
}

} // namespace

extern "C" {

/* thermal_gpu.cpp:17-72 (and :74-86 when mask != NULL).  The bedrock
 * variant is the literal thermal_with_bedrock kernel. */
int ref_thermal(float       *z,
                int          nx,
                int          ny,
                const float *talus,
                int          iterations,
                const float *bedrock,
                float       *deposition_map,
                const float *mask)
{
  if (!z || !talus || nx < 3 || ny < 3 || iterations < 0) return 1;
  const size_t       n = (size_t)nx * ny;
  std::vector<float> z0(z, z + n), a(z, z + n), b(n);
  for (int it = 0; it < iterations; it++)
  {
    if (bedrock)
      run_inplace(a.data(), b.data(), nullptr, nx, ny, [&](float *zw)
                  { hmref::thermal_with_bedrock(zw, talus, bedrock, nx, ny, it); });
    else
      run_inplace(a.data(), b.data(), nullptr, nx, ny,
                  [&](float *zw) { hmref::thermal(zw, talus, nx, ny, it); });
    std::swap(a, b);
  }
  extrapolate_borders(a.data(), nx, ny);
  if (deposition_map)
    for (size_t k = 0; k < n; k++) deposition_map[k] = std::max(a[k] - z0[k], 0.f);
  if (mask)
    for (size_t k = 0; k < n; k++) z[k] = z0[k] * (1.f - mask[k]) + a[k] * mask[k];
  else
    std::memcpy(z, a.data(), n * sizeof(float));
  return 0;
}

/* thermal_gpu.cpp:98-130 */
int ref_thermal_auto_bedrock(float       *z,
                             int          nx,
                             int          ny,
                             const float *talus,
                             int          iterations,
                             float       *deposition_map)
{
  if (!z || !talus || nx < 3 || ny < 3 || iterations < 0) return 1;
  const size_t       n = (size_t)nx * ny;
  std::vector<float> z0(z, z + n), a(z, z + n), b(n), bed(n, 0.f);
  for (int it = 0; it < iterations; it++)
  {
    run_inplace(a.data(), b.data(), bed.data(), nx, ny, [&](float *zw)
                { hmref::thermal_auto_bedrock(zw, talus, bed.data(), z0.data(), nx, ny, it); });
    std::swap(a, b);
  }
  extrapolate_borders(a.data(), nx, ny);
  if (deposition_map)
    for (size_t k = 0; k < n; k++) deposition_map[k] = std::max(a[k] - z0[k], 0.f);
  std::memcpy(z, a.data(), n * sizeof(float));
  return 0;
}

/* deposition.cpp:19-66 over the reference's thermal kernel (ref_thermal) */
int ref_sediment_deposition(float       *z,
                            int          nx,
                            int          ny,
                            const float *talus,
                            float        max_deposition,
                            int          iterations,
                            int          thermal_subiterations,
                            float       *deposition_map,
                            const float *mask)
{
  if (!z || !talus || nx < 3 || ny < 3 || iterations < 0 || thermal_subiterations < 0) return 1;
  const size_t       n = (size_t)nx * ny;
  const float        step = max_deposition / (int)iterations;
  std::vector<float> smap(n, 0.f), ztot(n);
  for (int it = 0; it < iterations; it++)
  {
    for (size_t k = 0; k < n; k++) smap[k] = smap[k] + step;
    for (size_t k = 0; k < n; k++) ztot[k] = z[k] + smap[k];
    int rc = ref_thermal(ztot.data(), nx, ny, talus, thermal_subiterations, nullptr, nullptr, nullptr);
    if (rc) return rc;
    for (size_t k = 0; k < n; k++) smap[k] = std::max(ztot[k] - z[k], 0.f);
  }
  for (size_t k = 0; k < n; k++)
  {
    const float zf = z[k] + smap[k];
    z[k] = mask ? z[k] * (1.f - mask[k]) + zf * mask[k] : zf;
    if (deposition_map) deposition_map[k] = smap[k];
  }
  return 0;
}

/* deposition.cpp:68-113 over the reference's thermal kernel: the talus
 * preparation from gradient_talus (gradient.cpp:217-243, in-place pair
 * sweeps from zero), ref_thermal with a deposition map, and the post
 * filter (z = input + deposition; hmap::laplace with its defaults sigma
 * 0.125 and 3 steps, filters.cpp:290-324, on the mask, then on a copy of z
 * blended in by that mask) */
int ref_sediment_layer(float       *z,
                       int          nx,
                       int          ny,
                       const float *talus_layer,
                       const float *talus_upper_limit,
                       int          iterations,
                       int          apply_post_filter,
                       float       *deposition_map)
{
  if (!z || !talus_layer || !talus_upper_limit || nx < 3 || ny < 3 || iterations < 0) return 1;
  const size_t       n = (size_t)nx * ny;
  auto               at = [nx](int i, int j) { return (size_t)j * nx + i; };
  std::vector<float> zb(z, z + n), g(n, 0.f), tr(talus_layer, talus_layer + n), fm(n, 1.f), map(n);
  for (int j = 0; j < ny; j++)
    for (int i = 1; i < nx - 1; i += 2)
    {
      const float d = std::abs(z[at(i, j)] - z[at(i + 1, j)]);
      g[at(i, j)] = std::max(g[at(i, j)], d);
      g[at(i - 1, j)] = std::max(g[at(i - 1, j)], g[at(i, j)]);
      g[at(i + 1, j)] = d;
    }
  for (int j = 1; j < ny - 1; j += 2)
    for (int i = 0; i < nx; i++)
    {
      const float d = std::abs(z[at(i, j)] - z[at(i, j + 1)]);
      g[at(i, j)] = std::max(g[at(i, j)], d);
      g[at(i, j - 1)] = std::max(g[at(i, j - 1)], g[at(i, j)]);
      g[at(i, j + 1)] = d;
    }
  for (size_t k = 0; k < n; k++)
    if (g[k] > talus_upper_limit[k])
    {
      fm[k] = 0.f;
      tr[k] = 4.f * (g[k] - talus_upper_limit[k]) + talus_upper_limit[k];
    }
  int rc = ref_thermal(z, nx, ny, tr.data(), iterations, nullptr, map.data(), nullptr);
  if (rc) return rc;
  if (apply_post_filter)
  {
    auto laplace = [&](std::vector<float> &a) {
      std::vector<float> delta(n);
      for (int it = 0; it < 3; it++)
      {
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < nx; i++)
          {
            float sum = 0.f;
            for (int dj = -1; dj <= 1; dj++)
              for (int di = -1; di <= 1; di++)
                if (di != 0 || dj != 0) sum += a[at(std::clamp(i + di, 0, nx - 1), std::clamp(j + dj, 0, ny - 1))];
            delta[at(i, j)] = sum - 8.f * a[at(i, j)];
          }
        for (size_t k = 0; k < n; k++) a[k] += 0.125f * delta[k];
      }
    };
    for (size_t k = 0; k < n; k++) z[k] = zb[k] + map[k];
    laplace(fm);
    std::vector<float> zs(z, z + n);
    laplace(zs);
    for (size_t k = 0; k < n; k++) z[k] = z[k] * (1.f - fm[k]) + zs[k] * fm[k];
  }
  if (deposition_map) std::memcpy(deposition_map, map.data(), n * sizeof(float));
  return 0;
}

/* snow_simulation.cpp:140-152 and its clamp_min(s, 0) over the
 * reference's thermal kernel: mask = clamp_max_smooth(s / snow_depth, 1)
 * (range.cpp:98-110, k = 0.2), z_w = z + s, talus = ratio *
 * gradient_norm(z_w) (gradient.cpp:124-135, 182-215; math.cpp:142-151),
 * masked thermal on z_w, s = max(z_w - z, 0) */
int ref_snow_post_filter(const float *z,
                         float       *s,
                         int          nx,
                         int          ny,
                         float        snow_depth,
                         int          iterations,
                         float        thermal_talus_ratio)
{
  if (!z || !s || nx < 3 || ny < 3 || iterations < 0) return 1;
  const size_t       n = (size_t)nx * ny;
  auto               at = [nx](int i, int j) { return (size_t)j * nx + i; };
  std::vector<float> mask(n), zw(n), dx(n), dy(n), talus(n);
  for (size_t k = 0; k < n; k++)
  {
    const float x = s[k] / snow_depth, kk = 0.2f, vmax = 1.f;
    const float h = std::max(kk - std::abs(x - vmax), 0.f) / kk;
    mask[k] = std::min(x, vmax) - h * h * h * kk / 6.f;
    zw[k] = z[k] + s[k];
  }
  for (int j = 0; j < ny; j++)
  {
    for (int i = 1; i < nx - 1; i++) dx[at(i, j)] = 0.5f * (zw[at(i + 1, j)] - zw[at(i - 1, j)]);
    dx[at(0, j)] = zw[at(1, j)] - zw[at(0, j)];
    dx[at(nx - 1, j)] = zw[at(nx - 1, j)] - zw[at(nx - 2, j)];
  }
  for (int j = 1; j < ny - 1; j++)
    for (int i = 0; i < nx; i++) dy[at(i, j)] = 0.5f * (zw[at(i, j + 1)] - zw[at(i, j - 1)]);
  for (int i = 0; i < nx; i++)
  {
    dy[at(i, 0)] = zw[at(i, 1)] - zw[at(i, 0)];
    dy[at(i, ny - 1)] = zw[at(i, ny - 1)] - zw[at(i, ny - 2)];
  }
  for (size_t k = 0; k < n; k++) talus[k] = thermal_talus_ratio * std::sqrt(dx[k] * dx[k] + dy[k] * dy[k]);
  int rc = ref_thermal(zw.data(), nx, ny, talus.data(), iterations, nullptr, nullptr, mask.data());
  if (rc) return rc;
  for (size_t k = 0; k < n; k++)
  {
    const float d = zw[k] - z[k];
    s[k] = d > 0.f ? d : 0.f;
  }
  return 0;
}

/* thermal_gpu.cpp:221-396: thermal_ridge / _scree / _schott / _olsen
 * (rule 0..3 as hmo_thermal_sibling), the masked overloads via
 * apply_with_mask */
int ref_thermal_sibling(int          rule,
                        float       *z,
                        int          nx,
                        int          ny,
                        const float *talus,
                        const float *zmax,
                        float        intensity,
                        int          iterations,
                        float       *deposition_map,
                        const float *mask)
{
  if (!z || !talus || nx < 3 || ny < 3 || iterations < 0 || rule < 0 || rule > 3) return 1;
  if (rule == 1 && !zmax) return 1;
  if (rule == 3 && (nx < 7 || ny < 7)) return 1;
  const size_t       n = (size_t)nx * ny;
  std::vector<float> z0(z, z + n), a(z, z + n), b(n);
  for (int it = 0; it < iterations; it++)
  {
    switch (rule)
    {
    case 0: run_inplace(a.data(), b.data(), nullptr, nx, ny, [&](float *zw) { hmref::thermal_ridge(zw, talus, nx, ny); }); break;
    case 1:
      run_inplace(a.data(), b.data(), nullptr, nx, ny, [&](float *zw) { hmref::thermal_scree(zw, talus, zmax, nx, ny); });
      break;
    case 2:
      run_inplace(a.data(), b.data(), nullptr, nx, ny,
                  [&](float *zw) { hmref::thermal_schott(zw, talus, nx, ny, intensity); });
      break;
    default:
      run_inplace(a.data(), b.data(), nullptr, nx, ny, [&](float *zw) { hmref::thermal_olsen(zw, talus, nx, ny); }, 3);
    }
    std::swap(a, b);
  }
  extrapolate_borders(a.data(), nx, ny);
  if (deposition_map && rule != 3)
    for (size_t k = 0; k < n; k++)
      deposition_map[k] = rule == 1 ? std::max(a[k] - z0[k], 0.f) : std::abs(a[k] - z0[k]);
  if (mask)
    for (size_t k = 0; k < n; k++) z[k] = z0[k] * (1.f - mask[k]) + a[k] * mask[k];
  else
    std::memcpy(z, a.data(), n * sizeof(float));
  return 0;
}

/* hydraulic_vpipes_gpu.cpp:15-178.  Separate input and output images per
 * pass, as the driver binds them; Array::sum is the serial float
 * accumulate of methods.cpp:428-431.  The kernels hard-code gravity and
 * pipe length to 1, so p->gravity, p->pipe_length and p->pipe_area are
 * not used here; the driver-level extensions rain_per_step and
 * initial_water are. */
int ref_vpipes(float                   *z,
               int                      nx,
               int                      ny,
               const hmo_vpipes_params *p,
               const float             *rain_map,
               float                   *water_depth,
               float                   *sediment,
               float                   *vel_u,
               float                   *vel_v)
{
  if (!z || !p || nx < 1 || ny < 1 || p->iterations < 0) return 1;
  const size_t       n = (size_t)nx * ny;
  std::vector<float> rain(n, 1.f);
  if (rain_map) rain.assign(rain_map, rain_map + n);
  const float        init_depth = p->initial_water < 0.f ? p->water_height : p->initial_water;
  std::vector<float> d(n, init_depth), d1(n), d2(n), s(n, 0.f), fl(n, 0.f), fr(n, 0.f), ft(n, 0.f),
      fb(n, 0.f), u(n, 0.f), v(n, 0.f);
  std::vector<float> fl_o(n), fr_o(n), ft_o(n), fb_o(n), z_o(n), s_o(n);
  for (size_t k = 0; k < n; k++) d[k] *= rain[k];
  const float water_volume_init = std::accumulate(d.begin(), d.end(), 0.f);
  const float rain_map_volume = std::accumulate(rain.begin(), rain.end(), 0.f);

  auto img = [&](std::vector<float> &a) { return hmref::hm_image{a.data(), nx, ny}; };

  for (int it = 0; it < p->iterations; it++)
  {
    for (size_t k = 0; k < n; k++) d1[k] = d[k] + p->rain_per_step * rain[k];

    hmref::hm_image iz{z, nx, ny}, i_fl = img(fl), i_fr = img(fr), i_ft = img(ft), i_fb = img(fb),
                    i_d1 = img(d1), o_fl = img(fl_o), o_fr = img(fr_o), o_ft = img(ft_o), o_fb = img(fb_o),
                    i_d2 = img(d2), i_u = img(u), i_v = img(v), i_s = img(s), o_z = img(z_o),
                    o_s = img(s_o);

#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
    {
      hmref::g_gid1 = j;
      for (int i = 0; i < nx; i++)
      {
        hmref::g_gid0 = i;
        hmref::hydraulic_vpipes_flow_pass(&iz, &i_fl, &i_fr, &i_ft, &i_fb, &i_d1, &o_fl, &o_fr, &o_ft,
                                          &o_fb, nx, ny, p->dt, p->flux_diffusion ? 1 : 0,
                                          p->flux_diffusion_strength);
      }
    }
    fl.swap(fl_o);
    fr.swap(fr_o);
    ft.swap(ft_o);
    fb.swap(fb_o);
    i_fl = img(fl), i_fr = img(fr), i_ft = img(ft), i_fb = img(fb);

#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
    {
      hmref::g_gid1 = j;
      for (int i = 0; i < nx; i++)
      {
        hmref::g_gid0 = i;
        hmref::hydraulic_vpipes_water_pass(&iz, &i_fl, &i_fr, &i_ft, &i_fb, &i_d1, &i_d2, &i_u, &i_v,
                                           nx, ny, p->dt, p->water_height);
      }
    }

#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
    {
      hmref::g_gid1 = j;
      for (int i = 0; i < nx; i++)
      {
        hmref::g_gid0 = i;
        hmref::hydraulic_vpipes_erosion_pass(&iz, &i_d2, &i_u, &i_v, &i_s, &o_z, &o_s, nx, ny,
                                             p->water_height, p->k_capacity, p->k_erode, p->k_depose,
                                             p->k_discharge_exp, p->downcutting_max_depth_ratio);
      }
    }
    std::memcpy(z, z_o.data(), n * sizeof(float));
    o_s = img(s_o);

#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
    {
      hmref::g_gid1 = j;
      for (int i = 0; i < nx; i++)
      {
        hmref::g_gid0 = i;
        hmref::hydraulic_vpipes_sediment_transport_pass(&i_u, &i_v, &o_s, &i_s, nx, ny, p->dt);
      }
    }

    const float keep = 1.f - p->dt * p->evap_rate;
    for (size_t k = 0; k < n; k++) d[k] = d2[k] * keep;
    if (p->maintain_water_volume)
    {
      float water_to_add = water_volume_init - std::accumulate(d.begin(), d.end(), 0.f);
      for (size_t k = 0; k < n; k++) d[k] += water_to_add * rain[k] / rain_map_volume;
    }
  }

  if (water_depth) std::memcpy(water_depth, d.data(), n * sizeof(float));
  if (sediment) std::memcpy(sediment, s.data(), n * sizeof(float));
  if (vel_u) std::memcpy(vel_u, u.data(), n * sizeof(float));
  if (vel_v) std::memcpy(vel_v, v.data(), n * sizeof(float));
  return 0;
}

/* flow_simulation, HighMap/src/hydrology/flow_simulation.cpp:26-110, with
 * the reference's flow and water pass kernels; dry-out as
 * water_depth.cpp:40-66 after Array::max (methods.cpp) */
int ref_flow_simulation(const float *z,
                        int          nx,
                        int          ny,
                        float        water_height,
                        const float *depth_map,
                        int          iterations,
                        float        dt,
                        int          flux_diffusion,
                        float        flux_diffusion_strength,
                        float        dry_out_ratio,
                        float       *water_depth)
{
  if (!z || !depth_map || !water_depth || nx < 1 || ny < 1 || iterations < 0) return 1;
  const size_t       n = (size_t)nx * ny;
  std::vector<float> zz(z, z + n), d(n), fl(n, 0.f), fr(n, 0.f), ft(n, 0.f), fb(n, 0.f), u(n), v(n);
  std::vector<float> fl_o(n), fr_o(n), ft_o(n), fb_o(n), d_o(n);
  for (size_t k = 0; k < n; k++) d[k] = water_height * depth_map[k];
  auto img = [&](std::vector<float> &a) { return hmref::hm_image{a.data(), nx, ny}; };
  for (int it = 0; it < iterations; it++)
  {
    hmref::hm_image iz = img(zz), i_fl = img(fl), i_fr = img(fr), i_ft = img(ft), i_fb = img(fb), i_d = img(d),
                    o_fl = img(fl_o), o_fr = img(fr_o), o_ft = img(ft_o), o_fb = img(fb_o), o_d = img(d_o),
                    i_u = img(u), i_v = img(v);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
    {
      hmref::g_gid1 = j;
      for (int i = 0; i < nx; i++)
      {
        hmref::g_gid0 = i;
        hmref::hydraulic_vpipes_flow_pass(&iz, &i_fl, &i_fr, &i_ft, &i_fb, &i_d, &o_fl, &o_fr, &o_ft, &o_fb, nx,
                                          ny, dt, flux_diffusion ? 1 : 0, flux_diffusion_strength);
      }
    }
    fl.swap(fl_o);
    fr.swap(fr_o);
    ft.swap(ft_o);
    fb.swap(fb_o);
    i_fl = img(fl), i_fr = img(fr), i_ft = img(ft), i_fb = img(fb);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
    {
      hmref::g_gid1 = j;
      for (int i = 0; i < nx; i++)
      {
        hmref::g_gid0 = i;
        hmref::hydraulic_vpipes_water_pass(&iz, &i_fl, &i_fr, &i_ft, &i_fb, &i_d, &o_d, &i_u, &i_v, nx, ny, dt,
                                           water_height);
      }
    }
    d.swap(d_o);
  }
  if (dry_out_ratio != 0.f)
  {
    const float dmax = *std::max_element(d.begin(), d.end());
    for (size_t k = 0; k < n; k++)
    {
      d[k] -= dry_out_ratio * dmax;
      d[k] = std::max(0.f, d[k]);
    }
  }
  std::memcpy(water_depth, d.data(), n * sizeof(float));
  return 0;
}

/* thermal_gpu.cpp:154-219,249-272: thermal_flatten (rule 4), thermal_inflate
 * (rule 5), thermal_rib (rule 6), as hmo_thermal_relief; the masked
 * overloads via apply_with_mask */
int ref_thermal_relief(int          rule,
                       float       *z,
                       int          nx,
                       int          ny,
                       const float *talus,
                       float        sigma_inf,
                       float        sigma_sup,
                       int          iterations,
                       const float *mask)
{
  if (!z || rule < 4 || rule > 6 || iterations < 0 || (rule != 6 && !talus)) return 1;
  const int nmin = rule == 5 ? 3 : 5;
  if (nx < nmin || ny < nmin) return 1;
  const size_t       n = (size_t)nx * ny;
  std::vector<float> a(z, z + n), b(n);
  for (int it = 0; it < iterations; it++)
  {
    if (rule == 4)
      run_inplace(a.data(), b.data(), nullptr, nx, ny,
                  [&](float *zw) { hmref::thermal_flatten(zw, talus, nx, ny, sigma_inf, sigma_sup); }, 2);
    else if (rule == 5)
      run_inplace(a.data(), b.data(), nullptr, nx, ny, [&](float *zw) { hmref::thermal_inflate(zw, talus, nx, ny); });
    else
      run_inplace(a.data(), b.data(), nullptr, nx, ny, [&](float *zw) { hmref::thermal_rib(zw, nx, ny); });
    std::swap(a, b);
  }
  extrapolate_borders_n(a.data(), nx, ny, rule == 6 ? 3 : 1);
  for (size_t k = 0; k < n; k++) z[k] = mask ? z[k] * (1.f - mask[k]) + a[k] * mask[k] : a[k];
  return 0;
}

/* flow_simulation.cpp:112-157 over shallow_viscous_flow.cl: the adaptive
 * dt of helper_vflow_compute_adaptive_dt (:16-24) every 10 steps, h_in ->
 * h_out per step, then water_depth_dry_out (water_depth.cpp:40-66) */
int ref_flow_simulation_viscous(const float *z,
                                int          nx,
                                int          ny,
                                float        water_height,
                                const float *depth_map,
                                int          iterations,
                                float        dt,
                                float        dry_out_ratio,
                                float        viscosity,
                                float        power,
                                float       *water_depth)
{
  if (!z || !depth_map || !water_depth || nx < 1 || ny < 1 || iterations < 0) return 1;
  const size_t       n = (size_t)nx * ny;
  std::vector<float> zz(z, z + n), d(n), d_o(n);
  for (size_t k = 0; k < n; k++) d[k] = water_height * depth_map[k];
  for (int it = 0; it < iterations; ++it)
  {
    if (it % 10 == 0)
    {
      const float hmax = *std::max_element(d.begin(), d.end());
      const float mobility = std::pow(hmax, power) / viscosity;
      dt = 0.2f / std::fmax(mobility, 1e-6f);
    }
    hmref::hm_image iz{zz.data(), nx, ny}, i_d{d.data(), nx, ny}, o_d{d_o.data(), nx, ny};
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
    {
      hmref::g_gid1 = j;
      for (int i = 0; i < nx; i++)
      {
        hmref::g_gid0 = i;
        hmref::shallow_viscous_flow(&iz, &i_d, &o_d, nx, ny, dt, viscosity, power);
      }
    }
    d.swap(d_o);
  }
  if (dry_out_ratio != 0.f)
  {
    const float dmax = *std::max_element(d.begin(), d.end());
    for (size_t k = 0; k < n; k++)
    {
      d[k] -= dry_out_ratio * dmax;
      d[k] = std::max(0.f, d[k]);
    }
  }
  std::memcpy(water_depth, d.data(), n * sizeof(float));
  return 0;
}

int ref_num_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

} // extern "C"
