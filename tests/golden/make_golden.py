"""Generate tests/golden/*.npz from the reference's own kernel text.

The reference has no golden vectors or known-answer tests for either
solver, so these fixtures are outputs of the reference's OpenCL kernels
(HighMap/src/gpu_opencl/kernels/thermal.cl, hydraulic_vpipes.cl, whose flow and
water passes also drive flow_simulation, and the sibling talus kernels
thermal_ridge.cl, thermal_scree.cl, thermal_schott.cl, thermal_olsen.cl) compiled
for the CPU by oracle/build_oracle.py and driven by oracle/ref_harness.cpp
(Jacobi form).  Run in a checkout where the reference tree is present:

    python tests/golden/make_golden.py [thermal] [config1] [vpipes] [flow_simulation] [siblings] [deposition]
                                     [layer] [snow] [relief] [viscous]

Each .npz holds the inputs, the parameters and the outputs of one case.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from highmap_b200.inputs import fbm  # noqa: E402
from oracle import pyoracle as po  # noqa: E402


# where _save writes (the fixtures' own directory; a test regenerates into a
# temporary one to check that the committed files are what this script makes)
OUT_DIR = HERE


def _save(name, **arrays):
    path = os.path.join(OUT_DIR, name + ".npz")
    np.savez_compressed(path, **arrays)
    print("wrote", path)


def thermal_cases():
    nx, ny = 64, 48
    z = fbm(nx, ny, seed=1)
    talus = (0.5 + fbm(nx, ny, seed=3)) / nx
    talus_u = np.full_like(z, 1.0 / nx)
    mask = fbm(nx, ny, seed=5)

    zo, depo = po.ref_thermal(z, talus_u, 100, deposition=True)
    _save("thermal_uniform", z=z, talus=talus_u, iterations=np.int32(100), out_z=zo, out_depo=depo)

    zo, depo = po.ref_thermal(z, talus, 60, deposition=True)
    _save("thermal_talus_map", z=z, talus=talus, iterations=np.int32(60), out_z=zo, out_depo=depo)

    bed = (0.3 * z).astype(np.float32)
    zo, depo = po.ref_thermal(z, talus, 40, bedrock=bed, deposition=True)
    _save("thermal_bedrock_literal", z=z, talus=talus, bedrock=bed, iterations=np.int32(40), out_z=zo,
          out_depo=depo)

    zo, depo = po.ref_thermal(z, talus, 40, mask=mask, deposition=True)
    _save("thermal_masked", z=z, talus=talus, mask=mask, iterations=np.int32(40), out_z=zo, out_depo=depo)

    zo, depo = po.ref_thermal_auto_bedrock(z, talus_u * 4, 60, deposition=True)
    _save("thermal_auto_bedrock", z=z, talus=talus_u * 4, iterations=np.int32(60), out_z=zo, out_depo=depo)

    # odd, non-square, minimal sizes
    for (nx2, ny2) in ((3, 3), (5, 17), (33, 7)):
        z2 = fbm(nx2, ny2, seed=7, kw=2.0)
        zo, depo = po.ref_thermal(z2, np.full_like(z2, 0.01), 9, deposition=True)
        _save("thermal_small_%dx%d" % (nx2, ny2), z=z2, talus=np.full_like(z2, 0.01), iterations=np.int32(9),
              out_z=zo, out_depo=depo)


def vpipes_cases():
    nx, ny = 48, 40
    z = fbm(nx, ny, seed=2)
    rain = (0.5 + fbm(nx, ny, seed=9)).astype(np.float32)
    cases = {
        # defaults of erosion.hpp:1206-1223, 25 iterations
        "vpipes_defaults": (dict(iterations=25), None),
        "vpipes_rain_map": (dict(iterations=25), rain),
        "vpipes_no_maintain": (dict(iterations=30, maintain_water_volume=0), None),
        "vpipes_rain_per_step": (dict(iterations=40, maintain_water_volume=0, flux_diffusion=0, dt=0.1,
                                      k_capacity=0.05, k_erode=0.01, k_depose=0.01, evap_rate=0.01,
                                      rain_per_step=1e-4, initial_water=0.0), None),
        "vpipes_exp_half": (dict(iterations=20, maintain_water_volume=0, k_discharge_exp=0.5), None),
    }
    for name, (kw, rmap) in cases.items():
        p = po.VpipesParams.make(**kw)
        zo, d, s, u, v = po.ref_vpipes(z, p, rain_map=rmap)
        arrays = dict(z=z, params=np.array(json.dumps(p.as_dict())), out_z=zo, out_water=d, out_sediment=s,
                      out_u=u, out_v=v)
        if rmap is not None:
            arrays["rain_map"] = rmap
        _save(name, **arrays)


def flow_simulation_cases():
    nx, ny = 56, 44
    z = fbm(nx, ny, seed=6)
    depth_map = fbm(nx, ny, seed=7)
    cases = {
        # defaults of hydrology.hpp:875-882 (dt 0.5, flux diffusion 0.01, no dry-out)
        "flow_simulation_defaults": dict(water_height=0.01, iterations=60, dt=0.5, flux_diffusion=True,
                                         flux_diffusion_strength=0.01, dry_out_ratio=0.0),
        "flow_simulation_dry_out": dict(water_height=0.02, iterations=40, dt=0.3, flux_diffusion=False,
                                        flux_diffusion_strength=0.01, dry_out_ratio=0.1),
    }
    for name, kw in cases.items():
        out = po.ref_flow_simulation(z, depth_map=depth_map, **kw)
        _save(name, z=z, depth_map=depth_map, params=np.array(json.dumps(kw)), out_water=out)


def sibling_cases():
    nx, ny = 52, 46
    z = fbm(nx, ny, seed=8)
    talus = ((0.3 + fbm(nx, ny, seed=9)) / nx).astype(np.float32)
    zmax = (z + 0.2).astype(np.float32)
    for rule, name, kw in ((po.RIDGE, "thermal_ridge", dict(iterations=30)),
                           (po.SCREE, "thermal_scree", dict(iterations=30, zmax=zmax)),
                           (po.SCHOTT, "thermal_schott", dict(iterations=30, intensity=0.2)),
                           (po.OLSEN, "thermal_olsen", dict(iterations=30))):
        zo, depo = po.ref_thermal_sibling(rule, z, talus, deposition=rule != po.OLSEN, **kw)
        arrays = dict(z=z, talus=talus, iterations=np.int32(kw["iterations"]), out_z=zo)
        if depo is not None:
            arrays["out_depo"] = depo
        if "zmax" in kw:
            arrays["zmax"] = zmax
        if "intensity" in kw:
            arrays["intensity"] = np.float32(kw["intensity"])
        _save(name, **arrays)


def deposition_cases():
    nx, ny = 50, 42
    z = fbm(nx, ny, seed=10)
    talus = ((0.3 + fbm(nx, ny, seed=11)) / nx).astype(np.float32)
    zo, depo = po.ref_sediment_deposition(z, talus, max_deposition=0.02, iterations=4, thermal_subiterations=8)
    _save("sediment_deposition", z=z, talus=talus, params=np.array(json.dumps(
        dict(max_deposition=0.02, iterations=4, thermal_subiterations=8))), out_z=zo, out_depo=depo)


def layer_cases():
    # sediment_layer: about half of the cells steeper than the upper limit
    for (nx, ny, seed, iters, post) in ((50, 42, 30, 25, True), (37, 29, 33, 15, False)):
        z = fbm(nx, ny, seed=seed)
        tl = ((0.5 + fbm(nx, ny, seed=seed + 1)) / nx).astype(np.float32)
        tu = ((3.0 + 2.0 * fbm(nx, ny, seed=seed + 2)) / nx).astype(np.float32)
        zo, depo = po.ref_sediment_layer(z, tl, tu, iters, post)
        _save("sediment_layer_%s" % ("post" if post else "nopost"), z=z, talus_layer=tl, talus_upper_limit=tu,
              iterations=np.int32(iters), apply_post_filter=np.int32(post), out_z=zo, out_depo=depo)


def snow_cases():
    # snow_simulation's post-filter on a snow cover of about a tenth of the relief
    nx, ny = 56, 44
    z = fbm(nx, ny, seed=40)
    s = (0.08 * fbm(nx, ny, seed=41)).astype(np.float32)
    so = po.ref_snow_post_filter(z, s, 0.05, 30, 0.2)
    _save("snow_post_filter", z=z, s=s, snow_depth=np.float32(0.05), iterations=np.int32(30),
          thermal_talus_ratio=np.float32(0.2), out_s=so)


def relief_cases():
    # thermal_flatten (sigma_inf 0.5, sigma_sup 0.2), thermal_inflate, thermal_rib; rib and flatten also masked
    nx, ny = 52, 38
    z = fbm(nx, ny, seed=50)
    talus = ((0.5 + fbm(nx, ny, seed=51)) / nx).astype(np.float32)
    mask = fbm(nx, ny, seed=52)
    for name, rule, kw in (("thermal_flatten", po.FLATTEN, dict(sigma_inf=0.5, sigma_sup=0.2)),
                           ("thermal_inflate", po.INFLATE, {}), ("thermal_rib", po.RIB, {})):
        for m in (None, mask):
            if m is not None and rule == po.INFLATE:
                continue
            zo = po.ref_thermal_relief(rule, z, talus, 15, mask=m, **kw)
            arrays = dict(z=z, talus=talus, iterations=np.int32(15), rule=np.int32(rule), out_z=zo,
                          sigma_inf=np.float32(kw.get("sigma_inf", 0.5)), sigma_sup=np.float32(kw.get("sigma_sup", 0.0)))
            if m is not None:
                arrays["mask"] = m
            _save(name + ("_masked" if m is not None else ""), **arrays)


def viscous_cases():
    # flow_simulation_viscous on inputs where the film stays stable (water conserved), with and without dry-out
    nx, ny = 128, 96
    z = fbm(nx, ny, seed=11)
    dm = fbm(nx, ny, seed=12)
    for dry in (0.0, 0.1):
        out = po.ref_flow_simulation_viscous(z, 0.05, dm, 60, 0.5, dry, 1.0, 2.5)
        _save("flow_simulation_viscous%s" % ("_dry" if dry else ""), z=z, depth_map=dm, water_height=np.float32(0.05),
              iterations=np.int32(60), dry_out_ratio=np.float32(dry), viscosity=np.float32(1.0),
              power=np.float32(2.5), out_d=out)


def _digest(a):
    """sha256 of an array's bytes, as 32 uint8 values."""
    import hashlib
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), dtype=np.uint8).copy()


def config1_cases():
    """The thermal benchmark configuration run on the CPU, verbatim: a
    256 x 256 fBm heightmap (seed 1, base wavenumber 4, 8 octaves,
    persistence 0.5, lacunarity 2, remapped to [0, 1]), uniform talus
    1/256, no bedrock, 100 iterations, heights and deposition map.  At
    768 KB the arrays themselves would dwarf the other fixtures, so the
    fixture keeps sha256 digests of the input and of the reference text's
    two outputs; the test regenerates the input and checks its digest
    first."""
    n = 256
    z = fbm(n, n, seed=1)
    talus = np.float32(1.0 / n)
    zo, depo = po.ref_thermal(z, np.full_like(z, talus), 100, deposition=True)
    _save("config1_thermal_256", z_sha256=_digest(z), talus=talus, iterations=np.int32(100),
          out_z_sha256=_digest(zo), out_depo_sha256=_digest(depo))


GROUPS = {"thermal": thermal_cases, "config1": config1_cases, "vpipes": vpipes_cases, "flow_simulation": flow_simulation_cases,
          "siblings": sibling_cases, "deposition": deposition_cases,
          "layer": layer_cases, "snow": snow_cases, "relief": relief_cases,
          "viscous": viscous_cases}

if __name__ == "__main__":
    if not po.ref_available():
        sys.exit("the reference checker oracle/_ref/libhm_ref.so could not be built")
    # all groups, or the ones named on the command line
    for g in sys.argv[1:] or list(GROUPS):
        GROUPS[g]()
