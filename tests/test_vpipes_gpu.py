"""GPU parity of the virtual-pipes solver against the oracle, via the C-ABI.

Bit-exact where both sides evaluate the same fp32 operations (every case
without the water-volume top-up and with discharge exponent 1: the GPU
reproduces the reference's one-rounding-per-operation arithmetic, fp64
hypot included).  Two cases differ by construction and are held to the
vpipes tolerance (max abs error <= 1e-3 of the height range) on z and
sediment instead: maintain_water_volume, whose grid-wide fp64 sum is
reduced in a different order on the two sides, and exponents other than 1,
where the C library's powf (not correctly rounded) and the GPU's fp64 pow
can differ in the last bit.
"""
import json
import os

import numpy as np
import pytest

from highmap_b200.inputs import fbm
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-3  # of the height range, vpipes

CONFIG2 = dict(maintain_water_volume=0, flux_diffusion=0, dt=0.1, k_capacity=0.05, k_erode=0.01, k_depose=0.01,
               evap_rate=0.01, gravity=9.81, pipe_area=1.0, pipe_length=1.0, rain_per_step=1e-4,
               initial_water=0.0, water_height=1e-2)


def _run_gpu(gpu, z0, pkw, rain=None):
    z = z0.copy()
    outs = [np.empty_like(z) for _ in range(4)]
    kw = dict(pkw)
    it = kw.pop("iterations", 50)
    gpu.hydraulic_vpipes(z, iterations=it, rain_map=rain, water_depth=outs[0], sediment=outs[1], vel_u=outs[2],
                         vel_v=outs[3], **kw)
    return (z, *outs)


def _check(got, want, z0, exact):
    rng = float(z0.max() - z0.min()) or 1.0
    names = ("z", "water", "sediment", "u", "v")
    errs = {n: float(np.abs(g.astype(np.float64) - w).max()) for n, g, w in zip(names, got, want)}
    assert errs["z"] <= TOL * rng, errs
    assert errs["sediment"] <= TOL * rng, errs
    if exact:
        for n, g, w in zip(names, got, want):
            assert np.array_equal(g, w), "%s not bit-exact: %s" % (n, errs)


@pytest.mark.parametrize("name", ["vpipes_no_maintain", "vpipes_rain_per_step", "vpipes_exp_half",
                                  "vpipes_defaults", "vpipes_rain_map"])
def test_golden(gpu, name):
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    p = json.loads(str(g["params"]))
    got = _run_gpu(gpu, g["z"], p, rain=g.get("rain_map"))
    want = tuple(g[k] for k in ("out_z", "out_water", "out_sediment", "out_u", "out_v"))
    _check(got, want, g["z"], exact=not p["maintain_water_volume"] and p["k_discharge_exp"] == 1.0)


@pytest.mark.parametrize("shape", [(128, 128), (97, 131), (256, 64), (5, 300)])
@pytest.mark.parametrize("case", ["config2", "defaults", "no_maintain_diffusion", "rain_map", "pipe_length"])
def test_against_oracle(gpu, shape, case):
    ny, nx = shape
    z0 = fbm(nx, ny, seed=2)
    rain = None
    if case == "config2":
        pkw = dict(CONFIG2, iterations=60)
    elif case == "defaults":
        pkw = dict(iterations=30)
    elif case == "no_maintain_diffusion":
        pkw = dict(iterations=30, maintain_water_volume=0)
    elif case == "rain_map":
        pkw = dict(iterations=30)
        rain = (0.25 + fbm(nx, ny, seed=12)).astype(np.float32)
    else:
        pkw = dict(iterations=30, maintain_water_volume=0, pipe_length=0.75, gravity=2.0, pipe_area=0.5)
    want = po.vpipes(z0, po.VpipesParams.make(**pkw), rain_map=rain)
    got = _run_gpu(gpu, z0, pkw, rain)
    _check(got, want, z0, exact=not pkw.get("maintain_water_volume", 1))


def test_deterministic(gpu):
    z0 = fbm(300, 220, seed=3)
    a = _run_gpu(gpu, z0, dict(iterations=40))
    b = _run_gpu(gpu, z0, dict(iterations=40))
    for x, y in zip(a, b):
        assert x.tobytes() == y.tobytes()


def test_device_api_matches_host_api(gpu):
    import torch
    z0 = fbm(512, 256, seed=7)
    pkw = dict(CONFIG2, iterations=50)
    h = _run_gpu(gpu, z0, pkw)
    dz = torch.from_numpy(z0.copy()).cuda()
    outs = [torch.empty_like(dz) for _ in range(4)]
    gpu.hydraulic_vpipes_device(dz, gpu.vpipes_params(**pkw), None, *outs)
    torch.cuda.synchronize()
    for x, y in zip((dz, *outs), h):
        assert np.array_equal(x.cpu().numpy(), y)


def test_full_size_config_properties(gpu):
    """4096^2 with the plain drop-in benchmark's vpipes configuration:
    finite, deterministic, water depth non-negative, and a band checked
    bit-exact against the oracle after a few iterations."""
    import torch
    n = 4096
    z0 = fbm(n, n, seed=2)
    it = 200
    p = dict(CONFIG2, iterations=it)
    dz = torch.from_numpy(z0).cuda()
    a = dz.clone()
    wa = torch.empty_like(dz)
    sa = torch.empty_like(dz)
    gpu.hydraulic_vpipes_device(a, gpu.vpipes_params(**p), None, wa, sa)
    b = dz.clone()
    gpu.hydraulic_vpipes_device(b, gpu.vpipes_params(**p))
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    assert bool(torch.isfinite(a).all()) and bool(torch.isfinite(wa).all()) and bool(torch.isfinite(sa).all())
    assert float(wa.min()) >= 0.0
    # band check: the top 712 rows run alone reach the same values in their
    # first 512 rows after 8 iterations (influence of the band's artificial
    # bottom edge travels about one row per iteration).  The band starts at
    # row 0 so every cell keeps its coordinates: the advection pass samples at
    # j - dt * v, whose rounding depends on the magnitude of j.
    iters = 8
    c = dz.clone()
    gpu.hydraulic_vpipes_device(c, gpu.vpipes_params(**dict(CONFIG2, iterations=iters)))
    torch.cuda.synchronize()
    rows, band = 512, 712
    want = po.vpipes(z0[:band], po.VpipesParams.make(**dict(CONFIG2, iterations=iters)))[0]
    got = c.cpu().numpy()[:rows]
    assert np.array_equal(got, want[:rows])


FAST = dict(maintain_water_volume=0, flux_diffusion=1, dt=0.5, gravity=40.0, initial_water=0.05, iterations=12)


@pytest.mark.parametrize("launch", [(128, 2, 32), (128, 2, 128), (256, 2, 64), (128, 3, 48), (256, 3, 256)])
@pytest.mark.parametrize("case", ["config2", "fast_water", "defaults"])
@pytest.mark.parametrize("nx", [333, 334])
def test_launch_shapes(gpu, launch, case, nx):
    """Every launch shape of the fused step gives the oracle's bits, for an
    odd and an even row length.  The fast-water case moves sediment further than the staged advection
    radius, so its samples go through the exact recomputation from global
    memory."""
    ny = 300
    z0 = fbm(nx, ny, seed=5)
    pkw = {"config2": dict(CONFIG2, iterations=40), "fast_water": FAST, "defaults": dict(iterations=20)}[case]
    want = po.vpipes(z0, po.VpipesParams.make(**pkw))
    gpu.vpipes_set_launch(*launch)
    try:
        got = _run_gpu(gpu, z0, pkw)
    finally:
        gpu.vpipes_set_launch(0)
    _check(got, want, z0, exact=not pkw.get("maintain_water_volume", 1))


def test_unaligned_device_buffer(gpu):
    """A z that is not 8-byte aligned (a view one element into a buffer)
    still matches the oracle."""
    import torch
    ny, nx = 120, 256
    z0 = fbm(nx, ny, seed=8)
    pkw = dict(CONFIG2, iterations=30)
    want = po.vpipes(z0, po.VpipesParams.make(**pkw))
    buf = torch.zeros(ny * nx + 1, device="cuda")
    z = buf[1:].view(ny, nx)
    z.copy_(torch.from_numpy(z0))
    assert z.data_ptr() % 8 != 0
    gpu.hydraulic_vpipes_device(z, gpu.vpipes_params(**pkw))
    torch.cuda.synchronize()
    assert np.array_equal(z.cpu().numpy(), want[0])


@pytest.mark.parametrize("shape", [(37, 260), (20, 40), (300, 44), (64, 4096), (129, 132)])
@pytest.mark.parametrize("case", ["config2", "fast_water", "defaults", "rain_map"])
def test_tiled_staging(gpu, shape, case):
    """The tiled step with its tiles fetched by TMA (row length a multiple
    of 4, at least 40 x 20) and by cp.async gives the same bits, and the
    oracle's where the oracle is bit-exact.  The shapes leave partial tiles
    on the right and bottom edges, where the TMA boxes read past the grid
    and the clamp-to-edge halo is rebuilt in shared memory."""
    ny, nx = shape
    z0 = fbm(nx, ny, seed=9)
    rain = None
    pkw = {"config2": dict(CONFIG2, iterations=40), "fast_water": FAST, "defaults": dict(iterations=20),
           "rain_map": dict(iterations=20)}[case]
    if case == "rain_map":
        rain = (0.25 + fbm(nx, ny, seed=13)).astype(np.float32)
    want = po.vpipes(z0, po.VpipesParams.make(**pkw), rain_map=rain)
    got = {}
    try:
        for algo in (gpu.VPIPES_TILED, gpu.VPIPES_TILED_CP_ASYNC):
            gpu.vpipes_set_algorithm(algo)
            got[algo] = _run_gpu(gpu, z0, pkw, rain)
    finally:
        gpu.vpipes_set_algorithm(gpu.VPIPES_AUTO)
    for a, b in zip(got[gpu.VPIPES_TILED], got[gpu.VPIPES_TILED_CP_ASYNC]):
        assert np.array_equal(a, b)
    _check(got[gpu.VPIPES_TILED], want, z0, exact=not pkw.get("maintain_water_volume", 1))


@pytest.mark.parametrize("iterations", [1, 2, 3, 8])
@pytest.mark.parametrize("case", ["config2", "fast_water"])
def test_folded_advection_step_counts(gpu, iterations, case):
    """Every step after the first advects the previous step's sediment
    inside its own tile (its staged s1 box, or s1 in memory for samples
    beyond it, which fast water forces), and the last step's advection runs
    after the loop: every step count, the first step alone included, gives
    the oracle's bits with TMA and with cp.async staging."""
    z0 = fbm(132, 129, seed=21)
    pkw = dict({"config2": CONFIG2, "fast_water": FAST}[case], iterations=iterations)
    want = po.vpipes(z0, po.VpipesParams.make(**pkw))
    got = {}
    try:
        for algo in (gpu.VPIPES_TILED, gpu.VPIPES_TILED_CP_ASYNC):
            gpu.vpipes_set_algorithm(algo)
            got[algo] = _run_gpu(gpu, z0, pkw)
    finally:
        gpu.vpipes_set_algorithm(gpu.VPIPES_AUTO)
    for a, b in zip(got[gpu.VPIPES_TILED], got[gpu.VPIPES_TILED_CP_ASYNC]):
        assert np.array_equal(a, b)
    _check(got[gpu.VPIPES_TILED], want, z0, exact=True)
