"""Two vpipes steps per launch (k_vp_tb2, HM_VPIPES_TILED_TB2) against the
oracle and against the one-step tiled kernels, via the C-ABI.

The two-step tile computes the pair's first step again on a 4-cell halo and
gathers the second step's advected sediment from it; taps beyond the halo
(fast water) recompute the first step's eroded sediment at that cell from
global memory.  Every case must give the oracle's bits where the oracle is
bit-exact, and the one-step kernels' bits everywhere (the volume top-up
runs one step per launch, so it only checks the fallback).
"""
import numpy as np
import pytest

from highmap_b200.inputs import fbm
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
TOL = 1e-3  # of the height range, vpipes

CONFIG2 = dict(maintain_water_volume=0, flux_diffusion=0, dt=0.1, k_capacity=0.05, k_erode=0.01, k_depose=0.01,
               evap_rate=0.01, gravity=9.81, pipe_area=1.0, pipe_length=1.0, rain_per_step=1e-4,
               initial_water=0.0, water_height=1e-2)
# water fast enough to carry sediment beyond the staged halo
FAST = dict(maintain_water_volume=0, flux_diffusion=1, dt=0.5, gravity=40.0, initial_water=0.05, iterations=12)

CASES = {
    "config2": dict(CONFIG2, iterations=41),
    "fast_water": FAST,
    "diffusion": dict(iterations=21, maintain_water_volume=0),
    "rain_map": dict(iterations=20, maintain_water_volume=0, rain_per_step=1e-3),
    "pipe_length": dict(iterations=20, maintain_water_volume=0, pipe_length=0.75, gravity=2.0, pipe_area=0.5),
    "maintain": dict(iterations=15),
}


def _run(gpu, algo, z0, pkw, rain=None):
    z = z0.copy()
    outs = [np.empty_like(z) for _ in range(4)]
    kw = dict(pkw)
    it = kw.pop("iterations")
    gpu.vpipes_set_algorithm(algo)
    try:
        gpu.hydraulic_vpipes(z, iterations=it, rain_map=rain, water_depth=outs[0], sediment=outs[1], vel_u=outs[2],
                             vel_v=outs[3], **kw)
    finally:
        gpu.vpipes_set_algorithm(gpu.VPIPES_AUTO)
    return (z, *outs)


def _compare(got, ref, want, z0, exact):
    names = ("z", "water", "sediment", "u", "v")
    for n, g, r in zip(names, got, ref):
        assert np.array_equal(g, r), "%s differs from the one-step kernels" % n
    rng = float(z0.max() - z0.min()) or 1.0
    errs = {n: float(np.abs(g.astype(np.float64) - w).max()) for n, g, w in zip(names, got, want)}
    assert errs["z"] <= TOL * rng and errs["sediment"] <= TOL * rng, errs
    if exact:
        for n, g, w in zip(names, got, want):
            assert np.array_equal(g, w), "%s not bit-exact with the oracle: %s" % (n, errs)


# small grids take 16 x 8 tiles; (333, 650) has enough 32 x 16 tiles for that shape, with ragged edges
@pytest.mark.parametrize("shape", [(128, 128), (97, 131), (256, 64), (5, 300), (20, 40), (37, 260), (333, 650)])
@pytest.mark.parametrize("case", sorted(CASES))
def test_two_step_tiles(gpu, shape, case):
    ny, nx = shape
    z0 = fbm(nx, ny, seed=31)
    pkw = CASES[case]
    rain = (0.25 + fbm(nx, ny, seed=32)).astype(np.float32) if case == "rain_map" else None
    want = po.vpipes(z0, po.VpipesParams.make(**pkw), rain_map=rain)
    ref = _run(gpu, gpu.VPIPES_TILED, z0, pkw, rain)
    got = _run(gpu, gpu.VPIPES_TILED_TB2, z0, pkw, rain)
    _compare(got, ref, want, z0, exact=not pkw.get("maintain_water_volume", 1))


@pytest.mark.parametrize("iterations", [1, 2, 3, 4, 5, 8, 9])
@pytest.mark.parametrize("case", ["config2", "fast_water"])
def test_step_counts(gpu, iterations, case):
    """Pairs start at the second step; an even count leaves the last step
    alone, an odd count ends on a pair whose second step writes the velocity
    outputs and is followed by the final advection."""
    z0 = fbm(132, 129, seed=33)
    pkw = dict(CASES[case], iterations=iterations)
    want = po.vpipes(z0, po.VpipesParams.make(**pkw))
    ref = _run(gpu, gpu.VPIPES_TILED, z0, pkw)
    got = _run(gpu, gpu.VPIPES_TILED_TB2, z0, pkw)
    _compare(got, ref, want, z0, exact=True)


def test_exponent_matches_one_step(gpu):
    """Discharge exponent 0.5 (fp64 pow on the GPU): the two-step path
    equals the one-step kernels bit for bit."""
    z0 = fbm(200, 150, seed=34)
    pkw = dict(iterations=17, maintain_water_volume=0, k_discharge_exp=0.5)
    want = po.vpipes(z0, po.VpipesParams.make(**pkw))
    ref = _run(gpu, gpu.VPIPES_TILED, z0, pkw)
    got = _run(gpu, gpu.VPIPES_TILED_TB2, z0, pkw)
    _compare(got, ref, want, z0, exact=False)


def test_large_grid_matches_one_step(gpu):
    """1024 x 768 at the plain drop-in benchmark's parameters: the two-step
    path equals the one-step kernels bit for bit after 101 steps."""
    import torch
    z0 = fbm(1024, 768, seed=35)
    p = gpu.vpipes_params(**dict(CONFIG2, iterations=101))
    res = []
    for algo in (gpu.VPIPES_TILED, gpu.VPIPES_TILED_TB2):
        dz = torch.from_numpy(z0.copy()).cuda()
        s = torch.empty_like(dz)
        gpu.vpipes_set_algorithm(algo)
        try:
            gpu.hydraulic_vpipes_device(dz, p, None, None, s)
            torch.cuda.synchronize()
        finally:
            gpu.vpipes_set_algorithm(gpu.VPIPES_AUTO)
        res.append((dz.cpu().numpy(), s.cpu().numpy()))
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])
