"""GPU parity of flow_simulation (the water-only use of the pipe model,
HighMap/src/hydrology/flow_simulation.cpp:26-110) against the oracle,
through the C-ABI.  The flow and water passes are evaluated with the
reference's fp32 roundings, so the bar is bit-exact equality, checked
also against fixtures made from the reference's own kernel text."""
import json
import os

import numpy as np
import pytest

from highmap_b200.inputs import fbm
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-3  # of the initial water depth range, as for vpipes


def _assert_parity(got, want):
    rng = float(want.max() - want.min()) or 1.0
    err = float(np.abs(got.astype(np.float64) - want).max())
    assert err <= TOL * rng, "max abs err %.3g" % err
    assert np.array_equal(got, want), "within tolerance (%.3g) but not bit-exact" % err


@pytest.mark.parametrize("name", ["flow_simulation_defaults", "flow_simulation_dry_out"])
def test_golden(gpu, name):
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    kw = json.loads(str(g["params"]))
    got = gpu.flow_simulation(g["z"], depth_map=g["depth_map"], **kw)
    _assert_parity(got, g["out_water"])


@pytest.mark.parametrize("shape", [(128, 128), (97, 131), (40, 256), (5, 300), (130, 260)])
@pytest.mark.parametrize("case", ["defaults", "no_diffusion_dry", "long"])
def test_against_oracle(gpu, shape, case):
    ny, nx = shape
    z = fbm(nx, ny, seed=31)
    dm = fbm(nx, ny, seed=32)
    kw = {"defaults": dict(iterations=40),
          "no_diffusion_dry": dict(iterations=40, dt=0.3, flux_diffusion=False, dry_out_ratio=0.15),
          "long": dict(iterations=300, dt=0.5, flux_diffusion=True, flux_diffusion_strength=0.02)}[case]
    want = po.flow_simulation(z, 0.01, dm, **kw)
    got = gpu.flow_simulation(z, 0.01, dm, **kw)
    _assert_parity(got, want)


def test_zero_iterations_and_dry_out(gpu):
    z = fbm(64, 64, seed=33)
    dm = fbm(64, 64, seed=34)
    got = gpu.flow_simulation(z, 0.02, dm, 0, dry_out_ratio=0.5)
    want = po.flow_simulation(z, 0.02, dm, 0, dry_out_ratio=0.5)
    assert np.array_equal(got, want)
    assert (got >= 0).all() and float(got.max()) > 0


def test_device_api_matches_host_api(gpu):
    import torch
    z = fbm(300, 200, seed=35)
    dm = fbm(300, 200, seed=36)
    h = gpu.flow_simulation(z, 0.01, dm, 60, dry_out_ratio=0.05)
    dz = torch.from_numpy(z).cuda()
    ddm = torch.from_numpy(dm).cuda()
    out = torch.empty_like(dz)
    gpu.flow_simulation_device(dz, 0.01, ddm, 60, out, dry_out_ratio=0.05)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), h)


def test_bad_arguments_raise(gpu):
    z = np.zeros((8, 8), np.float32)
    with pytest.raises(gpu.HMError):
        gpu.flow_simulation(z, 0.01, z, -1)
    with pytest.raises(gpu.HMError):
        gpu.flow_simulation(z, 0.01, z, 3, dt=0.0)


def test_full_size_band(gpu):
    """4096^2, 100 steps: the top 256 rows checked bit-exact against the
    oracle run on a band with a halo wider than the information reach (the
    flow pass and the water pass each reach one cell, so two per step)."""
    n, it = 4096, 100
    z = fbm(n, n, seed=2)
    dm = fbm(n, n, seed=3)
    got = gpu.flow_simulation(z, 0.01, dm, it)
    r1 = 256
    h = 2 * it + 8
    want = po.flow_simulation(z[:r1 + h], 0.01, dm[:r1 + h], it)
    assert np.array_equal(got[:r1], want[:r1])
    assert np.isfinite(got).all() and (got >= 0).all()
