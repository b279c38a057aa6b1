"""GPU parity of flow_simulation_viscous (HighMap/src/hydrology/
flow_simulation.cpp:112-157, kernel shallow_viscous_flow.cl) against the
oracle, through the C-ABI.

The face mobilities use pow, which neither the reference (OpenCL pow, glibc
powf on the oracle's side) nor this library rounds correctly in general:
the GPU evaluates pow in fp64 and rounds once, equal to powf except where
the exact power lies within about 2^-52 of a float rounding boundary, and
a last-bit difference in one face then diffuses to the cells around it.
The bar is therefore a tolerance on the water depth, written below (the
share of cells that differ at all is reported on failure)."""
import os

import numpy as np
import pytest

from highmap_b200.inputs import fbm
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-3  # of the deepest water of the oracle's result


def _assert_close(got, want):
    scale = float(np.abs(want).max()) or 1.0
    err = float(np.abs(got.astype(np.float64) - want).max())
    differ = float((got != want).mean())
    assert err <= TOL * scale, "max abs err %.3g > %.3g (%.2g of the cells differ)" % (err, TOL * scale, differ)


@pytest.mark.parametrize("case", ["flow_simulation_viscous", "flow_simulation_viscous_dry"])
def test_golden(gpu, case):
    g = dict(np.load(os.path.join(GOLDEN, case + ".npz")))
    out = gpu.flow_simulation_viscous(g["z"], float(g["water_height"]), g["depth_map"], int(g["iterations"]), 0.5,
                                      float(g["dry_out_ratio"]), float(g["viscosity"]), float(g["power"]))
    _assert_close(out, g["out_d"])


@pytest.mark.parametrize("shape", [(96, 128), (130, 257), (256, 256), (1, 300), (300, 1), (2, 2)])
@pytest.mark.parametrize("params", [(0.0, 1.0, 2.5), (0.1, 1.0, 2.5), (0.0, 2.0, 1.5)])
def test_against_oracle(gpu, shape, params):
    """Rows and columns of one cell exercise the clamp-to-edge reads on
    both sides at once."""
    ny, nx = shape
    rs = np.random.RandomState(71)
    z = fbm(nx, ny, seed=71) if min(shape) > 8 else rs.rand(ny, nx).astype(np.float32)
    dm = fbm(nx, ny, seed=72) if min(shape) > 8 else rs.rand(ny, nx).astype(np.float32)
    dry, visc, power = params
    want = po.flow_simulation_viscous(z, 0.05, dm, 47, 0.5, dry, visc, power)
    got = gpu.flow_simulation_viscous(z, 0.05, dm, 47, 0.5, dry, visc, power)
    _assert_close(got, want)


@pytest.mark.parametrize("iters", [0, 1, 9, 10, 11])
def test_few_iterations(gpu, iters):
    """The time step is re-derived at steps 0, 10, 20, ...; with no steps
    the result is water_height * depth_map (after the dry-out)."""
    z = fbm(80, 64, seed=73)
    dm = fbm(80, 64, seed=74)
    for dry in (0.0, 0.2):
        want = po.flow_simulation_viscous(z, 0.05, dm, iters, 0.5, dry)
        got = gpu.flow_simulation_viscous(z, 0.05, dm, iters, 0.5, dry)
        _assert_close(got, want)


def test_negative_depth_map(gpu):
    """The deepest water is taken over signed values (an all-negative depth
    map gives a negative maximum, as Array::max does)."""
    z = fbm(64, 48, seed=75)
    dm = (-0.5 - fbm(64, 48, seed=76)).astype(np.float32)
    for iters in (0, 3):
        want = po.flow_simulation_viscous(z, 0.05, dm, iters, 0.5, 0.1)
        got = gpu.flow_simulation_viscous(z, 0.05, dm, iters, 0.5, 0.1)
        _assert_close(got, want)


def test_water_is_conserved(gpu):
    """1024^2, 200 steps: where no cell is clamped at zero the fluxes cancel
    pairwise, so the total water stays what it was (a size-independent
    check beside the oracle comparison)."""
    n = 1024
    z = fbm(n, n, seed=77)
    dm = fbm(n, n, seed=78)
    got = gpu.flow_simulation_viscous(z, 0.05, dm, 200)
    m0 = float((np.float32(0.05) * dm).astype(np.float64).sum())
    m1 = float(got.astype(np.float64).sum())
    assert abs(m1 - m0) <= 1e-5 * m0
    assert (got >= 0).all()


def test_device_api_matches_host_api(gpu):
    import torch
    z = fbm(300, 200, seed=79)
    dm = fbm(300, 200, seed=80)
    host = gpu.flow_simulation_viscous(z, 0.05, dm, 33, 0.5, 0.05)
    dev = torch.device("cuda", 0)
    out = torch.empty((200, 300), dtype=torch.float32, device=dev)
    gpu.flow_simulation_viscous_device(torch.from_numpy(z).to(dev), 0.05, torch.from_numpy(dm).to(dev), 33, out, 0.5,
                                       0.05)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), host)


def test_rejects_bad_arguments(gpu):
    from highmap_b200 import _lib
    z = fbm(32, 32, seed=81)
    with pytest.raises(_lib.HMError):
        gpu.flow_simulation_viscous(z, 0.05, z, -1)
