"""GPU parity of thermal_flatten, thermal_inflate and thermal_rib
(HighMap/src/erosion/thermal_gpu.cpp:154-219,249-272, kernels
thermal_flatten.cl, thermal_inflate.cl, thermal_rib.cl) against the oracle,
through the C-ABI.  Bit-exact, with the thermal tolerance reported on
failure."""
import os

import numpy as np
import pytest

from highmap_b200.inputs import fbm
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-4  # of the height range, thermal


def _assert_parity(got, want, z0):
    fin = np.isfinite(z0)
    rng = float(z0[fin].max() - z0[fin].min()) or 1.0
    ok = np.isfinite(want)
    err = float(np.abs(got[ok].astype(np.float64) - want[ok]).max()) if ok.any() else 0.0
    assert err <= TOL * rng, "max abs err %.3g > %.3g" % (err, TOL * rng)
    assert np.array_equal(got, want, equal_nan=True), "within tolerance (%.3g) but not bit-exact" % err


def _run(gpu, rule, z, talus, iters, sigma_inf=0.5, sigma_sup=0.0, mask=None):
    if rule == po.FLATTEN:
        gpu.thermal_flatten(z, talus, iters, sigma_inf, sigma_sup, mask=mask)
    elif rule == po.INFLATE:
        gpu.thermal_inflate(z, talus, iters, mask=mask)
    else:
        gpu.thermal_rib(z, iters, mask=mask)


@pytest.mark.parametrize("case", ["thermal_flatten", "thermal_flatten_masked", "thermal_inflate", "thermal_rib",
                                  "thermal_rib_masked"])
def test_golden(gpu, case):
    g = dict(np.load(os.path.join(GOLDEN, case + ".npz")))
    z = g["z"].copy()
    _run(gpu, int(g["rule"]), z, g["talus"], int(g["iterations"]), float(g["sigma_inf"]), float(g["sigma_sup"]),
         g.get("mask"))
    _assert_parity(z, g["out_z"], g["z"])


@pytest.mark.parametrize("rule", [po.FLATTEN, po.INFLATE, po.RIB])
@pytest.mark.parametrize("shape", [(256, 256), (130, 257), (9, 300), (5, 5), (6, 9), (64, 63)])
@pytest.mark.parametrize("masked", [False, True])
def test_against_oracle(gpu, rule, shape, masked):
    """Even and odd widths take the column-pair and single-column sweeps;
    5 x 5 is the smallest grid flatten's 2-cell border and rib's 3-deep
    extrapolation allow."""
    ny, nx = shape
    rs = np.random.RandomState(91 + rule)
    z0 = fbm(nx, ny, seed=92) if min(shape) > 8 else rs.rand(ny, nx).astype(np.float32)
    talus = ((0.3 + fbm(nx, ny, seed=93)) / nx).astype(np.float32) if min(shape) > 8 else np.full_like(z0, 0.1)
    mask = rs.rand(ny, nx).astype(np.float32) if masked else None
    iters = 3 if rule == po.RIB else 19
    want = po.thermal_relief(rule, z0, talus, iters, 0.5, 0.25, mask=mask)
    z = z0.copy()
    _run(gpu, rule, z, talus, iters, 0.5, 0.25, mask)
    _assert_parity(z, want, z0)


@pytest.mark.parametrize("rule", [po.FLATTEN, po.INFLATE, po.RIB])
@pytest.mark.parametrize("iters", [0, 1, 2])
def test_few_iterations(gpu, rule, iters):
    z0 = fbm(96, 80, seed=94)
    talus = np.full_like(z0, 0.8 / 96)
    want = po.thermal_relief(rule, z0, talus, iters, 0.4, 0.1)
    z = z0.copy()
    _run(gpu, rule, z, talus, iters, 0.4, 0.1)
    _assert_parity(z, want, z0)


@pytest.mark.parametrize("sigmas", [(0.5, 0.0), (0.0, 0.5), (0.3, 0.7)])
def test_flatten_sigmas(gpu, sigmas):
    """Cells below and above their talus take sigma_inf and sigma_sup."""
    z0 = fbm(120, 90, seed=95)
    talus = ((0.5 + fbm(120, 90, seed=96)) * 2.0 / 120).astype(np.float32)
    want = po.thermal_relief(po.FLATTEN, z0, talus, 23, *sigmas)
    z = z0.copy()
    gpu.thermal_flatten(z, talus, 23, *sigmas)
    _assert_parity(z, want, z0)


def test_nan_cells(gpu):
    z0 = fbm(64, 48, seed=97)
    z0[10, 21] = np.nan
    z0[31, 6] = np.nan
    talus = np.full_like(z0, 0.6 / 64)
    for rule in (po.FLATTEN, po.INFLATE, po.RIB):
        want = po.thermal_relief(rule, z0, talus, 5, 0.5, 0.2)
        z = z0.copy()
        _run(gpu, rule, z, talus, 5, 0.5, 0.2)
        _assert_parity(z, want, z0)


def test_device_api_matches_host_api(gpu):
    import torch
    z0 = fbm(300, 200, seed=98)
    talus = ((0.5 + fbm(300, 200, seed=99)) / 300).astype(np.float32)
    mask = fbm(300, 200, seed=100)
    dev = torch.device("cuda", 0)
    for rule in (po.FLATTEN, po.INFLATE, po.RIB):
        z_h = z0.copy()
        _run(gpu, rule, z_h, talus, 11, 0.5, 0.2, mask)
        z_d = torch.from_numpy(z0.copy()).to(dev)
        gpu.thermal_relief_device(rule, z_d, torch.from_numpy(talus).to(dev) if rule != po.RIB else None, 11, 0.5,
                                  0.2, mask=torch.from_numpy(mask).to(dev))
        torch.cuda.synchronize()
        assert np.array_equal(z_d.cpu().numpy(), z_h)


def test_rejects_bad_arguments(gpu):
    from highmap_b200 import _lib
    import torch
    z = fbm(32, 32, seed=101)
    small = np.zeros((4, 4), np.float32)
    with pytest.raises(_lib.HMError):
        gpu.thermal_flatten(small.copy(), small, 3)  # flatten needs nx, ny >= 5
    with pytest.raises(_lib.HMError):
        gpu.thermal_rib(small.copy(), 3)  # rib extrapolates 3 cells deep
    with pytest.raises(_lib.HMError):
        gpu.thermal_inflate(z.copy(), z, -1)
    dev = torch.device("cuda", 0)
    zd = torch.from_numpy(z).to(dev)
    with pytest.raises(_lib.HMError):
        gpu.thermal_relief_device(po.OLSEN, zd, zd, 3)
    with pytest.raises(_lib.HMError):
        gpu.thermal_stencil_device(po.FLATTEN, zd, zd, 3)


def test_full_size_band(gpu):
    """2048^2, 60 flatten and inflate steps: a top band checked bit-exact
    against the oracle on the band plus a halo wider than the reach (two
    cells per flatten step, one per inflate step)."""
    n = 2048
    z0 = fbm(n, n, seed=102)
    talus = ((0.5 + fbm(n, n, seed=103)) / n).astype(np.float32)
    for rule, iters in ((po.FLATTEN, 60), (po.INFLATE, 60)):
        z = z0.copy()
        _run(gpu, rule, z, talus, iters, 0.5, 0.2)
        r1, h = 128, 2 * iters + 8
        want = po.thermal_relief(rule, z0[:r1 + h], talus[:r1 + h], iters, 0.5, 0.2)
        assert np.array_equal(z[:r1], want[:r1])
