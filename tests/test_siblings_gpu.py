"""GPU parity of the sibling talus stencils (thermal_ridge, thermal_scree,
thermal_schott, thermal_olsen; HighMap/src/erosion/thermal_gpu.cpp:221-396)
against the oracle, through the C-ABI.  Bar: bit-exact (the oracle is
itself bit-exact with the reference's kernel text), with the thermal
tolerance (1e-4 of the height range) reported on failure."""
import os

import numpy as np
import pytest

from highmap_b200.inputs import fbm
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-4  # of the height range, thermal
RULES = {"ridge": po.RIDGE, "scree": po.SCREE, "schott": po.SCHOTT, "olsen": po.OLSEN}


def _assert_parity(got, want, z0):
    rng = float(z0.max() - z0.min()) or 1.0
    err = float(np.abs(got.astype(np.float64) - want).max())
    assert err <= TOL * rng, "max abs err %.3g > %.3g" % (err, TOL * rng)
    assert np.array_equal(got, want), "within tolerance (%.3g) but not bit-exact" % err


def _run(gpu, name, z, talus, iterations, zmax=None, intensity=0.2, depo=None, mask=None):
    if name == "ridge":
        gpu.thermal_ridge(z, talus, iterations, deposition_map=depo, mask=mask)
    elif name == "scree":
        gpu.thermal_scree(z, talus, zmax, iterations, deposition_map=depo, mask=mask)
    elif name == "schott":
        gpu.thermal_schott(z, talus, iterations, intensity=intensity, deposition_map=depo, mask=mask)
    else:
        gpu.thermal_olsen(z, talus, iterations, mask=mask)


@pytest.mark.parametrize("name", list(RULES))
def test_golden(gpu, name):
    g = dict(np.load(os.path.join(GOLDEN, "thermal_%s.npz" % name)))
    z = g["z"].copy()
    depo = np.empty_like(z) if "out_depo" in g else None
    _run(gpu, name, z, g["talus"], int(g["iterations"]), zmax=g.get("zmax"),
         intensity=float(g["intensity"]) if "intensity" in g else 0.2, depo=depo)
    _assert_parity(z, g["out_z"], g["z"])
    if depo is not None:
        _assert_parity(depo, g["out_depo"], g["z"])


@pytest.mark.parametrize("shape", [(256, 256), (130, 257), (9, 300), (7, 7), (64, 33)])
@pytest.mark.parametrize("masked", [False, True])
@pytest.mark.parametrize("name", list(RULES))
def test_against_oracle(gpu, name, shape, masked):
    ny, nx = shape
    z0 = fbm(nx, ny, seed=41)
    talus = ((0.3 + fbm(nx, ny, seed=42)) / nx).astype(np.float32)
    zmax = (z0 + 0.25).astype(np.float32)
    mask = fbm(nx, ny, seed=43) if masked else None
    rule = RULES[name]
    want, want_d = po.thermal_sibling(rule, z0, talus, 23, zmax=zmax, intensity=0.15,
                                      deposition=rule != po.OLSEN, mask=mask)
    z = z0.copy()
    depo = np.empty_like(z) if rule != po.OLSEN else None
    _run(gpu, name, z, talus, 23, zmax=zmax, intensity=0.15, depo=depo, mask=mask)
    _assert_parity(z, want, z0)
    if depo is not None:
        _assert_parity(depo, want_d, z0)


@pytest.mark.parametrize("name", list(RULES))
def test_device_api_matches_host_api(gpu, name):
    import torch
    z0 = fbm(300, 200, seed=44)
    talus = ((0.3 + fbm(300, 200, seed=45)) / 300).astype(np.float32)
    zmax = (z0 + 0.25).astype(np.float32)
    rule = RULES[name]
    h = z0.copy()
    hd = np.empty_like(z0) if rule != po.OLSEN else None
    _run(gpu, name, h, talus, 17, zmax=zmax, depo=hd)
    dz = torch.from_numpy(z0.copy()).cuda()
    dd = torch.empty_like(dz) if rule != po.OLSEN else None
    gpu.thermal_stencil_device(rule, dz, torch.from_numpy(talus).cuda(), 17,
                               zmax=torch.from_numpy(zmax).cuda() if rule == po.SCREE else None,
                               deposition_map=dd)
    torch.cuda.synchronize()
    assert np.array_equal(dz.cpu().numpy(), h)
    if hd is not None:
        assert np.array_equal(dd.cpu().numpy(), hd)


def test_bad_arguments_raise(gpu):
    z = np.zeros((6, 6), np.float32)
    with pytest.raises(gpu.HMError):
        gpu.thermal_olsen(z, z, 3)  # olsen needs 7 x 7
    z = np.zeros((8, 8), np.float32)
    with pytest.raises(gpu.HMError):
        gpu.thermal_ridge(z, z, -1)


def test_full_size_band(gpu):
    """4096^2, 100 iterations of each: the top 256 rows bit-exact against the
    oracle on a band with a halo wider than the information reach (olsen
    reaches two cells per step, the others one)."""
    n, it = 4096, 100
    z0 = fbm(n, n, seed=2)
    talus = ((0.5 + fbm(n, n, seed=3)) / n).astype(np.float32)
    zmax = (z0 + 0.25).astype(np.float32)
    r1 = 256
    h = 2 * it + 8
    for name, rule in RULES.items():
        z = z0.copy()
        _run(gpu, name, z, talus, it, zmax=zmax)
        want, _ = po.thermal_sibling(rule, z0[:r1 + h], talus[:r1 + h], it, zmax=zmax[:r1 + h])
        assert np.array_equal(z[:r1], want[:r1]), name
