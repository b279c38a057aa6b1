"""GPU parity of sediment_deposition (HighMap/src/erosion/deposition.cpp:19-66,
layers of sediment each settled by short thermal solves) against the
oracle, through the C-ABI.  Bit-exact, with the thermal tolerance reported
on failure."""
import json
import os

import numpy as np
import pytest

from highmap_b200.inputs import fbm
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-4


def _assert_parity(got, want, z0):
    rng = float(z0.max() - z0.min()) or 1.0
    err = float(np.abs(got.astype(np.float64) - want).max())
    assert err <= TOL * rng, "max abs err %.3g" % err
    assert np.array_equal(got, want), "within tolerance (%.3g) but not bit-exact" % err


def test_golden(gpu):
    g = dict(np.load(os.path.join(GOLDEN, "sediment_deposition.npz")))
    kw = json.loads(str(g["params"]))
    z = g["z"].copy()
    depo = np.empty_like(z)
    gpu.sediment_deposition(z, g["talus"], deposition_map=depo, **kw)
    _assert_parity(z, g["out_z"], g["z"])
    _assert_parity(depo, g["out_depo"], g["z"])


@pytest.mark.parametrize("shape", [(256, 256), (130, 257), (9, 300)])
@pytest.mark.parametrize("masked", [False, True])
@pytest.mark.parametrize("its", [(5, 10), (1, 3), (0, 10), (3, 0)])
def test_against_oracle(gpu, shape, masked, its):
    ny, nx = shape
    z0 = fbm(nx, ny, seed=51)
    talus = ((0.3 + fbm(nx, ny, seed=52)) / nx).astype(np.float32)
    mask = fbm(nx, ny, seed=53) if masked else None
    want, want_d = po.sediment_deposition(z0, talus, 0.02, its[0], its[1], mask=mask)
    z = z0.copy()
    depo = np.empty_like(z)
    gpu.sediment_deposition(z, talus, depo, 0.02, its[0], its[1], mask=mask)
    _assert_parity(z, want, z0)
    _assert_parity(depo, want_d, z0)


def test_device_api_matches_host_api(gpu):
    import torch
    z0 = fbm(300, 200, seed=54)
    talus = ((0.3 + fbm(300, 200, seed=55)) / 300).astype(np.float32)
    h = z0.copy()
    hd = np.empty_like(z0)
    gpu.sediment_deposition(h, talus, hd, 0.015, 4, 12)
    dz = torch.from_numpy(z0.copy()).cuda()
    dd = torch.empty_like(dz)
    gpu.sediment_deposition_device(dz, torch.from_numpy(talus).cuda(), dd, 0.015, 4, 12)
    torch.cuda.synchronize()
    assert np.array_equal(dz.cpu().numpy(), h)
    assert np.array_equal(dd.cpu().numpy(), hd)
