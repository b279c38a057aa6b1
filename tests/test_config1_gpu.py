"""The thermal benchmark configuration, verbatim, on the GPU.

256 x 256 fBm heightmap (seed 1, base wavenumber 4, 8 octaves,
persistence 0.5, lacunarity 2, remapped to [0, 1]), uniform talus 1/256,
no bedrock, 100 iterations, through the scalar-talus drop-in
(hmap::gpu::thermal(Array&, float talus, int, Array*, Array*),
HighMap/src/erosion/thermal_gpu.cpp:88-96).  Final heights and deposition
map must equal the reference's kernel text bit for bit (digests in
tests/golden/config1_thermal_256.npz) and the oracle; the report the
reference's tests would give -- max / mean absolute error as a fraction of
the height range, and mass drift -- is checked against the thermal
tolerance (1e-4 of the range) for the GPU against the fp32 oracle and
against an fp64 run of the same scheme.
"""
import hashlib
import os

import numpy as np
import pytest

from highmap_b200.inputs import fbm
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "config1_thermal_256.npz")
TOL = 1e-4  # of the height range, thermal


def _digest(a):
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), dtype=np.uint8)


def _drift(z, z0):
    z0 = z0.astype(np.float64)
    return abs(float(z.astype(np.float64).sum() - z0.sum())) / float(np.abs(z0).sum())


def test_config1_verbatim(gpu):
    g = dict(np.load(GOLDEN))
    z0 = fbm(256, 256, seed=1)
    assert np.array_equal(_digest(z0), g["z_sha256"]), "input generator changed"
    talus = float(g["talus"])
    assert talus == 1.0 / 256
    z = z0.copy()
    depo = np.empty_like(z)
    gpu.thermal(z, talus, int(g["iterations"]), deposition_map=depo)

    # the reference's kernel text (digests) and the oracle, bit for bit
    assert np.array_equal(_digest(z), g["out_z_sha256"])
    assert np.array_equal(_digest(depo), g["out_depo_sha256"])
    want_z, want_d = po.thermal(z0, np.float32(talus), 100, deposition=True)
    assert np.array_equal(z, want_z) and np.array_equal(depo, want_d)

    # error report against the fp32 oracle and an fp64 run of the scheme
    rng = float(z0.max() - z0.min())
    z64, d64 = po.thermal(z0, np.float32(talus), 100, deposition=True, dtype=np.float64)
    for got, want in ((z, want_z), (z, z64), (depo, d64)):
        err = np.abs(got.astype(np.float64) - want.astype(np.float64))
        assert err.max() <= TOL * rng, "max abs err %.3g of range" % (err.max() / rng)
        assert err.mean() <= TOL * rng
    # the border extrapolation moves material, so the drift is the scheme's
    # own (the same in fp32 and fp64), not the kernels'
    assert abs(_drift(z, z0) - _drift(z64, z0)) <= 1e-6
