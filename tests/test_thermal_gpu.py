"""GPU parity of the thermal solver against the oracle, through the C-ABI.

The GPU kernels evaluate the reference's fp32 arithmetic one rounding per
operation, so the bar here is bit-exact equality with the oracle (which is
itself bit-exact with the reference's kernel text, tests/test_oracle.py);
the thermal tolerance (max abs error <= 1e-4 of the height range) is
checked as well so a failure reports its size.
"""
import json
import os

import numpy as np
import pytest

from highmap_b200.inputs import fbm
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-4  # of the height range, thermal


def _assert_parity(got, want, z0):
    rng = float(z0.max() - z0.min()) or 1.0
    err = float(np.abs(got.astype(np.float64) - want).max())
    assert err <= TOL * rng, "max abs err %.3g > %.3g" % (err, TOL * rng)
    assert np.array_equal(got, want), "within tolerance (%.3g) but not bit-exact" % err


@pytest.mark.parametrize("name", ["thermal_uniform", "thermal_talus_map", "thermal_masked",
                                  "thermal_small_3x3", "thermal_small_5x17", "thermal_small_33x7"])
def test_golden(gpu, name):
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    z = g["z"].copy()
    depo = np.empty_like(z)
    gpu.thermal(z, g["talus"], int(g["iterations"]), deposition_map=depo, mask=g.get("mask"))
    _assert_parity(z, g["out_z"], g["z"])
    _assert_parity(depo, g["out_depo"], g["z"])


def test_golden_bedrock_literal(gpu):
    g = dict(np.load(os.path.join(GOLDEN, "thermal_bedrock_literal.npz")))
    z = g["z"].copy()
    depo = np.empty_like(z)
    gpu.thermal(z, g["talus"], int(g["iterations"]), bedrock=g["bedrock"], deposition_map=depo,
                bedrock_mode=gpu.BEDROCK_LITERAL)
    _assert_parity(z, g["out_z"], g["z"])
    _assert_parity(depo, g["out_depo"], g["z"])


@pytest.mark.parametrize("time_block", [1, 0, 2, 4, 8])
@pytest.mark.parametrize("shape", [(256, 256), (130, 257), (77, 190), (9, 300)])
@pytest.mark.parametrize("variant", ["map", "scalar", "bedrock", "literal", "mask"])
def test_against_oracle(gpu, shape, variant, time_block):
    ny, nx = shape
    z0 = fbm(nx, ny, seed=2)
    talus = ((0.5 + fbm(nx, ny, seed=3)) / nx).astype(np.float32)
    kw = dict(deposition=True)
    gkw = {}
    iters = 37
    if variant == "scalar":
        talus_arg = np.float32(1.0 / nx)
        talus_o = np.full_like(z0, talus_arg)
    else:
        talus_arg = talus_o = talus
    if variant in ("bedrock", "literal"):
        bed = (0.3 * z0 + 0.2 * fbm(nx, ny, seed=8)).astype(np.float32)
        kw["bedrock"] = gkw["bedrock"] = bed
        mode = po.BEDROCK_LITERAL if variant == "literal" else po.BEDROCK_INTENDED
        kw["bedrock_mode"] = gkw["bedrock_mode"] = mode
    if variant == "mask":
        kw["mask"] = gkw["mask"] = fbm(nx, ny, seed=6)
    want_z, want_d = po.thermal(z0, talus_o, iters, **kw)
    z = z0.copy()
    depo = np.empty_like(z)
    gpu.thermal(z, float(talus_arg) if variant == "scalar" else talus_arg, iters, deposition_map=depo,
                time_block=time_block, **gkw)
    _assert_parity(z, want_z, z0)
    _assert_parity(depo, want_d, z0)


@pytest.mark.parametrize("iters", [0, 1, 2, 3])
def test_few_iterations(gpu, iters):
    z0 = fbm(64, 40, seed=9)
    want, _ = po.thermal(z0, 0.01, iters)
    z = z0.copy()
    gpu.thermal(z, 0.01, iters)
    _assert_parity(z, want, z0)


def test_deterministic(gpu):
    z0 = fbm(300, 200, seed=4)
    a = z0.copy()
    b = z0.copy()
    gpu.thermal(a, 1 / 300, 50)
    gpu.thermal(b, 1 / 300, 50)
    assert a.tobytes() == b.tobytes()


def test_device_api_matches_host_api(gpu):
    import torch
    z0 = fbm(512, 384, seed=5)
    talus = ((0.5 + fbm(512, 384, seed=6)) / 512).astype(np.float32)
    bed = (0.3 * z0).astype(np.float32)
    h = z0.copy()
    gpu.thermal(h, talus, 25, bedrock=bed)
    dz = torch.from_numpy(z0.copy()).cuda()
    gpu.thermal_device(dz, torch.from_numpy(talus).cuda(), 25, bedrock=torch.from_numpy(bed).cuda())
    torch.cuda.synchronize()
    assert np.array_equal(dz.cpu().numpy(), h)


@pytest.mark.parametrize("offset", [0, 1])
@pytest.mark.parametrize("nx", [512, 390, 391])
def test_device_buffer_alignment(gpu, offset, nx):
    """Even rows on 8-byte aligned grids go through the column-pair sweep,
    odd rows or grids one float off alignment through the one-column
    sweep; every case gives the oracle's bits."""
    import torch
    ny = 70
    z0 = fbm(nx, ny, seed=7)
    talus = ((0.5 + fbm(nx, ny, seed=8)) / nx).astype(np.float32)
    bed = (0.3 * z0).astype(np.float32)
    want, _ = po.thermal(z0, talus, 21, bedrock=bed)

    def dev(x):
        buf = torch.zeros(x.size + 1, device="cuda")
        t = buf[offset:offset + x.size].view(x.shape)
        t.copy_(torch.from_numpy(x))
        return t
    dz, dt, db = dev(z0), dev(talus), dev(bed)
    gpu.thermal_device(dz, dt, 21, bedrock=db, time_block=1)
    torch.cuda.synchronize()
    assert np.array_equal(dz.cpu().numpy(), want)


def test_bad_arguments_raise(gpu):
    z = np.zeros((2, 8), np.float32)
    with pytest.raises(gpu.HMError):
        gpu.thermal(z, 0.1, 3)
    z = np.zeros((8, 8), np.float32)
    with pytest.raises(gpu.HMError):
        gpu.thermal(z, 0.1, -1)


def test_full_size_config_properties(gpu):
    """4096^2 with the configuration of the plain drop-in benchmark (talus
    map, bedrock 0.3 z, 500 iterations): bedrock respected, deterministic,
    and a 512-row band checked bit-exact against the oracle after 40
    iterations (a band 2*40 rows taller than its checked middle, so the
    band's own border cannot reach it)."""
    import torch
    n = 4096
    z0 = fbm(n, n, seed=2)
    talus = ((0.5 + fbm(n, n, seed=3)) / n).astype(np.float32)
    bed = (0.3 * z0).astype(np.float32)
    dz = torch.from_numpy(z0).cuda()
    dt = torch.from_numpy(talus).cuda()
    db = torch.from_numpy(bed).cuda()
    a = dz.clone()
    gpu.thermal_device(a, dt, 500, bedrock=db)
    b = dz.clone()
    gpu.thermal_device(b, dt, 500, bedrock=db)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    ai = a[1:-1, 1:-1]
    assert bool((ai >= db[1:-1, 1:-1]).all())
    # band check
    iters = 40
    c = dz.clone()
    gpu.thermal_device(c, dt, iters, bedrock=db)
    torch.cuda.synchronize()
    r0, r1 = 1800, 1800 + 512
    band = slice(r0 - iters - 1, r1 + iters + 1)
    want, _ = po.thermal(z0[band], talus[band], iters, bedrock=bed[band])
    got = c.cpu().numpy()[r0:r1, 1:-1]
    assert np.array_equal(got, want[iters + 1:iters + 1 + 512, 1:-1])
