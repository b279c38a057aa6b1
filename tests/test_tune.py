"""The launch-shape autotuner: tuned shapes are valid candidates, results
do not depend on them, and the table survives a save / load round trip."""
import numpy as np
import pytest

from highmap_b200.inputs import fbm
from oracle import pyoracle as po


def test_load_skips_invalid_lines(built_lib, tmp_path):
    from highmap_b200 import tune
    p = tmp_path / "shapes.txt"
    p.write_text("# header\n"
                 "vpipes 9 9 128 2 64 0 0.100\n"
                 "vpipes 10 10 999 2 64 0 0.100\n"      # unsupported threads per CTA
                 "thermal 9 9 0 0 128 8 0.050\n"
                 "thermal 9 8 0 0 128 99 0.050\n"       # unsupported block depth
                 "batch 0 0 2 0 16 0 0.300\n"
                 "batch 0 0 7 0 16 0 0.300\n"           # unsupported CTAs per SM
                 "garbage line\n")
    tune.clear()
    assert tune.load(str(p)) == 3
    out = tmp_path / "out.txt"
    tune.save(str(out))
    lines = [l for l in out.read_text().splitlines() if not l.startswith("#")]
    assert sorted(l.split()[0] for l in lines) == ["batch", "thermal", "vpipes"]
    assert "batch 0 0 2 0 16 0" in out.read_text()
    tune.clear()


def test_load_time_block_and_one_tile_entries(built_lib, tmp_path):
    """Vpipes entries of the tiled kernels keep their steps per launch (0, 1
    or 2; others are refused), and a batch entry with 0 CTAs per SM (one CTA
    per tile of a round) is accepted."""
    from highmap_b200 import tune
    p = tmp_path / "shapes.txt"
    p.write_text("vpipes 10 10 0 0 0 2 0.200\n"
                 "vpipes 11 11 0 0 0 3 0.200\n"         # unsupported steps per launch
                 "batch 0 0 0 0 32 0 0.300\n")
    tune.clear()
    try:
        assert tune.load(str(p)) == 2
        out = tmp_path / "out.txt"
        tune.save(str(out))
        text = out.read_text()
        assert "vpipes 10 10 0 0 0 2" in text and "vpipes 11 11" not in text
        assert "batch 0 0 0 0 32 0" in text
    finally:
        tune.clear()


@pytest.mark.gpu
def test_autotune_then_parity(gpu, tmp_path):
    from highmap_b200 import tune
    tune.clear()
    rv = tune.autotune(tune.VPIPES, 300, 260, steps=6)
    rt = tune.autotune(tune.THERMAL, 300, 260, steps=6)
    assert (rv["tpb"], rv["radius"], rv["rows"]) == (0, 0, 0) or (
        rv["tpb"] in (128, 256) and rv["radius"] in (2, 3) and rv["rows"] >= 32)
    assert rt["time_block"] in (1, 2, 4, 8)
    assert rv["ms_per_step"] > 0 and rt["ms_per_step"] > 0
    # the tuned shapes are used for this size class; results stay the oracle's
    z0 = fbm(300, 260, seed=3)
    z = z0.copy()
    gpu.thermal(z, 1 / 300, 21)
    want, _ = po.thermal(z0, np.full_like(z0, 1 / 300, dtype=np.float32), 21)
    assert np.array_equal(z, want)
    cfg = dict(maintain_water_volume=0, flux_diffusion=0, dt=0.1, gravity=9.81, rain_per_step=1e-4,
               initial_water=0.0, iterations=30)
    z = z0.copy()
    gpu.hydraulic_vpipes(z, **cfg)
    want = po.vpipes(z0, po.VpipesParams.make(**cfg))[0]
    assert np.array_equal(z, want)
    p = tmp_path / "t.txt"
    tune.save(str(p))
    tune.clear()
    assert tune.load(str(p)) == 2
    tune.clear()


@pytest.mark.gpu
def test_autotune_batch_then_bit_identical(gpu):
    """The batched form's tuner picks a valid occupancy and thermal tile
    height; a batch run with that choice still equals solo solves."""
    import torch

    from highmap_b200 import batch as B
    from highmap_b200 import tune
    tune.clear()
    r = tune.autotune(tune.BATCH, 512, 512, steps=4)
    assert r["tpb"] in (0, 1, 2, 3, 4) and r["rows"] in (8, 16, 32) and r["ms_per_step"] > 0
    assert r["candidates"] == 15
    specs = [("thermal", 200, 136, 23), ("vpipes", 264, 136, 17), ("vpipes", 96, 40, 9), ("thermal", 72, 520, 31)]
    zs, jobs, solo = [], [], []
    cfg = dict(maintain_water_volume=0, flux_diffusion=0, dt=0.1, gravity=9.81, rain_per_step=1e-4,
               initial_water=0.0)
    for k, (kind, nx, ny, it) in enumerate(specs):
        z0 = torch.from_numpy(fbm(nx, ny, seed=30 + k)).cuda()
        z = z0.clone()
        zs.append(z)
        jobs.append(B.thermal_job(z, 1.0 / nx, it) if kind == "thermal" else B.vpipes_job(z, it, **cfg))
        w = z0.clone()
        if kind == "thermal":
            gpu.thermal_device(w, 1.0 / nx, it)
        else:
            gpu.hydraulic_vpipes_device(w, gpu.vpipes_params(**dict(cfg, iterations=it)))
        solo.append(w)
    B.run(jobs, use_graph=True)
    torch.cuda.synchronize()
    for z, w in zip(zs, solo):
        assert torch.equal(z, w)
    tune.clear()
