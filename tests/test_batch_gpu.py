"""Batched form: many heightmaps of uneven sizes and iteration counts in one
batch give, job by job, the oracle's results (bit-exact where the single
solves are; within the vpipes tolerance with the water-volume top-up)."""
import numpy as np
import pytest

from highmap_b200.inputs import fbm
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

CONFIG2 = dict(maintain_water_volume=0, flux_diffusion=0, dt=0.1, k_capacity=0.05, k_erode=0.01, k_depose=0.01,
               evap_rate=0.01, gravity=9.81, pipe_area=1.0, pipe_length=1.0, rain_per_step=1e-4,
               initial_water=0.0, water_height=1e-2)
FAST = dict(maintain_water_volume=0, flux_diffusion=1, dt=0.5, gravity=40.0, initial_water=0.05)


def _specs():
    """(kind, nx, ny, iterations, options) of a mixed batch."""
    return [
        ("thermal", 130, 257, 37, dict(talus="map", bedrock=True, depo=True)),
        ("thermal", 64, 64, 5, dict(talus=0.02)),
        ("thermal", 3, 3, 4, dict(talus=0.01)),
        ("thermal", 300, 90, 0, dict(talus=0.01, depo=True)),
        ("vpipes", 333, 300, 40, dict(params=CONFIG2)),
        ("vpipes", 128, 200, 25, dict(params=dict(), outputs=True)),
        ("vpipes", 131, 97, 33, dict(params=dict(maintain_water_volume=0), rain=True, outputs=True)),
        ("vpipes", 250, 250, 12, dict(params=FAST, outputs=True)),
        ("vpipes", 40, 40, 0, dict(params=dict(), outputs=True)),
    ]


def _make(specs, seed0=30):
    import torch
    from highmap_b200 import batch as B
    jobs, cases = [], []
    for k, (kind, nx, ny, it, o) in enumerate(specs):
        z0 = fbm(nx, ny, seed=seed0 + k)
        z = torch.from_numpy(z0.copy()).cuda()
        case = dict(kind=kind, z0=z0, z=z, it=it, o=o)
        if kind == "thermal":
            if o["talus"] == "map":
                t = ((0.5 + fbm(nx, ny, seed=seed0 + 100 + k)) / nx).astype(np.float32)
                case["talus"] = t
                talus = torch.from_numpy(t).cuda()
            else:
                case["talus"] = np.float32(o["talus"])
                talus = float(o["talus"])
            bed = None
            if o.get("bedrock"):
                case["bed"] = (0.3 * z0).astype(np.float32)
                bed = torch.from_numpy(case["bed"]).cuda()
            depo = torch.empty_like(z) if o.get("depo") else None
            case["depo"] = depo
            jobs.append(B.thermal_job(z, talus, it, bedrock=bed, deposition_map=depo))
        else:
            rain = None
            if o.get("rain"):
                case["rain"] = (0.25 + fbm(nx, ny, seed=seed0 + 200 + k)).astype(np.float32)
                rain = torch.from_numpy(case["rain"]).cuda()
            outs = [torch.empty_like(z) for _ in range(4)] if o.get("outputs") else [None] * 4
            case["outs"] = outs
            jobs.append(B.vpipes_job(z, it, rain, *outs, **o["params"]))
        cases.append(case)
    return jobs, cases


def _verify(cases):
    for c in cases:
        z0, it, o = c["z0"], c["it"], c["o"]
        got = c["z"].cpu().numpy()
        rng = float(z0.max() - z0.min())
        if c["kind"] == "thermal":
            talus = c["talus"] if isinstance(c["talus"], np.ndarray) else np.full_like(z0, c["talus"])
            want, depo = po.thermal(z0, talus, it, bedrock=c.get("bed"), deposition=True)
            assert np.array_equal(got, want), (z0.shape, it)
            if c["depo"] is not None:
                assert np.array_equal(c["depo"].cpu().numpy(), depo)
        else:
            p = po.VpipesParams.make(**dict(o["params"], iterations=it))
            want = po.vpipes(z0, p, rain_map=c.get("rain"))
            exact = not p.maintain_water_volume
            if exact:
                assert np.array_equal(got, want[0]), (z0.shape, it)
            else:
                assert np.abs(got - want[0]).max() <= 1e-3 * rng
            if o.get("outputs"):
                for t, w in zip(c["outs"], want[1:]):
                    g = t.cpu().numpy()
                    if exact:
                        assert np.array_equal(g, w), (z0.shape, it)
                    else:
                        assert np.abs(g - w).max() <= 1e-3 * max(rng, float(np.abs(w).max()))


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_run_matches_oracle(gpu, use_graph):
    import torch
    from highmap_b200 import batch as B
    jobs, cases = _make(_specs())
    B.run(jobs, use_graph=use_graph)
    torch.cuda.synchronize()
    _verify(cases)


@pytest.mark.parametrize("per_sm", [0, 4, 1])
def test_round_launch_modes(gpu, tmp_path, per_sm):
    """The rounds launched as one CTA per tile (per_sm 0) or as persistent
    CTAs (1 or 4 per SM), chosen through a launch-shape table: every job
    still gives the oracle's bits."""
    import torch
    from highmap_b200 import batch as B
    from highmap_b200 import tune
    t = tmp_path / "batch.txt"
    t.write_text("batch 0 0 %d 0 16 0 1.0\n" % per_sm)
    tune.clear()
    try:
        assert tune.load(str(t)) == 1
        for use_graph in (True, False):
            jobs, cases = _make(_specs(), seed0=90)
            B.run(jobs, use_graph=use_graph)
            torch.cuda.synchronize()
            _verify(cases)
    finally:
        tune.clear()


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_run_with_large_jobs(gpu, use_graph):
    """Jobs of at least 2^20 cells run through the plain solvers on a side
    stream beside the rounds of the smaller ones (here also grids of 2^18
    cells and more, batched); every job still gives the oracle's bits (the
    oracle on the large grids is bounded by the iteration counts)."""
    import torch
    from highmap_b200 import batch as B
    specs = [("thermal", 1024, 1024, 9, dict(talus="map", bedrock=True, depo=True)),
             ("vpipes", 1032, 1024, 6, dict(params=CONFIG2, outputs=True)),
             ("vpipes", 1024, 1040, 5, dict(params=dict(), outputs=True)),
             ("thermal", 600, 520, 7, dict(talus=0.02)),
             ("vpipes", 512, 512, 11, dict(params=FAST, outputs=True)),
             ("thermal", 96, 80, 12, dict(talus=0.02)),
             ("vpipes", 120, 88, 14, dict(params=CONFIG2, outputs=True))]
    jobs, cases = _make(specs, seed0=70)
    B.run(jobs, use_graph=use_graph)
    torch.cuda.synchronize()
    _verify(cases)


def test_cancelled_job_leaves_the_others_exact(gpu):
    """A job released before it finishes (a cancelled request) leaves the
    rounds at once; the jobs beside it finish with the oracle's bits and the
    batch's device memory returns to what the others hold."""
    import torch
    from highmap_b200 import batch as B
    specs = [("vpipes", 200, 136, 30, dict(params=CONFIG2, outputs=True)),
             ("vpipes", 264, 200, 40, dict(params=CONFIG2)),
             ("thermal", 160, 120, 35, dict(talus="map", bedrock=True, depo=True)),
             ("thermal", 320, 96, 45, dict(talus=0.02))]
    jobs, cases = _make(specs, seed0=80)
    b = B.Batch()
    ids = [b.add(j) for j in jobs]
    b.step(6)
    cancelled = (ids[1], ids[3])
    for i in cancelled:
        assert not b.status(i)[1]
        b.release(i)
    keep = [k for k in range(len(ids)) if ids[k] not in cancelled]
    assert b.bytes_in_use() == sum(B.job_bytes(jobs[k]) for k in keep)
    while any(not b.status(ids[k])[1] for k in keep):
        b.step(5)
    b.synchronize()
    torch.cuda.synchronize()
    _verify([cases[k] for k in keep])
    b.close()


def test_evict_and_restore_is_bit_identical(gpu):
    """Jobs moved to host memory mid-run (eviction under an HBM budget) and
    admitted again later go on from the step they had reached: every job,
    evicted or not, ends with the oracle's bits, and the evicted jobs stop
    counting against the batch's device memory while they are out."""
    import torch
    from highmap_b200 import batch as B
    specs = [("vpipes", 200, 136, 30, dict(params=CONFIG2, outputs=True)),
             ("vpipes", 136, 120, 26, dict(params=dict(), outputs=True)),
             ("thermal", 160, 120, 35, dict(talus="map", bedrock=True, depo=True)),
             ("thermal", 96, 200, 28, dict(talus=0.02))]
    jobs, cases = _make(specs, seed0=90)
    b = B.Batch()
    ids = [b.add(j) for j in jobs]
    b.step(7)
    full = b.bytes_in_use()
    snaps = {}
    for k in (1, 2):
        steps_before = b.status(ids[k])[0]
        snaps[k] = b.evict(ids[k])
        assert b.status(ids[k]) == (steps_before, False)
    assert b.bytes_in_use() == full - B.job_bytes(jobs[1]) - B.job_bytes(jobs[2])
    b.step(9)  # the others advance; the evicted two do not
    assert b.status(ids[1])[0] == 7 and b.status(ids[2])[0] == 7
    for k in (2, 1):
        b.restore(ids[k], snaps[k])
    assert b.bytes_in_use() == full
    while any(not b.status(i)[1] for i in ids):
        b.step(6)
    b.synchronize()
    torch.cuda.synchronize()
    _verify(cases)
    b.close()


def test_staggered_admission(gpu):
    """Jobs admitted at different rounds (as the served form admits them)
    still each see their own step sequence."""
    import torch
    from highmap_b200 import batch as B
    specs = _specs()
    jobs, cases = _make(specs, seed0=60)
    b = B.Batch()
    ids = []
    order = [4, 0, 5, 1, 6, 2, 7, 3, 8]
    for n, k in enumerate(order):
        ids.append(b.add(jobs[k]))
        b.step(3 + n)
    while any(not b.status(i)[1] for i in ids):
        b.step(7)
    b.synchronize()
    torch.cuda.synchronize()
    for i in ids:
        steps, done = b.status(i)
        assert done
    _verify(cases)
    before = b.bytes_in_use()
    assert before > 0
    for i in ids:
        b.release(i)
    assert b.bytes_in_use() == 0
    b.close()


def test_vpipes_admitted_after_thermal_only_rounds(gpu):
    """A vpipes job admitted after rounds in which only thermal jobs ran
    (its predecessor finished and was released, as in the served form)
    starts with a clean deferred-advection list: the rounds without vpipes
    tiles re-arm the list's count, so no entry of the released job is
    replayed.  Both later jobs match the oracle."""
    import torch
    from highmap_b200 import batch as B
    specs = [("vpipes", 250, 250, 12, dict(params=FAST, outputs=True)),
             ("thermal", 300, 300, 60, dict(talus=0.01)),
             ("vpipes", 260, 240, 15, dict(params=FAST, outputs=True))]
    jobs, cases = _make(specs, seed0=90)
    b = B.Batch()
    first = b.add(jobs[0])
    therm = b.add(jobs[1])
    while not b.status(first)[1]:
        b.step(1)
    b.synchronize()
    b.release(first)
    b.step(5)  # thermal only
    second = b.add(jobs[2])
    while not (b.status(therm)[1] and b.status(second)[1]):
        b.step(4)
    b.synchronize()
    torch.cuda.synchronize()
    _verify(cases[1:])
    b.close()


def test_job_bytes_accounts_state(gpu):
    import torch
    from highmap_b200 import batch as B
    z = torch.zeros((100, 120), device="cuda")
    jt = B.thermal_job(z, 0.01, 10)
    jv = B.vpipes_job(z, 10)
    assert B.job_bytes(jt) >= 120 * 100 * 4
    assert B.job_bytes(jv) >= 13 * 120 * 100 * 4


def test_served_loop_completes_every_request(gpu):
    """The served form's loop on the device: a short Poisson stream, the
    larger requests through the plain lane beside the batch; every request
    completes once and the work is counted once."""
    from highmap_b200 import forms as F
    reqs = F.serve_requests(12, 200.0, seed=5, lo=64, hi=1024, it_lo=5, it_hi=60)
    pool = F.FieldPool(count=2, side=1024)
    lat, cells, total = F.serve(reqs, pool, large_cells=512 * 512, rounds_per_tick=8)
    assert sorted(lat) == [r["id"] for r in reqs]
    assert all(v >= 0 for v in lat.values())
    assert any(r["nx"] * r["ny"] >= 512 * 512 for r in reqs) and any(r["nx"] * r["ny"] < 512 * 512 for r in reqs)
    assert cells == sum(r["nx"] * r["ny"] * r["iterations"] for r in reqs)
    assert total > 0
