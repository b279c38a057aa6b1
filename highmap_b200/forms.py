"""Workloads and measurement of the batched and served forms.

Batched form: many heightmaps of uneven sizes and iteration counts run as
one batch (hm_batch_run, one CUDA graph) against the same jobs solved one
call at a time with the plain device path (hm_thermal_device /
hm_vpipes_device), both on device-resident inputs.

Served form: a request loop, as an interactive node-graph editor would
drive it: requests arrive as a Poisson stream; small ones are admitted
into an open batch while their device state fits an HBM budget, advance
together a few rounds per tick (continuous batching) on a high-priority
stream and are retired when done, while large ones, which fill the GPU on
their own, run one at a time through the plain path on a low-priority
stream beside them; latency is completion minus arrival.  The same stream
served first-come first-served by the plain path is the comparison
point.

Inputs are seeded synthetic fBm fields (highmap_b200.inputs).
"""
from __future__ import annotations

import heapq
import math
import time

import numpy as np

from . import batch as B
from . import gpu as G
from .inputs import fbm

VPIPES_BASE = dict(maintain_water_volume=0, flux_diffusion=0, dt=0.1, k_capacity=0.05, k_erode=0.01,
                   k_depose=0.01, evap_rate=0.01, gravity=9.81, pipe_area=1.0, pipe_length=1.0,
                   initial_water=0.0, water_height=1e-2)


# ---------------------------------------------------------------- batched

def batch_specs(n_jobs=256, seed=0, lo=128, hi=2048):
    """Job list of the batched configuration: sides log-uniform in [lo, hi]
    rounded to multiples of 8, aspect ratio up to 2:1, half thermal (talus
    uniform in [0.5, 2] / nx) and half vpipes (rain uniform in [5e-5, 5e-4]
    per step), iterations uniform in [50, 1000], fBm seeds 100 + k."""
    rng = np.random.default_rng(seed)
    specs = []
    for k in range(n_jobs):
        a = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        ratio = rng.uniform(1.0, 2.0)
        if rng.uniform() < 0.5:
            nx, ny = a, a / ratio
        else:
            nx, ny = a / ratio, a
        nx = int(min(hi, max(lo, round(nx / 8) * 8)))
        ny = int(min(hi, max(lo, round(ny / 8) * 8)))
        kind = "thermal" if k % 2 == 0 else "vpipes"
        it = int(rng.integers(50, 1001))
        talus = float(rng.uniform(0.5, 2.0)) / nx
        rain = float(rng.uniform(5e-5, 5e-4))
        specs.append(dict(kind=kind, nx=nx, ny=ny, iterations=it, talus=talus, rain=rain, seed=100 + k))
    return specs


def _inputs(specs):
    return [fbm(s["nx"], s["ny"], seed=s["seed"]) for s in specs]


def _job(s, z):
    if s["kind"] == "thermal":
        return B.thermal_job(z, s["talus"], s["iterations"])
    return B.vpipes_job(z, s["iterations"], **dict(VPIPES_BASE, rain_per_step=s["rain"]))


def _plain(s, z, ctx, stream):
    if s["kind"] == "thermal":
        G.thermal_device(z, s["talus"], s["iterations"], ctx=ctx, stream=stream)
    else:
        p = G.vpipes_params(**dict(VPIPES_BASE, rain_per_step=s["rain"], iterations=s["iterations"]))
        G.hydraulic_vpipes_device(z, p, ctx=ctx, stream=stream)


def _peak_rates(ctx, stream, side=2048, iters=200):
    """Cell-updates/s of one large plain solve of each kind (the plain
    path's speed where launches are not the limit)."""
    import torch
    out = {}
    z0 = torch.from_numpy(fbm(side, side, seed=99)).cuda()
    for kind in ("thermal", "vpipes"):
        s = dict(kind=kind, nx=side, ny=side, iterations=iters, talus=1.0 / side, rain=1e-4)
        z = z0.clone()
        _plain(s, z, ctx, stream)
        z = z0.clone()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _plain(s, z, ctx, stream)
        e1.record()
        torch.cuda.synchronize()
        out[kind] = side * side * iters / (e0.elapsed_time(e1) * 1e-3)
    return out


def run_batch_benchmark(n_jobs=256, seed=0):
    """Aggregate cell-updates/s of the batched run and of plain per-job
    calls on the same jobs, every job's result compared bit for bit.

    Also the ceiling of the ratio on this job mix: the plain path runs a
    large grid near its own per-cell speed, so batching can only win back
    what plain calls lose on grids too small to fill the GPU.  ideal_s is
    the whole mix at the per-cell speed of one large plain solve of each
    kind; plain_s / ideal_s bounds any batched form's speed-up, and the
    per-size breakdown shows where plain calls lose time."""
    import torch
    specs = batch_specs(n_jobs, seed)
    fields = _inputs(specs)
    host = [torch.from_numpy(f) for f in fields]
    cells = sum(s["nx"] * s["ny"] * s["iterations"] for s in specs)
    ctx = G.Context(torch.cuda.current_device())
    stream = torch.cuda.current_stream().cuda_stream
    peak = _peak_rates(ctx, stream)

    # plain: one call per job, device-resident inputs, each timed
    big = max(specs, key=lambda s: s["nx"] * s["ny"])
    for kind in ("thermal", "vpipes"):  # warm the workspace at the largest size
        _plain(dict(big, kind=kind, iterations=2), host[0].new_zeros((big["ny"], big["nx"])).cuda(), ctx, stream)
    torch.cuda.synchronize()
    zs = [h.cuda() for h in host]
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in specs]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for s, z, (a, b) in zip(specs, zs, ev):
        a.record()
        _plain(s, z, ctx, stream)
        b.record()
    e1.record()
    torch.cuda.synchronize()
    plain_s = e0.elapsed_time(e1) * 1e-3
    per_job = [a.elapsed_time(b) * 1e-3 for a, b in ev]

    # batched: every job in one graph-captured batch
    zb = [h.cuda() for h in host]
    jobs = [_job(s, z) for s, z in zip(specs, zb)]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    B.run(jobs, use_graph=True, ctx=ctx)
    torch.cuda.synchronize()
    batch_s = time.perf_counter() - t0
    mismatched = [k for k, (a, b) in enumerate(zip(zb, zs)) if not torch.equal(a, b)]
    del zs, zb
    ctx.close()

    ideal_s = sum(s["nx"] * s["ny"] * s["iterations"] / peak[s["kind"]] for s in specs)
    bands = []
    for lo, hi in ((0, 256 * 256), (256 * 256, 512 * 512), (512 * 512, 1024 * 1024), (1024 * 1024, 1 << 30)):
        idx = [k for k, s in enumerate(specs) if lo <= s["nx"] * s["ny"] < hi]
        if not idx:
            continue
        w = sum(specs[k]["nx"] * specs[k]["ny"] * specs[k]["iterations"] for k in idx)
        t = sum(per_job[k] for k in idx)
        ideal = sum(specs[k]["nx"] * specs[k]["ny"] * specs[k]["iterations"] / peak[specs[k]["kind"]] for k in idx)
        bands.append({"cells_from": lo, "cells_below": hi, "jobs": len(idx), "share_of_work": w / cells,
                      "plain_s": t, "share_of_plain_time": t / plain_s, "plain_over_ideal": t / ideal})
    return {
        "jobs": n_jobs, "cell_updates": cells,
        "batched_cell_updates_per_s": cells / batch_s, "plain_cell_updates_per_s": cells / plain_s,
        "speedup": plain_s / batch_s, "batched_s": batch_s, "plain_s": plain_s,
        "batched_includes": "admission, state init, graph capture and instantiation, all rounds (host clock)",
        "plain_includes": "one device call per job, back to back (CUDA events)",
        "peak_plain_cell_updates_per_s_2048": peak,
        "ideal_s_at_peak_rates": ideal_s, "speedup_ceiling": plain_s / ideal_s,
        "by_size": bands,
        "jobs_compared": n_jobs, "jobs_bit_identical": n_jobs - len(mismatched), "mismatched_jobs": mismatched,
    }


# ---------------------------------------------------------------- served

def serve_requests(n, rate, seed=0, lo=256, hi=4096, it_lo=20, it_hi=2000):
    """Request stream of the served configuration: Poisson arrivals at
    `rate` per second, sides log-uniform in [lo, hi] (multiples of 8),
    50/50 thermal / vpipes, iterations log-uniform in [it_lo, it_hi]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    for rid in range(n):
        t += rng.exponential(1.0 / rate)
        side = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        side = int(max(lo, min(hi, round(side / 8) * 8)))
        it = int(round(math.exp(rng.uniform(math.log(it_lo), math.log(it_hi)))))
        kind = "thermal" if rng.uniform() < 0.5 else "vpipes"
        reqs.append(dict(id=rid, arrival=t, kind=kind, nx=side, ny=side, iterations=it, talus=1.0 / side,
                         rain=1e-4, seed=rid))
    return reqs


class FieldPool:
    """Device-resident source heightmaps: a few large fBm fields; request k
    takes a window of field k % count at an offset drawn from its id."""

    def __init__(self, count=4, side=4096, seed=7):
        import torch
        self.fields = [torch.from_numpy(fbm(side, side, seed=seed + k)).cuda() for k in range(count)]
        self.side = side

    def take(self, rid, nx, ny):
        f = self.fields[rid % len(self.fields)]
        rng = np.random.default_rng(rid)
        ox = int(rng.integers(0, self.side - nx + 1))
        oy = int(rng.integers(0, self.side - ny + 1))
        return f[oy:oy + ny, ox:ox + nx].contiguous()


def _bytes_plain(r):
    """Device workspace a plain solve of request r needs (its grid and the
    solver's scratch), for the admission budget."""
    n = r["nx"] * r["ny"] * 4
    return n * (2 if r["kind"] == "thermal" else 17)


class CudaLanes:
    """The device side of the served loop: an open batch (hm_batch_*) on a
    high-priority stream, and the large lane, plain device calls on a
    low-priority stream.  Jobs are windows of the field pool."""

    def __init__(self, pool):
        import torch
        self._torch = torch
        dev = torch.cuda.current_device()
        self.pool = pool
        self.batch = B.Batch(G.Context(dev))
        self.big_ctx = G.Context(dev)
        self.big_stream = torch.cuda.Stream(priority=0)  # lowest priority

    def start_large(self, r):
        """Launch request r on the large lane; returns a handle."""
        z = self.pool.take(r["id"], r["nx"], r["ny"])
        self._torch.cuda.current_stream().synchronize()
        _plain(r, z, self.big_ctx, self.big_stream.cuda_stream)
        ev = self._torch.cuda.Event()
        ev.record(self.big_stream)
        return (z, ev)

    def large_done(self, handle):
        return handle[1].query()

    def large_bytes(self, r):
        return _bytes_plain(r)

    def make_job(self, r):
        z = self.pool.take(r["id"], r["nx"], r["ny"])
        return (z, _job(r, z))

    def job_bytes(self, job):
        return B.job_bytes(job[1])

    def add(self, job):
        # the window copy runs on torch's stream, the batch on its own
        self._torch.cuda.current_stream().synchronize()
        return self.batch.add(job[1])

    def bytes_in_use(self):
        return self.batch.bytes_in_use()

    def step(self, rounds):
        self.batch.step(rounds)
        self.batch.synchronize()

    def status(self, jid):
        return self.batch.status(jid)

    def release(self, jid):
        self.batch.release(jid)

    def close(self):
        self.batch.close()
        self.big_ctx.close()


def serve(reqs, pool, budget_bytes=120 << 30, rounds_per_tick=64, large_cells=1024 * 1024, lanes=None,
          clock=time.perf_counter, sleep=time.sleep, on_done=None):
    """Size-aware continuous batching: returns per-request latencies (s) and
    totals.

    Requests of at least `large_cells` cells fill the GPU on their own:
    they go, first come first served, through the plain device path on a
    low-priority stream (one at a time; their state stays in the solver's
    workspace).  Smaller requests are admitted into an open batch, in
    arrival order, while their device state and the large lane's fit the
    HBM budget (the first into an empty batch always), advance together a
    few rounds per tick on the batch's high-priority stream, which runs
    beside the large solve, and retire when done.  A tick runs until the
    next batched job completes, at most `rounds_per_tick` rounds (which
    bounds how long an arrival waits for admission).  `lanes` is the device
    side (CudaLanes over `pool` by default); `clock` and `sleep` the time
    source; `on_done(request, handle)` (optional) sees every completed
    request with its lane's handle, whose first item is the result grid."""
    own = lanes is None
    if own:
        lanes = CudaLanes(pool)
    pending = list(reqs)
    waiting = []     # arrived small requests, not admitted (FIFO)
    big_queue = []   # arrived large requests (FIFO)
    big = None       # (request, handle) of the running large solve
    active = {}      # job id -> (request, job)
    lat = {}
    t0 = clock()
    cells = 0
    while pending or waiting or active or big_queue or big:
        now = clock() - t0
        while pending and pending[0]["arrival"] <= now:
            r = pending.pop(0)
            (big_queue if r["nx"] * r["ny"] >= large_cells else waiting).append(r)
        # the large lane: start the next large solve when the lane is free
        if big is not None and lanes.large_done(big[1]):
            r = big[0]
            lat[r["id"]] = clock() - t0 - r["arrival"]
            cells += r["nx"] * r["ny"] * r["iterations"]
            if on_done:
                on_done(r, big[1])
            big = None
        if big is None and big_queue:
            r = big_queue.pop(0)
            big = (r, lanes.start_large(r))
        big_bytes = lanes.large_bytes(big[0]) if big is not None else 0
        while waiting:
            r = waiting[0]
            job = lanes.make_job(r)
            if active and lanes.bytes_in_use() + lanes.job_bytes(job) + big_bytes > budget_bytes:
                break
            waiting.pop(0)
            active[lanes.add(job)] = (r, job)
        if not active:
            if big is not None:
                sleep(0.0002)
            elif pending:
                sleep(max(0.0, min(0.01, pending[0]["arrival"] - now)))
            continue
        nearest = min(r["iterations"] - lanes.status(jid)[0] for jid, (r, _) in active.items())
        lanes.step(max(1, min(nearest, rounds_per_tick)))
        done_t = clock() - t0
        for jid in list(active):
            if lanes.status(jid)[1]:
                r, job = active.pop(jid)
                lat[r["id"]] = done_t - r["arrival"]
                cells += r["nx"] * r["ny"] * r["iterations"]
                if on_done:
                    on_done(r, job)
                lanes.release(jid)
    total = clock() - t0
    if own:
        lanes.close()
    return lat, cells, total


def serve_plain(reqs, pool):
    """First-come first-served, one plain call per request."""
    import torch
    ctx = G.Context(torch.cuda.current_device())
    stream = torch.cuda.current_stream().cuda_stream
    lat = {}
    t0 = time.perf_counter()
    cells = 0
    for r in reqs:
        now = time.perf_counter() - t0
        if r["arrival"] > now:
            time.sleep(r["arrival"] - now)
        z = pool.take(r["id"], r["nx"], r["ny"])
        _plain(r, z, ctx, stream)
        torch.cuda.synchronize()
        lat[r["id"]] = time.perf_counter() - t0 - r["arrival"]
        cells += r["nx"] * r["ny"] * r["iterations"]
    total = time.perf_counter() - t0
    ctx.close()
    return lat, cells, total


def _pct(v, q):
    return float(np.percentile(np.asarray(v), q)) if v else None


def run_serve_benchmark(n_requests=10000, rates=(40.0, 120.0), seed=0, sample_every=100):
    """Throughput and p50/p99 latency of the served form and of the plain
    path (first come first served, one call per request) for each arrival
    rate, on the same request stream.  Every `sample_every`-th request's
    served result is kept and compared with the same request solved alone
    by the plain path: bit-identical count and max abs difference as a
    fraction of the request's input height range."""
    import torch
    pool = FieldPool()
    out = []
    for rate in rates:
        reqs = serve_requests(n_requests, rate, seed)
        kept = {}

        def keep(r, handle):
            if r["id"] % sample_every == 0:
                kept[r["id"]] = (r, handle[0])
        lat_b, cells_b, tot_b = serve(reqs, pool, on_done=keep)
        torch.cuda.synchronize()
        lat_p, cells_p, tot_p = serve_plain(reqs, pool)
        # served results against the plain path, request by request
        ctx = G.Context(torch.cuda.current_device())
        same, worst = 0, 0.0
        for rid, (r, z) in sorted(kept.items()):
            z0 = pool.take(r["id"], r["nx"], r["ny"])
            w = z0.clone()
            _plain(r, w, ctx, torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            rng = float(z0.max() - z0.min()) or 1.0
            worst = max(worst, float((w - z).abs().max()) / rng)
            same += int(torch.equal(w, z))
        ctx.close()
        lb, lp = list(lat_b.values()), list(lat_p.values())
        out.append({
            "rate_per_s": rate, "requests": n_requests, "completed": {"served": len(lb), "plain": len(lp)},
            "served": {"cell_updates_per_s": cells_b / tot_b, "p50_s": _pct(lb, 50), "p99_s": _pct(lb, 99),
                       "wall_s": tot_b},
            "plain": {"cell_updates_per_s": cells_p / tot_p, "p50_s": _pct(lp, 50), "p99_s": _pct(lp, 99),
                      "wall_s": tot_p},
            "throughput_ratio": (cells_b / tot_b) / (cells_p / tot_p),
            "vs_plain": {"sampled": len(kept), "bit_identical": same, "max_abs_of_range": worst},
        })
        del kept
        torch.cuda.empty_cache()
    return {"sweep": out}
