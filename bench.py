"""Benchmark of the plain GPU drop-ins at 4096^2 fp32.

Workload of one step (the reference's headline configuration): on one
4096 x 4096 fBm heightmap (seed 2, kw 4, 8 octaves, remapped to [0, 1])
  * thermal: talus map (0.5 + fBm seed 3) / 4096, bedrock 0.3 z,
    500 iterations, then the border extrapolation;
  * vpipes: water starts at 0, rain 1e-4 per step, dt 0.1, pipe area 1,
    gravity 9.81, k_capacity 0.05, k_erode = k_depose = 0.01, evaporation
    0.01, no volume top-up, no flux diffusion, 1000 iterations.
Metric: cell-updates/s = cells x (500 + 1000) per step / step time.

value  : inputs resident in HBM, CUDA events on the launch stream, max over
         ranks.
e2e    : the same step through the host-buffer C-ABI (hm_thermal, hm_vpipes)
         from pinned host memory: uploads and downloads inside the timing.
roofline: the dominant kernel (vpipes, 56 algorithmic bytes per
         cell-update) timed live with CUDA events inside the timed region.
cpu_baseline: the reference's kernel text compiled for the CPU
         (oracle/_ref, all host threads) on a bounded sample, scaled to the
         same metric.

Multi-GPU: the solvers do not shard (one heightmap per call); every rank
runs an independent replica (scaling "weak"), value = all ranks' cell
updates / max-over-ranks time.

`--impl reference` times the reference's CPU implementation of the path
(oracle/_ref) on the host cores with the same metric; under torchrun only
rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_SIDE = 4096
THERMAL_ITERS = 500
VPIPES_ITERS = 1000
VPIPES_BYTES = 56.0   # algorithmic bytes per vpipes cell-update (7 fields in + out)
THERMAL_BYTES = 16.0  # z, talus, bedrock in; z out
CONFIG2_VPIPES = dict(maintain_water_volume=0, flux_diffusion=0, dt=0.1, k_capacity=0.05, k_erode=0.01,
                      k_depose=0.01, evap_rate=0.01, gravity=9.81, pipe_area=1.0, pipe_length=1.0,
                      rain_per_step=1e-4, initial_water=0.0, water_height=1e-2)
METRIC = "cell-updates/s at 4096^2 fp32 (thermal 500 + vpipes 1000 iterations per step)"


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--size", type=int, default=N_SIDE)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--form", choices=["plain", "batch", "serve", "sweep", "extras", "parity", "tblock"],
                    default="plain",
                    help="plain: the drop-in headline; batch: 256 mixed jobs batched vs plain calls; "
                         "serve: Poisson request stream, continuous batching vs plain FIFO; "
                         "sweep: thermal and vpipes at 1024^2..16384^2, 200 iterations, rates and errors; "
                         "extras: thermal_auto_bedrock, flow_simulation and the sibling talus stencils at 4096^2; "
                         "parity: thermal x500 and vpipes x1000 at 4096^2, GPU vs the reference's kernel text and "
                         "fp64 on the host cores; tblock: vpipes at one and at two steps per launch (temporal "
                         "blocking) on the --sizes grids, device-timed, with the autotuner's pick")
    ap.add_argument("--parity-part", choices=["all", "gpu", "host"], default="all",
                    help="parity form: both sides, or only the GPU or host side (sha256 digests link the two)")
    ap.add_argument("--sizes", default="1024,2048,4096,8192,16384", help="grid sides of the sweep form")
    ap.add_argument("--jobs", type=int, default=256, help="jobs of the batch form")
    ap.add_argument("--requests", type=int, default=10000, help="requests per rate of the serve form")
    ap.add_argument("--rates", default="40,120", help="arrival rates (requests/s) of the serve form")
    ap.add_argument("--vpipes-launch", default=None,
                    help="fused vpipes launch shape 'tpb,radius,rows' (default: built-in choice)")
    a = ap.parse_args()
    if a.warmup < 3:
        ap.error("--warmup must be >= 3")
    return a


def _config(n):
    return {
        "workload": "plain drop-ins, %dx%d fp32: thermal (talus map, bedrock 0.3 z) x%d + vpipes x%d"
                    % (n, n, THERMAL_ITERS, VPIPES_ITERS),
        "grid": [n, n],
        "thermal": {"iterations": THERMAL_ITERS, "talus": "(0.5 + fbm seed 3) / nx", "bedrock": "0.3 z",
                    "bedrock_mode": "intended"},
        "vpipes": dict(CONFIG2_VPIPES, iterations=VPIPES_ITERS),
        "inputs": "fBm seed 2 remapped to [0,1] (synthetic, seeded)",
        "l2": "inputs larger than L2 (state 7 x 64 MiB for vpipes, 4 x 64 MiB for thermal)",
        "parallelism": "replicas",
    }


def _inputs(n):
    import numpy as np

    from highmap_b200.inputs import fbm
    z = fbm(n, n, seed=2)
    talus = ((0.5 + fbm(n, n, seed=3)) / n).astype(np.float32)
    bed = (0.3 * z).astype(np.float32)
    return z, talus, bed


# ---------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples of the benchmark GPU during the timed region."""

    Q = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
        except Exception:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=5)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9 or (self.uuid and f[0] != self.uuid):
                continue
            try:
                sm.append(float(f[1].split()[0]))
                smax.append(float(f[2].split()[0]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _vp_kernels(shape):
    """Kernels of one vpipes step for the launch shape in use."""
    if shape and shape.get("tpb"):
        return "k_vp_fused + k_vp_fixup"
    return ("k_vp_step_tma: the previous step's advection folded into this step's tile (the first step is "
            "k_vp_fwe_tma, the last step's advection k_vp_advect)")


def _traffic():
    """DRAM bytes (read + write) of one vpipes step kernel launch at 4096^2
    from the committed ncu summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            t = json.load(f)
        return t.get("vpipes_bytes_per_step_4096")
    except Exception:
        return None


# ---------------------------------------------------------------- cpu

def _cpu_rates(n, budget_s=12.0, use_ref=True):
    """Cell-update rates of the CPU implementation on a bounded sample:
    a few thermal and vpipes iterations on the full n x n inputs, about
    budget_s seconds of work in all.  The per-iteration cost is sized from
    runs of 1 and 3 iterations, so fixed per-call costs (copies, thread
    start-up) do not shrink the sample."""
    import numpy as np

    from oracle import pyoracle as po
    z, talus, bed = _inputs(n)
    if use_ref and po.ref_available():
        kind, th, vp, cores = "reference", po.ref_thermal, po.ref_vpipes, None
    else:
        kind, th, vp, cores = "port", po.thermal, po.vpipes, None

    def t_thermal(k):
        t = time.perf_counter()
        th(z, talus, k, bedrock=bed) if kind == "reference" else th(z, talus, k, bedrock=bed)
        return time.perf_counter() - t

    def t_vpipes(k):
        p = po.VpipesParams.make(**dict(CONFIG2_VPIPES, iterations=k))
        t = time.perf_counter()
        vp(z, p)
        return time.perf_counter() - t

    # per-iteration cost from 1 and 3 iterations, then the sample itself
    t1 = max((t_thermal(3) - t_thermal(1)) / 2, 1e-4)
    v1 = max((t_vpipes(3) - t_vpipes(1)) / 2, 1e-4)
    kt = max(1, int(0.35 * budget_s / t1))
    kv = max(1, int(0.65 * budget_s / v1))
    tt = t_thermal(kt)
    tv = t_vpipes(kv)
    cells = float(n) * n
    rate_t = cells * kt / tt
    rate_v = cells * kv / tv
    cores = po.num_threads()
    return kind, cores, rate_t, rate_v, kt, kv, tt + tv


def _composite(cells, rate_t, rate_v):
    step_s = cells * THERMAL_ITERS / rate_t + cells * VPIPES_ITERS / rate_v
    return cells * (THERMAL_ITERS + VPIPES_ITERS) / step_s


REF_THERMAL_EXTRA = 8  # thermal iterations a reference step adds beyond its 1-iteration call
REF_VPIPES_EXTRA = 4   # vpipes iterations likewise


def run_reference(a):
    """The reference's CPU implementation of the path (its kernel text
    compiled for the host, oracle/_ref; the restatement where that library
    is absent) on all host threads.

    A full step of the workload (500 thermal + 1000 vpipes iterations at
    4096^2) takes minutes on the host, so each timed step is a bounded
    sample of it: one thermal call of 1 iteration and one of
    1 + REF_THERMAL_EXTRA, one vpipes call of 1 and one of
    1 + REF_VPIPES_EXTRA, all on the full inputs.  The per-iteration cost
    of each solver is the difference of the two calls, summed over the
    timed steps, so a call's fixed costs (copies of the inputs, buffer
    set-up, thread start-up) are not charged to its iterations; the
    metric is the composite rate of 500 + 1000 iterations at those
    per-iteration costs.  `ms_per_step` is the measured time of one sample
    step; the time a full workload step would take is extrapolated
    (`workload_ms_per_step_extrapolated`)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import pyoracle as po
    n = a.size
    cells = float(n) * n
    z, talus, bed = _inputs(n)
    use_ref = po.ref_available()
    kind = "reference" if use_ref else "port"
    th = po.ref_thermal if use_ref else po.thermal
    vp = po.ref_vpipes if use_ref else po.vpipes
    mt, mv = REF_THERMAL_EXTRA, REF_VPIPES_EXTRA
    pv_short = po.VpipesParams.make(**dict(CONFIG2_VPIPES, iterations=1))
    pv_long = po.VpipesParams.make(**dict(CONFIG2_VPIPES, iterations=1 + mv))

    def timed(fn):
        t = time.perf_counter()
        fn()
        return time.perf_counter() - t

    def step():
        t1 = timed(lambda: th(z, talus, 1, bedrock=bed))
        tk = timed(lambda: th(z, talus, 1 + mt, bedrock=bed))
        v1 = timed(lambda: vp(z, pv_short))
        vk = timed(lambda: vp(z, pv_long))
        return tk - t1, vk - v1, t1 + tk + v1 + vk

    for _ in range(a.warmup):
        step()
    dt_th = dt_vp = wall = 0.0
    for _ in range(a.steps):
        x, y, w = step()
        dt_th += x
        dt_vp += y
        wall += w
    # guard against a difference at the timer's resolution
    rate_t = cells * mt * a.steps / max(dt_th, 1e-9)
    rate_v = cells * mv * a.steps / max(dt_vp, 1e-9)
    value = _composite(cells, rate_t, rate_v)
    cores = po.num_threads()
    sample = ("each step: thermal calls of 1 and %d iterations and vpipes calls of 1 and %d iterations on the full "
              "%dx%d inputs; per-iteration cost = difference of the two calls (fixed per-call costs excluded), "
              "extrapolated to %d + %d iterations" % (1 + mt, 1 + mv, n, n, THERMAL_ITERS, VPIPES_ITERS))
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * wall / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": _config(n),
        "extrapolated": True,
        "workload_ms_per_step_extrapolated": 1e3 * cells * (THERMAL_ITERS + VPIPES_ITERS) / value,
        "per_solver": {"thermal_cell_updates_per_s": rate_t, "vpipes_cell_updates_per_s": rate_v,
                       "thermal_iterations_differenced": mt * a.steps,
                       "vpipes_iterations_differenced": mv * a.steps},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": cores, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)
    return 0


# ---------------------------------------------------------------- ours

def run_ours(a):
    import numpy as np
    import torch
    import torch.distributed as dist

    from highmap_b200 import gpu as G

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    if not G.init_opencl():
        raise RuntimeError("no usable device: " + G.L.lib().hm_last_error().decode())
    ctx = G.Context(local)
    n = a.size
    cells = float(n) * n
    z, talus, bed = _inputs(n)
    dev = torch.device("cuda", local)
    z0_d = torch.from_numpy(z).to(dev)
    talus_d = torch.from_numpy(talus).to(dev)
    bed_d = torch.from_numpy(bed).to(dev)
    z_th = torch.empty_like(z0_d)
    z_vp = torch.empty_like(z0_d)
    # launch shapes picked by the autotuner for this grid size (part of warm-up)
    from highmap_b200 import tune
    tuned = {"vpipes": tune.autotune(tune.VPIPES, n, n, steps=20, ctx=ctx),
             "thermal": tune.autotune(tune.THERMAL, n, n, steps=40, ctx=ctx)}
    if a.vpipes_launch:  # an explicit shape overrides the tuned one (the tuner clears overrides)
        shape = [int(x) for x in a.vpipes_launch.split(",")]
        G.vpipes_set_launch(*shape)
        tuned["vpipes"] = {"tpb": shape[0], "radius": shape[1], "rows": shape[2], "override": True}
    pv = G.vpipes_params(**dict(CONFIG2_VPIPES, iterations=VPIPES_ITERS))
    stream = torch.cuda.Stream(device=dev)

    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(a.steps)]

    def step(e=None):
        if e:
            e[0].record(stream)
        z_th.copy_(z0_d)
        G.thermal_device(z_th, talus_d, THERMAL_ITERS, bedrock=bed_d, ctx=ctx, stream=stream.cuda_stream)
        if e:
            e[1].record(stream)
        z_vp.copy_(z0_d)
        G.hydraulic_vpipes_device(z_vp, pv, ctx=ctx, stream=stream.cuda_stream)
        if e:
            e[2].record(stream)

    with torch.cuda.stream(stream):
        for _ in range(a.warmup):
            step()
    torch.cuda.synchronize()

    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
        if not uuid.startswith("GPU-"):
            uuid = "GPU-" + uuid
    except Exception:
        uuid = None
    clocks = ClockSampler(uuid)
    clocks.start()
    time.sleep(0.5)

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    G.launch_count_reset()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    # NVTX range "timed": lets a profiler's launch list select exactly these steps
    torch.cuda.nvtx.range_push("timed")
    with torch.cuda.stream(stream):
        t_start.record(stream)
        for k in range(a.steps):
            step(ev[k])
        t_end.record(stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    launches = G.launch_count()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()

    elapsed_ms = t_start.elapsed_time(t_end)
    th_ms = sum(e[0].elapsed_time(e[1]) for e in ev)
    vp_ms = sum(e[1].elapsed_time(e[2]) for e in ev)
    from highmap_b200.replicas import job_rate, max_over_ranks
    elapsed_ms, th_ms, vp_ms = max_over_ranks([elapsed_ms, th_ms, vp_ms], dist if world > 1 else None, dev)

    value = job_rate(world, a.steps, cells * (THERMAL_ITERS + VPIPES_ITERS), elapsed_ms)
    ms_per_step = elapsed_ms / a.steps

    peak, peak_kind = _peaks()
    vp_step_s = vp_ms * 1e-3 / (a.steps * VPIPES_ITERS)
    th_step_s = th_ms * 1e-3 / (a.steps * THERMAL_ITERS)
    achieved = VPIPES_BYTES * cells / vp_step_s / 1e9
    th_achieved = THERMAL_BYTES * cells / th_step_s / 1e9
    traffic = _traffic()

    # e2e through the host-buffer C-ABI, pinned host memory
    e2e = None
    if not a.no_e2e:
        zp = torch.empty((n, n), dtype=torch.float32, pin_memory=True).numpy()
        tp = torch.empty((n, n), dtype=torch.float32, pin_memory=True).numpy()
        bp = torch.empty((n, n), dtype=torch.float32, pin_memory=True).numpy()
        tp[...] = talus
        bp[...] = bed
        vkw = dict(CONFIG2_VPIPES)

        def e2e_step():
            zp[...] = z
            t0 = time.perf_counter()
            G.thermal(zp, tp, THERMAL_ITERS, bedrock=bp, ctx=ctx)
            t1 = time.perf_counter()
            zp[...] = z
            t2 = time.perf_counter()
            G.hydraulic_vpipes(zp, iterations=VPIPES_ITERS, ctx=ctx, **vkw)
            t3 = time.perf_counter()
            return (t1 - t0) + (t3 - t2)

        for _ in range(a.warmup):
            e2e_step()
        if world > 1:
            dist.barrier()
        tot = sum(e2e_step() for _ in range(a.steps))
        tot = max_over_ranks([tot], dist if world > 1 else None, dev)[0]
        e2e = {"value": job_rate(world, a.steps, cells * (THERMAL_ITERS + VPIPES_ITERS), 1e3 * tot),
               "unit": "cell-updates/s",
               "h2d_bytes_per_step": int(4 * cells * 4), "d2h_bytes_per_step": int(2 * cells * 4),
               "ms_per_step": 1e3 * tot / a.steps}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        kind, cores, rt, rv, kt, kv, secs = _cpu_rates(n)
        cpu = {"value": _composite(cells, rt, rv), "unit": "cell-updates/s", "cores": cores, "kind": kind,
               "sample": "%d thermal + %d vpipes iterations on the full %dx%d inputs (%.1f s of CPU time), "
                         "scaled to %d + %d iterations" % (kt, kv, n, n, secs, THERMAL_ITERS, VPIPES_ITERS),
               "thermal_cell_updates_per_s": rt, "vpipes_cell_updates_per_s": rv}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": _config(n),
            "per_solver": {
                "thermal_cell_updates_per_s": world * a.steps * cells * THERMAL_ITERS / (th_ms * 1e-3),
                "vpipes_cell_updates_per_s": world * a.steps * cells * VPIPES_ITERS / (vp_ms * 1e-3),
                "thermal_roofline": {"bound": "hbm", "achieved": th_achieved, "peak": peak, "unit": "GB/s",
                                     "frac": th_achieved / peak, "bytes_per_cell_update": THERMAL_BYTES},
            },
            "roofline": {"bound": "hbm", "kernel": "vpipes step (%s)" % _vp_kernels(tuned["vpipes"]), "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "bytes_per_cell_update": VPIPES_BYTES},
            "e2e": e2e, "cpu_baseline": cpu, "clocks": clk, "gpu_launches": launches,
            "launch_shapes": tuned,
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------- sweep

SWEEP_ITERS = 200
SWEEP_FULL_CHECK = 2048  # sides up to this are checked against the oracle on the whole grid
SWEEP_BAND = 256         # larger sides: the top SWEEP_BAND rows, run by the oracle with a halo


def _errors(got, want, z0):
    """max / mean absolute error (as a fraction of the input height range),
    the relative L1 distance of HighMap's array comparison
    (HighMap/src/dbg/assert.cpp:47-70: sum|a-b| / min(sum|a|, sum|b|)) and
    whether the two fields are bit-identical."""
    import numpy as np
    g = got.astype(np.float64)
    w = want.astype(np.float64)
    d = np.abs(g - w)
    rng = float(z0.max() - z0.min()) or 1.0
    den = min(float(np.abs(g).sum()), float(np.abs(w).sum()))
    return {"max_abs_of_range": float(d.max()) / rng, "mean_abs_of_range": float(d.mean()) / rng,
            "rel_l1": float(d.sum()) / den if den else float(d.sum()), "bit_exact": bool(np.array_equal(got, want))}


def run_sweep(a):
    """Thermal and vpipes (the plain drop-in configuration's parameters) on
    square grids, 200 iterations each, seeds 10.. by size: device-timed
    cell-updates/s and algorithmic GB/s against the measured copy bandwidth,
    the autotuner's launch shapes, mass drift, and errors of the GPU result
    against the fp32 oracle and the fp64 oracle (whole grid up to 2048^2;
    above, the top 256 rows, which the oracle recomputes on a band with a
    halo wider than the information reach)."""
    import numpy as np
    import torch

    from highmap_b200 import gpu as G
    from highmap_b200 import tune
    from highmap_b200.inputs import fbm
    from oracle import pyoracle as po
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if not G.init_opencl():
        raise RuntimeError("no usable device: " + G.L.lib().hm_last_error().decode())
    ctx = G.Context(local)
    dev = torch.device("cuda", local)
    peak, peak_kind = _peaks()
    sizes = [int(x) for x in a.sizes.split(",")]
    it = SWEEP_ITERS
    pv = dict(CONFIG2_VPIPES)
    rows = []
    for k, n in enumerate(sizes):
        seed = 10 + k
        z0 = fbm(n, n, seed=seed)
        talus = ((0.5 + fbm(n, n, seed=seed + 100)) / n).astype(np.float32)
        bed = (0.3 * z0).astype(np.float32)
        shapes = {"vpipes": tune.autotune(tune.VPIPES, n, n, steps=20, ctx=ctx),
                  "thermal": tune.autotune(tune.THERMAL, n, n, steps=40, ctx=ctx)}
        zd = torch.from_numpy(z0).to(dev)
        td = torch.from_numpy(talus).to(dev)
        bd = torch.from_numpy(bed).to(dev)
        zt = torch.empty_like(zd)
        zv = torch.empty_like(zd)
        wd = torch.empty_like(zd)
        sd = torch.empty_like(zd)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        for rep in range(2):  # the first pass warms up
            zt.copy_(zd)
            zv.copy_(zd)
            torch.cuda.synchronize()
            e[0].record()
            G.thermal_device(zt, td, it, bedrock=bd, ctx=ctx)
            e[1].record()
            e[2].record()
            G.hydraulic_vpipes_device(zv, G.vpipes_params(**dict(pv, iterations=it)), None, wd, sd, ctx=ctx)
            e[3].record()
            torch.cuda.synchronize()
        cells = float(n) * n
        t_th = e[0].elapsed_time(e[1]) * 1e-3
        t_vp = e[2].elapsed_time(e[3]) * 1e-3
        got_t = zt.cpu().numpy()
        got_v, got_w, got_s = zv.cpu().numpy(), wd.cpu().numpy(), sd.cpu().numpy()
        row = {"n": n, "seed": seed, "launch_shapes": shapes,
               "thermal": {"cell_updates_per_s": cells * it / t_th,
                           "gb_per_s": THERMAL_BYTES * cells * it / t_th / 1e9,
                           "frac": THERMAL_BYTES * cells * it / t_th / 1e9 / peak,
                           "mass_drift": abs(float(got_t.astype(np.float64).sum() - z0.astype(np.float64).sum())) /
                           float(np.abs(z0.astype(np.float64)).sum())},
               "vpipes": {"cell_updates_per_s": cells * it / t_vp,
                          "gb_per_s": VPIPES_BYTES * cells * it / t_vp / 1e9,
                          "frac": VPIPES_BYTES * cells * it / t_vp / 1e9 / peak,
                          # terrain + suspended sediment (the water itself is not conserved: rain and
                          # evaporation); erosion moves material between the two, advection resamples s
                          "material_drift": abs(float((got_v.astype(np.float64) + got_s).sum()) -
                                                float(z0.astype(np.float64).sum())) /
                          float(np.abs(z0.astype(np.float64)).sum()),
                          "water_depth_max": float(got_w.max())}}
        # errors against the oracle: whole grid, or the top band with a halo
        if n <= SWEEP_FULL_CHECK:
            r1, sl = n, slice(None)
        else:
            r1, sl = SWEEP_BAND + it + 16, slice(0, SWEEP_BAND)
        scope = "whole grid" if n <= SWEEP_FULL_CHECK else "rows 0..%d (oracle on %d rows)" % (SWEEP_BAND - 1, r1)
        ref_t32, _ = po.thermal(z0[:r1], talus[:r1], it, bedrock=bed[:r1])
        ref_t64, _ = po.thermal(z0[:r1], talus[:r1], it, bedrock=bed[:r1], dtype=np.float64)
        pp = po.VpipesParams.make(**dict(pv, iterations=it))
        ref_v32 = po.vpipes(z0[:r1], pp)[0]
        ref_v64 = po.vpipes(z0[:r1], pp, dtype=np.float64)[0]
        row["thermal"]["vs_oracle_fp32"] = _errors(got_t[sl], ref_t32[sl], z0)
        row["thermal"]["vs_oracle_fp64"] = _errors(got_t[sl], ref_t64[sl], z0)
        row["vpipes"]["vs_oracle_fp32"] = _errors(got_v[sl], ref_v32[sl], z0)
        row["vpipes"]["vs_oracle_fp64"] = _errors(got_v[sl], ref_v64[sl], z0)
        row["checked"] = scope
        rows.append(row)
        print(json.dumps({"sweep_row": row}), flush=True)
        del zd, td, bd, zt, zv, wd, sd
        torch.cuda.empty_cache()
    out = {"metric": "cell-updates/s and GB/s vs the HBM roofline, thermal and vpipes, 200 iterations per size",
           "value": max(r["vpipes"]["cell_updates_per_s"] for r in rows), "unit": "cell-updates/s", "n_gpus": 1,
           "higher_is_better": True, "dtype": "f32", "data": "synthetic", "form": "sweep",
           "config": {"workload": "size sweep", "sizes": sizes, "iterations": it, "peak_gbs": peak,
                      "peak_kind": peak_kind, "bytes_per_cell_update": {"thermal": THERMAL_BYTES,
                                                                          "vpipes": VPIPES_BYTES}},
           "rows": rows}
    print(json.dumps(out), flush=True)
    ctx.close()
    return 0


# ---------------------------------------------------------------- parity

def _material(z, s=None):
    """fp64 sum of the terrain (plus suspended sediment for vpipes)."""
    import numpy as np
    t = float(z.astype(np.float64).sum())
    return t + (float(s.astype(np.float64).sum()) if s is not None else 0.0)


def _digest(x):
    import hashlib

    import numpy as np
    return hashlib.sha256(np.ascontiguousarray(x).tobytes()).hexdigest()


def run_parity(a):
    """The plain drop-in configuration at full length on the full grid,
    GPU against the reference's kernel text on the host cores and against
    an fp64 run of the same scheme: thermal (talus map, bedrock 0.3 z,
    500 iterations) and vpipes (1000 iterations) at 4096^2.

    Thermal runs twice: in the bedrock mode the benchmark measures (update,
    then clamp to the bedrock), compared with the fp32 and fp64 oracle (the
    reference text has only the literal mode), and in the reference's
    literal mode, compared with the reference text itself.  Vpipes runs
    twice too: with the benchmark's gravity 9.81, compared with the fp32
    and fp64 oracle (the reference text hard-codes gravity 1, so it cannot
    run this configuration), and with everything else the same but gravity
    1, compared with the reference text itself.  Each
    comparison reports max and mean |difference| as a fraction of the
    input's height range, the relative L1 distance of HighMap's array
    comparison and bit-exactness; mass drift is |sum z_T - sum z_0| /
    sum |z_0| for thermal, the same over terrain plus suspended sediment
    for vpipes (rain and evaporation change the water itself).

    --parity-part gpu runs only the GPU solves and host runs only the
    host-side ones (reference text, fp32 and fp64 oracle and every
    statistic against fp64); each prints sha256 digests of its outputs.
    Where a GPU digest equals the host digest of the same field the two
    results are bit-identical, so every statistic of the host result holds
    for the GPU's.  `all` (the default) runs both and compares directly."""
    import numpy as np

    from oracle import pyoracle as po
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    part = a.parity_part
    n = a.size
    z0, talus, bed = _inputs(n)
    base = _material(z0)
    den = float(np.abs(z0.astype(np.float64)).sum())

    def drift(m):
        return abs(m - base) / den

    out = {"metric": "max/mean abs error (fraction of the height range) and mass drift after the full iteration "
                     "counts, GPU vs the reference's kernel text and vs fp64",
           "unit": "fraction of height range", "higher_is_better": False, "n_gpus": 1, "dtype": "f32",
           "data": "synthetic", "form": "parity", "parity_part": part,
           "tolerance_of_range": {"thermal": 1e-4, "vpipes": 1e-3},
           "config": dict(_config(n), workload="plain drop-ins at full length, %dx%d: thermal x%d, vpipes x%d"
                          % (n, n, THERMAL_ITERS, VPIPES_ITERS)),
           "input_sha256": _digest(z0)}
    gpu = host = None
    if part in ("all", "gpu"):
        import torch

        from highmap_b200 import gpu as G
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        if not G.init_opencl():
            raise RuntimeError("no usable device: " + G.L.lib().hm_last_error().decode())
        ctx = G.Context(int(os.environ.get("LOCAL_RANK", "0")))
        t0 = time.perf_counter()
        # host buffers through the C-ABI, as a caller of the drop-in would
        z_int = z0.copy()
        G.thermal(z_int, talus, THERMAL_ITERS, bedrock=bed, ctx=ctx)
        z_lit = z0.copy()
        G.thermal(z_lit, talus, THERMAL_ITERS, bedrock=bed, bedrock_mode=G.BEDROCK_LITERAL, ctx=ctx)
        gpu = {"thermal_intended": z_int, "thermal_literal": z_lit}
        for tag, kw in (("vpipes", CONFIG2_VPIPES), ("vpipes_g1", dict(CONFIG2_VPIPES, gravity=1.0))):
            z_vp = z0.copy()
            s_vp = np.empty_like(z0)
            w_vp = np.empty_like(z0)
            G.hydraulic_vpipes(z_vp, iterations=VPIPES_ITERS, water_depth=w_vp, sediment=s_vp, ctx=ctx, **kw)
            gpu.update({tag + "_z": z_vp, tag + "_sediment": s_vp, tag + "_water": w_vp})
        ctx.close()
        out["gpu"] = {"seconds": time.perf_counter() - t0,
                      "sha256": {k: _digest(v) for k, v in gpu.items()},
                      "mass_drift": {"thermal_intended": drift(_material(z_int)),
                                     "thermal_literal": drift(_material(z_lit)),
                                     "vpipes_material": drift(_material(gpu["vpipes_z"], gpu["vpipes_sediment"])),
                                     "vpipes_g1_material": drift(_material(gpu["vpipes_g1_z"],
                                                                           gpu["vpipes_g1_sediment"]))}}
    if part in ("all", "host"):
        if not po.ref_available():
            raise RuntimeError("the reference's kernel text (oracle/_ref/libhm_ref.so) is not built")
        t1 = time.perf_counter()
        o32_int, _ = po.thermal(z0, talus, THERMAL_ITERS, bedrock=bed)
        o64_int, _ = po.thermal(z0, talus, THERMAL_ITERS, bedrock=bed, dtype=np.float64)
        r_lit, _ = po.ref_thermal(z0, talus, THERMAL_ITERS, bedrock=bed)
        o64_lit, _ = po.thermal(z0, talus, THERMAL_ITERS, bedrock=bed, bedrock_mode=po.BEDROCK_LITERAL,
                                dtype=np.float64)
        pp = po.VpipesParams.make(**dict(CONFIG2_VPIPES, iterations=VPIPES_ITERS))
        o32_vp = po.vpipes(z0, pp)
        o64_vp = po.vpipes(z0, pp, dtype=np.float64)
        pg1 = po.VpipesParams.make(**dict(CONFIG2_VPIPES, gravity=1.0, iterations=VPIPES_ITERS))
        r_g1 = po.ref_vpipes(z0, pg1)
        o64_g1 = po.vpipes(z0, pg1, dtype=np.float64)
        host = {"thermal_intended": o32_int, "thermal_literal": r_lit, "vpipes_z": o32_vp[0],
                "vpipes_sediment": o32_vp[2], "vpipes_water": o32_vp[1], "vpipes_g1_z": r_g1[0],
                "vpipes_g1_sediment": r_g1[2], "vpipes_g1_water": r_g1[1]}
        out["host"] = {
            "seconds": time.perf_counter() - t1, "cores": po.num_threads(),
            "what": {"thermal_intended": "fp32 oracle (pinned to the reference text in every mode it has)",
                     "thermal_literal": "reference kernel text",
                     "vpipes_*": "fp32 oracle (gravity 9.81 is an extension the reference text lacks)",
                     "vpipes_g1_*": "reference kernel text (gravity 1)"},
            "sha256": {k: _digest(v) for k, v in host.items()},
            "vs_fp64": {"thermal_intended": _errors(o32_int, o64_int, z0),
                        "thermal_literal": _errors(r_lit, o64_lit, z0),
                        "vpipes_z": _errors(o32_vp[0], o64_vp[0], z0),
                        "vpipes_sediment": _errors(o32_vp[2], o64_vp[2], z0),
                        "vpipes_g1_z": _errors(r_g1[0], o64_g1[0], z0),
                        "vpipes_g1_sediment": _errors(r_g1[2], o64_g1[2], z0)},
            "mass_drift": {"thermal_intended": drift(_material(o32_int)),
                           "thermal_intended_fp64": drift(_material(o64_int)),
                           "thermal_literal": drift(_material(r_lit)),
                           "vpipes_material": drift(_material(o32_vp[0], o32_vp[2])),
                           "vpipes_material_fp64": drift(_material(o64_vp[0], o64_vp[2])),
                           "vpipes_g1_material": drift(_material(r_g1[0], r_g1[2])),
                           "vpipes_g1_material_fp64": drift(_material(o64_g1[0], o64_g1[2]))},
            "water_depth_max": {"vpipes": float(o32_vp[1].max()), "vpipes_g1": float(r_g1[1].max())}}
    ok = True
    if gpu is not None and host is not None:
        cmp = {k: _errors(gpu[k], host[k], z0) for k in gpu}
        out["gpu_vs_host"] = cmp
        ok = all(cmp[k]["max_abs_of_range"] <= (1e-4 if k.startswith("thermal") else 1e-3) for k in cmp)
        out["within_tolerance"] = ok
        out["value"] = cmp["vpipes_z"]["max_abs_of_range"]
    print(json.dumps(out), flush=True)
    return 0 if ok else 1


# ---------------------------------------------------------------- extras

AUTO_BEDROCK_BYTES = 16.0  # z in and out, talus, z0 (the bedrock grid is folded away)
FLOW_BYTES = 44.0          # z, depth and four fluxes in; depth and four fluxes out


def run_extras(a):
    """thermal_auto_bedrock (talus map, 500 iterations), flow_simulation
    (depth map, 1000 iterations, reference defaults), sediment_deposition
    (20 layers x 25 steps), sediment_layer and the snow post-filter (500
    steps each), the sibling talus stencils ridge, scree (zmax = z +
    0.25), schott and olsen and the relatives flatten, inflate and rib (200
    iterations each) and flow_simulation_viscous (1000 steps) on the 4096^2
    inputs:
    device-timed cell-updates/s against the HBM roofline, and the
    reference's kernel text on the host cores on a bounded sample (a few
    iterations on the full grid, scaled)."""
    import numpy as np
    import torch

    from highmap_b200 import gpu as G
    from oracle import pyoracle as po
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if not G.init_opencl():
        raise RuntimeError("no usable device: " + G.L.lib().hm_last_error().decode())
    ctx = G.Context(local)
    dev = torch.device("cuda", local)
    peak, peak_kind = _peaks()
    n = a.size
    cells = float(n) * n
    z, talus, _ = _inputs(n)
    from highmap_b200.inputs import fbm
    depth_map = fbm(n, n, seed=4)
    zd = torch.from_numpy(z).to(dev)
    td = torch.from_numpy(talus).to(dev)
    dm = torch.from_numpy(depth_map).to(dev)
    w = torch.empty_like(zd)
    zt = torch.empty_like(zd)
    rows = {}
    for name, iters, bpc, run in (
            ("thermal_auto_bedrock", 500, AUTO_BEDROCK_BYTES,
             lambda k: G.thermal_auto_bedrock_device(zt, td, k, ctx=ctx)),
            ("flow_simulation", 1000, FLOW_BYTES,
             lambda k: G.flow_simulation_device(zd, 0.01, dm, k, w, ctx=ctx))):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        for rep in range(a.warmup + 1):
            zt.copy_(zd)
            torch.cuda.synchronize()
            e0.record()
            run(iters)
            e1.record()
            torch.cuda.synchronize()
        t = e0.elapsed_time(e1) * 1e-3
        rate = cells * iters / t
        rows[name] = {"iterations": iters, "cell_updates_per_s": rate, "bytes_per_cell_update": bpc,
                      "gb_per_s": rate * bpc / 1e9, "frac": rate * bpc / 1e9 / peak, "peak": peak,
                      "peak_kind": peak_kind}
    # sediment_deposition: 20 layers of 25 thermal steps (talus map) each
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for rep in range(a.warmup + 1):
        zt.copy_(zd)
        torch.cuda.synchronize()
        e0.record()
        G.sediment_deposition_device(zt, td, None, 0.01, 20, 25, ctx=ctx)
        e1.record()
        torch.cuda.synchronize()
    t = e0.elapsed_time(e1) * 1e-3
    rate = cells * 500 / t
    rows["sediment_deposition"] = {"iterations": 500, "cell_updates_per_s": rate, "bytes_per_cell_update": 12.0,
                                   "gb_per_s": rate * 12.0 / 1e9, "frac": rate * 12.0 / 1e9 / peak, "peak": peak,
                                   "peak_kind": peak_kind, "layers": 20, "thermal_subiterations": 25}
    # sediment_layer (500 thermal steps, post-filter on) and the snow
    # post-filter (500 masked thermal steps): thermal cell-updates/s at the
    # 12 B of a talus-map step, the preparation and filter passes included
    upper = ((3.0 + 2.0 * fbm(n, n, seed=5)) / n).astype(np.float32)
    snow = (0.08 * fbm(n, n, seed=6)).astype(np.float32)
    ud = torch.from_numpy(upper).to(dev)
    sd = torch.from_numpy(snow).to(dev)
    s_w = torch.empty_like(sd)
    for name, run in (("sediment_layer", lambda: G.sediment_layer_device(zt, td, ud, 500, True, ctx=ctx)),
                      ("snow_post_filter", lambda: G.snow_post_filter_device(zd, s_w, 0.05, 500, 0.2, ctx=ctx))):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        for rep in range(a.warmup + 1):
            zt.copy_(zd)
            s_w.copy_(sd)
            torch.cuda.synchronize()
            e0.record()
            run()
            e1.record()
            torch.cuda.synchronize()
        t = e0.elapsed_time(e1) * 1e-3
        rate = cells * 500 / t
        rows[name] = {"iterations": 500, "cell_updates_per_s": rate, "bytes_per_cell_update": 12.0,
                      "gb_per_s": rate * 12.0 / 1e9, "frac": rate * 12.0 / 1e9 / peak, "peak": peak,
                      "peak_kind": peak_kind}
    # sibling talus stencils, 200 iterations each
    zmax = (z + 0.25).astype(np.float32)
    zmd = torch.from_numpy(zmax).to(dev)
    sib = (("thermal_ridge", G.RIDGE, 12.0), ("thermal_scree", G.SCREE, 16.0), ("thermal_schott", G.SCHOTT, 12.0),
           ("thermal_olsen", G.OLSEN, 12.0))
    for name, rule, bpc in sib:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        for rep in range(a.warmup + 1):
            zt.copy_(zd)
            torch.cuda.synchronize()
            e0.record()
            G.thermal_stencil_device(rule, zt, td, 200, zmax=zmd if rule == G.SCREE else None, ctx=ctx)
            e1.record()
            torch.cuda.synchronize()
        t = e0.elapsed_time(e1) * 1e-3
        rate = cells * 200 / t
        rows[name] = {"iterations": 200, "cell_updates_per_s": rate, "bytes_per_cell_update": bpc,
                      "gb_per_s": rate * bpc / 1e9, "frac": rate * bpc / 1e9 / peak, "peak": peak,
                      "peak_kind": peak_kind}
    # thermal_flatten (sigma_inf 0.5, sigma_sup 0.2), thermal_inflate and
    # thermal_rib, 200 iterations each (rib: no talus read)
    rel = (("thermal_flatten", G.FLATTEN, 12.0), ("thermal_inflate", G.INFLATE, 12.0), ("thermal_rib", G.RIB, 8.0))
    for name, rule, bpc in rel:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        for rep in range(a.warmup + 1):
            zt.copy_(zd)
            torch.cuda.synchronize()
            e0.record()
            G.thermal_relief_device(rule, zt, td if rule != G.RIB else None, 200, 0.5, 0.2, ctx=ctx)
            e1.record()
            torch.cuda.synchronize()
        t = e0.elapsed_time(e1) * 1e-3
        rate = cells * 200 / t
        rows[name] = {"iterations": 200, "cell_updates_per_s": rate, "bytes_per_cell_update": bpc,
                      "gb_per_s": rate * bpc / 1e9, "frac": rate * bpc / 1e9 / peak, "peak": peak,
                      "peak_kind": peak_kind}
    # flow_simulation_viscous, 1000 steps (depth map, water height 0.01):
    # 12 B per step (z and the depth read, the depth written; neighbours in
    # cache), the adaptive time step and the dry-out included
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for rep in range(a.warmup + 1):
        torch.cuda.synchronize()
        e0.record()
        G.flow_simulation_viscous_device(zd, 0.01, dm, 1000, w, 0.5, 0.0, 1.0, 2.5, ctx=ctx)
        e1.record()
        torch.cuda.synchronize()
    t = e0.elapsed_time(e1) * 1e-3
    rate = cells * 1000 / t
    rows["flow_simulation_viscous"] = {"iterations": 1000, "cell_updates_per_s": rate, "bytes_per_cell_update": 12.0,
                                       "gb_per_s": rate * 12.0 / 1e9, "frac": rate * 12.0 / 1e9 / peak, "peak": peak,
                                       "peak_kind": peak_kind}
    # the reference's kernel text on the host cores, a few iterations
    refs = [("thermal_auto_bedrock", lambda k: po.ref_thermal_auto_bedrock(z, talus, k)),
            ("flow_simulation", lambda k: po.ref_flow_simulation(z, 0.01, depth_map, k))]
    for name, rule, _ in sib:
        refs.append((name, lambda k, rule=rule: po.ref_thermal_sibling(rule, z, talus, k, zmax=zmax)))
    refs.append(("sediment_deposition", lambda k: po.ref_sediment_deposition(z, talus, 0.01, 1, k)))
    refs.append(("sediment_layer", lambda k: po.ref_sediment_layer(z, talus, upper, k, True)))
    refs.append(("snow_post_filter", lambda k: po.ref_snow_post_filter(z, snow, 0.05, k, 0.2)))
    for name, rule, _ in rel:
        refs.append((name, lambda k, rule=rule: po.ref_thermal_relief(rule, z, talus, k, 0.5, 0.2)))
    refs.append(("flow_simulation_viscous", lambda k: po.ref_flow_simulation_viscous(z, 0.01, depth_map, k)))
    for name, fn in refs:
        fn(1)
        k = 4 if name in ("flow_simulation", "thermal_olsen", "thermal_flatten", "flow_simulation_viscous") else 8
        t0 = time.perf_counter()
        fn(k)
        t = time.perf_counter() - t0
        rows[name]["cpu_baseline"] = {"value": cells * k / t, "unit": "cell-updates/s", "cores": po.num_threads(),
                                      "kind": "reference", "sample": "%d iterations on the full %dx%d inputs" %
                                      (k, n, n)}
    out = {"metric": "cell-updates/s at %d^2, thermal_auto_bedrock, flow_simulation, deposition callers, "
                     "sibling talus stencils" % n,
           "value": rows["flow_simulation"]["cell_updates_per_s"], "unit": "cell-updates/s", "n_gpus": 1,
           "higher_is_better": True, "dtype": "f32", "data": "synthetic", "form": "extras",
           "config": {"workload": "auto-bedrock thermal (talus map) x500, flow simulation (depth map fBm seed 4, "
                                  "water height 0.01, dt 0.5, flux diffusion 0.01) x1000", "grid": [n, n]},
           "rows": rows}
    print(json.dumps(out), flush=True)
    ctx.close()
    return 0


def run_tblock(a):
    """Vpipes (the plain drop-in configuration's parameters, 200 iterations)
    with one step per launch (HM_VPIPES_TILED) and with two
    (HM_VPIPES_TILED_TB2) on square grids: device time per step,
    cell-updates/s, algorithmic GB/s against the measured copy bandwidth,
    whether the two give the same bits, and which the autotuner keeps.  One
    JSON line per size."""
    import numpy as np
    import torch

    from highmap_b200 import gpu as G
    from highmap_b200 import tune
    from highmap_b200.inputs import fbm
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if not G.init_opencl():
        raise RuntimeError("no usable device: " + G.L.lib().hm_last_error().decode())
    ctx = G.Context(local)
    dev = torch.device("cuda", local)
    peak, peak_kind = _peaks()
    it = SWEEP_ITERS
    p = G.vpipes_params(**dict(CONFIG2_VPIPES, iterations=it))
    for k, n in enumerate(int(x) for x in a.sizes.split(",")):
        z0 = torch.from_numpy(fbm(n, n, seed=10 + k)).to(dev)
        algos = (("one_step", G.VPIPES_TILED), ("two_steps", G.VPIPES_TILED_TB2))
        ms = {name: [] for name, _ in algos}
        res = {}
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        try:
            for rep in range(3):  # the first pass warms up
                for name, algo in algos:
                    G.vpipes_set_algorithm(algo)
                    z = z0.clone()
                    sd = torch.empty_like(z)
                    torch.cuda.synchronize()
                    e0.record()
                    G.hydraulic_vpipes_device(z, p, None, None, sd, ctx=ctx)
                    e1.record()
                    torch.cuda.synchronize()
                    if rep:
                        ms[name].append(e0.elapsed_time(e1) / it)
                    res[name] = (z.cpu().numpy(), sd.cpu().numpy())
        finally:
            G.vpipes_set_algorithm(G.VPIPES_AUTO)
        same = all(np.array_equal(x, y) for x, y in zip(res["one_step"], res["two_steps"]))
        tuned = tune.autotune(tune.VPIPES, n, n, steps=20, ctx=ctx)
        row = {"form": "tblock", "grid": [n, n], "iterations": it, "bit_identical": bool(same),
               "tuned_time_block": 2 if (tuned["tpb"] == 0 and tuned["time_block"] == 2) else 1,
               "tuned": tuned, "peak_gbs": peak, "peak_kind": peak_kind}
        for name, _ in algos:
            t = min(ms[name])
            rate = n * n / (t * 1e-3)
            row[name] = {"ms_per_step": t, "cell_updates_per_s": rate, "algorithmic_gbs": rate * 56 / 1e9,
                         "frac": rate * 56 / 1e9 / peak}
        row["two_over_one_time"] = row["two_steps"]["ms_per_step"] / row["one_step"]["ms_per_step"]
        print(json.dumps(row), flush=True)
    ctx.close()
    return 0


def run_form(a):
    """The batched or served form on one GPU (rank 0 of a torchrun launch
    runs it; the others exit)."""
    import torch

    from highmap_b200 import forms
    from highmap_b200 import gpu as G
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if not G.init_opencl():
        raise RuntimeError("no usable device: " + G.L.lib().hm_last_error().decode())
    if a.form == "batch":
        r = forms.run_batch_benchmark(n_jobs=a.jobs)
        out = {"metric": "aggregate cell-updates/s, %d mixed thermal/vpipes jobs (128..2048, 50..1000 iterations), "
                         "batched vs plain per-job calls" % a.jobs,
               "value": r["batched_cell_updates_per_s"], "unit": "cell-updates/s", "n_gpus": 1,
               "higher_is_better": True, "dtype": "f32", "data": "synthetic", "form": "batch",
               "config": {"workload": "batched form", "jobs": a.jobs, "sizes": "log-uniform 128..2048, x8, aspect<=2",
                          "iterations": "uniform 50..1000", "kinds": "half thermal, half vpipes"},
               "detail": r}
    else:
        rates = tuple(float(x) for x in a.rates.split(","))
        r = forms.run_serve_benchmark(n_requests=a.requests, rates=rates)
        best = max(r["sweep"], key=lambda x: x["served"]["cell_updates_per_s"])
        out = {"metric": "served cell-updates/s and p50/p99 latency, Poisson requests (256..4096, 20..2000 "
                         "iterations), continuous batching vs plain FIFO",
               "value": best["served"]["cell_updates_per_s"], "unit": "cell-updates/s", "n_gpus": 1,
               "higher_is_better": True, "dtype": "f32", "data": "synthetic", "form": "serve",
               "config": {"workload": "served form", "requests_per_rate": a.requests,
                          "budget_bytes": 120 << 30, "rates_per_s": list(rates)},
               "detail": r}
    print(json.dumps(out), flush=True)
    return 0


def main():
    a = _args()
    if a.impl == "reference":
        return run_reference(a)
    if a.form == "sweep":
        return run_sweep(a)
    if a.form == "extras":
        return run_extras(a)
    if a.form == "parity":
        return run_parity(a)
    if a.form == "tblock":
        return run_tblock(a)
    if a.form != "plain":
        return run_form(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
