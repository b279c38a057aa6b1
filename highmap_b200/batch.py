"""Batched solves: many heightmaps of uneven sizes and iteration counts
advanced together on one GPU (hm_batch_* of include/hm_erosion.h).

The reference has no batch interface; a node graph calls
hmap::gpu::thermal / hydraulic_vpipes once per node.  Here jobs are
described by device tensors (torch CUDA tensors), admitted into a batch,
and advanced by rounds: one round is one step of every active job, run as
one persistent kernel over the packed tiles of all jobs.  Results are
bit-identical to solving each job alone.
"""
from __future__ import annotations

import ctypes as C

from . import _lib as L
from .gpu import Context, default_context, vpipes_params

THERMAL = L.HM_JOB_THERMAL
VPIPES = L.HM_JOB_VPIPES


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _check_grid(t, name, shape):
    import torch
    if t is None:
        return
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32 or not t.is_contiguous():
        raise TypeError("%s must be a contiguous float32 CUDA tensor" % name)
    if tuple(t.shape) != tuple(shape):
        raise ValueError("%s has shape %s, expected %s" % (name, tuple(t.shape), tuple(shape)))


def thermal_job(z, talus, iterations, bedrock=None, deposition_map=None, bedrock_mode=L.HM_BEDROCK_INTENDED):
    """A thermal job on device tensors; ``talus`` is a tensor or a float."""
    ny, nx = z.shape
    _check_grid(z, "z", (ny, nx))
    j = L.Job()
    j.kind, j.nx, j.ny, j.iterations = THERMAL, nx, ny, int(iterations)
    j.z = _p(z)
    if isinstance(talus, (int, float)):
        j.talus, j.talus_value = None, float(talus)
    else:
        _check_grid(talus, "talus", (ny, nx))
        j.talus = _p(talus)
    _check_grid(bedrock, "bedrock", (ny, nx))
    _check_grid(deposition_map, "deposition_map", (ny, nx))
    j.bedrock, j.bedrock_mode, j.deposition_map = _p(bedrock), int(bedrock_mode), _p(deposition_map)
    j._keep = (z, talus, bedrock, deposition_map)
    return j


def vpipes_job(z, iterations, rain_map=None, water_depth=None, sediment=None, vel_u=None, vel_v=None, **params):
    """A virtual-pipes job on device tensors; ``params`` as vpipes_params."""
    ny, nx = z.shape
    _check_grid(z, "z", (ny, nx))
    for name, t in (("rain_map", rain_map), ("water_depth", water_depth), ("sediment", sediment),
                    ("vel_u", vel_u), ("vel_v", vel_v)):
        _check_grid(t, name, (ny, nx))
    j = L.Job()
    j.kind, j.nx, j.ny, j.iterations = VPIPES, nx, ny, int(iterations)
    j.z = _p(z)
    j.vpipes = vpipes_params(**params)
    j.rain_map, j.water_depth, j.sediment = _p(rain_map), _p(water_depth), _p(sediment)
    j.vel_u, j.vel_v = _p(vel_u), _p(vel_v)
    j._keep = (z, rain_map, water_depth, sediment, vel_u, vel_v)
    return j


def job_bytes(job) -> int:
    return int(L.lib().hm_batch_job_bytes(C.byref(job)))


class Batch:
    """An open batch (hm_batch): admit jobs, advance rounds, release."""

    def __init__(self, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self._h = C.c_void_p()
        L.check(L.lib().hm_batch_create(self.ctx.handle, C.byref(self._h)))
        self._jobs = {}

    def add(self, job) -> int:
        jid = C.c_int()
        L.check(L.lib().hm_batch_add(self._h, C.byref(job), C.byref(jid)))
        self._jobs[jid.value] = job
        return jid.value

    def step(self, rounds: int) -> None:
        L.check(L.lib().hm_batch_step(self._h, int(rounds)))

    def synchronize(self) -> None:
        L.check(L.lib().hm_batch_synchronize(self._h))

    def status(self, job_id: int):
        s, f = C.c_int(), C.c_int()
        L.check(L.lib().hm_batch_job_status(self._h, int(job_id), C.byref(s), C.byref(f)))
        return s.value, bool(f.value)

    def release(self, job_id: int) -> None:
        L.check(L.lib().hm_batch_release(self._h, int(job_id)))
        self._jobs.pop(job_id, None)

    def bytes_in_use(self) -> int:
        return int(L.lib().hm_batch_bytes_in_use(self._h))

    def evict(self, job_id: int):
        """Move an unfinished job's device state to host memory (a numpy
        byte array); the job leaves the rounds until ``restore``."""
        import numpy as np
        snap = np.empty(int(L.lib().hm_batch_snapshot_bytes(self._h, int(job_id))), dtype=np.uint8)
        L.check(L.lib().hm_batch_evict(self._h, int(job_id), snap.ctypes.data_as(C.c_void_p)))
        return snap

    def restore(self, job_id: int, snapshot) -> None:
        """Admit an evicted job again from its snapshot; it goes on from the
        step it had reached."""
        L.check(L.lib().hm_batch_restore(self._h, int(job_id), snapshot.ctypes.data_as(C.c_void_p)))

    @property
    def round(self) -> int:
        return int(L.lib().hm_batch_round(self._h))

    def close(self):
        if self._h:
            L.lib().hm_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run(jobs, use_graph: bool = True, ctx: Context | None = None) -> None:
    """Every job to completion in one batched pass (one CUDA graph)."""
    ctx = ctx or default_context()
    arr = (L.Job * len(jobs))(*jobs)
    L.check(L.lib().hm_batch_run(ctx.handle, arr if jobs else None, len(jobs), 1 if use_graph else 0))
