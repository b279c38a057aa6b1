"""The launch-shape autotuner (hm_autotune of include/hm_erosion.h).

``autotune(kind, nx, ny)`` times every candidate launch shape of a solver on
a synthetic terrain of that size and keeps the fastest for its size class;
solves that leave the choice to the library then use it.  ``BATCH`` tunes
the batched form (persistent CTAs per SM, thermal tile rows) on a synthetic
mixed batch with sides up to max(nx, ny); batches created afterwards use it.  ``save`` /
``load`` keep the table between processes.
"""
from __future__ import annotations

import ctypes as C

from . import _lib as L
from .gpu import Context, default_context

THERMAL = L.HM_JOB_THERMAL
VPIPES = L.HM_JOB_VPIPES
BATCH = 3  # HM_TUNE_BATCH: the batched form's CTAs per SM (tpb) and thermal tile rows (rows)


def autotune(kind: int, nx: int, ny: int, steps: int = 20, ctx: Context | None = None) -> dict:
    ctx = ctx or default_context()
    r = L.TuneResult()
    L.check(L.lib().hm_autotune(ctx.handle, int(kind), int(nx), int(ny), int(steps), C.byref(r)))
    return {f: getattr(r, f) for f, _ in r._fields_}


def save(path: str) -> None:
    L.check(L.lib().hm_autotune_save(str(path).encode()))


def load(path: str) -> int:
    n = C.c_int()
    L.check(L.lib().hm_autotune_load(str(path).encode(), C.byref(n)))
    return n.value


def clear() -> None:
    L.lib().hm_autotune_clear()
