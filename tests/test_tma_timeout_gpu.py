"""The one device-side wait on the path -- a vpipes tile waiting for its
TMA boxes -- is bounded, and running out is reported, not hung on.

The test hook hm_debug_tma_expect_extra arms every tile's barrier with 16
bytes more than its boxes deliver: every load still lands in shared
memory, but the barrier's phase cannot complete.  Each tile's wait then
runs out (a second per window, two windows), the tile sets the step's
error word and returns without writing, and hm_vpipes reports
HM_ERR_TIMEOUT with the caller's heights untouched.  Nothing faults; the
next call on the same context, with the hook off, is bit-exact with the
oracle.
"""
import time

import numpy as np
import pytest

from highmap_b200 import _lib as L
from highmap_b200.inputs import fbm
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

PARAMS = dict(iterations=3, maintain_water_volume=0, flux_diffusion=0, dt=0.1, k_capacity=0.05, k_erode=0.01,
              k_depose=0.01, evap_rate=0.01, gravity=9.81, rain_per_step=1e-4, initial_water=0.0)


@pytest.mark.parametrize("iterations, maintain", [(1, 0), (2, 0), (2, 1)])
def test_tma_wait_runs_out_and_reports_timeout(gpu, iterations, maintain):
    """One iteration runs only the first step's kernel (k_vp_fwe_tma); two
    add a later step's kernel (k_vp_step_tma, whose boxes arrive in two
    groups on two barriers).  With the volume top-up a tile that gave up
    still adds zero to the grid-wide sum, so the step's last tile finishes
    the sum instead of waiting for it."""
    # 64 x 40: TMA staging applies (nx a multiple of 4, nx >= 40, ny >= 24)
    z0 = fbm(64, 40, seed=12)
    ctx = gpu.Context(0)
    try:
        gpu.vpipes_set_algorithm(gpu.VPIPES_TILED)
        gpu.debug_tma_expect_extra(16)
        z = z0.copy()
        t = time.perf_counter()
        with pytest.raises(L.HMError) as e:
            gpu.hydraulic_vpipes(z, ctx=ctx, **dict(PARAMS, iterations=iterations, maintain_water_volume=maintain))
        elapsed = time.perf_counter() - t
        assert e.value.status == L.HM_ERR_TIMEOUT
        assert "timed out" in str(e.value)
        assert elapsed < 30.0, "the bounded wait took %.1f s" % elapsed
        assert np.array_equal(z, z0), "a timed-out call must leave the caller's heights as they were"
    finally:
        gpu.debug_tma_expect_extra(0)
    try:
        z = z0.copy()
        sed = np.empty_like(z)
        gpu.hydraulic_vpipes(z, sediment=sed, ctx=ctx, **PARAMS)
        wz, _, ws, _, _ = po.vpipes(z0, po.VpipesParams.make(**PARAMS))
        assert np.array_equal(z, wz) and np.array_equal(sed, ws)
    finally:
        gpu.vpipes_set_algorithm(gpu.VPIPES_AUTO)
        ctx.close()


def test_hook_rejects_bad_sizes(gpu):
    for bad in (8, 4097 * 16, 5000):
        with pytest.raises(L.HMError) as e:
            gpu.debug_tma_expect_extra(bad)
        assert e.value.status == L.HM_ERR_INVALID_ARGUMENT
    gpu.debug_tma_expect_extra(0)
