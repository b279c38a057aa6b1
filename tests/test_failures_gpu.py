"""Host-side failure cases of the device path, made without a GPU fault.

* A solve whose device workspace cannot be allocated -- a 65000 x 65000
  vpipes solve needs 19 grids of 16.9 GB, more than the device has --
  returns HM_ERR_OUT_OF_MEMORY before any kernel runs, and the same context
  then solves a small grid bit-exactly (its workspace grows again from
  nothing).
* A batched job cancelled before it finishes is covered in
  tests/test_batch_gpu.py (test_cancelled_job_leaves_the_others_exact).
"""
import numpy as np
import pytest

from highmap_b200 import _lib as L
from highmap_b200.inputs import fbm
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

CONFIG2 = dict(maintain_water_volume=0, flux_diffusion=0, dt=0.1, k_capacity=0.05, k_erode=0.01, k_depose=0.01,
               evap_rate=0.01, gravity=9.81, rain_per_step=1e-4, initial_water=0.0)


def test_workspace_out_of_memory_then_recovery(gpu):
    import torch
    n = 65000
    free, total = torch.cuda.mem_get_info()
    need = 19 * n * n * 4
    assert need > total, "the device would hold the workspace; the case would not fail"
    if free < n * n * 4 + (1 << 30):
        pytest.skip("not enough free device memory for the 16.9 GB grid itself")
    ctx = gpu.Context(torch.cuda.current_device())
    z = torch.empty((n, n), dtype=torch.float32, device="cuda")
    with pytest.raises(L.HMError) as e:
        gpu.hydraulic_vpipes_device(z, gpu.vpipes_params(**dict(CONFIG2, iterations=1)), ctx=ctx)
    assert e.value.status == L.HM_ERR_OUT_OF_MEMORY
    assert "cudaMalloc" in str(e.value)
    del z
    torch.cuda.empty_cache()
    # the context is still usable
    z0 = fbm(96, 72, seed=4)
    zt = torch.from_numpy(z0).cuda()
    gpu.hydraulic_vpipes_device(zt, gpu.vpipes_params(**dict(CONFIG2, iterations=9)), ctx=ctx)
    torch.cuda.synchronize()
    want = po.vpipes(z0, po.VpipesParams.make(**dict(CONFIG2, iterations=9)))[0]
    assert np.array_equal(zt.cpu().numpy(), want)
    ctx.close()
