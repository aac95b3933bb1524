"""The row-staged kernel's bounded wait on its bulk copies (rowstep.cuh).

The test hook lbm_debug_row_wait_extra_bytes makes the kernel announce 16
bytes more on its shared-memory barrier than its copies bring: every copy
lands, but the barrier's phase can never complete, as if a copy never
arrived.  Each block's wait gives up after one second of the GPU's global
timer, waits once more (bounded) for copies still on their way, sets the
case's error flag and leaves.  The host learns it from the next
lbm_get_observables (LBM_ERR_CUDA), the CUDA context stays usable, and a
fresh case then steps and matches the node kernel.  The grid has 8 rows
(8 blocks, one wave), so the run-out costs about two seconds.
"""
import ctypes as C
import time

import numpy as np
import pytest

from helpers import relerr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_row_kernel_wait_runs_out_and_reports(lbm):
    import torch

    p = lbm.make_params(32, 4, 2, rayleigh=1e5, sides=lbm.SIDES_PERIODIC, storage="f32")
    L = lbm.lib()
    with lbm.Case(p) as c:
        c.set_step_kernel(lbm.KERNEL_ROW)
        c.init_conduction(3, 1e-2)
        assert L.lbm_debug_row_wait_extra_bytes(c.handle, 8) == lbm.ERR_ARG   # not a multiple of 16
        assert L.lbm_debug_row_wait_extra_bytes(c.handle, 16) == lbm.OK
        t0 = time.perf_counter()
        c.step(1)                                   # enqueued; the launch itself succeeds
        torch.cuda.synchronize()                    # the kernel ends (its waits are bounded)
        waited = time.perf_counter() - t0
        o = lbm.LbmObservables()
        rc = L.lbm_get_observables(c.handle, C.byref(o), None)
        assert rc == lbm.ERR_CUDA
        assert "gave up waiting" in L.lbm_last_error().decode()
    assert 0.5 < waited < 30.0, waited
    # the context is still usable: a fresh case steps on the row kernel and
    # matches the node kernel
    got = {}
    for kind in (lbm.KERNEL_ROW, lbm.KERNEL_NODE):
        with lbm.Case(p) as c:
            c.set_step_kernel(kind)
            c.init_conduction(3, 1e-2)
            c.step(4)
            got[kind] = c.store_ref_state(("f", "g"))
            assert c.observables()["diverged"] == 0
    for k in ("f", "g"):
        assert relerr(got[lbm.KERNEL_ROW][k], got[lbm.KERNEL_NODE][k]) <= 2e-6, k
    assert np.isfinite(got[lbm.KERNEL_ROW]["f"]).all()
