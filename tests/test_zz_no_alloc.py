"""The no-allocation observables entry point (lbm_observables_noalloc).

It serves callers that may not allocate device memory through this library
(a stream being captured into a CUDA graph, an HBM budget fixed up front, a
thread that must not block in cudaMalloc/cudaFree): they pass their own
population buffers and an output struct in their own device memory, and the
reduction keeps its partial sums in a fixed array inside the library.

The test copies a case's state (through the native checkpoint) into buffers
it owns, calls the entry point twice in a row on two different states (the
second call reuses the array the first one left behind, and runs on a side
stream) and checks each result against lbm_get_observables on the same
state, in every storage format (16-bit: the one interleaved array of (f, g)
pairs, g passed as f + 1 element).  This file is named so that pytest
collects it last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("nu_bulk", "nu_top", "nu_bottom", "ke", "re", "ux_mean", "uy_mean", "uz_mean", "phi_mean")


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _own_buffers(lbm, case, torch):
    """Device tensors holding the populations and phi_prev of `case`, as the
    caller's own memory: (f, g, phi_prev, pop_stride, element bytes).  For
    16-bit storage f and g are one array of (f, g) pairs; the tensor `g` is
    then the same array and the call passes g = f + 1 element."""
    p = case.params
    nodes = p.lx * p.ly * p.lz
    ps = (nodes + 127) // 128 * 128
    sb = lbm.STORAGE_BYTES[p.storage]
    pop = 27 * ps * sb
    carry = ps * (8 if p.storage == lbm.STORE_F64 else 4)
    host = np.empty(case.checkpoint_bytes(), dtype=np.uint8)
    case.save_state(host)
    torch.cuda.synchronize()
    head = host.size - 2 * pop - carry
    pp = torch.from_numpy(host[head + 2 * pop:].copy()).cuda()
    if sb == 2:   # interleaved pairs: one region of 2 * pop bytes
        fg = torch.from_numpy(host[head:head + 2 * pop].copy()).cuda()
        return fg, fg, pp, ps, sb
    f = torch.from_numpy(host[head:head + pop].copy()).cuda()
    g = torch.from_numpy(host[head + pop:head + 2 * pop].copy()).cuda()
    return f, g, pp, ps, sb


def _call(lbm, p, f, g, pp, ps, sb, n, out, stream=None):
    g_ptr = f.data_ptr() + sb if sb == 2 else g.data_ptr()
    lbm.observables_noalloc(p, f.data_ptr(), g_ptr, pp.data_ptr(), ps, n % 2 == 1, n, out.data_ptr(),
                            stream=stream)


# Reduced observables of the same state agree to rounding (the FP64 sums
# run in the same kernel, so in practice bitwise)
TOL = 1e-12


@pytest.mark.parametrize("storage", ["f64", "f32", "f16s", "bf16s"])
def test_noalloc_matches_get_observables_twice(lbm, storage):
    import torch

    p = lbm.make_params(40, 24, 32, rayleigh=1e5, sides=lbm.SIDES_WALL, storage=storage)
    out = torch.zeros(C.sizeof(lbm.LbmObservables), dtype=torch.uint8, device="cuda")
    side = torch.cuda.Stream()
    with lbm.Case(p) as case:
        case.init_conduction(17, 1e-2)
        # two calls in a row: 7 steps (swapped layout), then 8 (natural); the
        # second on a side stream
        for steps, stream in ((7, None), (1, side)):
            case.step(steps)
            want = case.observables()
            f, g, pp, ps, sb = _own_buffers(lbm, case, torch)
            n = case.step_count
            if stream is not None:
                stream.wait_stream(torch.cuda.current_stream())
            _call(lbm, p, f, g, pp, ps, sb, n, out, stream)
            torch.cuda.synchronize()
            got = lbm.LbmObservables.from_buffer_copy(out.cpu().numpy().tobytes()).as_dict()
            assert got["step"] == n
            assert got["diverged"] == 0
            for k in KEYS:
                assert abs(got[k] - want[k]) <= TOL * max(1.0, abs(want[k])), (storage, k, got[k], want[k])


def test_noalloc_rejects_bad_arguments(lbm):
    p = lbm.make_params(8, 8, 8, storage="f32")
    rc = lbm.lib().lbm_observables_noalloc(C.byref(p), None, None, None, 512, 0, 0, None, None)
    assert rc == lbm.ERR_ARG
    rc = lbm.lib().lbm_observables_noalloc(C.byref(p), C.c_void_p(16), C.c_void_p(16), C.c_void_p(16),
                                           100, 0, 0, C.c_void_p(16), None)
    assert rc == lbm.ERR_ARG   # stride below the node count
