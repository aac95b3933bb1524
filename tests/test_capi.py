"""Host-side checks of the C ABI library that need no GPU: it loads, exports
every entry point include/lbm_ddf.h declares, derives parameters as the
reference does, and rejects bad arguments with a status instead of exiting."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in os.listdir(os.path.join(ROOT, "include")) if h.endswith(".h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(lbm_\w+)\s*\(", txt, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_exports_every_declared_symbol(lbm):
    names = declared_functions()
    assert "lbm_step" in names and "lbm_create" in names
    L = C.CDLL(lbm.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_abi_version(lbm):
    assert lbm.lib().lbm_abi_version() == 3


def test_largest_16bit_case_accepted(lbm):
    """512 x 512 x 1024 in FP16S (268 M nodes) is within the pair index range."""
    p = lbm.make_params(512, 512, 1024, storage="f16s")
    assert lbm.lib().lbm_derive(C.byref(p), C.byref(lbm.LbmDerived())) == lbm.OK


def test_derive_matches_reference_globals(lbm, oracle_mod):
    """src/globals.cu:13-23, via the oracle's restatement."""
    for (lx, ly, lz, ra, pr) in [(64, 64, 64, 1e5, 0.71), (256, 256, 256, 1e7, 0.71), (512, 256, 512, 1e8, 4.38)]:
        d = lbm.derive(lbm.make_params(lx, ly, lz, rayleigh=ra, prandtl=pr))
        o = oracle_mod.make_params(lx, ly, lz, rayleigh=ra, prandtl=pr)
        for k in ("visc", "tau", "u0", "diff", "tauc", "t0"):
            assert d[k] == getattr(o, k), k
    # free-fall velocity 0.1 and the tau values quoted for 64^3 / 256^3
    d = lbm.derive(lbm.make_params(64, 64, 64, rayleigh=1e5))
    assert abs(d["u0"] - 0.1) < 1e-15
    assert abs(d["tau"] - 0.5512) < 1e-4 and abs(d["tauc"] - 0.5721) < 1e-4


def test_reference_default_beta(lbm):
    rs = lbm.RunSurface(LX=400, LY=400, LZ=400)
    d = lbm.derive(rs.params())
    assert abs(rs.params().beta - 0.1 / (400 * 5.0)) == 0.0
    assert abs(d["u0"] - np.sqrt(0.02)) < 1e-15


@pytest.mark.parametrize("bad", [
    dict(lx=1), dict(ly=2), dict(lz=0), dict(sides=7), dict(storage=9), dict(rayleigh=-1.0),
    dict(prandtl=0.0), dict(t_hot=0.0), dict(gravity=0.0),
    dict(lx=800, ly=800, lz=800, storage=2),   # 16-bit pair rows beyond 32-bit indexing
])
def test_bad_params_rejected(lbm, bad):
    p = lbm.make_params(8, 8, 8)
    for k, v in bad.items():
        setattr(p, k, v)
    d = lbm.LbmDerived()
    rc = lbm.lib().lbm_derive(C.byref(p), C.byref(d))
    assert rc == lbm.ERR_ARG
    assert lbm.lib().lbm_last_error()
    h = C.c_void_p()
    assert lbm.lib().lbm_create(C.byref(p), C.byref(h)) == lbm.ERR_ARG
    assert not h.value


def test_too_many_nodes_rejected(lbm):
    p = lbm.make_params(2048, 2048, 1024)
    assert lbm.lib().lbm_derive(C.byref(p), C.byref(lbm.LbmDerived())) == lbm.ERR_ARG


def test_case_bytes(lbm):
    for st, b in lbm.STORAGE_BYTES.items():
        p = lbm.make_params(256, 256, 256, storage=st)
        n = 256 ** 3
        need = lbm.case_bytes(p)
        pops = 2 * 27 * n * b
        assert pops < need < pops + n * 8 + 10 ** 6


def test_null_case_is_an_error(lbm):
    L = lbm.lib()
    assert L.lbm_step(None, 1, None) == lbm.ERR_ARG
    assert L.lbm_destroy(None) == lbm.OK
    out = (lbm.LbmObservables * 2)()
    assert L.lbm_step_observed(None, 1, out, None) == lbm.ERR_ARG
    assert L.lbm_step_observed_async(None, 1, C.cast(out, C.c_void_p), None) == lbm.ERR_ARG
    t = np.zeros(8, dtype=np.float32)
    assert L.lbm_init_temperature(None, t.ctypes.data_as(C.c_void_p), None) == lbm.ERR_ARG
    assert L.lbm_init_conduction(None, 1, 1e-3, None) == lbm.ERR_ARG
    assert L.lbm_get_observables(None, C.byref(out[0]), None) == lbm.ERR_ARG
    assert "NULL" in L.lbm_last_error().decode()


def test_fastdiv_host_emulation():
    """FastDiv of lattice.cuh (Granlund-Montgomery), emulated exactly."""
    rng = np.random.default_rng(0)

    def params(d):
        l = 0
        while (1 << l) < d:
            l += 1
        m = (((1 << 32) * ((1 << l) - d)) // d + 1) & 0xFFFFFFFF
        return m, l

    for d in [1, 2, 3, 5, 7, 12, 48, 64, 96, 100, 127, 192, 255, 256, 400, 511, 512, 1000, 4095, 65536, 2 ** 20 + 3]:
        m, l = params(d)
        ns = np.concatenate([np.arange(0, 5000), rng.integers(0, 2 ** 31 - 1, 20000), [2 ** 31 - 1]])
        for n in ns.tolist():
            q = (((n * m) >> 32) + n) >> l
            assert q == n // d, (d, n)


def test_no_gpu_create_fails_cleanly(lbm):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    h = C.c_void_p()
    rc = lbm.lib().lbm_create(C.byref(lbm.make_params(8, 8, 8)), C.byref(h))
    assert rc in (lbm.ERR_CUDA, lbm.ERR_NOMEM)
    assert not h.value


def test_noalloc_argument_checks_need_no_gpu(lbm):
    """lbm_observables_noalloc rejects, before touching a device, a 16-bit
    call whose g is not f's partner element or whose stride would overflow
    the 32-bit pair index (9 * pop_stride >= 2^32), and an FP32 stride above
    2^40; the rejections name the rule."""
    L = lbm.lib()
    out = C.c_void_p(4096)
    pp = C.c_void_p(8192)
    for st in ("f16s", "bf16s"):
        p = lbm.make_params(8, 8, 8, storage=st)
        f = 1 << 20
        # g elsewhere than f + 1 element
        rc = L.lbm_observables_noalloc(C.byref(p), C.c_void_p(f), C.c_void_p(f + 4096), pp, 512, 0, 0, out, None)
        assert rc == lbm.ERR_ARG and "f + 1 element" in L.lbm_last_error().decode()
        # 477,218,589 is the smallest stride whose nine pair rows overflow
        # 32-bit indices
        big = 477_218_589
        assert 9 * (big - 1) < 2 ** 32 <= 9 * big
        rc = L.lbm_observables_noalloc(C.byref(p), C.c_void_p(f), C.c_void_p(f + 2), pp, big, 0, 0, out, None)
        assert rc == lbm.ERR_ARG and "pop_stride" in L.lbm_last_error().decode()
        rc = L.lbm_observables_noalloc(C.byref(p), C.c_void_p(f), C.c_void_p(f + 2), pp, 2 ** 33, 0, 0, out, None)
        assert rc == lbm.ERR_ARG
    p = lbm.make_params(8, 8, 8, storage="f32")
    rc = L.lbm_observables_noalloc(C.byref(p), C.c_void_p(1 << 20), C.c_void_p(1 << 21), pp, 2 ** 40 + 1, 0, 0,
                                   out, None)
    assert rc == lbm.ERR_ARG and "pop_stride" in L.lbm_last_error().decode()
    rc = L.lbm_observables_noalloc(C.byref(p), C.c_void_p(1 << 20), C.c_void_p(1 << 21), pp, 100, 0, 0, out, None)
    assert rc == lbm.ERR_ARG   # below the node count
