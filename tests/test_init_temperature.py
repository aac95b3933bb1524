"""Starting a case from the caller's temperature field (C ABI
lbm_init_temperature, Case.init_temperature).

The host generator lbm_ddf_b200.conduction_temperature is pinned on the CPU
against the oracle's conduction start (oracle/lbm_oracle.c
orc_init_conduction): g_i = w_i T bit for bit.  On the GPU, the conduction
field passed to init_temperature must give lbm_init_conduction's state:

  FP64 storage      bitwise equal fields, before and after 25 steps;
  FP32 storage      field-relative error <= 1e-5 after 25 steps (the field
                    arrives rounded to float32; init_conduction rounds w_i T
                    from the FP64 value);
  FP16S / BF16S     <= 5e-3 / 4e-2 (the 16-bit parity bounds).
"""
import numpy as np
import pytest

from helpers import relerr

LX, LY, LZ = 16, 12, 10
SEED, AMP = 7, 1e-3


def test_conduction_temperature_is_the_oracles(oracle_mod):
    import lbm_ddf_b200 as lbm

    p = oracle_mod.make_params(LX, LY, LZ)
    o = oracle_mod.Oracle(p)
    o.init_rest()
    w = 2.0 * o.field("g")[:, 0, 0, 0].copy()   # rest state: g_i = w_i / 2
    o.init_conduction(SEED, AMP)
    g = o.field("g").copy()
    o.close()
    t = lbm.conduction_temperature(LX, LY, LZ, SEED, AMP).reshape(LZ, LY, LX)
    assert np.array_equal(g, w[:, None, None, None] * t[None])


def test_conduction_temperature_noise_is_the_oracles(oracle_mod):
    import lbm_ddf_b200 as lbm

    t = lbm.conduction_temperature(5, 4, 3, seed=123, amplitude=1.0, t_hot=0.0, t_cold=0.0)
    u = np.array([oracle_mod.noise_uniform(123, i) for i in range(60)])
    assert np.array_equal(t, 2.0 * u - 1.0)


def _run(lbm, p, start, steps):
    with lbm.Case(p) as c:
        start(c)
        s0 = c.store_ref_state(("f", "g", "phi"))
        c.step(steps)
        s1 = c.store_ref_state()
        obs = c.observables()
    return s0, s1, obs


def _params(lbm, storage, periodic):
    sides = lbm.SIDES_PERIODIC if periodic else lbm.SIDES_WALL
    return lbm.make_params(LX, LY, LZ, sides=sides, storage=storage)


@pytest.fixture()
def gpu(lbm):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return lbm


@pytest.mark.gpu
@pytest.mark.parametrize("periodic", [True, False])
def test_f64_temperature_start_is_bitwise_the_conduction_start(gpu, periodic):
    lbm = gpu
    p = _params(lbm, "f64", periodic)
    t = lbm.conduction_temperature(LX, LY, LZ, SEED, AMP)
    a0, a1, oa = _run(lbm, p, lambda c: c.init_conduction(SEED, AMP), 25)
    b0, b1, ob = _run(lbm, p, lambda c: c.init_temperature(t), 25)
    for k in a0:
        assert np.array_equal(a0[k], b0[k]), k
    for k in a1:
        assert np.array_equal(a1[k], b1[k]), k
    for k in ("nu_bulk", "nu_top", "nu_bottom", "ke"):
        assert oa[k] == ob[k], k


@pytest.mark.gpu
@pytest.mark.parametrize("storage,tol", [("f32", 1e-5), ("f16s", 5e-3), ("bf16s", 4e-2)])
@pytest.mark.parametrize("periodic", [True, False])
def test_reduced_precision_temperature_start(gpu, storage, tol, periodic):
    lbm = gpu
    p = _params(lbm, storage, periodic)
    t = lbm.conduction_temperature(LX, LY, LZ, SEED, AMP, dtype=np.float32)
    _, a1, _ = _run(lbm, p, lambda c: c.init_conduction(SEED, AMP), 25)
    _, b1, _ = _run(lbm, p, lambda c: c.init_temperature(t), 25)
    for k in ("f", "g", "phi", "uy"):
        assert relerr(b1[k], a1[k]) <= tol, (k, relerr(b1[k], a1[k]))


@pytest.mark.gpu
@pytest.mark.parametrize("storage,dtype", [("f32", np.float32), ("f64", np.float64), ("f16s", np.float32)])
def test_temperature_from_pinned_and_device_tensors(gpu, storage, dtype):
    """Pageable host memory is copied in first; page-locked host memory and
    device memory are read by the init kernel itself: the same state."""
    import torch

    lbm = gpu
    p = _params(lbm, storage, False)
    t = lbm.conduction_temperature(LX, LY, LZ, SEED, AMP, dtype=dtype)
    ref = _run(lbm, p, lambda c: c.init_temperature(t), 5)[1]
    pinned = torch.from_numpy(t).pin_memory()
    dev = torch.from_numpy(t).cuda()
    stream = torch.cuda.Stream()
    for src, st in ((pinned, stream), (dev, None)):
        got = _run(lbm, p, lambda c: c.init_temperature(src, stream=st), 5)[1]
        for k in ref:
            assert np.array_equal(got[k], ref[k]), k


@pytest.mark.gpu
def test_temperature_argument_checks(gpu):
    import torch

    lbm = gpu
    with lbm.Case(_params(lbm, "f32", True)) as c:
        with pytest.raises(ValueError):
            c.init_temperature(np.zeros(LX * LY * LZ - 1))
        with pytest.raises(ValueError):
            c.init_temperature(torch.zeros(LX * LY * LZ, dtype=torch.float64))
        with pytest.raises(lbm.LbmError):
            c.step(1)   # a rejected start leaves the case uninitialised
        c.init_temperature(np.full(LX * LY * LZ, 0.5))   # converted to float32
        c.step(1)
