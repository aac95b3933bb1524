"""Observables reduced inside the step kernels (lbm_step_observed) against
the separate reduction (lbm_get_observables) of the same states.

The step kernels reduce the moments they compute anyway, in FP64, in another
order than lbm_get_observables: FP64 rounding apart.  For 16-bit BGK cases
lbm_get_observables forms each node's moments exactly as the split step
kernel does (the same loads and partial sums), so this holds there too."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("nu_bulk", "nu_top", "nu_bottom", "ke", "re", "ux_mean", "uy_mean", "uz_mean", "phi_mean")


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _close(got, want, rel, ab):
    for k in KEYS:
        assert abs(got[k] - want[k]) <= rel * abs(want[k]) + ab, (k, got[k], want[k])


@pytest.mark.parametrize("storage", ["f64", "f32", "f16s", "bf16s"])
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("collision", ["bgk", "regularized"])
@pytest.mark.parametrize("shape", [(24, 20, 16), (64, 12, 10)])
def test_step_observed_matches_get_observables(lbm, storage, periodic, collision, shape):
    """Rows of 24 nodes: warps straddle rows and planes; rows of 64: whole
    warps, a closed box's inner warps on the path without boundary tests."""
    p = lbm.make_params(*shape, rayleigh=1e6, storage=storage,
                        sides=lbm.SIDES_PERIODIC if periodic else lbm.SIDES_WALL)
    with lbm.Case(p) as a, lbm.Case(p) as b:
        for c in (a, b):
            c.set_collision(collision)
            c.init_conduction(21, 1e-2)
            c.step(30)
        want = []
        for _ in range(5):
            want.append(b.observables())
            b.step(1)
        got = a.step_observed(5)
        assert a.step_count == b.step_count == 35
        sa, sb = a.store_ref_state(("f", "g", "phi")), b.store_ref_state(("f", "g", "phi"))
    rel, ab = 1e-11, 1e-15
    for g, w in zip(got, want):
        assert g["step"] == w["step"] and g["diverged"] == 0
        _close(g, w, rel, ab)
    # the steps themselves are those of lbm_step
    for k in sa:
        if storage == "f64":
            assert np.array_equal(sa[k], sb[k]), k
        else:
            assert np.max(np.abs(sa[k] - sb[k])) <= 1e-6 * np.max(np.abs(sb[k])), k


def test_step_observed_rest_state_and_chunks(lbm):
    """From the reference's rest state (its first step collides with the
    stored phi = 0.5), in chunks of 1, 2 and 4 steps."""
    p = lbm.make_params(16, 12, 10, storage="f64", sides=lbm.SIDES_WALL)
    with lbm.Case(p) as a, lbm.Case(p) as b:
        a.init_rest()
        b.init_rest()
        got = a.step_observed(1) + a.step_observed(2) + a.step_observed(4)
        want = []
        for _ in range(7):
            want.append(b.observables())
            b.step(1)
        assert [g["step"] for g in got] == list(range(7))
        for g, w in zip(got, want):
            _close(g, w, 1e-11, 1e-15)
        assert a.observables() == b.observables()


def test_step_observed_rules(lbm):
    p = lbm.make_params(64, 8, 8, storage="f32", sides=lbm.SIDES_PERIODIC)
    with lbm.Case(p) as c:
        c.init_conduction(1)
        assert c.step_observed(0) == []
        c.set_step_kernel(lbm.KERNEL_ROW)
        with pytest.raises(lbm.LbmError):
            c.step_observed(1)


@pytest.mark.parametrize("storage", ["f64", "f32", "f16s"])
def test_step_observed_async_matches_blocking(lbm, storage):
    """lbm_step_observed_async enqueues the same steps and copies: the
    records equal lbm_step_observed's bit for bit once the stream has
    passed the calls, in chunks of 1 and 3 steps."""
    import torch

    p = lbm.make_params(24, 20, 16, rayleigh=1e6, storage=storage, sides=lbm.SIDES_PERIODIC)
    stream = torch.cuda.Stream()
    buf = lbm.ObservablesBuffer(10)
    with lbm.Case(p) as a, lbm.Case(p) as b:
        for c in (a, b):
            c.init_conduction(5, 1e-2)
            c.step(20)
        want = b.step_observed(4) + b.step_observed(6)
        for i in range(4):
            a.step_observed_async(1, buf, first=i, stream=stream)
        a.step_observed_async(3, buf, first=4, stream=stream)
        a.step_observed_async(3, buf, first=7, stream=stream)
        stream.synchronize()
        got = [buf[i] for i in range(10)]
        assert got == want
        assert a.observables() == b.observables()


def test_step_observed_async_rules(lbm):
    p = lbm.make_params(32, 8, 8, storage="f32", sides=lbm.SIDES_PERIODIC)
    buf = lbm.ObservablesBuffer(2)
    with lbm.Case(p) as c:
        with pytest.raises(lbm.LbmError):
            c.step_observed_async(1, buf)   # not initialised
        c.init_conduction(1)
        with pytest.raises(ValueError):
            c.step_observed_async(3, buf)
        with pytest.raises(ValueError):
            c.step_observed_async(1, buf, first=2)
        c.step_observed_async(2, buf)
        c.step_observed_async(0, buf)
        c.set_step_kernel(lbm.KERNEL_ROW)
        with pytest.raises(lbm.LbmError):
            c.step_observed_async(1, buf)
        import torch

        torch.cuda.synchronize()
        assert [buf[i]["step"] for i in range(2)] == [0, 1]
