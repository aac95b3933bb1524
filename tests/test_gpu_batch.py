"""Batches: many cases of different grids and parameters advanced by one
kernel launch per step (C ABI lbm_batch_*).

- each member equals the same case stepped alone by the single-case kernel
  (bitwise in FP64; FP32 to rounding, the two kernels being compiled apart);
- "alone = in the mix": a case in a batch of one and in a mixed batch gives
  bitwise the same state, in every storage format;
- graphs, odd step counts, membership changes and the autotuner do not
  change results.
"""
import numpy as np
import pytest

from helpers import relerr

pytestmark = pytest.mark.gpu

MIX = [(32, 32, 32, 1e5, 0.71), (48, 24, 40, 3e6, 4.38), (64, 32, 48, 1e4, 7.0), (40, 16, 24, 1e7, 0.71)]


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def make_cases(lbm, storage, specs=MIX, seed0=100):
    cases = []
    for i, (lx, ly, lz, ra, pr) in enumerate(specs):
        c = lbm.Case(lbm.make_params(lx, ly, lz, rayleigh=ra, prandtl=pr, sides=lbm.SIDES_PERIODIC, storage=storage))
        c.init_conduction(seed0 + i, 1e-2)
        cases.append(c)
    return cases


def states(cases, fields=("f", "g", "phi", "uy")):
    return [c.store_ref_state(fields) for c in cases]


@pytest.mark.parametrize("storage", ["f64", "f32", "f16s", "bf16s"])
def test_batch_equals_single_case_kernel(lbm, storage):
    steps = 9
    solo = make_cases(lbm, storage)
    for c in solo:
        c.step(steps)
    a = states(solo)
    mixed = make_cases(lbm, storage)
    with lbm.Batch(storage) as b:
        for c in mixed:
            b.add(c)
        b.step(4)
        b.step(5)
        assert all(c.step_count == steps for c in mixed)
        got = states(mixed)
    for x, y in zip(a, got):
        for k in x:
            if storage == "f64":
                assert np.array_equal(x[k], y[k]), k
            else:
                tol = {"f32": 2e-6, "f16s": 2e-3, "bf16s": 2e-2}[storage]
                assert relerr(y[k], x[k]) <= tol, k
    for c in solo + mixed:
        c.close()


@pytest.mark.parametrize("storage", ["f64", "f32", "f16s", "bf16s"])
def test_alone_equals_in_mix(lbm, storage):
    """A case's result is bitwise the same alone (batch of one) and in a mix."""
    steps = 10
    alone = make_cases(lbm, storage, MIX[1:2], seed0=7)[0]
    with lbm.Batch(storage) as b:
        b.add(alone)
        b.step(steps)
        want = alone.store_ref_state()
        want_obs = alone.observables()
    mix = make_cases(lbm, storage, MIX, seed0=6)      # member 1 has seed 7: the same case
    with lbm.Batch(storage) as b:
        for c in mix:
            b.add(c)
        b.step(steps)
        got = mix[1].store_ref_state()
        got_obs = mix[1].observables()
    for k in want:
        assert np.array_equal(want[k], got[k]), k
    assert want_obs == got_obs
    for c in mix + [alone]:
        c.close()


def test_graph_odd_steps_and_membership(lbm):
    """7 steps in one plain batch equal 3+1+3 graph steps, and a member that
    leaves after 2 steps and finishes in another batch."""
    storage = "f32"
    ref = make_cases(lbm, storage)
    with lbm.Batch(storage) as b:
        b.set_config(128, 0, use_graph=False)
        for c in ref:
            b.add(c)
        b.step(7)
        want = states(ref)
    cases = make_cases(lbm, storage)
    with lbm.Batch(storage) as a, lbm.Batch(storage) as b, lbm.Batch(storage) as c3:
        for x in (a, b, c3):
            x.set_config(128, 0, use_graph=True)
        a.add(cases[0])
        a.add(cases[1])
        for n in (3, 1, 3):
            a.step(n)
        b.add(cases[2])
        b.add(cases[3])
        b.step(2)
        b.remove(cases[3])
        b.step(5)
        c3.add(cases[3])
        c3.step(5)
        assert all(c.step_count == 7 for c in cases)
        got = states(cases)
    for x, y in zip(want, got):
        for k in x:
            assert np.array_equal(x[k], y[k]), k
    for c in ref + cases:
        c.close()


def test_persistent_shapes_and_autotune(lbm):
    """Every launch shape, and the autotuner's trial steps, advance the
    members exactly as the single-case kernel does (FP64: bitwise)."""
    storage = "f64"
    cases = make_cases(lbm, storage)
    with lbm.Batch(storage) as b:
        for c in cases:
            b.add(c)
        b.set_config(256, 8, use_graph=True)
        b.step(2)
        b.set_config(128, 2, use_graph=False)
        b.step(2)
        # 11 launches (10 tile-walk shapes and the per-case launch) x (2
        # warm-up + 2 timed) steps
        tuned = b.autotune(steps_per_trial=2)
        assert tuned["block"] in (128, 256) and tuned["blocks_per_sm"] in (0, 4, 8, 16, 32)
        assert tuned["ms_per_step"] > 0 and tuned["launch"] in ("tiles", "per_case")
        assert b.config()["block"] == tuned["block"] and b.launch == tuned["launch"]
        b.step(2)
        total = cases[0].step_count
        assert total == 2 + 2 + 44 + 2
        got = states(cases)
    ref = make_cases(lbm, storage)
    for c in ref:
        c.step(total)
    want = states(ref)
    for x, y in zip(want, got):
        for k in x:
            assert np.array_equal(x[k], y[k]), k
    for c in ref + cases:
        c.close()


def test_init_then_step_on_another_stream(lbm, oracle_mod):
    """Initialise on the default stream, step at once on a non-blocking
    stream: the steps must see the initialised state (the init calls return
    only when the state is written).  Repeated over fresh allocations, which
    may reuse a destroyed case's memory."""
    import torch

    s = torch.cuda.Stream()
    o = oracle_mod.Oracle(oracle_mod.make_params(32, 32, 32, rayleigh=5.2e4, prandtl=7.0, periodic_sides=True))
    o.init_conduction(56, 1e-3)
    o.step(4)
    want = o.field("f").copy()
    for rep in range(6):
        junk = lbm.Case(lbm.make_params(32, 32, 32, storage="f64"))
        junk.init_conduction(999, 0.5)
        junk.step(3)
        junk.close()
        with lbm.Case(lbm.make_params(32, 32, 32, rayleigh=5.2e4, prandtl=7.0, storage="f64")) as c:
            c.init_conduction(56, 1e-3)
            c.step(4, stream=s)
            s.synchronize()
            assert np.array_equal(c.store_ref_state(("f",))["f"], want), rep


@pytest.mark.parametrize("storage", ["f64", "f16s"])
def test_mixed_collision_models(lbm, storage):
    """Members with BGK and regularised collision in one batch: each equals
    the same case stepped alone (FP64 bitwise; the regularised update is
    written with explicit rounding, so its 16-bit members are bitwise too)."""
    models = ["regularized", "bgk", "regularized", "bgk"]
    solo = make_cases(lbm, storage)
    for c, m in zip(solo, models):
        c.set_collision(m)
        c.step(6)
    want = states(solo)
    cases = make_cases(lbm, storage)
    for c, m in zip(cases, models):
        c.set_collision(m)
    with lbm.Batch(storage) as b:
        for c in cases:
            b.add(c)
        b.step(6)
        got = states(cases)
    for m, x, y in zip(models, want, got):
        for k in x:
            if storage == "f64" or m == "regularized":
                assert np.array_equal(x[k], y[k]), (m, k)
            else:
                assert relerr(y[k], x[k]) <= 2e-3, k
    for c in solo + cases:
        c.close()


def test_member_rules(lbm):
    """A case belongs to one batch; calls that change a member's state are
    refused until it leaves; destroying a member removes it."""
    cases = make_cases(lbm, "f32", MIX[:3])
    with lbm.Batch("f32") as a, lbm.Batch("f32") as b:
        for c in cases:
            a.add(c)
        with pytest.raises(lbm.LbmError):
            b.add(cases[0])                  # already in another batch
        for call in (lambda c: c.step(1), lambda c: c.init_conduction(1), lambda c: c.set_collision("bgk")):
            with pytest.raises(lbm.LbmError) as e:
                call(cases[1])
            assert e.value.code == lbm.ERR_STATE
        cases[1].observables()               # reading is fine
        cases[2].close()                     # destroying a member removes it
        assert a.size()[0] == 2
        a.step(2)
        a.remove(cases[1])
        cases[1].step(1)
        b.add(cases[1])
        b.step(1)
        assert cases[0].step_count == 2 and cases[1].step_count == 4
    for c in cases[:2]:
        c.close()


def test_batch_rejections(lbm):
    with lbm.Batch("f32") as b:
        with lbm.Case(lbm.make_params(16, 8, 8, sides=lbm.SIDES_WALL, storage="f32")) as w:
            w.init_conduction(1)
            with pytest.raises(lbm.LbmError):
                b.add(w)                      # closed box
        with lbm.Case(lbm.make_params(16, 8, 8, storage="f16s")) as h:
            h.init_conduction(1)
            with pytest.raises(lbm.LbmError):
                b.add(h)                      # other storage
        with lbm.Case(lbm.make_params(16, 8, 8, storage="f32")) as r:
            r.init_rest()
            with pytest.raises(lbm.LbmError):
                b.add(r)                      # rest state: first step alone
            r.step(1)
            b.add(r)
            with pytest.raises(lbm.LbmError):
                b.add(r)                      # twice
            b.remove(r)
        with pytest.raises(lbm.LbmError):
            b.set_config(96, 0)


@pytest.mark.parametrize("storage", ["f64", "f16s"])
def test_batch_observables_equal_per_case(lbm, storage):
    """lbm_batch_observables (one asynchronous call for every member) gives
    bitwise what lbm_get_observables gives for each member, in member order,
    also after a removal."""
    import torch

    cases = make_cases(lbm, storage)
    with lbm.Batch(storage) as b:
        for c in cases:
            b.add(c)
        b.step(3)
        got = b.observables()
        assert [g["step"] for g in got] == [3] * len(cases)
        for c, g in zip(cases, got):
            assert g == c.observables()
        b.remove(cases[1])
        b.step(2)
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        got = b.observables(stream=s)
        rest = [c for i, c in enumerate(cases) if i != 1]
        for c, g in zip(rest, got):
            assert g == c.observables()
    for c in cases:
        c.close()


@pytest.mark.parametrize("storage", ["f64", "f32", "f16s", "bf16s"])
def test_per_case_launch_is_bitwise_lbm_step(lbm, storage):
    """LBM_BATCH_PER_CASE launches each member's own single-case kernel, so
    members end bitwise as lbm_step leaves them, in every storage format,
    with mixed collision models, members joining at different step parities
    (one in each AA layout), graphs of odd and even step counts, and a
    switch back to the tile walk part-way."""
    models = ["bgk", "regularized", "bgk", "bgk"]
    solo = make_cases(lbm, storage)
    for c, m in zip(solo, models):
        c.set_collision(m)
    solo[2].step(1)                            # one member starts in the other layout
    for c in solo:
        c.step(9)
    want = states(solo)
    cases = make_cases(lbm, storage)
    for c, m in zip(cases, models):
        c.set_collision(m)
    cases[2].step(1)
    with lbm.Batch(storage) as b:
        b.set_launch("per_case")
        assert b.launch == "per_case"
        for c in cases:
            b.add(c)
        b.step(3)
        b.step(1)
        b.set_config(128, 0, use_graph=False)
        b.step(2)
        b.set_config(128, 0, use_graph=True)
        b.set_launch("tiles")
        b.step(2)
        b.set_launch("per_case")
        b.step(1)
        got = states(cases)
        obs = b.observables()
    for i, (m, x, y) in enumerate(zip(models, want, got)):
        for k in x:
            if storage == "f32" or (storage in ("f16s", "bf16s") and m == "bgk"):
                # the two tile-walk steps round as the batch kernel does
                assert relerr(y[k], x[k]) <= {"f32": 2e-6, "f16s": 2e-3, "bf16s": 2e-2}[storage], (i, k)
            else:
                assert np.array_equal(x[k], y[k]), (i, m, k)
    assert [o["step"] for o in obs] == [c.step_count for c in cases]
    for c in solo + cases:
        c.close()


@pytest.mark.parametrize("storage", ["f32", "f16s"])
def test_per_case_launch_alone_is_bitwise(lbm, storage):
    """Without a tile-walk step in between, every member is bitwise the
    single-case run in every format."""
    solo = make_cases(lbm, storage)
    for c in solo:
        c.step(8)
    want = states(solo)
    cases = make_cases(lbm, storage)
    with lbm.Batch(storage) as b:
        b.set_launch("per_case")
        for c in cases:
            b.add(c)
        b.step(5)
        b.step(3)
        got = states(cases)
    for x, y in zip(want, got):
        for k in x:
            assert np.array_equal(x[k], y[k]), k
    for c in solo + cases:
        c.close()
