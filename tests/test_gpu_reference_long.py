"""The FP64 engine against the reference's own program over a long run at
the 64^3 benchmark grid: 10,000 steps at Ra 1e5 in the closed box, from the
same seeded state fed to both (the reference through its restart files).

The reference binary is built from the unmodified reference sources by
oracle/build_ref.py (with __graft_entry__.build()); without it the test is
skipped."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NAME = "c0_s10000"


def _series(txt):
    return np.array([[float(x) for x in l.split()] for l in txt.strip().splitlines() if l.strip()])


def test_f64_engine_equals_reference_program_10000_steps(lbm, oracle_mod):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from oracle import ref_run
    from oracle.ref_cases import REF_CASES

    if not os.path.exists(ref_run.binary(NAME)):
        pytest.skip("reference binary not built")
    c = REF_CASES[NAME]
    o = oracle_mod.Oracle(oracle_mod.make_params(c["lx"], c["ly"], c["lz"], rayleigh=c["rayleigh"],
                                                 prandtl=c["prandtl"]))
    o.init_conduction(31, 1e-3)
    st = {k: o.field(k).reshape(-1).copy() for k in ("rho", "ux", "uy", "uz", "phi", "f", "g")}
    ref = ref_run.run_case(NAME, st, timeout=900)
    p = lbm.make_params(c["lx"], c["ly"], c["lz"], rayleigh=c["rayleigh"], prandtl=c["prandtl"],
                        sides=lbm.SIDES_WALL, storage="f64")
    # the reference writes Nu when its absolute step is a multiple of NNUOUT
    marks = [s for s in range(c["continue_step"] + 1, c["nend"] + 1) if s % c["nnuout"] == 0]
    nu = []
    with lbm.Case(p) as case:
        case.load_ref_state(*(st[k] for k in ("rho", "ux", "uy", "uz", "phi", "f", "g")))
        at = c["continue_step"]
        for m in marks:
            case.step(m - at)
            at = m
            ob = case.observables()
            nu.append((ob["nu_bulk"], ob["nu_top"], ob["nu_bottom"]))
        case.step(c["nend"] - at)
        got = case.store_ref_state()
    for k in ("f", "g", "rho", "ux", "uy", "uz", "phi"):
        assert np.array_equal(got[k].reshape(-1), ref[k]), k + " not bitwise the reference's"
    # the reference's Nu file (src/output.cu:148-280): one row per NNUOUT steps,
    # printed with 7 significant digits
    want = _series(ref["nu_txt"])   # columns: step, 0, Nu_bulk, Nu_top, Nu_bottom
    assert want.shape == (len(nu), 5)
    assert list(want[:, 0]) == [float(m) for m in marks]
    np.testing.assert_allclose(np.array(nu), want[:, 2:], rtol=2e-6, atol=1e-20)


def test_reference_timing_runs_fed_through_pipes():
    """bench.py's reference arm feeds the seeded conduction state to the
    reference program through named pipes in place of its restart files
    (src/initial.cu:110-205 reads them with sequential fread); at 64^3 both
    timing runs complete and report a GPU time that grows with the steps."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from oracle import ref_run
    from oracle.ref_cases import REF_CASES, TIMING_SEED, TIMING_SETS

    short, long_ = TIMING_SETS["c0"]
    if not (os.path.exists(ref_run.binary(short)) and os.path.exists(ref_run.binary(long_))):
        pytest.skip("reference timing binaries not built")
    c = REF_CASES[long_]
    state = ref_run.conduction_restart(c["lx"], c["ly"], c["lz"], TIMING_SEED, 1e-3)
    ta = ref_run.time_case(short, restart=state, timeout=300)
    tb = ref_run.time_case(long_, restart=state, timeout=300)
    assert 0.0 <= ta < tb
