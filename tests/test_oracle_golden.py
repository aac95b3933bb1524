"""The CPU oracle against the reference program's own outputs.

The fixtures under tests/golden/ were written by the reference binary
(Summer536/LBM_DDF src/, rebuilt for sm_100a by oracle/build_ref.py) started
through its restart path from seeded states (tests/golden/make_golden.py).
This pins the oracle: with its default contraction model (the multiply-adds
nvcc fuses in the reference build, lbm_oracle.c) every population and every
macroscopic field is bitwise equal to the reference's after 1, 2, 50 and 1000
steps; the parity bounds (1e-12 field-relative, Nu 1e-10) are checked as
well, and the reference's printed Nu lines (7 significant digits) are
reproduced.
"""
import hashlib

import numpy as np
import pytest

from helpers import load_golden, nu_from_fields, parse_nu_txt, relerr
from oracle.ref_cases import REF_CASES

CASES = ["w12_s1", "w12_s2", "w12_rest50", "w12_s1000", "w24_s1000"]


def _oracle_for(oracle_mod, name):
    c = REF_CASES[name]
    p = oracle_mod.make_params(c["lx"], c["ly"], c["lz"], rayleigh=c["rayleigh"], prandtl=c["prandtl"])
    return oracle_mod.Oracle(p), c


def _start(o, g, c):
    if c["continue_step"] == 0:
        o.init_rest()
        return
    o.init_conduction(int(g["seed"]), float(g["amplitude"]))
    h = hashlib.sha256()
    for k in ("rho", "ux", "uy", "uz", "phi", "f", "g"):
        h.update(np.ascontiguousarray(o.field(k), dtype=np.float64).tobytes())
    assert h.hexdigest() == str(g["input_sha256"]), "regenerated input differs from the fixture's"
    # feed it through the restart semantics, as the reference read it
    st = {k: o.field(k).copy() for k in ("rho", "ux", "uy", "uz", "phi", "f", "g")}
    o.load_restart(**st)


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference(oracle_mod, name):
    g = load_golden(name)
    o, c = _oracle_for(oracle_mod, name)
    _start(o, g, c)
    steps = int(g["steps"])
    nnu = c.get("nnuout")
    nu_ref = parse_nu_txt(str(g["nu_txt"])) if nnu else None
    done = 0
    rows = []
    step0 = c["continue_step"]
    while done < steps:
        todo = steps - done
        if nnu:
            nxt = ((step0 + done) // nnu + 1) * nnu - step0
            todo = min(todo, nxt - done)
        o.step(todo)
        done += todo
        if nnu and (step0 + done) % nnu == 0:
            ob = o.observables()
            rows.append([step0 + done, 0.0, ob["nu_bulk"], ob["nu_top"], ob["nu_bottom"]])
    n = o.n
    if "sample_nodes" in g:
        nodes = g["sample_nodes"]
        f = o.field("f").reshape(27, n)[:, nodes]
        gg = o.field("g").reshape(27, n)[:, nodes]
    else:
        f = o.field("f").reshape(-1)
        gg = o.field("g").reshape(-1)
    assert relerr(f, g["f"].reshape(f.shape)) <= 1e-12
    assert relerr(gg, g["g"].reshape(gg.shape)) <= 1e-12
    assert np.array_equal(f.reshape(-1), g["f"].reshape(-1)), "f not bitwise equal"
    assert np.array_equal(gg.reshape(-1), g["g"].reshape(-1)), "g not bitwise equal"
    for k in ("rho", "ux", "uy", "uz", "phi"):
        assert relerr(o.field(k).reshape(-1), g[k]) <= 1e-12, k
        assert np.array_equal(o.field(k).reshape(-1), g[k]), k
    nu_o = nu_from_fields(o.field("uy"), o.field("phi"), c["lx"], c["ly"], c["lz"], o.params.diff)
    nu_r = nu_from_fields(g["uy"], g["phi"], c["lx"], c["ly"], c["lz"], o.params.diff)
    for a, b in zip(nu_o, nu_r):
        assert abs(a - b) <= 1e-10 * max(1.0, abs(b))
    if nnu:
        got = np.array(rows)
        assert got.shape == nu_ref.shape
        np.testing.assert_allclose(got[:, 0], nu_ref[:, 0])
        # %15.6E keeps 7 significant digits
        np.testing.assert_allclose(got[:, 2:], nu_ref[:, 2:], rtol=1e-6, atol=1e-12)


def test_oracle_nu_formula_matches_numpy(oracle_mod):
    """orc_observables' Nu equals the numpy restatement of src/output.cu:199-256."""
    o, c = _oracle_for(oracle_mod, "w24_s1000")
    o.init_conduction(3, 1e-3)
    o.step(20)
    ob = o.observables()
    nb, nt, nbot = nu_from_fields(o.field("uy"), o.field("phi"), c["lx"], c["ly"], c["lz"], o.params.diff)
    assert abs(ob["nu_bulk"] - nb) < 1e-12
    assert abs(ob["nu_top"] - nt) < 1e-12
    assert abs(ob["nu_bottom"] - nbot) < 1e-12


def test_contraction_model_is_needed(oracle_mod):
    """Without the fused multiply-adds the oracle is off by an ulp after one
    step, so the bitwise comparisons above do test the rounding model."""
    g = load_golden("w12_s1")
    default = oracle_mod.get_contract()
    try:
        oracle_mod.set_contract(0)
        o, c = _oracle_for(oracle_mod, "w12_s1")
        _start(o, g, c)
        o.step(1)
        assert not np.array_equal(o.field("g").reshape(-1), g["g"].reshape(-1))
        assert relerr(o.field("g").reshape(-1), g["g"].reshape(-1)) < 1e-15
    finally:
        oracle_mod.set_contract(default)


@pytest.mark.parametrize("grid,seed", [((12, 10, 8), 20240611), ((16, 12, 10), 1000), ((8, 5, 4), 7)])
def test_conduction_restart_bytes_match_oracle(oracle_mod, grid, seed):
    """oracle/ref_run.conduction_restart (the restart files that feed the
    reference program the seeded conduction state, in bench.py's reference
    arm) is bitwise the oracle's own orc_init_conduction state."""
    import numpy as np

    from oracle.ref_run import conduction_restart

    lx, ly, lz = grid
    o = oracle_mod.Oracle(oracle_mod.make_params(lx, ly, lz, rayleigh=1e7))
    o.init_conduction(seed, 1e-3)
    flow, fg = conduction_restart(lx, ly, lz, seed, 1e-3)
    want_flow = b"".join(o.field(k).reshape(-1).tobytes() for k in ("rho", "ux", "uy", "uz", "phi"))
    want_fg = o.field("f").reshape(-1).tobytes() + o.field("g").reshape(-1).tobytes()
    o.close()
    assert b"".join(flow()) == want_flow
    assert b"".join(fg()) == want_fg
