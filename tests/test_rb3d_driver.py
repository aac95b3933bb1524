"""The C++ host driver lbm_ddf_b200/rb3d: the reference's run surface
(src/parameters.h, src/main.cu) over the C ABI.

CPU: the parameters.h reader evaluates the reference's macro expressions and
derives tau, kappa, ... as src/globals.cu does.
GPU: started from the reference's own restart files (the ones the golden
fixtures were made from), rb3d writes the files the reference wrote:
fg%09d.dat and %09d.dat bitwise equal, the Nu / profile / statistics text
series equal to the printed digits.
"""
import os
import subprocess

import numpy as np
import pytest

from helpers import load_golden
from oracle.ref_cases import REF_CASES

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RB3D = os.path.join(ROOT, "lbm_ddf_b200", "rb3d")


def params_h(c, **extra) -> str:
    """A parameters.h in the reference's own format for case c."""
    lines = ["#ifndef PARAMETERS_H", "#define PARAMETERS_H", "",
             f"#define CONTINUE_STEP {c['continue_step']}",
             f"#define LX {c['lx']}", f"#define LY {c['ly']}", f"#define LZ {c['lz']}",
             "#define LXYZ (LX * LY * LZ)", "#define NPOP 27",
             f"#define NEND {c['nend']}", f"#define NDIAG {c.get('ndiag', 1000000000)}",
             f"#define NFLOWOUT {c.get('nflowout', 1000000000)}", f"#define NNUOUT {c.get('nnuout', 1000000000)}",
             f"#define RAYLEIGH {c['rayleigh']!r}", f"#define PRANDTL {c['prandtl']!r}",
             "#define T_HOT 1.0", "#define T_COLD 0.0", "#define GRAVITY 1.0",
             "#define BETA (0.01 / (LY * 1.0))  // free-fall velocity 0.1",
             "#define BLOCK_X 8", "#define BLOCK_Y 8", "#define BLOCK_Z 4", "", "#endif"]
    return "\n".join(lines) + "\n"


def dry(args):
    out = subprocess.run([RB3D, "--dry-run"] + args, capture_output=True, text=True, check=True).stdout
    return dict(line.split(" = ", 1) for line in out.strip().splitlines())


def test_dry_run_reference_defaults(lbm):
    v = dry([])
    assert float(v["LX"]) == 400 and float(v["NEND"]) == 1000
    assert float(v["BETA"]) == 0.1 / (400 * 5.0)
    assert v["dir"] == "Ra1.0e+07Pr0.71"


def test_params_file_expressions(lbm, oracle_mod, tmp_path):
    c = REF_CASES["w24_s1000"]
    f = tmp_path / "parameters.h"
    f.write_text(params_h(c))
    v = dry(["--params", str(f)])
    o = oracle_mod.make_params(c["lx"], c["ly"], c["lz"], rayleigh=c["rayleigh"], prandtl=c["prandtl"])
    assert float(v["BETA"]) == 0.01 / (c["ly"] * 1.0)
    for k in ("visc", "tau", "u0", "diff", "tauc", "t0"):
        assert float(v[k]) == getattr(o, k), k
    v = dry(["--params", str(f), "--LY", "2*LX", "--RAYLEIGH", "1e8"])
    assert float(v["LY"]) == 48 and float(v["RAYLEIGH"]) == 1e8


def _profile_rows(txt):
    """Rows of a Profile file (src/output.cu:328-368): a step line, then LY
    rows of 5 values; returns the 5-value rows with the step prepended."""
    rows, step = [], None
    for line in txt.strip().splitlines():
        v = line.split()
        if len(v) == 1:
            step = float(v[0])
        elif len(v) == 5:
            rows.append([float(x) for x in v] + [step])
    return np.array(rows)


def _series(txt):
    return np.array([[float(x) for x in l.split()] for l in txt.strip().splitlines() if l.strip()])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["w12_s1000", "w12_rest50"])
def test_rb3d_writes_the_reference_files(lbm, oracle_mod, tmp_path, name):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from oracle import ref_run

    c = REF_CASES[name]
    g = load_golden(name)
    d = tmp_path / ref_run.case_dir(c)
    if c["continue_step"] > 0:
        o = oracle_mod.Oracle(oracle_mod.make_params(c["lx"], c["ly"], c["lz"], rayleigh=c["rayleigh"],
                                                     prandtl=c["prandtl"]))
        o.init_conduction(int(g["seed"]), float(g["amplitude"]))
        ref_run.write_restart(str(d), c["continue_step"], *(o.field(k) for k in
                                                            ("rho", "ux", "uy", "uz", "phi", "f", "g")))
    (tmp_path / "parameters.h").write_text(params_h(c))
    r = subprocess.run([RB3D, "--params", "parameters.h"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "Simulation completed." in r.stdout
    n = c["lx"] * c["ly"] * c["lz"]
    st = ref_run.read_state(str(d), c["nend"], n)
    for k in ("f", "g", "rho", "ux", "uy", "uz", "phi"):
        assert np.array_equal(st[k], g[k].reshape(-1)), k
    nu_want = str(g["nu_txt"])
    p = d / ref_run.nu_name(c, "Nu")
    if nu_want:
        np.testing.assert_allclose(_series(p.read_text()), _series(nu_want), rtol=2e-6, atol=1e-20)
    prof_want = str(g["profile_txt"])
    p = d / ref_run.nu_name(c, "Profile")
    if prof_want:
        a, b = _profile_rows(p.read_text()), _profile_rows(prof_want)
        assert a.shape == b.shape
        np.testing.assert_allclose(a[:, :4], b[:, :4], rtol=2e-6, atol=1e-20)
        # phi_rms = sqrt(<phi^2> - <phi>^2) is rounding noise where a plane is
        # uniform; compare its square, a difference of O(1) sums
        assert np.all(np.abs(a[:, 4] ** 2 - b[:, 4] ** 2) <= 1e-13 + 5e-6 * b[:, 4] ** 2)
    want = str(g["statistics_txt"])
    p = d / "statistics.dat"
    if want:
        np.testing.assert_allclose(_series(p.read_text()), _series(want), rtol=2e-6, atol=1e-20)


def test_rb3d_rejects_unknown_collision(lbm):
    r = subprocess.run([RB3D, "--dry-run", "--collision", "mrt"], capture_output=True, text=True)
    assert r.returncode != 0 and "collision" in r.stderr


@pytest.mark.gpu
def test_rb3d_regularized_matches_library(lbm, tmp_path):
    """rb3d --collision regularized writes the state the library computes
    for the same case (FP64, closed box, seeded conduction start)."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from oracle import ref_run

    c = dict(continue_step=0, lx=16, ly=12, lz=10, nend=40, rayleigh=1e6, prandtl=0.71)
    (tmp_path / "parameters.h").write_text(params_h(c))
    r = subprocess.run([RB3D, "--params", "parameters.h", "--collision", "regularized", "--init", "conduction",
                        "--seed", "5", "--amplitude", "0.01"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    n = c["lx"] * c["ly"] * c["lz"]
    st = ref_run.read_state(str(tmp_path / ref_run.case_dir(c)), c["nend"], n)
    p = lbm.make_params(c["lx"], c["ly"], c["lz"], rayleigh=c["rayleigh"], prandtl=c["prandtl"],
                        beta=0.01 / c["ly"], sides=lbm.SIDES_WALL, storage="f64")
    with lbm.Case(p) as case:
        case.set_collision("regularized")
        case.init_conduction(5, 0.01)
        case.step(c["nend"])
        want = case.store_ref_state(("f", "g", "phi"))
    for k in ("f", "g", "phi"):
        assert np.array_equal(st[k], want[k].reshape(-1)), k
