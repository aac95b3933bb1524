"""Runs a reference binary built by oracle/build_ref.py.  TEST INFRASTRUCTURE.

The reference program (Summer536/LBM_DDF ``src/``) reads and writes its state
only through files in a directory named ``Ra%.1ePr%.2f`` (``src/output.cu:5``):

* restart input (``src/initial.cu:110-205``): ``%09d.dat`` = rho, ux, uy, uz,
  phi (N doubles each) and ``fg%09d.dat`` = f then g (27*N doubles each), raw
  native-endian, reference index order;
* at NEND (``src/main.cu:67-76``): the same two files for step NEND;
* every NNUOUT / NDIAG steps: ``Nu_<Ra>.txt`` (``src/output.cu:164-178,259``),
  ``Profile_<Ra>.txt`` and ``statistics.dat``.

``run_case`` writes the restart files, runs the binary in a scratch directory
and returns its outputs.  ``time_case`` runs a timing binary with its NEND
files pointed at /dev/null and returns the "GPU computation time" it prints
(``src/main.cu:92``), the sum of its per-step CUDA-event times.
"""
from __future__ import annotations

import os
import re
import subprocess
import tempfile

import numpy as np

try:
    from .ref_cases import REF_CASES
except ImportError:  # run from inside oracle/
    from ref_cases import REF_CASES

HERE = os.path.dirname(os.path.abspath(__file__))


def binary(name: str) -> str:
    return os.path.join(HERE, "_ref", "rb3d_" + name)


def case_dir(c: dict) -> str:
    return "Ra%.1ePr%.2f" % (c["rayleigh"], c["prandtl"])


def nu_name(c: dict, stem: str) -> str:
    """File-name rule of src/output.cu:164-178 / :298-312."""
    ra = c["rayleigh"]
    known = {1e5: "1e50", 5e5: "5e50", 1e6: "1e60", 5e6: "5e60", 1e7: "1e70", 1e8: "1e80"}
    return f"{stem}_{known[ra]}.txt" if ra in known else f"{stem}_%.2e.txt" % ra


def write_restart(directory: str, step: int, rho, ux, uy, uz, phi, f, g) -> None:
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, "%09d.dat" % step), "wb") as fh:
        for a in (rho, ux, uy, uz, phi):
            fh.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    with open(os.path.join(directory, "fg%09d.dat" % step), "wb") as fh:
        for a in (f, g):
            fh.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())


def read_state(directory: str, step: int, n: int) -> dict:
    flow = np.fromfile(os.path.join(directory, "%09d.dat" % step), dtype=np.float64)
    fg = np.fromfile(os.path.join(directory, "fg%09d.dat" % step), dtype=np.float64)
    assert flow.size == 5 * n and fg.size == 54 * n, (flow.size, fg.size, n)
    out = {k: flow[i * n:(i + 1) * n].copy() for i, k in enumerate(["rho", "ux", "uy", "uz", "phi"])}
    out["f"] = fg[: 27 * n].copy()
    out["g"] = fg[27 * n:].copy()
    return out


def run_case(name: str, restart: dict | None = None, timeout: float = 600.0) -> dict:
    """Runs case `name`; `restart` holds rho, ux, uy, uz, phi, f, g (flat,
    reference layout) when the case has continue_step > 0."""
    c = REF_CASES[name]
    n = c["lx"] * c["ly"] * c["lz"]
    with tempfile.TemporaryDirectory(prefix="lbmref_") as work:
        d = os.path.join(work, case_dir(c))
        if c["continue_step"] > 0:
            assert restart is not None, "case starts from a restart"
            write_restart(d, c["continue_step"], *(restart[k] for k in
                                                   ("rho", "ux", "uy", "uz", "phi", "f", "g")))
        proc = subprocess.run([binary(name)], cwd=work, capture_output=True, text=True,
                              timeout=timeout)
        if proc.returncode != 0:
            raise RuntimeError(f"reference {name} failed ({proc.returncode}): {proc.stderr[-2000:]}")
        out = read_state(d, c["nend"], n)
        out["stdout"] = proc.stdout
        for stem in ("Nu", "Profile"):
            p = os.path.join(d, nu_name(c, stem))
            out[stem.lower() + "_txt"] = open(p).read() if os.path.exists(p) else ""
        p = os.path.join(d, "statistics.dat")
        out["statistics_txt"] = open(p).read() if os.path.exists(p) else ""
        return out


def time_case(name: str, timeout: float = 900.0) -> float:
    """GPU seconds the reference reports for all of its steps of case `name`."""
    c = REF_CASES[name]
    with tempfile.TemporaryDirectory(prefix="lbmref_") as work:
        d = os.path.join(work, case_dir(c))
        os.makedirs(d)
        for fn in ("%09d.dat" % c["nend"], "fg%09d.dat" % c["nend"]):
            os.symlink(os.devnull, os.path.join(d, fn))
        proc = subprocess.run([binary(name)], cwd=work, capture_output=True, text=True,
                              timeout=timeout)
        if proc.returncode != 0:
            raise RuntimeError(f"reference {name} failed ({proc.returncode}): {proc.stderr[-2000:]}")
        m = re.search(r"GPU computation time:\s*([0-9.eE+-]+)", proc.stdout)
        if not m:
            raise RuntimeError("no GPU time in reference output: " + proc.stdout[-500:])
        return float(m.group(1))
