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
(``src/main.cu:92``), the sum of its per-step CUDA-event times; given a
restart state (``conduction_restart``) it feeds the two restart files
through named pipes, so a 256^3 state (8 GB of files) needs no disk.
"""
from __future__ import annotations

import os
import re
import subprocess
import tempfile
import threading

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


# D3Q27 weights in the order of src/initial.cu:71-83
_W = [8.0 / 27.0] + [2.0 / 27.0] * 6 + [1.0 / 54.0] * 12 + [1.0 / 216.0] * 8


def _splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return x ^ (x >> np.uint64(31))


def conduction_restart(lx: int, ly: int, lz: int, seed: int, amplitude: float = 1e-3, t_hot: float = 1.0,
                       t_cold: float = 0.0, gravity: float = 1.0, beta: float | None = None):
    """The seeded conduction state of orc_init_conduction (lbm_oracle.c) as
    the reference's two restart files, generated in pieces.

    Returns (flow, fg): functions that each yield the bytes of one file in
    order: ``%09d.dat`` = rho, ux, uy, uz, phi and ``fg%09d.dat`` = f, g
    (src/initial.cu:110-205), FP64, reference node order.  The state: T =
    T_hot - ((T_hot - T_cold) iy) / (LY - 1) + amplitude (2u - 1), u the
    oracle's counter-based noise; f = 0, g_i = w_i T; rho = 0, u = (0, F_y/2,
    0) with F_y = g beta (T - t0), phi = sum_i g_i in population order, as
    src/macrovar.cu:3-34 leaves them (tests/test_oracle_golden.py checks the
    bytes against the oracle's own state).  The engine's
    lbm_init_conduction(seed, amplitude) starts from the same state."""
    if beta is None:
        beta = 0.01 / (gravity * (t_hot - t_cold) * ly)
    n = lx * ly * lz
    key = _splitmix64(np.array([seed], dtype=np.uint64))[0]

    def temperature():
        with np.errstate(over="ignore"):
            r = _splitmix64(np.arange(n, dtype=np.uint64) + key)
        u = (r >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
        del r
        iy = np.broadcast_to(np.arange(ly, dtype=np.float64)[None, :, None], (lz, ly, lx)).reshape(-1)
        t = t_hot - ((t_hot - t_cold) * iy) / (ly - 1.0)
        return t + amplitude * (2.0 * u - 1.0)

    gb = gravity * beta
    t0 = 0.5 * (t_cold + t_hot)

    def flow():
        t = temperature()
        zeros = np.zeros(n)
        yield zeros.tobytes()                                    # rho
        yield zeros.tobytes()                                    # ux
        yield (0.0 + 0.5 * (gb * (t - t0))).tobytes()            # uy
        yield zeros.tobytes()                                    # uz
        phi = np.zeros(n)
        for w in _W:
            phi += w * t
        yield phi.tobytes()

    def fg():
        t = temperature()
        zeros = np.zeros(n).tobytes()
        for _ in range(27):
            yield zeros                                          # f
        for w in _W:
            yield (w * t).tobytes()                              # g

    return flow, fg


def _feed(path: str, chunks, errors: list):
    try:
        with open(path, "wb", buffering=0) as fh:    # blocks until the reader opens the pipe
            for b in chunks():
                fh.write(b)
    except BrokenPipeError:
        errors.append(path)


def time_case(name: str, timeout: float = 900.0, restart=None) -> float:
    """GPU seconds the reference reports for all of its steps of case `name`;
    `restart` = (flow, fg) from conduction_restart for cases that start from
    a restart (fed through named pipes)."""
    c = REF_CASES[name]
    with tempfile.TemporaryDirectory(prefix="lbmref_") as work:
        d = os.path.join(work, case_dir(c))
        os.makedirs(d)
        for fn in ("%09d.dat" % c["nend"], "fg%09d.dat" % c["nend"]):
            os.symlink(os.devnull, os.path.join(d, fn))
        feeders, errors = [], []
        if c["continue_step"] > 0:
            if restart is None:
                raise ValueError(f"{name} starts from a restart state")
            for fn, gen in zip(("%09d.dat" % c["continue_step"], "fg%09d.dat" % c["continue_step"]), restart):
                path = os.path.join(d, fn)
                os.mkfifo(path)
                th = threading.Thread(target=_feed, args=(path, gen, errors), daemon=True)
                th.start()
                feeders.append((path, th))
        try:
            proc = subprocess.run([binary(name)], cwd=work, capture_output=True, text=True, timeout=timeout)
        finally:
            for path, th in feeders:     # release a writer whose reader never came
                if th.is_alive():
                    try:
                        fd = os.open(path, os.O_RDONLY | os.O_NONBLOCK)
                        os.close(fd)
                    except OSError:
                        pass
                th.join(timeout=60)
        if proc.returncode != 0:
            raise RuntimeError(f"reference {name} failed ({proc.returncode}): {proc.stderr[-2000:]}")
        if errors:
            raise RuntimeError(f"reference {name} stopped reading its restart files: {errors}")
        m = re.search(r"GPU computation time:\s*([0-9.eE+-]+)", proc.stdout)
        if not m:
            raise RuntimeError("no GPU time in reference output: " + proc.stdout[-500:])
        return float(m.group(1))
