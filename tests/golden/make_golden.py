"""Generates the golden fixtures of tests/golden/ by running the reference.

Run on a machine with a B200 (the reference program is CUDA):

    python tests/golden/make_golden.py

For each parity case of oracle/ref_cases.py it builds the seeded input state,
feeds it to the reference binary ``oracle/_ref/rb3d_<case>`` through the
reference's restart path, and stores what the reference wrote at NEND:

* ``<case>.npz``: f, g (27*N) and rho, ux, uy, uz, phi (N), float64, reference
  layout; for the larger case only the macroscopic fields plus f and g at a
  fixed sample of nodes (``sample_nodes``) are kept, to stay small;
* the text outputs (Nu, profile, statistics) as strings;
* ``input_sha256``: a hash of the input state, so the tests can check that
  they regenerate the very same input.

Inputs: the conduction state of ``lbm_oracle.h`` (orc_init_conduction, seed
``SEED``, amplitude 1e-3) for restart cases — the oracle here only generates
the input, whose bytes are recorded — and the reference's own rest state
(init_arrays) for ``w12_rest50``.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Oracle, make_params  # noqa: E402
from oracle.ref_cases import REF_CASES  # noqa: E402
from oracle import ref_run  # noqa: E402

SEED = 20240611
AMPLITUDE = 1e-3
PARITY_CASES = ["w12_s1", "w12_s2", "w12_rest50", "w12_s1000", "w24_s1000"]
SAMPLED = {"w24_s1000": 256}


def input_state(name: str) -> dict | None:
    c = REF_CASES[name]
    if c["continue_step"] == 0:
        return None
    o = Oracle(make_params(c["lx"], c["ly"], c["lz"], rayleigh=c["rayleigh"], prandtl=c["prandtl"]))
    o.init_conduction(SEED, AMPLITUDE)
    st = {k: o.field(k).reshape(-1).copy() for k in ("rho", "ux", "uy", "uz", "phi", "f", "g")}
    o.close()
    return st


def state_hash(st: dict) -> str:
    h = hashlib.sha256()
    for k in ("rho", "ux", "uy", "uz", "phi", "f", "g"):
        h.update(np.ascontiguousarray(st[k], dtype=np.float64).tobytes())
    return h.hexdigest()


def sample_nodes(n: int, count: int) -> np.ndarray:
    rng = np.random.default_rng(12345)
    return np.sort(rng.choice(n, size=count, replace=False))


def main(argv=None) -> int:
    import argparse
    import shutil

    ap = argparse.ArgumentParser()
    ap.add_argument("--copy-to", default=None, help="also copy the fixtures to this directory")
    args = ap.parse_args(argv)
    for name in PARITY_CASES:
        c = REF_CASES[name]
        n = c["lx"] * c["ly"] * c["lz"]
        st = input_state(name)
        out = ref_run.run_case(name, restart=st)
        keep = dict(rho=out["rho"], ux=out["ux"], uy=out["uy"], uz=out["uz"], phi=out["phi"])
        if name in SAMPLED:
            nodes = sample_nodes(n, SAMPLED[name])
            keep["sample_nodes"] = nodes
            keep["f"] = out["f"].reshape(27, n)[:, nodes]
            keep["g"] = out["g"].reshape(27, n)[:, nodes]
        else:
            keep["f"] = out["f"]
            keep["g"] = out["g"]
        meta = dict(case=name, seed=SEED if st is not None else -1, amplitude=AMPLITUDE,
                    steps=c["nend"] - c["continue_step"],
                    input_sha256=state_hash(st) if st is not None else "",
                    nu_txt=out["nu_txt"], profile_txt=out["profile_txt"],
                    statistics_txt=out["statistics_txt"])
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **keep, **{k: np.array(v) for k, v in meta.items()})
        print("wrote", path, os.path.getsize(path), "bytes")
        if args.copy_to:
            os.makedirs(args.copy_to, exist_ok=True)
            shutil.copy(path, args.copy_to)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
