"""Shared helpers for the parity tests."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def relerr(a, b) -> float:
    """max |a - b| / max |b| (the field-relative error the tolerances use)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = float(np.max(np.abs(b))) if b.size else 0.0
    return float(np.max(np.abs(a - b))) / max(scale, 1e-300)


def load_golden(name: str) -> dict:
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        raise FileNotFoundError(f"golden fixture {path} missing (made by tests/golden/make_golden.py)")
    z = np.load(path, allow_pickle=False)
    return {k: z[k] for k in z.files}


def nu_from_fields(uy, phi, lx, ly, lz, diff, dT=1.0):
    """Nu_bulk, Nu_top, Nu_bottom of src/output.cu:199-256 from flat fields."""
    uy = np.asarray(uy).reshape(lz, ly, lx)
    phi = np.asarray(phi).reshape(lz, ly, lx)
    nu_bulk = 1.0 + float(np.mean(uy * phi)) * ly / (diff * dT)
    bot = (-3.0 * phi[:, 0, :] + 4.0 * phi[:, 1, :] - phi[:, 2, :]) / 2.0
    top = (3.0 * phi[:, ly - 1, :] - 4.0 * phi[:, ly - 2, :] + phi[:, ly - 3, :]) / 2.0
    return nu_bulk, -float(np.mean(top)) * ly / dT, -float(np.mean(bot)) * ly / dT


def parse_nu_txt(txt: str) -> np.ndarray:
    """Rows (step, 0, Nu_bulk, Nu_top, Nu_bottom) of a reference Nu file."""
    rows = [[float(v) for v in line.split()] for line in txt.strip().splitlines() if line.strip()]
    return np.array(rows, dtype=np.float64).reshape(-1, 5)
