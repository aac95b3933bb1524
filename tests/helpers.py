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


# ---- decaying shear wave (viscosity of a collision model) ------------------
#
# u_x(z) = U sin(k z), k = 2 pi / LZ, in a box with periodic x and z and the
# plates far away (LY = 48: the no-slip walls do not reach the mid-plane in
# the time measured), uniform temperature t0 and negligible buoyancy (g beta
# = 1e-10).  The Navier-Stokes solution decays as exp(-nu k^2 t); the lattice
# viscosity of BGK and of regularised BGK is nu = (tau - 1/2) / 3, up to
# discretisation error that vanishes as k -> 0.
SHEAR_GB = 1e-10


def shear_params(tau: float, ly: int, pr: float = 0.71) -> dict:
    """Run-surface values for a case whose tau_f is `tau`: Ra from
    src/globals.cu:13-16 solved for the viscosity (tau - 1/2) / 3."""
    visc = (tau - 0.5) / 3.0
    return dict(rayleigh=SHEAR_GB * 1.0 * ly ** 3 * pr / visc ** 2, prandtl=pr, beta=SHEAR_GB)


def shear_state(lx: int, ly: int, lz: int, amplitude: float = 1e-3) -> dict:
    """Equilibrium populations of the shear wave in the reference's restart
    layout (f a density deviation with rho = 0, g at T = 0.5 = t0)."""
    from oracle.oracle import CX, W

    k = 2.0 * np.pi / lz
    ux = np.broadcast_to((amplitude * np.sin(k * np.arange(lz)))[:, None, None], (lz, ly, lx)).copy()
    f = np.empty((27, lz, ly, lx))
    g = np.empty_like(f)
    for i in range(27):
        cu = 3.0 * (CX[i] * ux)
        p = cu + 0.5 * cu * cu - 1.5 * ux * ux
        f[i] = W[i] * p
        g[i] = W[i] * 0.5 * (1.0 + p)
    zero = np.zeros_like(ux)
    return dict(rho=zero, ux=ux, uy=zero, uz=zero, phi=zero + 0.5, f=f, g=g)


def shear_amplitude(ux: np.ndarray, ly: int, lz: int) -> float:
    """Projection of u_x on sin(k z) over the mid-plane y = LY / 2."""
    u = np.asarray(ux).reshape(lz, ly, -1)[:, ly // 2, :].mean(axis=1)
    return float(2.0 / lz * np.sum(u * np.sin(2.0 * np.pi / lz * np.arange(lz))))


def shear_steps(tau: float, lz: int) -> int:
    """Steps over which the amplitude falls by about e^-1/2."""
    k = 2.0 * np.pi / lz
    return int(0.5 / ((tau - 0.5) / 3.0 * k * k))
