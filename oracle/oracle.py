"""ctypes view of the CPU oracle (oracle/liblbm_oracle.so).

TEST INFRASTRUCTURE ONLY: the parity tests, ``__graft_entry__.smoke()`` and
``bench.py``'s cpu_baseline / reference legs use this module as the checker.
The product package ``lbm_ddf_b200`` never imports it.

The oracle restates the reference single-GPU step (Summer536/LBM_DDF ``src/``)
in FP64; see ``oracle/lbm_oracle.h`` for the per-function citations.  The
same transcription compiled in FP32 (``precision="f32"``,
liblbm_oracle_f32.so) is only a CPU baseline for bench.py, not a checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblbm_oracle.so")
LIB_PATHS = {"f64": LIB_PATH, "f32": os.path.join(HERE, "liblbm_oracle_f32.so")}
CTYPES = {"f64": C.c_double, "f32": C.c_float}
DTYPES = {"f64": np.float64, "f32": np.float32}

Q = 27
# D3Q27 order of src/initial.cu:71-73
CX = np.array([0, 1, 0, -1, 0, 0, 0, 1, -1, -1, 1, 1, 0, -1, 0, 1, 0, -1, 0, 1, -1, -1, 1, 1, -1, -1, 1])
CY = np.array([0, 0, 1, 0, -1, 0, 0, 1, 1, -1, -1, 0, 1, 0, -1, 0, 1, 0, -1, 1, 1, -1, -1, 1, 1, -1, -1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, 1, 1, -1, -1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1])
W = np.array([8.0 / 27.0] + [2.0 / 27.0] * 6 + [1.0 / 54.0] * 12 + [1.0 / 216.0] * 8)


class OrcParams(C.Structure):
    _fields_ = [
        ("lx", C.c_int32), ("ly", C.c_int32), ("lz", C.c_int32),
        ("periodic_sides", C.c_int32),
        ("rayleigh", C.c_double), ("prandtl", C.c_double),
        ("t_hot", C.c_double), ("t_cold", C.c_double),
        ("gravity", C.c_double), ("beta", C.c_double),
        ("visc", C.c_double), ("tau", C.c_double), ("u0", C.c_double),
        ("diff", C.c_double), ("tauc", C.c_double), ("t0", C.c_double),
    ]


_libs = {}


def build() -> str:
    """Compile the oracle with oracle/Makefile (gcc, OpenMP, no FP contraction)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib(precision: str = "f64"):
    if precision not in _libs:
        if not os.path.exists(LIB_PATHS[precision]):
            build()
        L = C.CDLL(LIB_PATHS[precision])
        P = C.POINTER(OrcParams)
        dp = C.POINTER(C.c_double)
        rp = C.POINTER(CTYPES[precision])
        L.orc_derive.argtypes = [P]
        L.orc_derive.restype = C.c_int
        L.orc_create.argtypes = [P]
        L.orc_create.restype = C.c_void_p
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_nodes.argtypes = [C.c_void_p]
        L.orc_nodes.restype = C.c_int64
        L.orc_field.argtypes = [C.c_void_p, C.c_int]
        L.orc_field.restype = rp
        L.orc_init_rest.argtypes = [C.c_void_p]
        L.orc_init_conduction.argtypes = [C.c_void_p, C.c_uint64, C.c_double]
        L.orc_noise_uniform.argtypes = [C.c_uint64, C.c_uint64]
        L.orc_noise_uniform.restype = C.c_double
        L.orc_set_populations.argtypes = [C.c_void_p, rp, rp, rp]
        L.orc_load_restart.argtypes = [C.c_void_p] + [rp] * 7
        L.orc_step.argtypes = [C.c_void_p, C.c_int]
        L.orc_observables.argtypes = [C.c_void_p, dp]
        L.orc_profile.argtypes = [C.c_void_p, dp]
        L.orc_threads.restype = C.c_int
        L.orc_set_contract.argtypes = [C.c_int]
        L.orc_set_collision.argtypes = [C.c_void_p, C.c_int]
        L.orc_get_collision.argtypes = [C.c_void_p]
        L.orc_get_contract.restype = C.c_int
        _libs[precision] = L
    return _libs[precision]


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


FIELDS = {"f": 0, "g": 1, "rho": 2, "ux": 3, "uy": 4, "uz": 5, "phi": 6,
          "force_x": 7, "force_y": 8, "force_z": 9}


def make_params(lx, ly, lz, rayleigh=1e5, prandtl=0.71, t_hot=1.0, t_cold=0.0,
                gravity=1.0, beta=None, periodic_sides=False) -> OrcParams:
    """Run-surface fields of src/parameters.h:8-26.  beta=None picks the
    free-fall velocity 0.1, i.e. beta = 0.01 / (gravity * dT * LY)."""
    if beta is None:
        beta = 0.01 / (gravity * (t_hot - t_cold) * ly)
    p = OrcParams(lx=lx, ly=ly, lz=lz, periodic_sides=int(bool(periodic_sides)),
                  rayleigh=rayleigh, prandtl=prandtl, t_hot=t_hot, t_cold=t_cold,
                  gravity=gravity, beta=beta)
    if lib().orc_derive(C.byref(p)) != 0:
        raise ValueError("bad grid for the oracle")
    return p


COLLISIONS = {"bgk": 0, "regularized": 1}


class Oracle:
    """One reference-layout case on the CPU: FP64 (the checker) or, with
    precision="f32", the FP32 build of the same transcription."""

    def __init__(self, params: OrcParams, precision: str = "f64"):
        self.params = params
        self.precision = precision
        self._L = lib(precision)
        self._h = self._L.orc_create(C.byref(params))
        if not self._h:
            raise MemoryError("orc_create failed")
        self.n = int(self._L.orc_nodes(self._h))
        self.shape = (params.lz, params.ly, params.lx)

    def close(self):
        if getattr(self, "_h", None):
            self._L.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def field(self, name: str) -> np.ndarray:
        """Live numpy view of a field (f and g are (27, LZ, LY, LX))."""
        ptr = self._L.orc_field(self._h, FIELDS[name])
        count = self.n * (Q if name in ("f", "g") else 1)
        a = np.ctypeslib.as_array(ptr, shape=(count,))
        return a.reshape((Q,) + self.shape if name in ("f", "g") else self.shape)

    def _rp(self, a):
        a = np.ascontiguousarray(a, dtype=DTYPES[self.precision])
        return a, a.ctypes.data_as(C.POINTER(CTYPES[self.precision]))

    def init_rest(self):
        self._L.orc_init_rest(self._h)

    def init_conduction(self, seed: int, amplitude: float = 1e-3):
        self._L.orc_init_conduction(self._h, C.c_uint64(seed), amplitude)

    def set_populations(self, f, g, phi_prev=None):
        f, fp = self._rp(f)
        g, gp = self._rp(g)
        pp = None
        if phi_prev is not None:
            phi_prev, pp = self._rp(phi_prev)
        self._L.orc_set_populations(self._h, fp, gp, pp)

    def load_restart(self, rho, ux, uy, uz, phi, f, g):
        arrs = [self._rp(a) for a in (rho, ux, uy, uz, phi, f, g)]
        self._L.orc_load_restart(self._h, *[p for _, p in arrs])

    def step(self, n: int = 1):
        self._L.orc_step(self._h, int(n))

    def set_collision(self, model: str):
        """'bgk' (the reference's) or 'regularized' (Latt and Chopard 2006)."""
        self._L.orc_set_collision(self._h, COLLISIONS[model])

    @property
    def collision(self) -> str:
        code = self._L.orc_get_collision(self._h)
        return next(k for k, v in COLLISIONS.items() if v == code)

    def observables(self) -> dict:
        out = np.zeros(10)
        self._L.orc_observables(self._h, _dp(out))
        keys = ["nu_bulk", "nu_top", "nu_bottom", "ke", "re", "ux_mean", "uy_mean",
                "uz_mean", "phi_mean", "diverged"]
        return dict(zip(keys, out.tolist()))

    def profile(self) -> np.ndarray:
        out = np.zeros(5 * self.params.ly)
        self._L.orc_profile(self._h, _dp(out))
        return out.reshape(self.params.ly, 5)


NVCC_FUSION = None  # the default mask, read from the library on first use


def set_contract(mask) -> None:
    """Rounding model: a bit mask of fused multiply-add sites (lbm_oracle.c);
    True selects the mask that rounds as the nvcc-built reference does,
    False / 0 rounds every operation separately."""
    global NVCC_FUSION
    if NVCC_FUSION is None:
        NVCC_FUSION = get_contract()
    if mask is True:
        mask = NVCC_FUSION
    lib().orc_set_contract(int(mask))


def get_contract() -> int:
    return int(lib().orc_get_contract())


def threads() -> int:
    return int(lib().orc_threads())


def noise_uniform(seed: int, node: int) -> float:
    return float(lib().orc_noise_uniform(C.c_uint64(seed), C.c_uint64(node)))
