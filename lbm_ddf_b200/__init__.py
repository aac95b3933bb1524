"""B200-native double-distribution lattice Boltzmann engine for 3D
Rayleigh–Bénard convection — Python host side.

This module mirrors the run surface of Summer536/LBM_DDF's single-GPU path
(``src/parameters.h`` fields, ``initialize()``, the per-step launches of
``src/main.cu:27-46`` and the outputs of ``src/output.cu``) over the C ABI of
``include/lbm_ddf.h``, implemented by the in-tree CUDA library
``liblbm_ddf.so``.  There is no CPU fallback: importing works without a GPU,
but every call that touches device state fails with :class:`LbmError` when
the library or a device is missing.

Axes follow the reference: arrays are indexed ``[z, y, x]`` (x fastest) and
``y`` is vertical, hot plate below ``iy = 0``, cold plate above ``iy = LY-1``.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "liblbm_ddf.so")
Q = 27

# status codes (include/lbm_ddf.h)
OK, ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_DIVERGED, ERR_STATE = 0, -1, -2, -3, -4, -5
SIDES_WALL, SIDES_PERIODIC = 0, 1
STORE_F64, STORE_F32, STORE_F16S, STORE_BF16S = 0, 1, 2, 3
STORAGE_NAMES = {"f64": STORE_F64, "f32": STORE_F32, "f16s": STORE_F16S, "bf16s": STORE_BF16S}
STORAGE_BYTES = {STORE_F64: 8, STORE_F32: 4, STORE_F16S: 2, STORE_BF16S: 2}
KERNEL_AUTO, KERNEL_NODE, KERNEL_ROW = 0, 1, 2
COLLISION_BGK, COLLISION_REGULARIZED = 0, 1
BATCH_TILES, BATCH_PER_CASE = 0, 1
BATCH_LAUNCH_NAMES = {"tiles": BATCH_TILES, "per_case": BATCH_PER_CASE}
COLLISION_NAMES = {"bgk": COLLISION_BGK, "regularized": COLLISION_REGULARIZED}


class LbmError(RuntimeError):
    """A C-ABI call returned an error status (the reference would exit())."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class LbmParams(C.Structure):
    _fields_ = [
        ("lx", C.c_int32), ("ly", C.c_int32), ("lz", C.c_int32),
        ("sides", C.c_int32), ("storage", C.c_int32), ("device", C.c_int32),
        ("rayleigh", C.c_double), ("prandtl", C.c_double),
        ("t_hot", C.c_double), ("t_cold", C.c_double),
        ("gravity", C.c_double), ("beta", C.c_double),
    ]


class LbmDerived(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("visc", "tau", "u0", "diff", "tauc", "t0")]


class LbmObservables(C.Structure):
    _fields_ = [
        ("step", C.c_int64),
        ("nu_bulk", C.c_double), ("nu_top", C.c_double), ("nu_bottom", C.c_double),
        ("ke", C.c_double), ("re", C.c_double),
        ("ux_mean", C.c_double), ("uy_mean", C.c_double), ("uz_mean", C.c_double),
        ("phi_mean", C.c_double),
        ("diverged", C.c_int32), ("reserved", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


_lib = None
_dp = C.POINTER(C.c_double)


def lib() -> C.CDLL:
    """The engine library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise LbmError(ERR_STATE, f"CUDA library {LIB_PATH} is not built; run "
                                      "python -c 'import __graft_entry__ as g; g.build()'")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        P = C.POINTER(LbmParams)
        L.lbm_last_error.restype = C.c_char_p
        L.lbm_abi_version.restype = C.c_int
        L.lbm_derive.argtypes = [P, C.POINTER(LbmDerived)]
        L.lbm_case_bytes.argtypes = [P, C.POINTER(C.c_uint64)]
        L.lbm_create.argtypes = [P, C.POINTER(vp)]
        L.lbm_destroy.argtypes = [vp]
        L.lbm_init_rest.argtypes = [vp, vp]
        L.lbm_init_conduction.argtypes = [vp, C.c_uint64, C.c_double, vp]
        L.lbm_init_temperature.argtypes = [vp, vp, vp]
        L.lbm_load_ref_state.argtypes = [vp] + [_dp] * 7
        L.lbm_store_ref_state.argtypes = [vp] + [_dp] * 7
        L.lbm_step.argtypes = [vp, C.c_int32, vp]
        L.lbm_get_observables.argtypes = [vp, C.POINTER(LbmObservables), vp]
        L.lbm_step_observed.argtypes = [vp, C.c_int32, C.POINTER(LbmObservables), vp]
        L.lbm_step_observed_async.argtypes = [vp, C.c_int32, vp, vp]
        L.lbm_get_profile.argtypes = [vp, _dp, vp]
        L.lbm_get_params.argtypes = [vp, P, C.POINTER(LbmDerived), C.POINTER(C.c_int64)]
        L.lbm_checkpoint_bytes.argtypes = [vp, C.POINTER(C.c_uint64)]
        L.lbm_save_state.argtypes = [vp, vp, C.c_uint64, vp]
        L.lbm_restore_state.argtypes = [vp, vp, C.c_uint64, vp]
        L.lbm_set_step_kernel.argtypes = [vp, C.c_int32]
        L.lbm_get_step_kernel.argtypes = [vp, C.POINTER(C.c_int32)]
        L.lbm_set_collision.argtypes = [vp, C.c_int32]
        L.lbm_debug_row_wait_extra_bytes.argtypes = [vp, C.c_uint32]
        L.lbm_get_collision.argtypes = [vp, C.POINTER(C.c_int32)]
        L.lbm_batch_create.argtypes = [C.c_int, C.c_int32, C.POINTER(vp)]
        L.lbm_batch_destroy.argtypes = [vp]
        L.lbm_batch_add.argtypes = [vp, vp]
        L.lbm_batch_remove.argtypes = [vp, vp]
        L.lbm_batch_size.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_uint64)]
        L.lbm_batch_step.argtypes = [vp, C.c_int32, vp]
        L.lbm_batch_observables.argtypes = [vp, vp, vp]
        L.lbm_batch_set_launch.argtypes = [vp, C.c_int32]
        L.lbm_batch_get_launch.argtypes = [vp, C.POINTER(C.c_int32)]
        L.lbm_batch_set_config.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32]
        L.lbm_batch_get_config.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.lbm_batch_autotune.argtypes = [vp, C.c_int32, vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                         C.POINTER(C.c_double)]
        L.lbm_observables_noalloc.argtypes = [P, vp, vp, vp, C.c_uint64, C.c_int32, C.c_int64, vp, vp]
        L.lbm_selfcheck_division.argtypes = [C.c_int, C.c_double, C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64)]
        for name in ("lbm_derive", "lbm_case_bytes", "lbm_create", "lbm_destroy", "lbm_init_rest",
                     "lbm_init_conduction", "lbm_load_ref_state", "lbm_store_ref_state", "lbm_step",
                     "lbm_get_observables", "lbm_get_profile", "lbm_get_params", "lbm_checkpoint_bytes",
                     "lbm_save_state", "lbm_restore_state", "lbm_selfcheck_division",
                     "lbm_observables_noalloc", "lbm_set_step_kernel", "lbm_get_step_kernel",
                     "lbm_set_collision", "lbm_get_collision", "lbm_step_observed", "lbm_step_observed_async",
                     "lbm_batch_create", "lbm_batch_destroy", "lbm_batch_add", "lbm_batch_remove",
                     "lbm_batch_size", "lbm_batch_step", "lbm_batch_set_config", "lbm_batch_get_config",
                     "lbm_batch_autotune", "lbm_batch_observables", "lbm_debug_row_wait_extra_bytes",
                     "lbm_batch_set_launch", "lbm_batch_get_launch"):
            getattr(L, name).restype = C.c_int
        _lib = L
    return _lib


def check(rc: int) -> int:
    if rc != OK:
        raise LbmError(rc, lib().lbm_last_error().decode(errors="replace"))
    return rc


def _stream_handle(stream) -> C.c_void_p:
    """cudaStream_t from None, an int handle, or an object with .cuda_stream
    (e.g. torch.cuda.Stream)."""
    if stream is None:
        return C.c_void_p(0)
    if hasattr(stream, "cuda_stream"):
        return C.c_void_p(int(stream.cuda_stream))
    return C.c_void_p(int(stream))


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def _buffer(buf):
    """(address, size in bytes) of a numpy array or a torch tensor."""
    if hasattr(buf, "data_ptr"):
        return int(buf.data_ptr()), int(buf.numel() * buf.element_size())
    a = np.asarray(buf)
    return int(a.ctypes.data), int(a.nbytes)


@dataclass
class RunSurface:
    """The fields of the reference's src/parameters.h:5-31, as runtime values,
    plus the engine's side-wall mode, storage format and device."""
    LX: int = 400
    LY: int = 400
    LZ: int = 400
    NEND: int = 1000
    NDIAG: int = 10000
    NFLOWOUT: int = 10000
    NNUOUT: int = 10000
    CONTINUE_STEP: int = 0
    RAYLEIGH: float = 1.0e7
    PRANDTL: float = 0.71
    T_HOT: float = 1.0
    T_COLD: float = 0.0
    GRAVITY: float = 1.0
    BETA: float | None = None     # None: 0.1 / (LY * 5.0) as in src/parameters.h:26
    sides: int = SIDES_WALL
    storage: int = STORE_F64
    device: int = 0

    def params(self) -> LbmParams:
        beta = self.BETA if self.BETA is not None else 0.1 / (self.LY * 5.0)
        return LbmParams(lx=self.LX, ly=self.LY, lz=self.LZ, sides=self.sides, storage=self.storage,
                         device=self.device, rayleigh=self.RAYLEIGH, prandtl=self.PRANDTL,
                         t_hot=self.T_HOT, t_cold=self.T_COLD, gravity=self.GRAVITY, beta=beta)


def make_params(lx, ly, lz, rayleigh=1e5, prandtl=0.71, t_hot=1.0, t_cold=0.0, gravity=1.0,
                beta=None, sides=SIDES_PERIODIC, storage=STORE_F32, device=0) -> LbmParams:
    """Parameters with beta chosen for free-fall velocity 0.1 unless given
    (g*beta*dT*LY = 0.01)."""
    if isinstance(storage, str):
        storage = STORAGE_NAMES[storage]
    if beta is None:
        beta = 0.01 / (gravity * (t_hot - t_cold) * ly)
    return LbmParams(lx=lx, ly=ly, lz=lz, sides=sides, storage=storage, device=device,
                     rayleigh=rayleigh, prandtl=prandtl, t_hot=t_hot, t_cold=t_cold,
                     gravity=gravity, beta=beta)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser (Steele, Lea & Flood 2014) on a uint64 array."""
    x = x + np.uint64(0x9E3779B97F4A7C15)
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def conduction_temperature(lx: int, ly: int, lz: int, seed: int, amplitude: float = 1e-3,
                           t_hot: float = 1.0, t_cold: float = 0.0, dtype=np.float64) -> np.ndarray:
    """The temperature field lbm_init_conduction forms, on the host: the
    conduction profile T_hot - ((T_hot - T_cold) iy) / (LY - 1) plus
    amplitude (2u - 1), u = splitmix64(splitmix64(seed) + idx) / 2^64 (53
    bits), in the same FP64 operations, as a flat array in the reference's
    node order (x fastest).  Pass it (as float32 for non-FP64 storage) to
    Case.init_temperature, perturbed as a study needs."""
    n = lx * ly * lz
    key = _splitmix64(np.array([seed], dtype=np.uint64))[0]
    with np.errstate(over="ignore"):
        r = _splitmix64(np.arange(n, dtype=np.uint64) + key)
    u = (r >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    iy = np.broadcast_to(np.arange(ly, dtype=np.float64)[None, :, None], (lz, ly, lx)).reshape(-1)
    t = t_hot - ((t_hot - t_cold) * iy) / (ly - 1.0)
    t = t + amplitude * (2.0 * u - 1.0)
    return t.astype(dtype, copy=False)


def derive(p: LbmParams) -> dict:
    d = LbmDerived()
    check(lib().lbm_derive(C.byref(p), C.byref(d)))
    return {k: getattr(d, k) for k, _ in d._fields_}


def selfcheck_division(divisor: float, n: int = 1 << 24, seed: int = 1, device: int = 0) -> int:
    """Mismatches of the FP64 path's division by `divisor` against the GPU's
    correctly rounded division over n random dividends (expected 0)."""
    bad = C.c_uint64()
    check(lib().lbm_selfcheck_division(device, divisor, n, seed, C.byref(bad)))
    return int(bad.value)


def observables_noalloc(params: LbmParams, f_ptr: int, g_ptr: int, phi_prev_ptr: int, pop_stride: int,
                        swapped: bool, step: int, out_dev_ptr: int, stream=None) -> None:
    """Enqueue the observables reduction over caller-owned device buffers
    into the lbm_observables at device address out_dev_ptr, allocating
    nothing (the C ABI's lbm_observables_noalloc: for callers that must not
    allocate device memory, e.g. while capturing a CUDA graph).  Returns
    without synchronising."""
    check(lib().lbm_observables_noalloc(C.byref(params), C.c_void_p(f_ptr), C.c_void_p(g_ptr),
                                        C.c_void_p(phi_prev_ptr), pop_stride, int(bool(swapped)), int(step),
                                        C.c_void_p(out_dev_ptr), _stream_handle(stream)))


def case_bytes(p: LbmParams) -> int:
    b = C.c_uint64()
    check(lib().lbm_case_bytes(C.byref(p), C.byref(b)))
    return int(b.value)


class ObservablesBuffer:
    """n lbm_observables records in page-locked host memory (torch's pinned
    allocator), the destination of Case.step_observed_async."""

    def __init__(self, n: int):
        import torch

        self._mem = torch.empty(max(1, n) * C.sizeof(LbmObservables), dtype=torch.uint8, pin_memory=True)
        self._recs = (LbmObservables * max(1, n)).from_address(self._mem.data_ptr())
        self._n = n

    def __len__(self) -> int:
        return self._n

    def address(self, i: int) -> int:
        return self._mem.data_ptr() + i * C.sizeof(LbmObservables)

    def __getitem__(self, i: int) -> dict:
        if not 0 <= i < self._n:
            raise IndexError(i)
        return self._recs[i].as_dict()


class Case:
    """One Rayleigh–Bénard case resident in HBM (src/globals.cu's device
    arrays, owned by this object instead of process globals)."""

    def __init__(self, params: LbmParams):
        self.params = params
        h = C.c_void_p()
        check(lib().lbm_create(C.byref(params), C.byref(h)))
        self._h = h
        self.shape = (params.lz, params.ly, params.lx)
        self.n = params.lx * params.ly * params.lz
        self.derived = derive(params)

    def close(self):
        if getattr(self, "_h", None):
            lib().lbm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def step_count(self) -> int:
        s = C.c_int64()
        check(lib().lbm_get_params(self._h, None, None, C.byref(s)))
        return int(s.value)

    def init_rest(self, stream=None):
        check(lib().lbm_init_rest(self._h, _stream_handle(stream)))

    def init_conduction(self, seed: int, amplitude: float = 1e-3, stream=None):
        check(lib().lbm_init_conduction(self._h, C.c_uint64(seed), amplitude, _stream_handle(stream)))

    def init_temperature(self, temperature, stream=None):
        """Start from a temperature field (C ABI lbm_init_temperature): zero
        velocity, equilibrium populations.  `temperature` holds LZ*LY*LX
        values in the reference's node order (x fastest), float64 for F64
        storage and float32 otherwise: a numpy array or a torch tensor on the
        host (pinned for an asynchronous copy) or on this case's GPU."""
        want = np.float64 if self.params.storage == STORE_F64 else np.float32
        n = self.n
        if hasattr(temperature, "data_ptr"):
            if str(temperature.dtype) != "torch." + np.dtype(want).name or not temperature.is_contiguous():
                raise ValueError(f"temperature must be a contiguous {np.dtype(want).name} tensor")
            if temperature.numel() != n:
                raise ValueError(f"temperature has {temperature.numel()} values, the grid {n}")
            ptr = int(temperature.data_ptr())
            keep = temperature
        else:
            keep = np.ascontiguousarray(temperature, dtype=want).reshape(-1)
            if keep.size != n:
                raise ValueError(f"temperature has {keep.size} values, the grid {n}")
            ptr = int(keep.ctypes.data)
        check(lib().lbm_init_temperature(self._h, C.c_void_p(ptr), _stream_handle(stream)))
        del keep   # the call returns once the state is written

    def load_ref_state(self, rho, ux, uy, uz, phi, f, g):
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (rho, ux, uy, uz, phi, f, g)]
        check(lib().lbm_load_ref_state(self._h, *[_ptr(a) for a in arrs]))

    def store_ref_state(self, fields=("rho", "ux", "uy", "uz", "phi", "f", "g")) -> dict:
        out = {}
        ptrs = []
        for k in ("rho", "ux", "uy", "uz", "phi", "f", "g"):
            if k in fields:
                out[k] = np.empty(((Q,) if k in ("f", "g") else ()) + self.shape, dtype=np.float64)
                ptrs.append(_ptr(out[k]))
            else:
                ptrs.append(None)
        check(lib().lbm_store_ref_state(self._h, *ptrs))
        return out

    def step(self, n: int = 1, stream=None):
        check(lib().lbm_step(self._h, int(n), _stream_handle(stream)))

    def observables(self, stream=None, allow_diverged: bool = False) -> dict:
        o = LbmObservables()
        rc = lib().lbm_get_observables(self._h, C.byref(o), _stream_handle(stream))
        if rc != OK and not (allow_diverged and rc == ERR_DIVERGED):
            check(rc)
        return o.as_dict()

    def step_observed(self, n: int = 1, stream=None, allow_diverged: bool = False) -> list:
        """n steps; returns the observables of each state the steps started
        from (reduced inside the step kernels: no extra read of the state)."""
        out = (LbmObservables * max(1, n))()
        rc = lib().lbm_step_observed(self._h, int(n), out, _stream_handle(stream))
        if rc != OK and not (allow_diverged and rc == ERR_DIVERGED):
            check(rc)
        return [out[i].as_dict() for i in range(n)]

    def step_observed_async(self, n: int, out: "ObservablesBuffer", first: int = 0, stream=None):
        """Enqueue n steps and the copy of their observables into out[first ..
        first + n) (C ABI lbm_step_observed_async) and return at once; the
        entries are valid after the stream passes this call."""
        if n < 0 or first < 0 or first + n > len(out):
            raise ValueError("observables buffer too small")
        check(lib().lbm_step_observed_async(self._h, int(n), C.c_void_p(out.address(first)),
                                            _stream_handle(stream)))

    @property
    def step_kernel(self) -> int:
        k = C.c_int32()
        check(lib().lbm_get_step_kernel(self._h, C.byref(k)))
        return int(k.value)

    def set_step_kernel(self, kind: int):
        check(lib().lbm_set_step_kernel(self._h, int(kind)))

    @property
    def collision(self) -> str:
        m = C.c_int32()
        check(lib().lbm_get_collision(self._h, C.byref(m)))
        return next(k for k, v in COLLISION_NAMES.items() if v == m.value)

    def set_collision(self, model):
        """'bgk' (the reference's collision, the default) or 'regularized'."""
        check(lib().lbm_set_collision(self._h, COLLISION_NAMES.get(model, model)))

    def checkpoint_bytes(self) -> int:
        b = C.c_uint64()
        check(lib().lbm_checkpoint_bytes(self._h, C.byref(b)))
        return int(b.value)

    def save_state(self, buf, stream=None):
        """Enqueue a copy of the device state into `buf` (anything exposing a
        writable buffer or a data_ptr(), e.g. a pinned torch uint8 tensor);
        synchronise `stream` before reading it."""
        ptr, size = _buffer(buf)
        check(lib().lbm_save_state(self._h, C.c_void_p(ptr), size, _stream_handle(stream)))

    def restore_state(self, buf, stream=None):
        ptr, size = _buffer(buf)
        check(lib().lbm_restore_state(self._h, C.c_void_p(ptr), size, _stream_handle(stream)))

    def profile(self, stream=None) -> np.ndarray:
        out = np.empty(5 * self.params.ly, dtype=np.float64)
        check(lib().lbm_get_profile(self._h, _ptr(out), _stream_handle(stream)))
        return out.reshape(self.params.ly, 5)


class Batch:
    """Cases advanced together by one kernel launch per step (C ABI
    lbm_batch_*).  The batch does not own its cases."""

    def __init__(self, storage=STORE_F32, device: int = 0):
        if isinstance(storage, str):
            storage = STORAGE_NAMES[storage]
        h = C.c_void_p()
        check(lib().lbm_batch_create(device, storage, C.byref(h)))
        self._h = h
        self.members = []

    def close(self):
        if getattr(self, "_h", None):
            lib().lbm_batch_destroy(self._h)
            self._h = None
            self.members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add(self, case: "Case"):
        check(lib().lbm_batch_add(self._h, case.handle))
        self.members.append(case)

    def remove(self, case: "Case"):
        check(lib().lbm_batch_remove(self._h, case.handle))
        self.members.remove(case)

    def size(self):
        m, n = C.c_int32(), C.c_uint64()
        check(lib().lbm_batch_size(self._h, C.byref(m), C.byref(n)))
        return int(m.value), int(n.value)

    def step(self, n: int = 1, stream=None):
        check(lib().lbm_batch_step(self._h, int(n), _stream_handle(stream)))

    def observables_async(self, out: "ObservablesBuffer", stream=None):
        """Enqueue the observables of every member, in self.members order,
        into out[0 .. len(self.members)) (C ABI lbm_batch_observables) and
        return at once; the entries are valid after the stream passes this
        call (synchronise it or an event recorded after the call)."""
        if len(out) < len(self.members):
            raise ValueError("observables buffer too small")
        check(lib().lbm_batch_observables(self._h, C.c_void_p(out.address(0)), _stream_handle(stream)))

    def observables(self, stream=None) -> list:
        """Observables of every member (self.members order); waits for the stream."""
        import torch

        out = ObservablesBuffer(len(self.members))
        self.observables_async(out, stream)
        if stream is None:
            torch.cuda.synchronize()
        else:
            stream.synchronize()
        return [out[i] for i in range(len(self.members))]

    def set_config(self, block: int = 128, blocks_per_sm: int = 0, use_graph: bool = True):
        check(lib().lbm_batch_set_config(self._h, block, blocks_per_sm, int(bool(use_graph))))

    def set_launch(self, launch):
        """'tiles' (one persistent kernel walks every member's tiles; the
        default) or 'per_case' (each member's own single-case kernel, the
        members on parallel streams)."""
        check(lib().lbm_batch_set_launch(self._h, BATCH_LAUNCH_NAMES.get(launch, launch)))

    @property
    def launch(self) -> str:
        m = C.c_int32()
        check(lib().lbm_batch_get_launch(self._h, C.byref(m)))
        return next(k for k, v in BATCH_LAUNCH_NAMES.items() if v == m.value)

    def config(self) -> dict:
        b, p, g = C.c_int32(), C.c_int32(), C.c_int32()
        check(lib().lbm_batch_get_config(self._h, C.byref(b), C.byref(p), C.byref(g)))
        return {"block": b.value, "blocks_per_sm": p.value, "use_graph": bool(g.value), "launch": self.launch}

    def autotune(self, steps_per_trial: int = 4, stream=None) -> dict:
        b, p, ms = C.c_int32(), C.c_int32(), C.c_double()
        check(lib().lbm_batch_autotune(self._h, steps_per_trial, _stream_handle(stream), C.byref(b), C.byref(p),
                                       C.byref(ms)))
        return {"block": b.value, "blocks_per_sm": p.value, "ms_per_step": ms.value, "launch": self.launch}
