"""Test infrastructure only: ctypes bridges to the oracle and to the reference.

* ``Oracle``     -- oracle/liboracle.so, the C restatement of the reference path
  (zxh_oracle.c), usable on any machine.
* ``Reference``  -- oracle/_ref/libzxhref_<backend>.so, the unmodified reference
  ZXH-Sim core compiled from its own sources by oracle/Makefile (backends
  ``single``, ``omp``, and ``cuda`` which needs a GPU).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module; the product never does.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
GATE_DTYPE = np.dtype(
    [("type", "<u4"), ("cq", "<u4"), ("q", "<u4"), ("reserved", "<u4"),
     ("theta", "<f8"), ("lam", "<f8"), ("phi", "<f8")]
)


def oracle_path() -> Path:
    return HERE / "liboracle.so"


def ref_path(backend: str) -> Path:
    return HERE / "_ref" / f"libzxhref_{backend}.so"


def ref_available(backend: str) -> bool:
    return ref_path(backend).is_file()


def as_records(gates) -> np.ndarray:
    """Accepts a structured array or a list of (type, cq, q, theta, lam, phi)."""
    if isinstance(gates, np.ndarray) and gates.dtype == GATE_DTYPE:
        return np.ascontiguousarray(gates)
    rec = np.zeros(len(gates), GATE_DTYPE)
    for i, g in enumerate(gates):
        t, cq, q, th, la, ph = (list(g) + [0.0] * 6)[:6]
        rec[i] = (t, cq, q, 0, th, la, ph)
    return rec


_P = ctypes.c_void_p
_SZ = ctypes.c_size_t


class Oracle:
    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            path = oracle_path()
            if not path.is_file():
                raise RuntimeError(f"{path} missing: run `make -C oracle oracle`")
            L = ctypes.CDLL(str(path))
            L.zxo_create.restype = _P
            L.zxo_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
            L.zxo_destroy.argtypes = [_P]
            L.zxo_push.argtypes = [_P, _P, _SZ]
            L.zxo_execute.argtypes = [_P]
            L.zxo_required_M.argtypes = [_P]
            L.zxo_required_M.restype = _SZ
            L.zxo_get_state.argtypes = [_P, _P, ctypes.c_int]
            L.zxo_real_state.argtypes = [_P, _P, ctypes.POINTER(_SZ)]
            L.zxo_global_phase.argtypes = [_P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
            L.zxo_affine.argtypes = [_P, _P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(_SZ)]
            L.zxo_sample_gpu.argtypes = [_P, ctypes.c_uint64, _SZ, _P, _P]
            L.zxo_uniform.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_uint64]
            L.zxo_uniform.restype = ctypes.c_double
            cls._lib = L
        return cls._lib

    def __init__(self, n: int, disable_x: bool = False, eager_expand_all: bool = False):
        self.n = n
        self.h = self.lib().zxo_create(n, int(disable_x), int(eager_expand_all))
        if not self.h:
            raise ValueError("oracle supports 1..63 qubits")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib().zxo_destroy(self.h)
            self.h = None

    def push(self, gates) -> None:
        rec = as_records(gates)
        if self.lib().zxo_push(self.h, rec.ctypes.data, len(rec)) != 0:
            raise ValueError("oracle rejected a gate record")

    def execute(self) -> None:
        rc = self.lib().zxo_execute(self.h)
        if rc != 0:
            raise RuntimeError(f"oracle execute failed ({rc})")

    def required_M(self) -> int:
        return int(self.lib().zxo_required_M(self.h))

    def get_state(self, order: int = 0) -> np.ndarray:
        out = np.zeros(1 << self.n, np.complex128)
        self.lib().zxo_get_state(self.h, out.ctypes.data, order)
        return out

    def real_state(self) -> np.ndarray:
        m = _SZ(0)
        buf = np.zeros(1 << self.required_M(), np.complex128)
        self.lib().zxo_real_state(self.h, buf.ctypes.data, ctypes.byref(m))
        return buf[: 1 << m.value]

    def global_phase(self) -> complex:
        re, im = ctypes.c_double(), ctypes.c_double()
        self.lib().zxo_global_phase(self.h, ctypes.byref(re), ctypes.byref(im))
        return complex(re.value, im.value)

    def affine(self):
        rows = np.zeros(self.n, np.uint64)
        b = ctypes.c_uint64(0)
        m = _SZ(0)
        self.lib().zxo_affine(self.h, rows.ctypes.data, ctypes.byref(b), ctypes.byref(m))
        return rows, int(b.value), int(m.value)

    def sample(self, seed: int, shots: int):
        wc = (self.n + 63) // 64
        words = np.zeros(shots * wc, np.uint64)
        real = np.zeros(shots, np.uint64)
        self.lib().zxo_sample_gpu(self.h, seed, shots, words.ctypes.data, real.ctypes.data)
        return words.reshape(shots, wc), real

    @classmethod
    def uniform(cls, seed: int, stream: int, idx: int) -> float:
        return float(cls.lib().zxo_uniform(seed, stream, idx))


class Reference:
    """The reference ZXH-Sim core itself (one backend per shared library)."""

    _libs: dict = {}

    @classmethod
    def lib(cls, backend: str):
        if backend not in cls._libs:
            path = ref_path(backend)
            if not path.is_file():
                raise RuntimeError(f"{path} missing: run `make -C oracle ref` where the reference is present")
            L = ctypes.CDLL(str(path))
            L.zxhref_create.restype = _P
            L.zxhref_create.argtypes = [_SZ, ctypes.c_int, ctypes.c_int]
            L.zxhref_destroy.argtypes = [_P]
            L.zxhref_push.argtypes = [_P, _P, _SZ]
            L.zxhref_execute.argtypes = [_P]
            L.zxhref_required_M.argtypes = [_P]
            L.zxhref_required_M.restype = _SZ
            L.zxhref_get_state.argtypes = [_P, _P]
            L.zxhref_sample.argtypes = [_P, ctypes.c_uint64, _SZ, _P]
            L.zxhref_measure.argtypes = [_P, ctypes.c_uint64, _SZ]
            if backend == "cuda":
                L.zxhref_device_state.argtypes = [_P, ctypes.POINTER(_P), ctypes.POINTER(_SZ),
                                                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
                L.zxhref_device_sync.restype = ctypes.c_int
            cls._libs[backend] = L
        return cls._libs[backend]

    def __init__(self, n: int, disable_x: bool = False, eager_expand_all: bool = False, backend: str = "single"):
        self.n = n
        self.backend = backend
        self.L = self.lib(backend)
        self.h = self.L.zxhref_create(n, int(disable_x), int(eager_expand_all))

    def __del__(self):
        if getattr(self, "h", None):
            self.L.zxhref_destroy(self.h)
            self.h = None

    def push(self, gates) -> None:
        rec = as_records(gates)
        if self.L.zxhref_push(self.h, rec.ctypes.data, len(rec)) != 0:
            raise ValueError("reference rejected a gate record")

    def execute(self) -> None:
        self.L.zxhref_execute(self.h)

    def required_M(self) -> int:
        return int(self.L.zxhref_required_M(self.h))

    def get_state(self) -> np.ndarray:
        out = np.zeros(1 << self.n, np.complex128)
        self.L.zxhref_get_state(self.h, out.ctypes.data)
        return out

    def measure(self, seed: int, shots: int) -> None:
        """set_seed + measure only (the draw stays in the reference's cache)."""
        self.L.zxhref_measure(self.h, seed, shots)

    def device_state(self):
        """cuda backend: (device pointer, live real-address bits m, global phase) of the
        state after execute(); the 2^m complex128 amplitudes are in real-address order.
        None when the probe's layout checks fail."""
        ptr, m = _P(), _SZ(0)
        re, im = ctypes.c_double(), ctypes.c_double()
        if self.L.zxhref_device_state(self.h, ctypes.byref(ptr), ctypes.byref(m), ctypes.byref(re),
                                      ctypes.byref(im)) != 0:
            return None
        return int(ptr.value), int(m.value), complex(re.value, im.value)

    def device_sync(self) -> None:
        if self.L.zxhref_device_sync() != 0:
            raise RuntimeError("reference device synchronize failed")

    def sample(self, seed: int, shots: int) -> np.ndarray:
        wc = (self.n + 63) // 64
        words = np.zeros(max(1, shots * wc), np.uint64)
        self.L.zxhref_sample(self.h, seed, shots, words.ctypes.data)
        return words[: shots * wc].reshape(shots, wc)


def omp_threads() -> int:
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
