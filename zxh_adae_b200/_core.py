"""ctypes binding of libzxhb200.so (include/zxh_b200.h).

Mirrors the reference's pybind11 module ``zxhsim._core``
(src/zxh/src/pybind/bindings.cpp:79-118 of ZXH-Sim): the same class ``ZXH(n,
disable_x=False, eager_expand_all=False)`` with the same method names and
argument order, plus module functions ``init/finalize/active/rank/nprocs`` and
``PrintRes``. Where the reference aborts the process on an error
(src/zxh/src/runtime/runtime_general.cpp:79-89), this binding raises:
``ValueError`` for bad arguments and limits, ``RuntimeError`` for calls out of
order, CUDA errors and device-side timeouts, ``MemoryError`` for failed
allocations.

The library is required: importing this module without the built
``libzxhb200.so`` raises ImportError; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

__version__ = "0.1.0"

_HERE = Path(__file__).resolve().parent
_LIB_PATH = Path(os.environ.get("ZXH_B200_LIB", _HERE / "libzxhb200.so"))

if not _LIB_PATH.is_file():
    raise ImportError(
        f"{_LIB_PATH} is missing: build it with `make -C zxh_adae_b200/csrc` "
        "(or __graft_entry__.build()); the B200 path has no CPU fallback"
    )

_lib = ctypes.CDLL(str(_LIB_PATH))

from .records import (  # noqa: F401  (re-exported: the record layouts of include/zxh_b200.h)
    BARRIER, CP, CRZ, CX, GATE_DTYPE, RX, RZ, TERM_DTYPE, TERM_X, TERM_Z, TERM_ZZ, U3, H, P, X, Z, as_records,
    as_terms,
)

C64, C128 = 1, 2
ORDER_REFERENCE, ORDER_QUBIT = 0, 1

_P = ctypes.c_void_p
_SZ = ctypes.c_size_t
_D = ctypes.c_double
_U64 = ctypes.c_uint64


def _sig(name, args, res=ctypes.c_int):
    f = getattr(_lib, name)
    f.argtypes = args
    f.restype = res
    return f


_sig("zxh_version", [], ctypes.c_char_p)
_sig("zxh_last_error", [_P], ctypes.c_char_p)
_sig("zxh_create", [ctypes.POINTER(_P), _SZ, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int])
_sig("zxh_destroy", [_P])
_sig("zxh_set_seed", [_P, _U64])
_sig("zxh_clear_seed", [_P])
_sig("zxh_clear_gates", [_P])
_sig("zxh_barrier", [_P])
_sig("zxh_rz", [_P, _SZ, _D])
_sig("zxh_crz", [_P, _SZ, _SZ, _D])
_sig("zxh_cp", [_P, _SZ, _SZ, _D])
_sig("zxh_p", [_P, _SZ, _D])
_sig("zxh_z", [_P, _SZ])
_sig("zxh_x", [_P, _SZ])
_sig("zxh_cx", [_P, _SZ, _SZ])
_sig("zxh_h", [_P, _SZ])
_sig("zxh_u3", [_P, _SZ, _D, _D, _D])
_sig("zxh_rx", [_P, _SZ, _D])
_sig("zxh_push_gates", [_P, _P, _SZ])
_sig("zxh_execute", [_P])
_sig("zxh_apply", [_P, _P, _SZ])
_sig("zxh_apply_async", [_P, _P, _SZ])
_sig("zxh_sync", [_P])
_sig("zxh_flush", [_P])
_sig("zxh_measure", [_P, _SZ])
_sig("zxh_get_results", [_P, _P, _SZ])
_sig("zxh_measured_count", [_P, ctypes.POINTER(_SZ)])
_sig("zxh_counts", [_P, _P, _P, _SZ, ctypes.POINTER(_SZ)])
_sig("zxh_get_state", [_P, _P, _SZ, ctypes.c_int])
_sig("zxh_get_state_device", [_P, _P, _SZ, ctypes.c_int])
_sig("zxh_required_M", [_P, ctypes.POINTER(_SZ)])
_sig("zxh_num_qubits", [_P, ctypes.POINTER(_SZ)])
_sig("zxh_state_view", [_P, ctypes.POINTER(_P), ctypes.POINTER(_SZ), ctypes.POINTER(_SZ),
                        ctypes.POINTER(_D), ctypes.POINTER(_D)])
_sig("zxh_stream", [_P, ctypes.POINTER(_P)])
_sig("zxh_set_param", [_P, ctypes.c_char_p, ctypes.c_int])
_sig("zxh_plan_stats", [_SZ, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _SZ, _P])
_sig("zxh_device_info", [ctypes.c_int, ctypes.c_char_p, _SZ, ctypes.POINTER(ctypes.c_int)])
_sig("zxh_optimize_gates", [_SZ, ctypes.c_int, _P, _SZ, _P, _SZ, ctypes.POINTER(_SZ)])
_sig("zxh_last_stats", [_P, ctypes.POINTER(_U64), ctypes.POINTER(_U64), ctypes.POINTER(_D)])
_sig("zxh_expectation", [_P, _P, _SZ, ctypes.POINTER(_D)])
_sig("zxh_adjoint_gradient", [_P, _P, _SZ, _SZ, ctypes.POINTER(_D), _P, _SZ])
_sig("zxh_gate_count", [_P, ctypes.POINTER(_SZ)])
_sig("zxh_batch_create", [ctypes.POINTER(_P), _SZ, _P, _P, _P, _P, _P, ctypes.c_int, ctypes.c_int])
_sig("zxh_batch_destroy", [_P])
_sig("zxh_batch_last_error", [_P], ctypes.c_char_p)
_sig("zxh_batch_gradient_offsets", [_P, _P])
_sig("zxh_batch_run", [_P, ctypes.c_int, _P, _P, _SZ])
_sig("zxh_batch_set", [_P, ctypes.c_char_p, ctypes.c_int])
_sig("zxh_batch_get", [_P, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)])
_sig("zxh_batch_tune", [_P, ctypes.c_int])
_sig("zxh_batch_stats", [_P, ctypes.POINTER(_U64), ctypes.POINTER(_U64), ctypes.POINTER(_D), ctypes.POINTER(_U64)])

_ERRORS = {1: ValueError, 2: RuntimeError, 3: RuntimeError, 4: MemoryError, 5: ValueError, 6: RuntimeError}


def library_path() -> str:
    return str(_LIB_PATH)


def version() -> str:
    return _lib.zxh_version().decode()


def _raise(rc: int, handle) -> None:
    msg = _lib.zxh_last_error(handle).decode(errors="replace")
    raise _ERRORS.get(rc, RuntimeError)(msg or f"zxh error {rc}")


PASS_KINDS = ("product", "expand", "tile", "pair", "diagonal", "fast", "row", "grow")  # out[2..9]


def device_info(device: int = 0) -> tuple:
    """(name, SM count) of a CUDA device (zxh_device_info)."""
    buf = ctypes.create_string_buffer(256)
    sms = ctypes.c_int(0)
    rc = _lib.zxh_device_info(int(device), buf, 256, ctypes.byref(sms))
    if rc != 0:
        _raise(rc, None)
    return buf.value.decode(errors="replace"), int(sms.value)


def plan_stats(n: int, gates, dtype: str = "complex64", disable_x: bool = False,
               eager_expand_all: bool = False) -> dict:
    """Host-only dry run of execute() (no GPU needed): state bits and pass counts."""
    rec = as_records(gates)
    out = np.zeros(13, np.uint64)
    rc = _lib.zxh_plan_stats(int(n), int(bool(disable_x)), int(bool(eager_expand_all)),
                             C64 if dtype == "complex64" else C128, rec.ctypes.data, len(rec), out.ctypes.data)
    if rc != 0:
        _raise(rc, None)
    d = {"M": int(out[0]), "m": int(out[1]), "passes": int(out[10]), "walsh": int(out[11]), "span": int(out[12])}
    d.update({k: int(out[2 + i]) for i, k in enumerate(PASS_KINDS)})
    return d


def optimize_records(n: int, gates, level: int = 2) -> np.ndarray:
    """The host circuit compiler (zxh_optimize_gates): the reference's boundary
    scheduler (circ_optimizer.py:218-420) over gate records. Returns records equal
    to the input up to a global phase."""
    rec = as_records(gates)
    cnt = _SZ(0)
    rc = _lib.zxh_optimize_gates(int(n), int(level), rec.ctypes.data if len(rec) else None, len(rec), None, 0,
                                 ctypes.byref(cnt))
    if rc != 0:
        _raise(rc, None)
    out = np.zeros(cnt.value, GATE_DTYPE)
    rc = _lib.zxh_optimize_gates(int(n), int(level), rec.ctypes.data if len(rec) else None, len(rec),
                                 out.ctypes.data if len(out) else None, len(out), ctypes.byref(cnt))
    if rc != 0:
        _raise(rc, None)
    return out


# Module-level runtime calls of the reference (bindings.cpp:86-90). One process
# drives one or more GPUs through independent handles, so these only track state.
_active = False


def init() -> None:
    global _active
    _active = True


def finalize() -> None:
    global _active
    _active = False


def active() -> bool:
    return _active


def rank() -> int:
    return 0


def nprocs() -> int:
    return 1


def PrintRes(res, n: int) -> None:
    """Prints bitstring counts, qubit n-1 first (zxh.cpp:842-871)."""
    counts: dict = {}
    for row in res:
        s = "".join("1" if (i < len(row) and row[i]) else "0" for i in range(n - 1, -1, -1))
        counts[s] = counts.get(s, 0) + 1
    for k in sorted(counts):
        print(f"{k}: {counts[k]}")


class ZXH:
    """One simulator: a gate list, a device state and its sampler results.

    ``dtype`` selects complex128 (the reference's only type) or complex64
    amplitudes; ``device`` is the CUDA ordinal.
    """

    def __init__(self, n: int, disable_x: bool = False, eager_expand_all: bool = False, *,
                 dtype: str = "complex128", device: int = 0):
        if dtype not in ("complex64", "complex128"):
            raise ValueError("dtype must be 'complex64' or 'complex128'")
        h = _P()
        rc = _lib.zxh_create(ctypes.byref(h), int(n), int(bool(disable_x)), int(bool(eager_expand_all)),
                             C64 if dtype == "complex64" else C128, int(device))
        if rc != 0:
            _raise(rc, None)
        self._h = h
        self._n = int(n)
        self.dtype = np.dtype(dtype)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:  # the module may already be torn down at interpreter exit
            _lib.zxh_destroy(h)
            self._h = None

    def close(self) -> None:
        self.__del__()

    def _ck(self, rc: int) -> None:
        if rc != 0:
            _raise(rc, self._h)

    # --- recording (zxh.cpp:216-310) -------------------------------------------------
    def set_seed(self, seed: int) -> None:
        self._ck(_lib.zxh_set_seed(self._h, int(seed) & 0xFFFFFFFFFFFFFFFF))

    def clear_seed(self) -> None:
        self._ck(_lib.zxh_clear_seed(self._h))

    def clear_gates(self) -> None:
        self._ck(_lib.zxh_clear_gates(self._h))

    def Barrier(self) -> None:
        self._ck(_lib.zxh_barrier(self._h))

    def Rz(self, q: int, theta: float) -> None:
        self._ck(_lib.zxh_rz(self._h, q, theta))

    def CRz(self, cq: int, q: int, theta: float) -> None:
        self._ck(_lib.zxh_crz(self._h, cq, q, theta))

    def CP(self, cq: int, q: int, theta: float) -> None:
        self._ck(_lib.zxh_cp(self._h, cq, q, theta))

    def P(self, q: int, theta: float) -> None:
        self._ck(_lib.zxh_p(self._h, q, theta))

    def Z(self, q: int) -> None:
        self._ck(_lib.zxh_z(self._h, q))

    def X(self, q: int) -> None:
        self._ck(_lib.zxh_x(self._h, q))

    def CX(self, cq: int, q: int) -> None:
        self._ck(_lib.zxh_cx(self._h, cq, q))

    def H(self, q: int) -> None:
        self._ck(_lib.zxh_h(self._h, q))

    def U3(self, q: int, theta: float, lam: float, phi: float) -> None:
        """U3 with the reference's argument order (theta, lambda, phi) (zxh.h:36)."""
        self._ck(_lib.zxh_u3(self._h, q, theta, lam, phi))

    def Rx(self, q: int, theta: float) -> None:
        self._ck(_lib.zxh_rx(self._h, q, theta))

    def push_gates(self, gates) -> None:
        rec = as_records(gates)
        self._ck(_lib.zxh_push_gates(self._h, rec.ctypes.data, len(rec)))

    # --- running ---------------------------------------------------------------------
    def execute(self) -> None:
        self._ck(_lib.zxh_execute(self._h))

    def apply(self, gates) -> None:
        """Applies more gates to the current state without recording them. The
        phases left after the batch's last U3 rotations ride in the next apply's
        first window; reads of the state (get_state, state_view, measure,
        expectation) and flush() apply them first."""
        rec = as_records(gates)
        self._ck(_lib.zxh_apply(self._h, rec.ctypes.data, len(rec)))

    def apply_async(self, gates) -> None:
        """apply() without waiting for the GPU: the next call plans while this batch
        runs; errors surface at sync() or at the next other call."""
        rec = as_records(gates)
        self._ck(_lib.zxh_apply_async(self._h, rec.ctypes.data, len(rec)))

    def sync(self) -> None:
        """Waits for the apply_async work in flight."""
        self._ck(_lib.zxh_sync(self._h))

    def flush(self) -> None:
        """Applies the phases the last apply carried over (every call that reads the
        state does so itself); last_stats() then reports that pass."""
        self._ck(_lib.zxh_flush(self._h))

    def measure(self, shots: int) -> None:
        self._ck(_lib.zxh_measure(self._h, int(shots)))

    def measured_count(self) -> int:
        out = _SZ(0)
        self._ck(_lib.zxh_measured_count(self._h, ctypes.byref(out)))
        return int(out.value)

    def results_words(self, shots: int | None = None) -> np.ndarray:
        """Cached outcomes as uint64 words (bit q = qubit q), in draw order."""
        cnt = self.measured_count() if shots is None else int(shots)
        words = np.zeros(max(cnt, 1), np.uint64)
        self._ck(_lib.zxh_get_results(self._h, words.ctypes.data, cnt))
        return words[:cnt]

    def _rows(self, words: np.ndarray) -> list:
        n = self._n
        bits = ((words[:, None] >> np.arange(n, dtype=np.uint64)[None, :]) & np.uint64(1)).astype(bool)
        return [list(map(bool, r)) for r in bits]

    def get_results(self) -> list:
        """list[list[bool]] with entry q = qubit q (bindings.cpp:61-75)."""
        return self._rows(self.results_words())

    def Sampling(self, shots: int) -> list:
        self.measure(shots)
        return self._rows(self.results_words(shots))

    def counts_words(self) -> tuple:
        """(words, counts) of the last measure(): its distinct outcomes, counted on
        the device, sorted by word (bit q = qubit q)."""
        nu = _SZ(0)
        self._ck(_lib.zxh_counts(self._h, None, None, 0, ctypes.byref(nu)))
        k = int(nu.value)
        words = np.zeros(max(k, 1), np.uint64)
        cnt = np.zeros(max(k, 1), np.uint64)
        self._ck(_lib.zxh_counts(self._h, words.ctypes.data, cnt.ctypes.data, k, ctypes.byref(nu)))
        order = np.argsort(words[:k], kind="stable")
        words, cnt = words[:k][order], cnt[:k][order]
        if k > 1 and np.any(words[1:] == words[:-1]):  # a singular map (CX with control = target)
            words, inv = np.unique(words, return_inverse=True)
            cnt = np.bincount(inv, weights=cnt.astype(np.float64)).astype(np.uint64)
        return words, cnt

    def sample_counts(self, shots: int) -> dict:
        """Counts keyed by bitstrings with qubit n-1 first (bindings.cpp:36-54), in
        increasing key order as the reference's std::map."""
        self.measure(shots)
        keys, cnt = self.counts_words()
        n = self._n
        return {format(k, f"0{n}b"): c for k, c in zip(keys.tolist(), cnt.tolist())}

    def get_state(self, order: int = ORDER_REFERENCE) -> np.ndarray:
        """2^n amplitudes in the reference's get_state order (zxh.cpp:579-636)."""
        out = np.zeros(1 << self._n, self.dtype)
        self._ck(_lib.zxh_get_state(self._h, out.ctypes.data, out.size, int(order)))
        return out

    def get_state_device(self, ptr: int, elems: int, order: int = ORDER_REFERENCE) -> None:
        self._ck(_lib.zxh_get_state_device(self._h, ctypes.c_void_p(ptr), int(elems), int(order)))

    def required_M(self) -> int:
        out = _SZ(0)
        self._ck(_lib.zxh_required_M(self._h, ctypes.byref(out)))
        return int(out.value)

    def num_qubits(self) -> int:
        return self._n

    def state_view(self):
        """(device pointer, real bits m, bytes per amplitude, global phase)."""
        p, m, eb = _P(), _SZ(0), _SZ(0)
        gr, gi = _D(0.0), _D(0.0)
        self._ck(_lib.zxh_state_view(self._h, ctypes.byref(p), ctypes.byref(m), ctypes.byref(eb),
                                     ctypes.byref(gr), ctypes.byref(gi)))
        return int(p.value or 0), int(m.value), int(eb.value), complex(gr.value, gi.value)

    def stream(self) -> int:
        s = _P()
        self._ck(_lib.zxh_stream(self._h, ctypes.byref(s)))
        return int(s.value or 0)

    def set_param(self, name: str, value: int) -> None:
        """Pass-planner tuning knob (see zxh_set_param in include/zxh_b200.h)."""
        self._ck(_lib.zxh_set_param(self._h, name.encode(), int(value)))

    def last_stats(self) -> tuple:
        """(kernels launched, state passes, device ms) of the last execute/apply/measure."""
        k, p, ms = _U64(0), _U64(0), _D(0.0)
        self._ck(_lib.zxh_last_stats(self._h, ctypes.byref(k), ctypes.byref(p), ctypes.byref(ms)))
        return int(k.value), int(p.value), float(ms.value)

    # --- observables and gradients (no counterpart in the reference) -----------------
    def gate_count(self) -> int:
        """Recorded gates after lowering (CRz counts as P + CP)."""
        out = _SZ(0)
        self._ck(_lib.zxh_gate_count(self._h, ctypes.byref(out)))
        return int(out.value)

    def expectation(self, terms) -> float:
        """<psi|H|psi> of the current state for Z / ZZ / X terms, FP64-reduced on the GPU."""
        t = as_terms(terms)
        v = _D(0.0)
        self._ck(_lib.zxh_expectation(self._h, t.ctypes.data, len(t), ctypes.byref(v)))
        return float(v.value)

    def adjoint_gradient(self, terms, checkpoint_every: int = 0) -> tuple:
        """(<H>, d<H>/d theta per recorded gate) from one forward and one reverse
        sweep over the recorded gates; leaves the forward output as the state."""
        t = as_terms(terms)
        cnt = self.gate_count()
        g = np.zeros(max(cnt, 1), np.float64)
        v = _D(0.0)
        self._ck(_lib.zxh_adjoint_gradient(self._h, t.ctypes.data, len(t), int(checkpoint_every), ctypes.byref(v),
                                           g.ctypes.data, g.size))
        return float(v.value), g[:cnt]
