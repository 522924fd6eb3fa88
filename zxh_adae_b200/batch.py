"""Energies and adjoint gradients of many independent circuits in one launch.

Binds the ``zxh_batch_*`` entry points of include/zxh_b200.h (no counterpart in
the reference, which runs one circuit per ``ZXH`` object with process-global
device state). Each circuit has its own qubit count, gate records and observable
terms; the library compiles every circuit once into a chain of passes and runs
all chains either one launch at a time (``"sequential"``), in one persistent
kernel that takes tasks from a queue (``"persistent"``), or by replaying that
launch from a captured CUDA graph (``"graph"``). ``tune()`` times the persistent
launch over the gate-fusion depth, the task size (the tile of work one CTA
takes), the threads per CTA and the reverse passes' depth, keeps the fastest,
and can persist the choice (tuning.py).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _core
from ._core import _D, _P, _SZ, _U64, C64, C128, _lib, as_records, as_terms, device_info
from .tuning import KNOBS, TuneCache, batch_key

MODES = {"sequential": 0, "persistent": 1, "graph": 2}
_ERRORS = _core._ERRORS


def _raise(rc, handle):
    msg = _lib.zxh_batch_last_error(handle).decode(errors="replace")
    raise _ERRORS.get(rc, RuntimeError)(msg or f"zxh batch error {rc}")


class Batch:
    """``circuits``: iterable of ``(n, gate_records, terms)``."""

    def __init__(self, circuits, dtype: str = "complex64", device: int = 0):
        if dtype not in ("complex64", "complex128"):
            raise ValueError("dtype must be 'complex64' or 'complex128'")
        circuits = list(circuits)
        nq = np.array([int(c[0]) for c in circuits], np.uint32)
        recs = [as_records(c[1]) for c in circuits]
        terms = [as_terms(c[2]) for c in circuits]
        goff = np.zeros(len(circuits) + 1, np.uint64)
        goff[1:] = np.cumsum([len(r) for r in recs])
        toff = np.zeros(len(circuits) + 1, np.uint64)
        toff[1:] = np.cumsum([len(t) for t in terms])
        g = np.concatenate(recs) if recs else np.zeros(0, _core.GATE_DTYPE)
        t = np.concatenate(terms) if terms else np.zeros(0, _core.TERM_DTYPE)
        g = np.ascontiguousarray(g if len(g) else np.zeros(1, _core.GATE_DTYPE))
        t = np.ascontiguousarray(t if len(t) else np.zeros(1, _core.TERM_DTYPE))
        h = _P()
        rc = _lib.zxh_batch_create(ctypes.byref(h), len(circuits), nq.ctypes.data, goff.ctypes.data, g.ctypes.data,
                                   toff.ctypes.data, t.ctypes.data, C64 if dtype == "complex64" else C128, int(device))
        if rc != 0:
            _raise(rc, None)
        self._h = h
        self.count = len(circuits)
        self.nqubits = nq
        self.dtype = dtype
        self.device = int(device)
        off = np.zeros(self.count + 1, np.uint64)
        self._ck(_lib.zxh_batch_gradient_offsets(self._h, off.ctypes.data))
        self.grad_offsets = off.astype(np.int64)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.zxh_batch_destroy(h)
            self._h = None

    def close(self) -> None:
        self.__del__()

    def _ck(self, rc):
        if rc != 0:
            _raise(rc, self._h)

    def run(self, mode: str = "graph"):
        """(energies[count], flat gradients) -- circuit c's gradients are
        ``grads[grad_offsets[c]:grad_offsets[c + 1]]``, one per recorded gate."""
        e = np.zeros(self.count, np.float64)
        g = np.zeros(max(int(self.grad_offsets[-1]), 1), np.float64)
        self._ck(_lib.zxh_batch_run(self._h, MODES[mode], e.ctypes.data, g.ctypes.data, g.size))
        return e, g[: int(self.grad_offsets[-1])]

    def gradients(self, flat):
        return [flat[self.grad_offsets[c]:self.grad_offsets[c + 1]] for c in range(self.count)]

    def set(self, name: str, value: int) -> None:
        self._ck(_lib.zxh_batch_set(self._h, name.encode(), int(value)))

    def get(self, name: str) -> int:
        v = ctypes.c_int(0)
        self._ck(_lib.zxh_batch_get(self._h, name.encode(), ctypes.byref(v)))
        return int(v.value)

    def settings(self) -> dict:
        """The knob settings in use (tuning.KNOBS)."""
        return {k: self.get(k) for k in KNOBS}

    def tune(self, reps: int = 1, cache=None) -> dict:
        """Times the persistent launch over its knobs (zxh_batch_tune) and keeps
        the fastest. cache: a path (or TuneCache); settings found there for this
        batch's shape and GPU are applied without timing, and new ones are stored."""
        tc = cache if isinstance(cache, TuneCache) or cache is None else TuneCache(cache)
        key = batch_key(self.nqubits, self.dtype, *device_info(self.device)) if tc else None
        hit = tc.get(key) if tc else None
        if hit:
            for k in KNOBS:
                self.set(k, hit[k])
            return {**hit, "cached": True}
        self._ck(_lib.zxh_batch_tune(self._h, int(reps)))
        out = self.settings()
        if tc:
            tc.put(key, out)
        return {**out, "cached": False}

    def stats(self) -> tuple:
        """(ops, tasks, device ms of the last run)."""
        o, t, ms, by = _U64(0), _U64(0), _D(0.0), _U64(0)
        self._ck(_lib.zxh_batch_stats(self._h, ctypes.byref(o), ctypes.byref(t), ctypes.byref(ms), ctypes.byref(by)))
        return int(o.value), int(t.value), float(ms.value)

    def state_bytes(self) -> int:
        """Algorithmic state bytes of one run (the roofline numerator)."""
        by = _U64(0)
        self._ck(_lib.zxh_batch_stats(self._h, None, None, None, ctypes.byref(by)))
        return int(by.value)
