"""Record layouts of the C ABI (include/zxh_b200.h) as numpy dtypes.

Pure numpy: importing this module loads no native code, so gate lists can be
built (by the workload generators, for instance) without the CUDA library.

* ``GATE_DTYPE``: the 40-byte ``zxh_gate`` record; field meaning follows the
  reference's gate_t (src/zxh/include/zxhsim/defs.h:76-84), U3 parameters in
  ZXH's (theta, lambda, phi) order (src/zxh/include/zxhsim/zxh.h:36).
* gate codes: the reference's gate_type_t numbering (defs.h:61-74).
* ``TERM_DTYPE``: the 24-byte ``zxh_term`` observable term.
"""
from __future__ import annotations

import numpy as np

GATE_DTYPE = np.dtype(
    [("type", "<u4"), ("cq", "<u4"), ("q", "<u4"), ("reserved", "<u4"),
     ("theta", "<f8"), ("lam", "<f8"), ("phi", "<f8")]
)

BARRIER, Z, RZ, P, CRZ, CP, X, CX, H, U3, RX = 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11

TERM_DTYPE = np.dtype([("kind", "<u4"), ("q0", "<u4"), ("q1", "<u4"), ("reserved", "<u4"), ("coef", "<f8")])
TERM_Z, TERM_ZZ, TERM_X = 1, 2, 3


def as_records(gates) -> np.ndarray:
    """Gate records from a structured array or an iterable of
    ``(type, cq, q[, theta, lambda, phi])`` tuples."""
    if isinstance(gates, np.ndarray) and gates.dtype == GATE_DTYPE:
        return np.ascontiguousarray(gates)
    rows = list(gates)
    rec = np.zeros(len(rows), GATE_DTYPE)
    for i, g in enumerate(rows):
        t, cq, q, th, la, ph = (list(g) + [0.0] * 6)[:6]
        rec[i] = (t, cq, q, 0, th, la, ph)
    return rec


def as_terms(terms) -> np.ndarray:
    """Observable terms from a structured array or ``(kind, q0, q1, coef)`` tuples."""
    if isinstance(terms, np.ndarray) and terms.dtype == TERM_DTYPE:
        return np.ascontiguousarray(terms)
    rows = list(terms)
    out = np.zeros(len(rows), TERM_DTYPE)
    for i, (k, q0, q1, c) in enumerate(rows):
        out[i] = (k, q0, q1, 0, c)
    return out
