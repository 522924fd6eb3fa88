"""Test infrastructure only: CPU checks of the expectation and adjoint-gradient path.

The reference has no observables, so there is nothing of its own to restate
here. Parity of ``zxh_expectation`` / ``zxh_adjoint_gradient`` is anchored on the
reference's forward semantics instead: every energy below is computed from the
oracle's state (``Oracle.get_state``, bit-exact with the reference's serial
backend, zxh.cpp:579-636), and every derivative is a central difference or a
parameter shift of such energies. ``dense_adjoint`` restates the adjoint method
itself on a dense numpy state (qubit q = bit q), for the CPU tests of the
method's formulas; the product never imports this module.
"""
from __future__ import annotations

import math

import numpy as np

from .bridge import Oracle

TERM_Z, TERM_ZZ, TERM_X = 1, 2, 3


def qubit_order(state_ref: np.ndarray, n: int) -> np.ndarray:
    """Reference get_state order (qubit q at bit n-1-q) -> qubit q at bit q."""
    idx = np.arange(1 << n)
    rev = np.zeros_like(idx)
    for q in range(n):
        rev |= ((idx >> q) & 1) << (n - 1 - q)
    return state_ref[rev]


def terms_rows(terms):
    """(kind, q0, q1, coef) rows from a structured term array or tuples."""
    if isinstance(terms, np.ndarray) and terms.dtype.names:
        return [(int(t["kind"]), int(t["q0"]), int(t["q1"]), float(t["coef"])) for t in terms]
    return [tuple(t) for t in terms]


def energy_dense(psi: np.ndarray, n: int, terms) -> float:
    """<psi|H|psi> for (kind, q0, q1, coef) terms, psi in qubit order."""
    idx = np.arange(1 << n)
    p = np.abs(psi) ** 2
    e = 0.0
    for kind, q0, q1, c in terms_rows(terms):
        if kind == TERM_Z:
            e += c * float(np.sum(p * (1 - 2 * ((idx >> q0) & 1))))
        elif kind == TERM_ZZ:
            s = ((idx >> q0) ^ (idx >> q1)) & 1
            e += c * float(np.sum(p * (1 - 2 * s)))
        elif kind == TERM_X:
            e += c * float(np.real(np.vdot(psi, psi[idx ^ (1 << q0)])))
        else:
            raise ValueError(kind)
    return e


def oracle_state(n: int, records) -> np.ndarray:
    """The oracle's state after the gate records, in qubit order."""
    o = Oracle(n)
    o.push(records)
    o.execute()
    return qubit_order(o.get_state(), n)


def oracle_energy(n: int, records, terms) -> float:
    """<H> of the oracle's state after the gate records."""
    return energy_dense(oracle_state(n, records), n, terms)


def _oracle_shift(n, circ, params, terms, s, which):
    p = np.asarray(params, np.float64)
    ks = range(p.size) if which is None else which
    g = np.full(p.size, np.nan)
    for k in ks:
        d = np.zeros_like(p)
        d[k] = s
        g[k] = oracle_energy(n, circ.records(p + d), terms) - oracle_energy(n, circ.records(p - d), terms)
    return g


def oracle_central_difference(n: int, circ, params, terms, step: float = 1e-6, which=None) -> np.ndarray:
    """FP64 central differences of oracle energies for the parameters in `which`."""
    return _oracle_shift(n, circ, params, terms, step, which) / (2 * step)


def oracle_parameter_shift(n: int, circ, params, terms, which=None) -> np.ndarray:
    """(E(p + pi/2 e_k) - E(p - pi/2 e_k)) / 2 of oracle energies."""
    return _oracle_shift(n, circ, params, terms, math.pi / 2, which) / 2


# --- dense restatement of the adjoint method ----------------------------------------

def _u3(th, la, ph):
    c, s = math.cos(th / 2), math.sin(th / 2)
    return np.array([[c, -np.exp(1j * la) * s], [np.exp(1j * ph) * s, np.exp(1j * (ph + la)) * c]])


def _gate(g):
    """(kind, q, cq, matrix / diagonal / phase, generator) of a lowered record."""
    t, cq, q, th, la, ph = (int(g[0]), int(g[1]), int(g[2]), float(g[4]), float(g[5]), float(g[6]))
    if t == 9:
        return "u", q, None, np.array([[1, 1], [1, -1]]) / math.sqrt(2), None
    if t == 10:
        gen = None
        if la == 0.0 and ph == 0.0:
            gen = np.array([[0, -1j], [1j, 0]])
        elif la == math.pi / 2 and ph == -math.pi / 2:
            gen = np.array([[0, 1], [1, 0]])
        return "u", q, None, _u3(th, la, ph), gen
    if t == 7:
        return "u", q, None, np.array([[0, 1], [1, 0]]), None
    if t == 8:
        return "cx", q, cq, None, None
    if t in (2, 3, 4):
        th = math.pi if t == 2 else th
        d = np.array([np.exp(-0.5j * th), np.exp(0.5j * th)]) if t in (2, 3) else np.array([1, np.exp(1j * th)])
        gen = None if t == 2 else (np.array([1.0, -1.0]) if t == 3 else np.array([0.0, -2.0]))
        return "d", q, None, d, gen
    if t == 6:
        return "cp", q, cq, np.exp(1j * th), np.array([0.0, -2.0])
    if t == 1:
        return "b", 0, None, None, None
    raise ValueError(t)


def _apply(psi, n, kind, q, cq, m, inverse=False):
    idx = np.arange(1 << n)
    out = psi.copy()
    if kind == "u":
        if inverse:
            m = m.conj().T
        i0 = idx[((idx >> q) & 1) == 0]
        i1 = i0 | (1 << q)
        out[i0] = m[0, 0] * psi[i0] + m[0, 1] * psi[i1]
        out[i1] = m[1, 0] * psi[i0] + m[1, 1] * psi[i1]
    elif kind == "cx":
        on = ((idx >> cq) & 1) == 1
        out[on] = psi[idx[on] ^ (1 << q)]
    elif kind == "d":
        f = m[(idx >> q) & 1]
        out = psi * (f.conj() if inverse else f)
    elif kind == "cp":
        s = ((idx >> q) & (idx >> cq) & 1) == 1
        out[s] = psi[s] * (np.conj(m) if inverse else m)
    return out


def _hamiltonian_apply(psi, n, terms):
    idx = np.arange(1 << n)
    out = np.zeros_like(psi)
    for kind, q0, q1, c in terms_rows(terms):
        if kind == TERM_Z:
            out += c * (1 - 2 * ((idx >> q0) & 1)) * psi
        elif kind == TERM_ZZ:
            out += c * (1 - 2 * (((idx >> q0) ^ (idx >> q1)) & 1)) * psi
        else:
            out += c * psi[idx ^ (1 << q0)]
    return out


def dense_adjoint(n: int, records, terms):
    """(<H>, per-record gradient) by the adjoint method on a dense state: psi and
    lambda = H psi walk back over the gates, and for U_k = exp(-i theta G_k) the
    gradient is 2 Im<lambda|G_k|psi> taken on the states right after gate k, i.e.
    Im<lambda|Gen|psi> with Gen = Y, X, Z for RY, RX, RZ and -2 Pi_1 for P and CP."""
    psi = np.zeros(1 << n, complex)
    psi[0] = 1
    ops = [_gate(g) for g in records]
    for kind, q, cq, m, _ in ops:
        psi = _apply(psi, n, kind, q, cq, m)
    lam = _hamiltonian_apply(psi, n, terms)
    e = float(np.real(np.vdot(psi, lam)))
    idx = np.arange(1 << n)
    grads = np.zeros(len(ops))
    for k in range(len(ops) - 1, -1, -1):
        kind, q, cq, m, gen = ops[k]
        if gen is not None:
            if kind == "u":
                gpsi = _apply(psi, n, "u", q, None, gen)
            elif kind == "d":
                gpsi = gen[(idx >> q) & 1] * psi
            else:
                gpsi = np.where(((idx >> q) & (idx >> cq) & 1) == 1, gen[1], 0.0) * psi
            grads[k] = float(np.imag(np.vdot(lam, gpsi)))
        psi = _apply(psi, n, kind, q, cq, m, inverse=True)
        lam = _apply(lam, n, kind, q, cq, m, inverse=True)
    return e, grads
