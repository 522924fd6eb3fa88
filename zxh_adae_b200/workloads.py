"""Seeded synthetic circuits of the benchmark configurations.

The reference quotes its results on MQT-Bench circuits (not used here); these
generators stand in for them with the shapes, sizes and angle distributions of
the five configurations this path is measured on. Every generator takes one
integer seed and draws from ``numpy.random.default_rng(seed)`` in a fixed order,
so any run (ours, the oracle's, the reference's) sees the same gate list.

Records use the 40-byte layout of include/zxh_b200.h; U3 records carry
(theta, lambda, phi) in ZXH's argument order. This module and ``records`` load
no native code.
"""
from __future__ import annotations

import math

import numpy as np

from .records import BARRIER, CP, CX, H, P, RZ, U3, X, as_records

TWO_PI = 2.0 * math.pi


def plain_layers(n: int, layers: int, seed: int) -> np.ndarray:
    """H on every qubit, then `layers` x [U3 on every qubit; cp(alpha) on (i, i+1)].

    Draw order per layer: for each qubit (theta, phi, lambda), then the n-1 alphas.
    Configuration 1 is plain_layers(20, 10, seed) followed by 1024 shots.
    """
    rng = np.random.default_rng(seed)
    recs = [(H, 0, q) for q in range(n)]
    for _ in range(layers):
        ang = rng.uniform(0.0, TWO_PI, size=(n, 3))
        alpha = rng.uniform(0.0, TWO_PI, size=n - 1)
        for q in range(n):
            th, ph, la = ang[q]
            recs.append((U3, 0, q, th, la, ph))
        for i in range(n - 1):
            recs.append((CP, i, i + 1, alpha[i]))
    return as_records(recs)


def h_all(n: int) -> np.ndarray:
    return as_records([(H, 0, q) for q in range(n)])


def diag_batch(n: int, batch: int, seed: int) -> np.ndarray:
    """B gates: p on a uniform qubit or cp on a uniform ordered pair (50/50),
    angle uniform [0, 2 pi) (configuration 2, without the H header)."""
    rng = np.random.default_rng(seed)
    recs = []
    for _ in range(batch):
        kind = rng.integers(2)
        th = rng.uniform(0.0, TWO_PI)
        if kind == 0:
            recs.append((P, 0, int(rng.integers(n)), th))
        else:
            c = int(rng.integers(n))
            t = int(rng.integers(n - 1))
            t = t + 1 if t >= c else t
            recs.append((CP, c, t, th))
    return as_records(recs)


def cx_chain(n: int) -> np.ndarray:
    """CX(i, i+1) for i = 0..n-2, in order (the adjoint ansatz's entangling chain).
    After it every qubit's selector is the parity of a prefix of the real bits, so
    the p/cp gates of a following window have multi-bit selectors."""
    return as_records([(CX, i, i + 1) for i in range(n - 1)])


def cp_cascade(n: int) -> np.ndarray:
    """Controlled-phase cascade over all pairs j > i with angle pi / 2^(j - i)."""
    recs = []
    for i in range(n):
        for j in range(i + 1, n):
            recs.append((CP, i, j, math.pi / float(2 ** (j - i))))
    return as_records(recs)


def u3_layer(n: int, seed: int) -> np.ndarray:
    """U3 on every qubit, angles (theta, phi, lambda) uniform [0, 2 pi) drawn qubit
    by qubit: one U3 batch of configuration 3, without its cz matching."""
    rng = np.random.default_rng(seed)
    ang = rng.uniform(0.0, TWO_PI, size=(n, 3))
    return as_records([(U3, 0, q, ang[q][0], ang[q][2], ang[q][1]) for q in range(n)])


def u3_matching_layers(n: int, layers: int, seed: int) -> np.ndarray:
    """`layers` x [U3 on every qubit (angles uniform [0, 2 pi)); cz on a random
    perfect matching] after H on every qubit (configuration 3, first part).
    cz is recorded as CP(pi). Draw order per layer: angles (n x 3), then a
    permutation of the qubits whose consecutive pairs are matched."""
    rng = np.random.default_rng(seed)
    recs = [(H, 0, q) for q in range(n)]
    for _ in range(layers):
        ang = rng.uniform(0.0, TWO_PI, size=(n, 3))
        perm = rng.permutation(n)
        for q in range(n):
            th, ph, la = ang[q]
            recs.append((U3, 0, q, th, la, ph))
        for k in range(0, n - 1, 2):
            recs.append((CP, int(perm[k]), int(perm[k + 1]), math.pi))
    return as_records(recs)


def hidden_string(n_data: int, seed: int):
    """Hidden-string circuit on n_data + 1 qubits (ancilla = qubit n_data): H on
    every data qubit, X then H on the ancilla (preparing |->), CX from every data
    qubit whose secret bit is 1 onto the ancilla, H on the data qubits. The data
    register then reads the secret with certainty. (An H on the ancilla before
    its X would make H X H = Z act on |0>, cancel the phase kickback and lose the
    deterministic answer, so the ancilla gets X then H only.)
    Returns (records, secret)."""
    rng = np.random.default_rng(seed)
    secret = int(rng.integers(1, 1 << n_data))
    anc = n_data
    recs = [(H, 0, q) for q in range(n_data)]
    recs += [(X, 0, anc), (H, 0, anc)]
    for i in range(n_data):
        if (secret >> i) & 1:
            recs.append((CX, i, anc))
    recs += [(H, 0, q) for q in range(n_data)]
    return as_records(recs), secret


def random_circuit(n: int, count: int, seed: int, kinds=None) -> np.ndarray:
    """Random gate list over the whole native set (test workload)."""
    rng = np.random.default_rng(seed)
    kinds = kinds or [BARRIER, 2, RZ, P, 5, CP, X, CX, H, U3, 11]
    if n == 1:  # two-qubit gates need two distinct qubits
        kinds = [k for k in kinds if k not in (5, CP, CX)]
    recs = []
    for _ in range(count):
        t = int(kinds[rng.integers(len(kinds))])
        q = int(rng.integers(n))
        cq = int(rng.integers(n))
        if n > 1:
            while cq == q:
                cq = int(rng.integers(n))
        a = rng.uniform(0.0, TWO_PI, size=3)
        recs.append((t, cq, q, a[0], a[1], a[2]))
    return as_records(recs)


def batch_tfim(count: int, seed: int, nmin: int = 10, nmax: int = 22, layers: int = 20):
    """Configuration 5: `count` circuits, n uniform in {nmin..nmax}; each has
    `layers` x [U3(theta, phi, lambda) on every qubit; cp(alpha) on (i, i+1)] with
    angles uniform [0, 2 pi), and its own TFIM observable sum Z_i Z_{i+1} + h sum X_i,
    h uniform [0.5, 1.5]. U3 is recorded as P(lambda), RY(theta) = U3(theta, 0, 0),
    P(phi) (the same matrix, U = P(phi) RY(theta) P(lambda)) so that every angle is
    a parameter of the adjoint gradient; within a layer the P(lambda) of all qubits
    come first, then the RY, then the P(phi) (gates on different qubits commute).
    Returns a list of (n, records, terms, h).
    Draw order: n and h per circuit, then per layer (theta, phi, lambda) per qubit
    and the n - 1 alphas."""
    from .records import TERM_X, TERM_ZZ, as_terms

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(nmin, nmax + 1))
        h = float(rng.uniform(0.5, 1.5))
        recs = []
        for _ in range(layers):
            ang = rng.uniform(0.0, TWO_PI, size=(n, 3))
            alpha = rng.uniform(0.0, TWO_PI, size=n - 1)
            recs += [(P, 0, q, ang[q][2]) for q in range(n)]
            recs += [(U3, 0, q, ang[q][0], 0.0, 0.0) for q in range(n)]
            recs += [(P, 0, q, ang[q][1]) for q in range(n)]
            for i in range(n - 1):
                recs.append((CP, i, i + 1, alpha[i]))
        terms = as_terms([(TERM_ZZ, i, i + 1, 1.0) for i in range(n - 1)] + [(TERM_X, i, 0, h) for i in range(n)])
        out.append((n, as_records(recs), terms, h))
    return out

