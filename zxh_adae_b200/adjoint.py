"""Expectation values and adjoint gradients of parameterised circuits.

No counterpart in the reference (ZXH-Sim computes states and samples only). The
device work is ``zxh_adjoint_gradient`` of the C ABI: one forward pass of the
recorded gates, lambda = H psi, and one reverse sweep that uncomputes psi and
lambda with the inverse gates and reduces every d<H>/d theta in FP64 inside the
reverse passes. This module adds

* ``tfim_terms`` -- the transverse-field Ising observable sum J Z_i Z_{i+1} + h sum X_i
  (open boundary) as ``zxh_term`` records;
* ``hardware_efficient_ansatz`` -- L repetitions of [RY, RZ on every qubit, CX chain
  i -> i+1] plus a final RY/RZ layer (2 n (L + 1) parameters);
* ``Circuit`` -- gate records with a linear map from parameters to record angles;
* ``AdjointExpectation`` -- a ``torch.autograd.Function`` returning <H> whose
  backward is the adjoint gradient;
* ``finite_difference`` and ``parameter_shift`` -- the two checks, both run on the
  plain forward path (``execute`` + ``expectation``).
"""
from __future__ import annotations

import math

import numpy as np

from . import _core
from ._core import CRZ, CX, RX, RZ, TERM_X, TERM_ZZ, U3, as_records, as_terms


def tfim_terms(n: int, h: float = 1.0, j: float = 1.0) -> np.ndarray:
    """sum_i j Z_i Z_{i+1} (i < n-1) + h sum_i X_i."""
    rows = [(TERM_ZZ, i, i + 1, j) for i in range(n - 1)] + [(TERM_X, i, 0, h) for i in range(n)]
    return as_terms(rows)


class Circuit:
    """Gate records whose angles are ``theta[slot[k]] = coef[k] * params[param[k]]``.

    ``records`` may hold CRz and Rx records; they are lowered the way the library
    records them (CRz: P(-theta/2) on the control, then CP(theta), zxh.cpp:246-252;
    Rx: U3(theta, pi/2, -pi/2), zxh.cpp:303-310), so the per-record gradients of
    ``zxh_adjoint_gradient`` line up with ``base`` and ``gradient`` turns them into
    d<H>/d param."""

    def __init__(self, n: int, records, param_of_record):
        rec = as_records(records)
        pr = np.asarray(param_of_record, np.int64)
        if pr.shape != (len(rec),):
            raise ValueError("param_of_record needs one entry per record (-1 = fixed gate)")
        low = []
        slot, param, coef = [], [], []
        for i, r in enumerate(rec):
            p = int(pr[i])
            if r["type"] == CRZ:
                low.append((_core.P, 0, r["cq"], -0.5 * r["theta"], 0.0, 0.0))
                low.append((_core.CP, r["cq"], r["q"], r["theta"], 0.0, 0.0))
                if p >= 0:
                    slot += [len(low) - 2, len(low) - 1]
                    param += [p, p]
                    coef += [-0.5, 1.0]
                continue
            if r["type"] == RX:
                low.append((U3, 0, r["q"], r["theta"], math.pi / 2, -math.pi / 2))
            else:
                low.append(tuple(r[k] for k in ("type", "cq", "q", "theta", "lam", "phi")))
            if p >= 0:
                slot.append(len(low) - 1)
                param.append(p)
                coef.append(1.0)
        self.n = int(n)
        self.base = as_records(low)
        self.slot = np.asarray(slot, np.int64)
        self.param = np.asarray(param, np.int64)
        self.coef = np.asarray(coef, np.float64)
        self.nparams = int(self.param.max()) + 1 if len(self.param) else 0

    def records(self, params) -> np.ndarray:
        p = np.asarray(params, np.float64)
        if p.shape != (self.nparams,):
            raise ValueError(f"expected {self.nparams} parameters")
        rec = self.base.copy()
        rec["theta"][self.slot] = self.coef * p[self.param]
        return rec

    def gradient(self, per_gate: np.ndarray) -> np.ndarray:
        """Chain rule from per-record gradients to parameter gradients."""
        g = np.zeros(self.nparams, np.float64)
        np.add.at(g, self.param, self.coef * np.asarray(per_gate)[self.slot])
        return g


def hardware_efficient_ansatz(n: int, reps: int = 8) -> Circuit:
    """reps x [RY(q), RZ(q) on every qubit; CX(i, i+1) chain] + final RY/RZ layer.
    RY is the record U3(theta, 0, 0). Parameters: layer r holds RY angles of qubits
    0..n-1 at 2 n r + q and RZ angles at 2 n r + n + q."""
    rec, par = [], []
    for r in range(reps + 1):
        for q in range(n):
            rec.append((U3, 0, q, 0.0, 0.0, 0.0))
            par.append(2 * n * r + q)
        for q in range(n):
            rec.append((RZ, 0, q, 0.0))
            par.append(2 * n * r + n + q)
        if r < reps:
            for q in range(n - 1):
                rec.append((CX, q, q + 1))
                par.append(-1)
    return Circuit(n, rec, par)


def energy(sim, circ: Circuit, params, terms, device_ms: list | None = None) -> float:
    """<H> through the plain forward path: execute, then the expectation pass.
    device_ms, if given, receives the kernel milliseconds of both (CUDA events on
    the simulator's stream)."""
    sim.clear_gates()
    sim.push_gates(circ.records(params))
    sim.execute()
    ms = sim.last_stats()[2]
    e = sim.expectation(terms)
    if device_ms is not None:
        device_ms.append(ms + sim.last_stats()[2])
    return e


def adjoint(sim, circ: Circuit, params, terms, checkpoint_every: int = 0):
    """(<H>, d<H>/d params) from one forward and one reverse sweep."""
    sim.clear_gates()
    sim.push_gates(circ.records(params))
    e, g = sim.adjoint_gradient(terms, checkpoint_every)
    return e, circ.gradient(g)


def _shifted(sim, circ, params, terms, s, which, device_ms=None):
    p = np.asarray(params, np.float64)
    ks = range(p.size) if which is None else which
    g = np.full(p.size, np.nan)
    for k in ks:
        d = np.zeros_like(p)
        d[k] = s
        g[k] = energy(sim, circ, p + d, terms, device_ms) - energy(sim, circ, p - d, terms, device_ms)
    return g


def finite_difference(sim, circ: Circuit, params, terms, step: float = 1e-6, which=None) -> np.ndarray:
    """Central differences (E(p + s e_k) - E(p - s e_k)) / 2 s for the parameters
    in ``which`` (all by default; the others are NaN)."""
    return _shifted(sim, circ, params, terms, step, which) / (2 * step)


def parameter_shift(sim, circ: Circuit, params, terms, which=None, device_ms: list | None = None) -> np.ndarray:
    """(E(p + pi/2 e_k) - E(p - pi/2 e_k)) / 2: exact for RY, RZ, RX, P and CP
    parameters that feed one gate each (each is a single-frequency rotation).
    device_ms, if given, receives the kernel milliseconds of every energy."""
    if len(np.unique(circ.param)) != len(circ.param) or np.any(circ.coef != 1.0):
        raise ValueError("parameter shift needs every parameter on exactly one gate with coefficient 1")
    return _shifted(sim, circ, params, terms, math.pi / 2, which, device_ms) / 2


try:
    import torch

    class AdjointExpectation(torch.autograd.Function):
        """<H>(params) with the adjoint gradient as its backward.

        ``AdjointExpectation.apply(params, sim, circuit, terms, checkpoint_every)``;
        params is a 1-D tensor; the result is a 0-d float64 tensor on params' device."""

        @staticmethod
        def forward(ctx, params, sim, circ, terms, checkpoint_every=0):
            p = params.detach().to("cpu", torch.float64).numpy()
            e, g = adjoint(sim, circ, p, terms, checkpoint_every)
            ctx.save_for_backward(torch.as_tensor(g, dtype=params.dtype, device=params.device))
            return torch.tensor(e, dtype=torch.float64, device=params.device)

        @staticmethod
        def backward(ctx, gout):
            (g,) = ctx.saved_tensors
            return gout.to(g.dtype) * g, None, None, None, None

except ImportError:  # torch is optional for the C ABI and the numpy helpers
    AdjointExpectation = None


__all__ = ["tfim_terms", "Circuit", "hardware_efficient_ansatz", "energy", "adjoint", "finite_difference",
           "parameter_shift", "AdjointExpectation"]
