"""Circuit loader for the native ZXH gate set.

Same contract as the reference's ``load_circuit_transpiled``
(src/zxh/zxhsim/qasm.py:65-133 of ZXH-Sim): the circuit must already be lowered
to the native gates (src/zxh/zxhsim/gate_sets.py ZXH_NATIVE_GATES); ``u``/``u3``
parameters are reordered from (theta, phi, lambda) to ZXH's (theta, lambda, phi);
``reset`` clears the recorded gates; ``measure`` and ``id`` are skipped. The
circuit object is used through the Qiskit ``QuantumCircuit`` interface
(``.data``, ``.find_bit``) but Qiskit itself is not imported. Unlike the
reference, which calls one binding method per gate, records are collected and
pushed in one ``push_gates`` call.
"""
from __future__ import annotations

import math

import numpy as np

from . import _core

NATIVE_GATES = frozenset(
    ("barrier", "measure", "reset", "id", "x", "cx", "h", "z", "rz", "rx", "p", "u", "u3", "cp", "crz")
)


def _qubit_index(circuit, qubit) -> int:
    return circuit.find_bit(qubit).index


def _to_float(value) -> float:
    try:
        return float(value)
    except Exception as exc:  # symbolic parameters
        raise ValueError(f"Cannot evaluate symbolic parameter {value!r} to float.") from exc


def load_circuit_transpiled(sim, circuit) -> None:
    unsupported = sorted({inst.operation.name.lower() for inst in circuit.data} - NATIVE_GATES)
    if unsupported:
        raise NotImplementedError(
            f"Circuit contains gates outside the allowed set: {unsupported}. allowed_gates={sorted(NATIVE_GATES)}"
        )
    recs = []

    def flush():
        if recs:
            sim.push_gates(_core.as_records(recs))
            recs.clear()

    for inst in circuit.data:
        op = inst.operation
        name = op.name.lower()
        qs = [_qubit_index(circuit, q) for q in inst.qubits]
        if name in ("measure", "id"):
            continue
        if name == "reset":
            flush()
            sim.clear_gates()
            continue
        if name == "barrier":
            recs.append((_core.BARRIER, 0, 0))
        elif name == "x":
            recs.append((_core.X, 0, qs[0]))
        elif name == "cx":
            recs.append((_core.CX, qs[0], qs[1]))
        elif name == "h":
            recs.append((_core.H, 0, qs[0]))
        elif name == "z":
            recs.append((_core.Z, 0, qs[0]))
        elif name == "rz":
            recs.append((_core.RZ, 0, qs[0], _to_float(op.params[0])))
        elif name == "rx":
            recs.append((_core.RX, 0, qs[0], _to_float(op.params[0])))
        elif name == "p":
            recs.append((_core.P, 0, qs[0], _to_float(op.params[0])))
        elif name in ("u", "u3"):
            theta, phi, lam = (_to_float(v) for v in op.params[:3])
            recs.append((_core.U3, 0, qs[0], theta, lam, phi))
        elif name == "cp":
            recs.append((_core.CP, qs[0], qs[1], _to_float(op.params[0])))
        elif name == "crz":
            recs.append((_core.CRZ, qs[0], qs[1], _to_float(op.params[0])))
    flush()


# Gates the circuit compiler accepts (the reference's frontend set,
# src/zxh/zxhsim/gate_sets.py ZXH_FRONTEND_GATES); those outside NATIVE_GATES are
# lowered to native records first.
FRONTEND_GATES = NATIVE_GATES | frozenset(
    ("swap", "cz", "ry", "u1", "u2", "s", "sdg", "t", "tdg", "rzz", "ccz", "ccx")
)


def _ccz(c0: int, c1: int, t: int) -> list:
    """CCZ as 6 CX and 7 RZ(+-pi/4), equal to CCZ up to a global phase: the
    textbook Toffoli phase network the reference's compiler also emits
    (circ_optimizer.py:153-168)."""
    a = math.pi / 4.0
    seq = [("cx", c1, t), ("rz", t, -a), ("cx", c0, t), ("rz", t, a), ("cx", c1, t), ("rz", t, -a),
           ("cx", c0, t), ("rz", c1, a), ("rz", t, a), ("cx", c0, c1), ("rz", c0, a), ("rz", c1, -a),
           ("cx", c0, c1)]
    return [(_core.CX, x, y) if k == "cx" else (_core.RZ, 0, x, y) for k, x, y in seq]


def frontend_records(name: str, qs, params) -> list:
    """One frontend instruction as native gate records: the reference's lowering of
    swap / cz / rzz / ccz / ccx (circ_optimizer.py:171-209) and the standard
    definitions of ry, u1, u2, s, sdg, t, tdg. measure / reset / id give []."""
    C = _core
    p = [_to_float(v) for v in params]
    if name in ("measure", "reset", "id"):
        return []
    one = {
        "x": lambda: [(C.X, 0, qs[0])],
        "h": lambda: [(C.H, 0, qs[0])],
        "z": lambda: [(C.Z, 0, qs[0])],
        "rz": lambda: [(C.RZ, 0, qs[0], p[0])],
        "rx": lambda: [(C.RX, 0, qs[0], p[0])],
        "ry": lambda: [(C.U3, 0, qs[0], p[0], 0.0, 0.0)],
        "p": lambda: [(C.P, 0, qs[0], p[0])],
        "u1": lambda: [(C.P, 0, qs[0], p[0])],
        "u2": lambda: [(C.U3, 0, qs[0], math.pi / 2.0, p[1], p[0])],  # u2(phi, lambda)
        "s": lambda: [(C.P, 0, qs[0], math.pi / 2.0)],
        "sdg": lambda: [(C.P, 0, qs[0], -math.pi / 2.0)],
        "t": lambda: [(C.P, 0, qs[0], math.pi / 4.0)],
        "tdg": lambda: [(C.P, 0, qs[0], -math.pi / 4.0)],
        "u": lambda: [(C.U3, 0, qs[0], p[0], p[2], p[1])],  # (theta, phi, lambda) -> (theta, lambda, phi)
        "u3": lambda: [(C.U3, 0, qs[0], p[0], p[2], p[1])],
        "barrier": lambda: [(C.BARRIER, 0, 0)],
        "cx": lambda: [(C.CX, qs[0], qs[1])],
        "cp": lambda: [(C.CP, qs[0], qs[1], p[0])],
        "crz": lambda: [(C.CRZ, qs[0], qs[1], p[0])],
        "cz": lambda: [(C.CP, qs[0], qs[1], math.pi)],
        "swap": lambda: [(C.CX, qs[0], qs[1]), (C.CX, qs[1], qs[0]), (C.CX, qs[0], qs[1])],
        "rzz": lambda: [(C.CX, qs[0], qs[1]), (C.RZ, 0, qs[1], p[0]), (C.CX, qs[0], qs[1])],
        "ccz": lambda: _ccz(qs[0], qs[1], qs[2]),
        "ccx": lambda: [(C.H, 0, qs[2])] + _ccz(qs[0], qs[1], qs[2]) + [(C.H, 0, qs[2])],
    }
    if name not in one:
        raise NotImplementedError(
            f"Circuit contains gates outside the allowed set: {[name]}. allowed_gates={sorted(FRONTEND_GATES)}"
        )
    return one[name]()


def compile_circuit(circuit, n: int, optimize_level: int = 2):
    """The circuit as segments of compiled records: ``(records, reset_before)``.

    Frontend gates are lowered (frontend_records) and each stretch between
    measure / reset instructions (where the reference's scheduler flushes every
    qubit) goes through the host circuit compiler (``zxh_optimize_gates``, the
    reference's boundary scheduler at ``optimize_level``)."""
    segments, cur, reset = [], [], False

    def close():
        nonlocal cur, reset
        if cur or reset:
            recs = _core.optimize_records(n, cur, optimize_level) if cur else np.zeros(0, _core.GATE_DTYPE)
            segments.append((recs, reset))
        cur, reset = [], False

    for inst in circuit.data:
        name = inst.operation.name.lower()
        qs = [_qubit_index(circuit, q) for q in inst.qubits]
        if name in ("measure", "reset"):
            close()
            reset = name == "reset"
            continue
        cur.extend(frontend_records(name, qs, inst.operation.params))
    close()
    return segments


def load_circuit(sim, circuit, optimize_level: int | None = None) -> None:
    """The reference's ``load_circuit`` (qasm.py:54-62): compile the circuit with
    the boundary scheduler at ``optimize_level`` (default 0: gates re-emitted one
    by one, identities dropped), then record it on ``sim``."""
    level = 0 if optimize_level is None else int(optimize_level)
    for recs, reset in compile_circuit(circuit, sim.num_qubits(), level):
        if reset:
            sim.clear_gates()
        if len(recs):
            sim.push_gates(recs)


def bitrow_to_str(row) -> str:
    """Bit row (entry q = qubit q) as a string with qubit n-1 first (qasm.py:136-137)."""
    return "".join("1" if bit else "0" for bit in reversed(row))


def records(gates) -> np.ndarray:
    return _core.as_records(gates)
