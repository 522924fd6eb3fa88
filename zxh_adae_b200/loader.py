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


def bitrow_to_str(row) -> str:
    """Bit row (entry q = qubit q) as a string with qubit n-1 first (qasm.py:136-137)."""
    return "".join("1" if bit else "0" for bit in reversed(row))


def records(gates) -> np.ndarray:
    return _core.as_records(gates)
