"""CPU tests of the host circuit compiler (zxh_optimize_gates, loader.compile_circuit):
the reference's boundary-scheduler cases (src/zxh/tests/unit/test_circ_optimizer.py:
15-127, which compare Qiskit Operators) restated over gate records, with
equivalence checked on the oracle: the compiled circuit's unitary equals the
input's up to one global phase (every basis state is run through both), and
random circuits keep their state. No GPU."""
import math
from collections import Counter

import numpy as np
import pytest

import zxh_adae_b200 as zx
from oracle import observables as ob
from zxh_adae_b200 import workloads as wl
from zxh_adae_b200._core import plan_stats
from zxh_adae_b200.loader import compile_circuit, frontend_records

C = zx._core


def kinds(recs):
    return [int(r["type"]) for r in recs]


def unitary(n, recs):
    """Columns = the oracle's state (qubit q at bit q) for every basis input."""
    cols = []
    for k in range(1 << n):
        prep = [(C.X, 0, q) for q in range(n) if (k >> q) & 1]
        cols.append(ob.oracle_state(n, zx.as_records(prep + rec_tuples(recs))))
    return np.array(cols).T


def rec_tuples(recs):
    return [(int(r["type"]), int(r["cq"]), int(r["q"]), float(r["theta"]), float(r["lam"]), float(r["phi"]))
            for r in zx.as_records(recs)]


def equiv_up_to_phase(a, b, tol=1e-9):
    k = np.unravel_index(np.argmax(np.abs(a)), a.shape)
    ph = b[k] / a[k]
    ph /= abs(ph)
    return float(np.max(np.abs(b - ph * a))) <= tol


def opt_equiv(n, recs, level=2):
    out = zx.optimize_records(n, recs, level)
    assert equiv_up_to_phase(unitary(n, rec_tuples(recs)), unitary(n, rec_tuples(out)))
    return out


class _Op:
    def __init__(self, name, params=()):
        self.name, self.params = name, list(params)


class _Inst:
    def __init__(self, name, qubits, params=()):
        self.operation, self.qubits = _Op(name, params), qubits


class _Bit:
    def __init__(self, i):
        self.index = i


class _Circuit:
    """The slice of Qiskit's QuantumCircuit the compiler uses."""

    def __init__(self, insts):
        self.data = insts

    def find_bit(self, q):
        return _Bit(q)


def compiled(insts, n, level=2):
    segs = compile_circuit(_Circuit(insts), n, level)
    assert len(segs) == 1 and not segs[0][1]
    return segs[0][0]


def test_hh_cx_crossing_preserves_equivalence():
    g = [(C.H, 0, 0), (C.H, 0, 1), (C.CX, 0, 1), (C.H, 0, 0), (C.H, 0, 1)]
    out = opt_equiv(2, g)
    assert kinds(out) == [C.CX] and (int(out[0]["cq"]), int(out[0]["q"])) == (1, 0)


def test_optimizer_reduces_required_state_bits_when_h_pairs_cancel():
    g = zx.as_records([(C.H, 0, 0), (C.H, 0, 1), (C.CX, 0, 1), (C.H, 0, 0), (C.H, 0, 1)])
    assert plan_stats(2, zx.optimize_records(2, g, 0))["M"] == 2
    assert plan_stats(2, zx.optimize_records(2, g, 2))["M"] == 0


def test_zeroh_is_flushed_locally_at_cx_boundary():
    g = [(C.RZ, 0, 0, 0.3), (C.X, 0, 0), (C.RZ, 0, 1, -0.4), (C.CX, 0, 1)]
    out = opt_equiv(2, g)
    assert C.CP not in kinds(out)


def test_nonexact_oneh_is_flushed_locally_at_cx_boundary():
    g = [(C.RZ, 0, 1, 0.25), (C.H, 0, 1), (C.CX, 0, 1)]
    out = opt_equiv(2, g)
    assert kinds(out) == [C.U3, C.CX]


def test_double_exact_h_rule_preserves_equivalence():
    out = opt_equiv(2, [(C.H, 0, 0), (C.H, 0, 1), (C.CX, 0, 1)])
    assert kinds(out) == [C.CX, C.H, C.H] and (int(out[0]["cq"]), int(out[0]["q"])) == (1, 0)


def test_standalone_z_is_serialized_as_rz():
    assert kinds(opt_equiv(1, [(C.Z, 0, 0)])) == [C.RZ]


@pytest.mark.parametrize("name,qubits,params,expect", [
    ("swap", [0, 1], (), [C.CX, C.CX, C.CX]),
    ("cz", [0, 1], (), [C.CP]),
    ("rzz", [0, 1], (0.375,), [C.CX, C.RZ, C.CX]),
])
def test_two_qubit_frontend_gates_lower_inside_the_compiler(name, qubits, params, expect):
    out = compiled([_Inst(name, qubits, params)], 2)
    assert kinds(out) == expect
    want = {"swap": np.eye(4)[[0, 2, 1, 3]], "cz": np.diag([1, 1, 1, -1]),
            "rzz": np.diag(np.exp(-0.5j * 0.375 * np.array([1, -1, -1, 1])))}[name]
    assert equiv_up_to_phase(want.astype(complex), unitary(2, rec_tuples(out)))


def _ccz_matrix():
    return np.diag([1, 1, 1, 1, 1, 1, 1, -1]).astype(complex)


def test_ccz_is_lowered_to_cx_plus_rz_inside_the_compiler():
    out = compiled([_Inst("ccz", [0, 1, 2])], 3)
    counts = Counter(kinds(out))
    assert set(counts) == {C.CX, C.RZ} and counts[C.CX] == 6 and counts[C.RZ] == 7
    assert equiv_up_to_phase(_ccz_matrix(), unitary(3, rec_tuples(out)))


def test_ccx_is_lowered_to_h_cx_rz_inside_the_compiler():
    out = compiled([_Inst("ccx", [0, 1, 2])], 3)
    names = kinds(out)
    assert names.count(C.CX) == 6 and set(names) <= {C.H, C.U3, C.CX, C.RZ}
    ccx = np.eye(8, dtype=complex)[[0, 1, 2, 7, 4, 5, 6, 3]]  # flips qubit 2 where qubits 0 and 1 are set
    assert equiv_up_to_phase(ccx, unitary(3, rec_tuples(out)))


@pytest.mark.parametrize("name,params,mat", [
    ("ry", (0.7,), lambda t: np.array([[math.cos(t / 2), -math.sin(t / 2)], [math.sin(t / 2), math.cos(t / 2)]])),
    ("u1", (0.4,), lambda t: np.diag([1, np.exp(1j * t)])),
    ("s", (), lambda: np.diag([1, 1j])),
    ("sdg", (), lambda: np.diag([1, -1j])),
    ("t", (), lambda: np.diag([1, np.exp(0.25j * math.pi)])),
    ("tdg", (), lambda: np.diag([1, np.exp(-0.25j * math.pi)])),
    ("u2", (0.3, -1.1), lambda p, l: np.array([[1, -np.exp(1j * l)], [np.exp(1j * p), np.exp(1j * (p + l))]]) / math.sqrt(2)),
])
def test_single_qubit_frontend_gates(name, params, mat):
    for level in (0, 2):
        out = compiled([_Inst(name, [0], params)], 1, level)
        assert equiv_up_to_phase(np.asarray(mat(*params), complex), unitary(1, rec_tuples(out)))


def test_measure_and_reset_split_segments_and_unknown_gates_raise():
    insts = [_Inst("h", [0]), _Inst("measure", [0]), _Inst("h", [0]), _Inst("reset", [0]), _Inst("x", [1])]
    segs = compile_circuit(_Circuit(insts), 2, 2)
    assert [(kinds(r), reset) for r, reset in segs] == [([C.H], False), ([C.H], False), ([C.X], True)]
    with pytest.raises(NotImplementedError):
        compile_circuit(_Circuit([_Inst("cswap", [0, 1, 2])]), 3)
    with pytest.raises(ValueError):
        zx.optimize_records(2, [(C.CX, 1, 1)])
    with pytest.raises(ValueError):
        zx.optimize_records(2, [(C.H, 0, 2)])


def _random_frontend(n, count, seed):
    rng = np.random.default_rng(seed)
    insts = []
    one = ["h", "x", "z", "rz", "rx", "ry", "p", "s", "t", "u", "sdg"]
    for _ in range(count):
        r = rng.random()
        if r < 0.55:
            name = one[int(rng.integers(len(one)))]
            nparam = {"rz": 1, "rx": 1, "ry": 1, "p": 1, "u": 3}.get(name, 0)
            insts.append(_Inst(name, [int(rng.integers(n))], rng.uniform(-math.pi, math.pi, nparam)))
        elif r < 0.85:
            a, b = (int(v) for v in rng.choice(n, 2, replace=False))
            name = ["cx", "cx", "cp", "crz", "cz", "swap", "rzz"][int(rng.integers(7))]
            insts.append(_Inst(name, [a, b], rng.uniform(-math.pi, math.pi, 1) if name in ("cp", "crz", "rzz") else ()))
        elif r < 0.95 and n >= 3:
            a, b, c = (int(v) for v in rng.choice(n, 3, replace=False))
            insts.append(_Inst(["ccx", "ccz"][int(rng.integers(2))], [a, b, c]))
        else:
            insts.append(_Inst("barrier", list(range(n))))
    return insts


@pytest.mark.parametrize("seed", range(12))
def test_random_circuits_keep_their_state(seed):
    n = 2 + seed % 6
    insts = _random_frontend(n, 60, 4000 + seed)
    base = compiled(insts, n, 0)
    for level in (1, 2):
        out = compiled(insts, n, level)
        a, b = ob.oracle_state(n, base), ob.oracle_state(n, out)
        assert equiv_up_to_phase(a, b, 1e-9)
        assert plan_stats(n, out)["M"] <= plan_stats(n, base)["M"]


@pytest.mark.parametrize("seed", range(4))
def test_h_sandwiched_cx_chains_shrink_the_state(seed):
    # H on all, CX chains between H layers: the crossings leave the CX's reversed
    # and cancel the H pairs, so fewer state bits and passes are needed
    n = 8
    rng = np.random.default_rng(seed)
    recs = []
    for _ in range(3):
        recs += [(C.H, 0, q) for q in range(n)]
        for _ in range(6):
            a, b = (int(v) for v in rng.choice(n, 2, replace=False))
            recs.append((C.CX, a, b))
        recs += [(C.H, 0, q) for q in range(n)]
    out = opt_equiv(n, recs) if n <= 6 else zx.optimize_records(n, recs, 2)
    assert equiv_up_to_phase(ob.oracle_state(n, zx.as_records(recs)), ob.oracle_state(n, out))
    assert kinds(out).count(C.H) == 0
    assert plan_stats(n, out)["M"] == 0 < plan_stats(n, zx.as_records(recs))["M"]


def test_compiled_hidden_string_circuit_matches():
    g, _secret = wl.hidden_string(11, seed=5)
    n = 12
    out = zx.optimize_records(n, g, 2)
    assert equiv_up_to_phase(ob.oracle_state(n, zx.as_records(g)), ob.oracle_state(n, out))
    assert plan_stats(n, out)["M"] <= plan_stats(n, zx.as_records(g))["M"]
