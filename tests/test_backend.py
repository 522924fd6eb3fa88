"""The zxh backend's host logic (zxh_adae_b200/backend.py) against a fake
simulator: the steps of the reference's ZXHQiskitBackend._run_circuit / run /
ZXHJob (src/zxh/zxhsim/qiskit_backend.py:150-330) in their order, option checks,
circuit coercion, the cached simulator, and the result shape. No GPU."""
import pytest

from zxh_adae_b200 import _core
from zxh_adae_b200 import backend as bk


class _Inst:
    def __init__(self, name, qubits, params=()):
        self.operation = type("Op", (), {"name": name, "params": list(params)})()
        self.qubits = list(qubits)


class _Bit:
    def __init__(self, i):
        self.index = i


class _Circuit:
    def __init__(self, n, insts):
        self.num_qubits = n
        self.data = insts

    def find_bit(self, q):
        return _Bit(q)


class _FakeSim:
    def __init__(self, n, log):
        self.n, self.log, self.recs = n, log, []

    def num_qubits(self):
        return self.n

    def set_seed(self, s):
        self.log.append(("set_seed", s))

    def clear_seed(self):
        self.log.append(("clear_seed",))

    def clear_gates(self):
        self.log.append(("clear_gates",))
        self.recs = []

    def push_gates(self, rec):
        self.recs.extend(rec.tolist())

    def execute(self):
        self.log.append(("execute", len(self.recs)))

    def sample_counts(self, shots):
        self.log.append(("sample_counts", shots))
        return {"0" * self.n: shots}


class _Backend(bk.Backend):
    def __init__(self, **kw):
        super().__init__(**kw)
        self.log, self.made = [], 0

    def _make_sim(self, n):
        self.made += 1
        return _FakeSim(n, self.log)


def _bell():
    return _Circuit(2, [_Inst("h", [0]), _Inst("cx", [0, 1]), _Inst("measure", [0]), _Inst("measure", [1])])


def test_run_path_order_and_result():
    b = _Backend()
    job = b.run(_bell(), shots=100, seed_simulator=7)
    assert job.status() == "DONE"
    assert b.log == [("set_seed", 7), ("clear_gates",), ("execute", 2), ("sample_counts", 100)]
    res = job.result()
    assert res.backend_name == "zxh" and res.success
    assert res.get_counts() == {"00": 100} and res.results[0].shots == 100 and res.results[0].seed == 7
    assert res.results[0].metadata["sample_time"] >= 0.0
    with pytest.raises(bk.JobError):
        job.submit()


def test_seed_none_clears_the_seed_and_defaults():
    b = _Backend()
    b.run([_bell(), _bell()])
    assert b.log.count(("clear_seed",)) == 2 and ("sample_counts", 1) in b.log  # default shots = 1
    assert b.made == 1  # one cached simulator
    assert isinstance(b.run([_bell(), _bell()]).result().get_counts(), list)


def test_width_mismatch_and_bad_inputs():
    b = _Backend()
    b.run(_bell())
    with pytest.raises(bk.JobError):
        b.run(_Circuit(3, [_Inst("h", [0])]))
    with pytest.raises(bk.JobError):
        b.run(_bell(), disable_x=True)
    with pytest.raises(bk.JobError):
        b.run(_bell(), eager_expand_all=False)
    with pytest.raises(TypeError):
        b.run("not a circuit")
    with pytest.raises(TypeError):
        b.run([_bell(), 3])
    with pytest.raises(bk.JobError):
        bk.Job(b, [], {}).result()


def test_native_set_and_frontend_gates_through_the_compiler():
    b = _Backend()
    swap = _Circuit(2, [_Inst("h", [0]), _Inst("swap", [0, 1])])
    with pytest.raises(NotImplementedError):  # the reference's run takes transpiled circuits only
        b.run(swap)
    b.run(swap, optimize_level=2)
    assert b.log[-2][0] == "execute" and b.log[-2][1] > 0
    assert "swap" not in b.operation_names and "swap" in b.frontend_operation_names
    assert set(b.operation_names) <= set(b.frontend_operation_names)


def test_reset_clears_recorded_gates():
    b = _Backend()
    c = _Circuit(1, [_Inst("h", [0]), _Inst("reset", [0]), _Inst("x", [0])])
    b.run(c)
    assert b.log.count(("clear_gates",)) == 2 and b.log[-2] == ("execute", 1)


def test_make_zxh_backend_exported():
    import zxh_adae_b200 as zx
    b = zx.make_zxh_backend(disable_x=True, dtype="complex64")
    assert isinstance(b, bk.Backend) and b.name == "zxh"
    assert b._build["disable_x"] and b._build["dtype"] == "complex64"
    assert _core.ZXH.clear_seed  # the seed path the backend prefers exists on the simulator
