"""CPU tests of the host logic: the execute() walk and pass planner (dry run
through the C ABI, no GPU), calc_mem parity with the oracle, the Python loader,
and the multi-process replica plumbing of bench.py over gloo."""
import math
import os
import socket
import subprocess
import sys
import textwrap
from pathlib import Path

import numpy as np
import pytest

import zxh_adae_b200 as zx
from oracle.bridge import Oracle
from zxh_adae_b200 import workloads as wl
from zxh_adae_b200._core import plan_stats

ROOT = Path(__file__).resolve().parent.parent


def test_diag_batch_is_one_pass():
    st = plan_stats(30, np.concatenate([wl.h_all(30), wl.diag_batch(30, 4096, 1)]))
    assert st["M"] == 30 and st["product"] == 1 and st["passes"] == 1 and st["diagonal"] == 1


def test_window_after_cx_chain_is_one_walsh_pass():
    # after CX(i, i+1) on every i the selectors are prefix parities of the real
    # bits: the whole 4096-gate window is one Walsh-sum pass, not 128 split passes
    g = np.concatenate([wl.h_all(30), wl.cx_chain(30), wl.diag_batch(30, 4096, 1)])
    for dtype in ("complex64", "complex128"):
        st = plan_stats(30, g, dtype=dtype)
        assert st["walsh"] == 1 and st["passes"] == 1 and st["diagonal"] == 0, st
    # a window of single-bit selectors keeps the diagonal pass
    st = plan_stats(30, np.concatenate([wl.h_all(30), wl.diag_batch(30, 4096, 1)]))
    assert st["walsh"] == 0 and st["diagonal"] == 1


def test_u3_layer_splits_into_low_and_strided_passes():
    rng = np.random.default_rng(0)
    lay = zx.as_records([(zx._core.U3, 0, q, *rng.uniform(0, 6.28, 3)) for q in range(30)])
    # complex64: span passes, 13 gates on bits 0..12 and the 17 high-bit gates in
    # two strided passes (9 + 8, runs of 16 and 32 amplitudes); complex128: 12 gates
    # on bits 0..11 and two strided passes of 9 (runs of 8 amplitudes, 128 B)
    st = plan_stats(30, np.concatenate([wl.h_all(30), lay]), dtype="complex64")
    assert st["span"] == 3 and st["row"] == 0 and st["passes"] == 3
    st = plan_stats(30, np.concatenate([wl.h_all(30), lay]), dtype="complex128")
    assert st["span"] == 3 and st["row"] == 0 and st["passes"] == 3
    # 32 qubits: 13 + 10 + 9 (at most 10 high-bit gates per pass: runs of at
    # least 8 amplitudes)
    st = plan_stats(32, np.concatenate([wl.h_all(32), wl.u3_layer(32, 3)]))
    assert st["span"] == 3 and st["passes"] == 3


def test_small_windows_fuse_into_u3_passes():
    st = plan_stats(20, wl.plain_layers(20, 10, 1))
    assert st["diagonal"] == 0 and st["passes"] == 20  # 10 layers x (1 strided + 1 low span pass), cp chains fused
    st = plan_stats(20, wl.plain_layers(20, 10, 1), dtype="complex128")
    assert st["diagonal"] == 0 and st["passes"] == 20  # 10 layers x (1 strided + 1 low span pass)
    st = plan_stats(32, wl.u3_matching_layers(32, 4, 33))
    assert st["diagonal"] == 0 and st["passes"] == 12  # 3 span passes per layer, cz matchings fused


def test_prefix_of_first_touch_gates_is_one_product_pass():
    st = plan_stats(24, wl.h_all(24))
    assert st == {**st, "M": 24, "m": 24, "passes": 0, "product": 1}


def test_eager_expand_all_and_disable_x_plans():
    g = zx.as_records([(zx._core.H, 0, 0), (zx._core.CX, 0, 1), (zx._core.X, 0, 2), (zx._core.CX, 1, 2)])
    st = plan_stats(3, g, disable_x=True, eager_expand_all=True)
    assert st["M"] == 3
    st = plan_stats(3, g, disable_x=True)
    assert st["M"] == 3  # X/CX count as expansions under disable_x (calc_mem, zxh.cpp:655-663)


@pytest.mark.parametrize("seed", range(30))
def test_calc_mem_matches_oracle(seed):
    n = 2 + seed % 12
    g = wl.random_circuit(n, 80, 700 + seed)
    o = Oracle(n)
    o.push(g)
    assert plan_stats(n, g)["M"] == o.required_M()


def test_plan_rejects_bad_records():
    with pytest.raises(ValueError):
        plan_stats(3, zx.as_records([(zx._core.H, 0, 3)]))
    with pytest.raises(ValueError):
        plan_stats(3, zx.as_records([(99, 0, 0)]))
    with pytest.raises(ValueError):
        plan_stats(64, wl.h_all(2))


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
    """The slice of Qiskit's QuantumCircuit the loader uses."""

    def __init__(self, insts):
        self.data = insts

    def find_bit(self, q):
        return _Bit(q)


class _Recorder:
    def __init__(self):
        self.recs = []
        self.cleared = 0

    def push_gates(self, rec):
        self.recs.extend(rec.tolist())

    def clear_gates(self):
        self.cleared += 1


def test_loader_lowering_matches_reference_loader():
    # u/u3 parameters reorder (theta, phi, lambda) -> (theta, lambda, phi) as
    # qasm.py:114-121 does; measure/id are skipped; reset clears the gate list
    c = _Circuit([_Inst("h", [0]), _Inst("u", [1], (0.1, 0.2, 0.3)), _Inst("cp", [0, 1], (0.5,)),
                  _Inst("measure", [0]), _Inst("id", [1]), _Inst("crz", [1, 0], (0.7,)), _Inst("barrier", [0, 1]),
                  _Inst("rx", [0], (0.9,)), _Inst("reset", [0]), _Inst("x", [1])])
    r = _Recorder()
    zx.load_circuit_transpiled(r, c)
    kinds = [row[0] for row in r.recs]
    assert kinds == [zx._core.H, zx._core.U3, zx._core.CP, zx._core.CRZ, zx._core.BARRIER, zx._core.RX, zx._core.X]
    u = r.recs[1]
    assert u[2] == 1 and (u[4], u[5], u[6]) == (0.1, 0.3, 0.2)
    assert r.cleared == 1
    with pytest.raises(NotImplementedError):
        zx.load_circuit_transpiled(r, _Circuit([_Inst("swap", [0, 1])]))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_bench_replica_reduction_over_gloo():
    # two CPU ranks run bench.py's barrier and max-over-ranks helpers on gloo
    code = textwrap.dedent(
        f"""
        import os, sys
        sys.path.insert(0, {str(ROOT)!r})
        import torch.distributed as dist
        import bench
        dist.init_process_group("gloo", init_method="tcp://127.0.0.1:{_free_port()}",
                                rank=int(sys.argv[1]), world_size=2)
        bench.barrier(dist)
        v = bench.max_over_ranks(dist, 1.0 + int(sys.argv[1]), -1)
        assert v == 2.0, v
        bench.barrier(dist)
        dist.destroy_process_group()
        print("ok", sys.argv[1])
        """
    )
    procs = [subprocess.Popen([sys.executable, "-c", code, str(r)], stdout=subprocess.PIPE, stderr=subprocess.PIPE)
             for r in range(2)]
    outs = [p.communicate(timeout=120) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e.decode()[-2000:]
        assert b"ok" in o
