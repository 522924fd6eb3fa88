"""Phases carried from one apply to the next.

After its last U3 batch an apply leaves the real split's P(b) phases and global
phase pending; the next apply takes them into its first window, and every call
that reads the state (get_state, state_view, measure, expectation) or flush()
applies them first. These tests compare layer-by-layer applies, with reads and
other gate kinds between them, against the oracle run of the whole gate list.
Tolerances as in test_gpu_parity.py.
"""
import numpy as np
import pytest

import zxh_adae_b200 as zx
from oracle.bridge import Oracle
from oracle.observables import energy_dense
from zxh_adae_b200 import workloads as wl

pytestmark = pytest.mark.gpu
TOL = {"complex128": 1e-12, "complex64": 1e-6}
DTYPES = ["complex128", "complex64"]


def oracle_state(n, parts):
    o = Oracle(n)
    o.push(np.concatenate(parts))
    o.execute()
    return o


def err(s, o):
    return float(np.max(np.abs(s.get_state(0).astype(np.complex128) - o.get_state(0))))


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("n", [14, 17])
def test_u3_layers_applied_one_by_one(dtype, n):
    head = wl.h_all(n)
    layers = [wl.u3_layer(n, seed=70 + k) for k in range(4)]
    s = zx.ZXH(n, dtype=dtype)
    s.push_gates(head)
    s.execute()
    for k, layer in enumerate(layers):
        s.apply(layer)
        if k == 1:  # a read in between applies the carried phases; the next apply carries again
            assert err(s, oracle_state(n, [head] + layers[:2])) <= TOL[dtype]
    assert err(s, oracle_state(n, [head] + layers)) <= TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
def test_carried_phases_meet_other_gate_kinds(dtype):
    # after a U3 layer: CX transport (the map changes, the carried phases are on
    # real bits), a diagonal batch (merged into its window), a U3 batch after CX
    # (a general strided pass takes the phases as its prologue), X gates
    n = 16
    rng = np.random.default_rng(5)
    head = wl.h_all(n)
    parts = [
        wl.u3_layer(n, seed=1),
        zx.as_records([(zx._core.CX, i, i + 1) for i in range(0, n - 1, 2)]),
        wl.u3_layer(n, seed=2),
        wl.diag_batch(n, 50, seed=3),
        wl.u3_layer(n, seed=4),
        zx.as_records([(zx._core.CX, i, i + 1) for i in range(n - 1)]),
        zx.as_records([(zx._core.U3, 0, q, *rng.uniform(0, 2 * np.pi, 3)) for q in range(0, n, 3)]),
        zx.as_records([(zx._core.X, 0, q) for q in range(0, n, 4)]),
        wl.u3_layer(n, seed=6),
    ]
    s = zx.ZXH(n, dtype=dtype)
    s.push_gates(head)
    s.execute()
    for p in parts:
        s.apply(p)
    assert err(s, oracle_state(n, [head] + parts)) <= TOL[dtype]


def test_measure_after_apply_draws_the_oracle_stream():
    n = 15
    head = wl.h_all(n)
    layers = [wl.u3_layer(n, seed=20 + k) for k in range(3)]
    s = zx.ZXH(n, dtype="complex128")
    s.push_gates(head)
    s.execute()
    for layer in layers:
        s.apply(layer)
    o = oracle_state(n, [head] + layers)
    want, _ = o.sample(123, 5000)
    s.set_seed(123)
    s.measure(5000)
    assert np.array_equal(s.results_words(), want[:, 0])


@pytest.mark.parametrize("dtype", DTYPES)
def test_apply_async_and_state_view_and_expectation(dtype):
    import torch

    n = 16
    head = wl.h_all(n)
    layers = [wl.u3_layer(n, seed=40 + k) for k in range(3)]
    s = zx.ZXH(n, dtype=dtype)
    s.push_gates(head)
    s.execute()
    for layer in layers:
        s.apply_async(layer)
    s.sync()
    assert err(s, oracle_state(n, [head] + layers)) <= TOL[dtype]

    # the raw view holds the state with its phases applied: the same real-address
    # array as one execute() of the whole list (same walk, same real layout)
    def view(sim):
        ptr, m, eb, g = sim.state_view()

        class _CAI:
            __cuda_array_interface__ = {"shape": (1 << m,), "typestr": "<c8" if dtype == "complex64" else "<c16",
                                        "data": (ptr, False), "version": 3}
        return (torch.as_tensor(_CAI(), device="cuda").to(torch.complex128) * complex(g)).cpu().numpy()

    s.apply(wl.u3_layer(n, seed=50))
    whole = zx.ZXH(n, dtype=dtype)
    whole.push_gates(np.concatenate([head] + layers + [wl.u3_layer(n, seed=50)]))
    whole.execute()
    assert float(np.max(np.abs(view(s) - view(whole)))) <= TOL[dtype]
    whole.close()
    # expectation of sum Z_i Z_{i+1} + sum X_i after one more layer (carried again)
    more = wl.u3_layer(n, seed=99)
    s.apply(more)
    terms = [(zx._core.TERM_ZZ, i, i + 1, 1.0) for i in range(n - 1)] + \
        [(zx._core.TERM_X, i, 0, 0.7) for i in range(n)]
    e = s.expectation(terms)
    ref = energy_dense(oracle_state(n, [head] + layers + [wl.u3_layer(n, seed=50), more]).get_state(0), n, terms)
    assert abs(e - ref) <= (1e-10 if dtype == "complex128" else 1e-4)


@pytest.mark.parametrize("dtype", DTYPES)
def test_flush_runs_one_pass_then_nothing(dtype):
    n = 16
    s = zx.ZXH(n, dtype=dtype)
    s.push_gates(wl.h_all(n))
    s.execute()
    s.apply(wl.u3_layer(n, seed=8))
    s.flush()
    assert s.last_stats()[1] == 1  # the carried phases: one diagonal pass
    s.flush()
    assert s.last_stats()[:2] == (0, 0)
    o = oracle_state(n, [wl.h_all(n), wl.u3_layer(n, seed=8)])
    assert err(s, o) <= TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
def test_carried_phases_across_plan_knobs(dtype):
    # the phases one apply leaves are taken by the next whatever pass kind it plans:
    # span passes, register-row passes (span = 0), passes without the real split
    # (nothing carried further), the register form of the span pass, general
    # strided passes after a CX chain
    n = 16
    head = wl.h_all(n)
    layers = [wl.u3_layer(n, seed=60 + k) for k in range(6)]
    chain = zx.as_records([(zx._core.CX, i, i + 1) for i in range(n - 1)])
    s = zx.ZXH(n, dtype=dtype)
    s.push_gates(head)
    s.execute()
    s.apply(layers[0])
    s.set_param("span", 0)
    s.apply(layers[1])
    s.set_param("real_split", 0)
    s.apply(layers[2])
    s.set_param("real_split", 1)
    s.set_param("span", 1)
    s.set_param("span_land", 0)
    s.apply(layers[3])
    s.set_param("span_land", 1)
    s.apply(layers[4])
    s.apply(np.concatenate([chain, layers[5]]))
    assert err(s, oracle_state(n, [head] + layers[:5] + [chain, layers[5]])) <= TOL[dtype]
