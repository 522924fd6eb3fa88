"""Pins against ZXH-Sim's own GPU path: the unmodified reference CUDA backend,
compiled from its sources by oracle/Makefile (oracle/_ref/libzxhref_cuda.so),
run on the same GPU.

* the oracle's restatement of the reference GPU sampler draws exactly the
  reference GPU sampler's outcomes (same seed, same order);
* this library's amplitudes match the reference GPU path within 1e-12
  (complex128), and its samples equal the reference GPU samples.
"""
import numpy as np
import pytest

import zxh_adae_b200 as zx
from oracle.bridge import Oracle, Reference, ref_available
from zxh_adae_b200 import workloads as wl

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not ref_available("cuda"), reason="reference CUDA backend not built (oracle/_ref)"),
]

CASES = [
    ("plain12", 12, lambda: wl.plain_layers(12, 3, seed=1)),
    ("plain16", 16, lambda: wl.plain_layers(16, 2, seed=2)),
    ("random10", 10, lambda: wl.random_circuit(10, 120, seed=3)),
    ("diag14", 14, lambda: np.concatenate([wl.h_all(14), wl.diag_batch(14, 300, 4), wl.cp_cascade(14)])),
    ("hidden11", 12, lambda: wl.hidden_string(11, seed=5)[0]),
]


@pytest.mark.parametrize("name,n,make", CASES, ids=[c[0] for c in CASES])
def test_state_matches_reference_gpu(name, n, make):
    gates = make()
    r = Reference(n, backend="cuda")
    r.push(gates)
    r.execute()
    want = r.get_state()
    s = zx.ZXH(n, dtype="complex128")
    s.push_gates(gates)
    s.execute()
    assert np.max(np.abs(s.get_state() - want)) <= 1e-12
    s64 = zx.ZXH(n, dtype="complex64")
    s64.push_gates(gates)
    s64.execute()
    assert np.max(np.abs(s64.get_state().astype(np.complex128) - want)) <= 1e-6


@pytest.mark.parametrize("name,n,make", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("shots", [1, 1024, 30000])
def test_samples_match_reference_gpu(name, n, make, shots):
    gates = make()
    seed = 1000 + shots
    r = Reference(n, backend="cuda")
    r.push(gates)
    r.execute()
    want = r.sample(seed, shots)[:, 0]
    o = Oracle(n)
    o.push(gates)
    o.execute()
    assert np.array_equal(o.sample(seed, shots)[0][:, 0], want)
    s = zx.ZXH(n, dtype="complex128")
    s.push_gates(gates)
    s.execute()
    s.set_seed(seed)
    s.measure(shots)
    assert np.array_equal(s.results_words(), want)
