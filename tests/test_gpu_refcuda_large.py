"""Parity with ZXH-Sim's own GPU path at the benchmark sizes.

The unmodified reference CUDA backend (oracle/_ref/libzxhref_cuda.so, compiled
from its sources) and this library run the same gate lists on the same GPU; the
two real-address states are compared on the device (oracle/devstate.py), with
the global phases applied, in FP64:

* max |amp - reference| <= 1e-12 for complex128 and <= 1e-6 for complex64,
* the live real-address bits (the state's size after lazy expansion) equal,
* the fidelity error 1 - |<ours|ref>|^2 is reported (ZXH_PARITY_LOG=<file>
  appends one JSON line per case).

Shapes: configuration 2's diagonal batches (H on all, then B random p/cp with
B in {64, 256, 1024, 4096}) and the full controlled-phase cascade at 28 qubits,
a 4096-gate window after a CX chain (multi-bit selectors) at 26 qubits,
configuration 3's U3 + cz matching layers at 26 qubits and its hidden-string
circuit at 26+1 qubits, configuration 4's ansatz forward state at 24 qubits and
configuration 1 at 20 qubits. A 16-qubit case also goes through get_state in
the reference's output order, which pins the real-address comparison itself.
"""
import json
import math
import os

import numpy as np
import pytest

import zxh_adae_b200 as zx
from oracle import devstate
from oracle.bridge import Reference, ref_available
from zxh_adae_b200 import adjoint as ad
from zxh_adae_b200 import workloads as wl

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not ref_available("cuda"), reason="reference CUDA backend not built (oracle/_ref)"),
]

TOL = {"complex128": 1e-12, "complex64": 1e-6}


def _ansatz24():
    circ = ad.hardware_efficient_ansatz(24, 8)
    p = np.random.default_rng(2024).uniform(-math.pi, math.pi, circ.nparams)
    return circ.records(p)


CASES = [
    ("config2_B64_28q", 28, lambda: np.concatenate([wl.h_all(28), wl.diag_batch(28, 64, 11)])),
    ("config2_B256_28q", 28, lambda: np.concatenate([wl.h_all(28), wl.diag_batch(28, 256, 12)])),
    ("config2_B1024_28q", 28, lambda: np.concatenate([wl.h_all(28), wl.diag_batch(28, 1024, 13)])),
    ("config2_B4096_28q", 28, lambda: np.concatenate([wl.h_all(28), wl.diag_batch(28, 4096, 14)])),
    ("config2_cascade_28q", 28, lambda: np.concatenate([wl.h_all(28), wl.cp_cascade(28)])),
    # after a CX chain every selector is a prefix parity of the real bits: the
    # window is one Walsh-sum pass here, single-gate sweeps in the reference
    ("cxchain_B4096_26q", 26, lambda: np.concatenate([wl.h_all(26), wl.cx_chain(26), wl.diag_batch(26, 4096, 15)])),
    ("config3_u3cz4_26q", 26, lambda: wl.u3_matching_layers(26, 4, 33)),
    ("config3_hidden_27q", 27, lambda: wl.hidden_string(26, 34)[0]),
    ("config4_ansatz_24q", 24, _ansatz24),
    ("config1_20q", 20, lambda: wl.plain_layers(20, 10, 2024)),
]


def _log(rec: dict) -> None:
    path = os.environ.get("ZXH_PARITY_LOG")
    if path:
        with open(path, "a") as fh:
            fh.write(json.dumps(rec) + "\n")


def _reference(n, gates):
    r = Reference(n, backend="cuda")
    r.push(gates)
    r.execute()
    found = r.device_state()
    assert found is not None, "reference state probe failed its layout checks"
    return r, found


@pytest.mark.parametrize("name,n,make", CASES, ids=[c[0] for c in CASES])
def test_state_matches_reference_gpu_at_benchmark_sizes(name, n, make):
    gates = make()
    r, (rptr, rm, rphase) = _reference(n, gates)
    ref = devstate.device_view(rptr, rm, 16)
    for dtype in ("complex128", "complex64"):
        s = zx.ZXH(n, dtype=dtype)
        s.push_gates(gates)
        s.execute()
        ptr, m, eb, phase = s.state_view()
        assert m == rm, f"{name} {dtype}: live bits {m} vs the reference's {rm}"
        c = devstate.compare(devstate.device_view(ptr, m, eb), phase, ref, rphase)
        _log({"case": name, "qubits": n, "dtype": dtype, "gates": int(len(gates)), **c})
        assert c["max_abs"] <= TOL[dtype], f"{name} {dtype}: {c}"
        assert c["fidelity_err"] <= (1e-12 if dtype == "complex128" else 1e-9), f"{name} {dtype}: {c}"
        s.close()
    del r


def test_real_address_comparison_agrees_with_get_state():
    n = 16
    gates = np.concatenate([wl.plain_layers(n, 2, seed=8), wl.diag_batch(n, 500, 9)])
    r, (rptr, rm, rphase) = _reference(n, gates)
    want = r.get_state()
    s = zx.ZXH(n, dtype="complex128")
    s.push_gates(gates)
    s.execute()
    assert np.max(np.abs(s.get_state() - want)) <= 1e-12
    ptr, m, eb, phase = s.state_view()
    c = devstate.compare(devstate.device_view(ptr, m, eb), phase, devstate.device_view(rptr, rm, 16), rphase)
    assert m == rm and c["max_abs"] <= 1e-12
    assert abs(c["norm_b"] - 1.0) < 1e-12  # the probe found the whole (normalised) reference state
