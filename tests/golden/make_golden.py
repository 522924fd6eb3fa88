"""Generates the golden fixtures of this directory from the reference itself.

* states.npz    -- get_state() of the unmodified reference ZXH-Sim serial CPU
                   backend (oracle/_ref/libzxhref_single.so, compiled from the
                   reference's own sources by oracle/Makefile) for the circuits of
                   the reference's unit tests (src/zxh/tests/unit/test_measure_api.py)
                   and integration cases (src/zxh/tests/integration/cases/*.qasm),
                   written here as gate lists, plus seeded synthetic circuits.
* ref_gpu_samples.npz -- measure()/get_results() of the reference CUDA backend
                   (oracle/_ref/libzxhref_cuda.so) on a B200: packed outcome words
                   for fixed seeds. Needs a GPU: `python tests/golden/make_golden.py
                   --gpu-samples OUT.npz`.

Run from the repository root: `python tests/golden/make_golden.py`.
"""
from __future__ import annotations

import argparse
import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.bridge import GATE_DTYPE, Reference, as_records  # noqa: E402

BARRIER, Z, RZ, P, CRZ, CP, X, CX, H, U3, RX = 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11


def qiskit_u(q, theta, phi, lam):
    """Qiskit u(theta, phi, lambda) as a ZXH U3 record (theta, lambda, phi)."""
    return (U3, 0, q, theta, lam, phi)


def unit_cases():
    """Circuits of the reference's test_measure_api.py (n, flags, gates)."""
    return {
        "asym_basis_x0": (2, (False, False), [(X, 0, 0)]),
        "rz_pi": (1, (False, False), [(RZ, 0, 0, math.pi)]),
        "general_u": (2, (False, False), [qiskit_u(0, 0.3, 0.4, 0.5)]),
        "disable_x": (3, (True, False), [(H, 0, 0), (CX, 0, 1), (X, 0, 2), (CX, 1, 2), qiskit_u(1, 0.2, 0.4, 0.1)]),
        "eager_expand_all": (3, (False, True), [(H, 0, 0), (CP, 0, 1, 0.3), (CX, 1, 2), (RZ, 0, 2, 0.4)]),
        "disable_x_and_eager": (3, (True, True), [(H, 0, 0), (CX, 0, 1), (X, 0, 2), (CX, 1, 2), (H, 0, 2)]),
        "affine_111": (3, (False, False), [(X, 0, 0), (CX, 0, 1), (CX, 1, 2)]),
        "bell": (2, (False, False), [(H, 0, 0), (CX, 0, 1)]),
        "u3_cluster_00": (2, (False, False), [(H, 0, 0), (H, 0, 1), (X, 0, 0), (H, 0, 0), (H, 0, 1)]),
        "seed_repro": (3, (False, False), [(H, 0, 0), (CP, 0, 1, 0.37), (H, 0, 1), (CX, 1, 2)]),
        "crz_interference": (2, (False, False), [(X, 0, 0), (H, 0, 1), (CRZ, 0, 1, 0.6), (H, 0, 1)]),
        # integration cases (tests/integration/cases)
        "x_1_delta": (1, (False, False), [(X, 0, 0)]),
        "h_1_balanced": (1, (False, False), [(H, 0, 0)]),
        "bell_2_support": (2, (False, False), [(H, 0, 0), (CX, 0, 1)]),
        "u3_1_balanced": (1, (False, False), [qiskit_u(0, math.pi / 2, 0.0, 0.0)]),
        "h_11_delta": (11, (False, False), [(H, 0, q) for q in range(11)] * 2),
    }


def synthetic_cases():
    from zxh_adae_b200 import workloads as wl

    cases = {
        "plain_12q_3layers": (12, (False, False), wl.plain_layers(12, 3, seed=7)),
        "diag_10q": (10, (False, False), np.concatenate([wl.h_all(10), wl.diag_batch(10, 200, 3), wl.cp_cascade(10)])),
        "hidden_string_9": (10, (False, False), wl.hidden_string(9, seed=2)[0]),
    }
    for k in range(6):
        n = 3 + k
        cases[f"random_{n}q_{k}"] = (n, (False, False), wl.random_circuit(n, 60, seed=500 + k))
    return cases


def all_cases():
    c = unit_cases()
    c.update(synthetic_cases())
    return c


def pack(cases):
    out = {}
    for name, (n, (dx, ea), gates) in cases.items():
        rec = as_records(gates)
        r = Reference(n, dx, ea, backend="single")
        r.push(rec)
        r.execute()
        out[f"{name}__gates"] = rec.view(np.uint8)
        out[f"{name}__meta"] = np.array([n, int(dx), int(ea), r.required_M()], np.int64)
        out[f"{name}__state"] = r.get_state()
    return out


SAMPLE_CASES = [("bell", 4096, 20260407), ("seed_repro", 256, 31415926), ("crz_interference", 4096, 20260408),
                ("plain_12q_3layers", 1024, 7), ("hidden_string_9", 3000, 11), ("diag_10q", 20000, 5)]


def gpu_samples(path: Path):
    cases = all_cases()
    out = {}
    for name, shots, seed in SAMPLE_CASES:
        n, (dx, ea), gates = cases[name]
        r = Reference(n, dx, ea, backend="cuda")
        r.push(as_records(gates))
        r.execute()
        out[f"{name}__words"] = r.sample(seed, shots)[:, 0]
        out[f"{name}__seed"] = np.array([seed, shots], np.uint64)
    np.savez_compressed(path, **out)


def load_states(path: Path | None = None):
    """{name: (n, disable_x, eager, M, records, state)} from states.npz."""
    z = np.load(path or Path(__file__).with_name("states.npz"))
    names = sorted({k.split("__")[0] for k in z.files})
    res = {}
    for nm in names:
        meta = z[f"{nm}__meta"]
        rec = z[f"{nm}__gates"].view(GATE_DTYPE)
        res[nm] = (int(meta[0]), bool(meta[1]), bool(meta[2]), int(meta[3]), rec, z[f"{nm}__state"])
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpu-samples", type=Path, default=None)
    a = ap.parse_args()
    if a.gpu_samples:
        gpu_samples(a.gpu_samples)
        return
    np.savez_compressed(Path(__file__).with_name("states.npz"), **pack(all_cases()))


if __name__ == "__main__":
    main()
