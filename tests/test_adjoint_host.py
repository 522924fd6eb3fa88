"""CPU tests of the adjoint-gradient path's host side: the dense restatement of
the adjoint method against central differences and parameter shifts of oracle
energies, the circuit/parameter bookkeeping of zxh_adae_b200.adjoint, and the
forward plan of the 24-qubit ansatz (dry run, no GPU)."""
import math

import numpy as np
import pytest

from oracle import observables as ob
from zxh_adae_b200 import _core
from zxh_adae_b200 import adjoint as ad
from zxh_adae_b200._core import plan_stats


def mixed_circuit(n, seed):
    """Every gate kind of the library, with parameters on RY, RX, RZ, P, CP, CRz."""
    rng = np.random.default_rng(seed)
    rec, par = [], []
    k = 0
    for layer in range(3):
        for q in range(n):
            kind = rng.integers(6)
            if kind == 0:
                rec.append((_core.U3, 0, q, 0.0, 0.0, 0.0))  # RY
            elif kind == 1:
                rec.append((_core.RX, 0, q, 0.0))
            elif kind == 2:
                rec.append((_core.RZ, 0, q, 0.0))
            elif kind == 3:
                rec.append((_core.P, 0, q, 0.0))
            elif kind == 4:
                rec.append((_core.H, 0, q))
                par.append(-1)
                rec.append((_core.U3, 0, q, 0.0, 0.0, 0.0))
            else:
                rec.append((_core.U3, 0, q, 0.0, 0.0, 0.0))
            par.append(k)
            k += 1
        a, b = rng.choice(n, 2, replace=False)
        rec += [(_core.CX, int(a), int(b)), (_core.X, 0, int(rng.integers(n))), (_core.Z, 0, int(rng.integers(n)))]
        par += [-1, -1, -1]
        a, b = rng.choice(n, 2, replace=False)
        rec.append((_core.CP, int(a), int(b), 0.0))
        par.append(k)
        k += 1
        a, b = rng.choice(n, 2, replace=False)
        rec.append((_core.CRZ, int(a), int(b), 0.0))
        par.append(k)
        k += 1
        rec.append((_core.U3, 0, int(rng.integers(n)), 0.3, 0.2, 0.1))  # fixed general U3
        par.append(-1)
    return ad.Circuit(n, rec, par)


def random_terms(n, seed):
    rng = np.random.default_rng(seed)
    rows = []
    for _ in range(2 * n):
        k = int(rng.integers(1, 4))
        a, b = rng.choice(n, 2, replace=False)
        rows.append((k, int(a), int(b), float(rng.normal())))
    return _core.as_terms(rows)


@pytest.mark.parametrize("seed", range(3))
def test_dense_adjoint_matches_oracle_differences(seed):
    n = 4
    circ = mixed_circuit(n, seed) if seed else ad.hardware_efficient_ansatz(n, 2)
    terms = random_terms(n, seed) if seed else ad.tfim_terms(n)
    p = np.random.default_rng(seed).uniform(-math.pi, math.pi, circ.nparams)
    e, g = ob.dense_adjoint(n, circ.records(p), terms)
    assert abs(e - ob.oracle_energy(n, circ.records(p), terms)) < 1e-12
    grad = circ.gradient(g)
    assert np.max(np.abs(grad - ob.oracle_central_difference(n, circ, p, terms))) < 1e-7
    if np.all(circ.coef == 1.0):
        assert np.max(np.abs(grad - ob.oracle_parameter_shift(n, circ, p, terms))) < 1e-12


def test_crz_and_rx_lowering_in_circuit():
    c = ad.Circuit(2, [(_core.CRZ, 0, 1, 0.0), (_core.RX, 0, 1, 0.0), (_core.H, 0, 0)], [0, 1, -1])
    rec = c.records([0.8, 0.4])
    assert list(rec["type"]) == [_core.P, _core.CP, _core.U3, _core.H]
    assert rec["theta"][0] == -0.4 and rec["theta"][1] == 0.8 and rec["theta"][2] == 0.4
    assert rec["lam"][2] == math.pi / 2 and rec["phi"][2] == -math.pi / 2
    assert np.allclose(c.gradient(np.array([1.0, 2.0, 3.0, 0.0])), [-0.5 + 2.0, 3.0])
    with pytest.raises(ValueError):
        ad.parameter_shift(None, c, [0.0, 0.0], [])


def test_ansatz_and_observable_sizes():
    c = ad.hardware_efficient_ansatz(24, 8)
    assert c.nparams == 432 and len(c.base) == 9 * 48 + 8 * 23
    t = ad.tfim_terms(24)
    assert len(t) == 23 + 24 and t["coef"].sum() == 47.0


def test_ansatz_forward_plan_with_all_qubits_expanded():
    c = ad.hardware_efficient_ansatz(24, 8)
    st = plan_stats(24, c.records(np.linspace(-3, 3, 432)), dtype="complex64", eager_expand_all=True)
    assert st["M"] == 24 and st["m"] == 24 and st["product"] == 1 and st["passes"] > 0
