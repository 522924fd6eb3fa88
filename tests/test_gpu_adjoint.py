"""GPU parity of zxh_expectation and zxh_adjoint_gradient.

Energies are checked against the oracle's state (bit-exact with the reference's
forward semantics) and gradients against FP64 central differences (step 1e-6)
and parameter shifts of oracle energies, then against the same differences on
this library's own complex128 forward path at 24 qubits, the size of the
432-parameter ansatz."""
import math

import numpy as np
import pytest

from oracle import observables as ob
from tests.test_adjoint_host import mixed_circuit, random_terms
from zxh_adae_b200 import _core
from zxh_adae_b200 import adjoint as ad

pytestmark = pytest.mark.gpu


def _params(circ, seed):
    return np.random.default_rng(seed).uniform(-math.pi, math.pi, circ.nparams)


@pytest.mark.parametrize("n,seed", [(3, 0), (5, 1), (9, 2), (12, 3)])
def test_expectation_matches_oracle(n, seed):
    circ = mixed_circuit(n, seed)
    p = _params(circ, seed)
    terms = random_terms(n, seed)
    for dtype, tol in (("complex128", 1e-12), ("complex64", 2e-5)):
        s = _core.ZXH(n, dtype=dtype)
        s.push_gates(circ.records(p))
        s.execute()
        assert abs(s.expectation(terms) - ob.oracle_energy(n, circ.records(p), terms)) < tol * len(terms)


def test_expectation_drops_x_terms_outside_the_state():
    # qubit 2 is never touched: the lazily expanded state does not span it, and
    # <X_2> = 0 exactly; Z_2 still reads +1
    n = 4
    rec = [(_core.H, 0, 0), (_core.CX, 0, 1), (_core.U3, 0, 3, 0.7, 0.1, 0.2)]
    terms = _core.as_terms([(_core.TERM_X, 2, 0, 1.5), (_core.TERM_Z, 2, 0, 0.25), (_core.TERM_X, 3, 0, 1.0),
                            (_core.TERM_ZZ, 0, 1, 2.0)])
    s = _core.ZXH(n)
    s.push_gates(rec)
    s.execute()
    assert s.state_view()[1] < n
    assert abs(s.expectation(terms) - ob.oracle_energy(n, _core.as_records(rec), terms)) < 1e-12


@pytest.mark.parametrize("n,seed", [(4, 0), (7, 1), (10, 2)])
@pytest.mark.parametrize("adj_regs", [3, 4])
@pytest.mark.parametrize("staged", [0, 7])
def test_adjoint_matches_oracle_differences(n, seed, adj_regs, staged):
    circ = mixed_circuit(n, seed) if seed else ad.hardware_efficient_ansatz(n, 3)
    terms = random_terms(n, seed) if seed else ad.tfim_terms(n)
    p = _params(circ, seed)
    s = _core.ZXH(n)
    s.set_param("adj_regs", adj_regs)  # high-delta gates per reverse strided pass
    s.set_param("grow_staged", staged)  # strided passes staging their next item in shared memory
    e, g = ad.adjoint(s, circ, p, terms)
    assert abs(e - ob.oracle_energy(n, circ.records(p), terms)) < 1e-11
    fd = ob.oracle_central_difference(n, circ, p, terms)
    assert np.max(np.abs(g - fd)) < 1e-6
    if np.all(circ.coef == 1.0):
        assert np.max(np.abs(g - ob.oracle_parameter_shift(n, circ, p, terms))) < 1e-10


@pytest.mark.parametrize("dtype", ["complex128", "complex64"])
def test_checkpoints_do_not_change_the_gradient(dtype):
    n = 11
    circ = ad.hardware_efficient_ansatz(n, 4)
    terms = ad.tfim_terms(n, h=0.7)
    p = _params(circ, 5)
    s = _core.ZXH(n, dtype=dtype)
    e0, g0 = ad.adjoint(s, circ, p, terms, 0)
    tol = 1e-12 if dtype == "complex128" else 2e-5
    for k in (1, 5, 17, 10_000):
        e, g = ad.adjoint(s, circ, p, terms, k)
        assert abs(e - e0) < tol and np.max(np.abs(g - g0)) < tol, k
    ref = _core.ZXH(n)
    _, g128 = ad.adjoint(ref, circ, p, terms)
    assert np.max(np.abs(g0 - g128)) < (1e-12 if dtype == "complex128" else 1e-5)


def test_state_after_the_sweep_is_the_forward_output():
    n = 9
    circ = mixed_circuit(n, 7)
    p = _params(circ, 7)
    s = _core.ZXH(n)
    s.push_gates(circ.records(p))
    s.adjoint_gradient(random_terms(n, 7), 3)
    got = s.get_state()
    want = ob.oracle_state(n, circ.records(p))
    assert np.max(np.abs(ob.qubit_order(got, n) - want)) < 1e-12
    s.set_seed(3)
    s.measure(100)
    assert s.measured_count() == 100


def test_torch_autograd_function():
    torch = pytest.importorskip("torch")
    n = 6
    circ = ad.hardware_efficient_ansatz(n, 2)
    terms = ad.tfim_terms(n)
    s = _core.ZXH(n)
    x = torch.tensor(_params(circ, 11), dtype=torch.float64, requires_grad=True)
    e = ad.AdjointExpectation.apply(x, s, circ, terms, 4)
    (3.0 * e).backward()
    e_ref, g_ref = ad.adjoint(_core.ZXH(n), circ, x.detach().numpy(), terms)
    assert abs(float(e) - e_ref) < 1e-12
    assert torch.allclose(x.grad, torch.as_tensor(3.0 * g_ref), atol=1e-12)


def test_adjoint_24q_ansatz_c64_within_1e5_of_fp64_differences():
    # the 24-qubit, 432-parameter ansatz in complex64 against complex128 central
    # differences on the plain forward path, on a spread of parameters
    n = 24
    circ = ad.hardware_efficient_ansatz(n, 8)
    terms = ad.tfim_terms(n)
    p = _params(circ, 24)
    s64 = _core.ZXH(n, dtype="complex64")
    e, g = ad.adjoint(s64, circ, p, terms, 48)
    s128 = _core.ZXH(n, dtype="complex128")
    which = [0, 1, 23, 24, 47, 200, 215, 216, 383, 384, 407, 431]
    fd = ad.finite_difference(s128, circ, p, terms, 1e-6, which)
    assert abs(e - ad.energy(s128, circ, p, terms)) < 1e-5
    assert np.max(np.abs(g[which] - fd[which])) < 1e-5


def test_errors():
    s = _core.ZXH(3)
    with pytest.raises(RuntimeError):
        s.expectation([(_core.TERM_Z, 0, 0, 1.0)])
    s.push_gates([(_core.H, 0, 0)])
    with pytest.raises(ValueError):
        s.adjoint_gradient([(9, 0, 0, 1.0)])
    with pytest.raises(ValueError):
        s.adjoint_gradient([(_core.TERM_ZZ, 0, 5, 1.0)])
    g = np.zeros(1)
    v = _core.ctypes.c_double(0.0)
    t = _core.as_terms([(_core.TERM_Z, 0, 0, 1.0)])
    s.push_gates([(_core.H, 0, 1)])
    rc = _core._lib.zxh_adjoint_gradient(s._h, t.ctypes.data, 1, 0, _core.ctypes.byref(v), g.ctypes.data, 1)
    assert rc == 1  # two recorded gates, room for one gradient
