"""Sample counts of the GPU sampler against the exact complex128 probabilities.

complex128 draws equal the reference GPU sampler's shot for shot (the same
uniform stream, tests/test_gpu_refcuda.py); complex64 draws follow the same
stream through single-precision masses, so a shot whose uniform lands within
rounding of a CDF boundary may pick the neighbouring outcome. Their
distribution is checked with a chi-square goodness-of-fit test against the
probabilities of the oracle's complex128 state (pinned bit-exact to the
reference): bins of at least 20 expected draws, the test fails below a p-value
of 1e-4 (tests/chisq.py). Seeds are fixed, so each case is deterministic."""
import numpy as np
import pytest

import zxh_adae_b200 as zx
from oracle.bridge import Oracle
from tests.chisq import P_VALUE_FLOOR, bit_reverse_index, chi_square
from zxh_adae_b200 import workloads as wl

pytestmark = pytest.mark.gpu

CASES = [(10, 200_000, 31), (14, 500_000, 32), (18, 1_000_000, 33)]


@pytest.mark.parametrize("dtype", ["complex64", "complex128"])
@pytest.mark.parametrize("n,shots,seed", CASES, ids=[f"{c[0]}q_{c[1]}" for c in CASES])
def test_counts_fit_the_complex128_probabilities(dtype, n, shots, seed):
    gates = wl.plain_layers(n, 3, seed=seed)
    o = Oracle(n)
    o.push(gates)
    o.execute()
    p = np.abs(o.get_state()) ** 2
    s = zx.ZXH(n, dtype=dtype)
    s.push_gates(gates)
    s.execute()
    for draw_seed in (seed, seed + 1000):
        s.set_seed(draw_seed)
        s.measure(shots)
        r = chi_square(p, bit_reverse_index(s.results_words(), n))
        assert r["p_value"] > P_VALUE_FLOOR and r["min_expected"] >= 20.0, (dtype, n, r)
    s.close()
