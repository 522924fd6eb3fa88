"""The chi-square check of sample counts (tests/chisq.py), on the CPU.

The oracle's restatement of the reference GPU sampler draws from its own
state's probabilities; the check must accept those draws and must reject the
same draws held against a slightly different state (a mistake planted in the
oracle's input: one extra small rotation)."""
import numpy as np

from oracle.bridge import Oracle
from tests.chisq import P_VALUE_FLOOR, bit_reverse_index, chi_square
from zxh_adae_b200 import workloads as wl
from zxh_adae_b200.records import U3, as_records


def _probs(n, gates):
    o = Oracle(n)
    o.push(gates)
    o.execute()
    return o, np.abs(o.get_state()) ** 2


def test_chi_square_accepts_the_right_distribution():
    n = 10
    o, p = _probs(n, wl.plain_layers(n, 3, seed=21))
    for seed in (1, 2, 3):
        words, _ = o.sample(seed, 100_000)
        r = chi_square(p, bit_reverse_index(words[:, 0], n))
        assert r["p_value"] > P_VALUE_FLOOR and r["min_expected"] >= 20.0, r


def test_chi_square_rejects_a_planted_mistake():
    n = 10
    gates = wl.plain_layers(n, 3, seed=21)
    o, _ = _probs(n, gates)
    wrong = np.concatenate([gates, as_records([(U3, 0, 3, 0.08, 0.0, 0.0)])])
    _, p_wrong = _probs(n, wrong)
    words, _ = o.sample(5, 100_000)
    r = chi_square(p_wrong, bit_reverse_index(words[:, 0], n))
    assert r["p_value"] < 1e-8, r


def test_bit_reverse_index():
    w = np.array([0b0001, 0b0110, 0b1000], np.uint64)
    assert bit_reverse_index(w, 4).tolist() == [0b1000, 0b0110, 0b0001]
