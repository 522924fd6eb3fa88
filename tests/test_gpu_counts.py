"""GPU tests of zxh_counts: outcome counts of a draw, computed on the device.

The per-shot outcomes of the same draw (zxh_get_results, whose stream is pinned to
the reference sampler elsewhere) are the reference here: the device counts must
equal np.unique of those words exactly, for segments counted by the warp sort
(at most 32 shots), by the shared histogram (heavier ones), states smaller than
one segment, lazily expanded qubits and X-transported maps (nonzero offset)."""
import ctypes
from collections import Counter

import numpy as np
import pytest

import zxh_adae_b200 as zx
from zxh_adae_b200 import _core
from zxh_adae_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _want(s):
    return np.unique(s.results_words(), return_counts=True)


def _check(s, shots, seed=5):
    s.set_seed(seed)
    s.measure(shots)
    words, cnt = s.counts_words()
    kw, kc = _want(s)
    assert np.array_equal(words, kw) and np.array_equal(cnt, kc.astype(np.uint64))
    assert int(cnt.sum()) == shots
    return len(words)


def _h_u3(n, seed, dtype="complex64", skip=()):
    rng = np.random.default_rng(seed)
    g = [(_core.H, 0, q) for q in range(n) if q not in skip]
    g += [(_core.U3, 0, q, *rng.uniform(-0.6, 0.6, 3)) for q in range(n) if q not in skip]
    s = zx.ZXH(n, dtype=dtype)
    s.push_gates(g)
    s.execute()
    return s


@pytest.mark.parametrize("dtype", ["complex64", "complex128"])
def test_counts_light_segments(dtype):
    # 2^24 amplitudes, 4096 segments, ~5 shots each: the warp-sort path
    s = _h_u3(24, 1, dtype)
    assert _check(s, 20000) > 15000


@pytest.mark.parametrize("dtype", ["complex64", "complex128"])
def test_counts_heavy_segments(dtype):
    # 2^16 amplitudes, 16 segments with thousands of shots each: the histogram path
    s = _h_u3(16, 2, dtype)
    _check(s, 300000)


def test_counts_mixed_and_peaked():
    # a few heavy outcomes among a spread tail: both paths in one draw
    n = 18
    g = [(_core.H, 0, q) for q in range(n)] + [(_core.U3, 0, q, 0.9, 0.1, -0.3) for q in range(6)]
    g += [(_core.U3, 0, q, 2.6, 0.0, 0.0) for q in range(6, n)]  # close to |1> on the high qubits
    s = zx.ZXH(n)
    s.push_gates(g)
    s.execute()
    _check(s, 50000)


@pytest.mark.parametrize("n", [1, 3, 7, 12])
def test_counts_states_smaller_than_a_segment(n):
    s = _h_u3(n, 3)
    _check(s, 5000)
    _check(s, 20)


def test_counts_basis_state_and_ghz():
    n = 20
    s = zx.ZXH(n)
    s.push_gates([(_core.X, 0, q) for q in (1, 4, 19)])  # map offset only: one outcome
    s.execute()
    assert _check(s, 100000) == 1
    words, cnt = s.counts_words()
    assert int(words[0]) == (1 << 1) | (1 << 4) | (1 << 19) and int(cnt[0]) == 100000
    s = zx.ZXH(n)
    s.push_gates([(_core.H, 0, 0)] + [(_core.CX, q, q + 1) for q in range(n - 1)])
    s.execute()
    assert _check(s, 4096) == 2
    words, _ = s.counts_words()
    assert words.tolist() == [0, (1 << n) - 1]


def test_counts_singular_map_merges_words():
    # CX(0, 0) is accepted as in the reference and clears the map column of real
    # bit 0: both real indices read as word 0, and the two device counts merge
    s = zx.ZXH(6)
    s.push_gates([(_core.H, 0, 0), (_core.CX, 0, 0)])
    s.execute()
    s.set_seed(3)
    s.measure(1000)
    nu = _core._SZ(0)
    assert _core._lib.zxh_counts(s._h, None, None, 0, ctypes.byref(nu)) == 0 and nu.value == 2
    words, cnt = s.counts_words()
    assert words.tolist() == [0] and cnt.tolist() == [1000]
    assert s.sample_counts(1000) == {"000000": 1000}


def test_counts_lazy_qubits_and_transported_x():
    # untouched qubits stay outside the state; X and CX move through the map
    n = 26
    s = zx.ZXH(n)
    s.push_gates(wl.random_circuit(14, 300, 77))
    s.push_gates([(_core.X, 0, 20), (_core.CX, 3, 24), (_core.X, 0, 25)])
    s.execute()
    assert s.state_view()[1] < n
    _check(s, 30000)


def test_counts_30q_complex64_million_shots():
    s = _h_u3(30, 4)
    k = _check(s, 1_000_000)
    assert k > 900_000


def test_counts_api_edges():
    s = _h_u3(10, 6)
    nu = _core._SZ(0)
    # no draw since execute: nothing to count
    assert _core._lib.zxh_counts(s._h, None, None, 0, ctypes.byref(nu)) == 0 and nu.value == 0
    s.measure(0)
    assert _core._lib.zxh_counts(s._h, None, None, 0, ctypes.byref(nu)) == 0 and nu.value == 0
    s.set_seed(9)
    s.measure(3000)
    assert _core._lib.zxh_counts(s._h, None, None, 0, ctypes.byref(nu)) == 0
    k = int(nu.value)
    assert k > 100
    w = np.zeros(k, np.uint64)
    c = np.zeros(k, np.uint64)
    rc = _core._lib.zxh_counts(s._h, w.ctypes.data, c.ctypes.data, k - 1, ctypes.byref(nu))
    assert rc == 5 and nu.value == k  # ZXH_ERR_LIMIT
    assert _core._lib.zxh_counts(s._h, w.ctypes.data, None, k, ctypes.byref(nu)) == 1  # ZXH_ERR_ARG
    for _ in range(2):  # repeated calls give the same counts
        assert _core._lib.zxh_counts(s._h, w.ctypes.data, c.ctypes.data, k, ctypes.byref(nu)) == 0
        kw, kc = _want(s)
        o = np.argsort(w, kind="stable")
        assert np.array_equal(w[o], kw) and np.array_equal(c[o], kc.astype(np.uint64))
    # a new execute drops the draw
    s.execute()
    assert _core._lib.zxh_counts(s._h, None, None, 0, ctypes.byref(nu)) == 0 and nu.value == 0


def test_sample_counts_matches_sampling():
    s = _h_u3(12, 8)
    s.set_seed(123)
    counts = s.sample_counts(5000)
    s.set_seed(123)
    rows = s.Sampling(5000)
    assert counts == dict(Counter("".join("1" if b else "0" for b in reversed(r)) for r in rows))
    assert list(counts) == sorted(counts)


class _Inst:
    def __init__(self, name, qubits, params=()):
        self.operation = type("Op", (), {"name": name, "params": list(params)})()
        self.qubits = list(qubits)


class _Circuit:
    def __init__(self, n, insts):
        self.num_qubits = n
        self.data = insts

    def find_bit(self, q):
        return type("Bit", (), {"index": q})()


def test_backend_run_on_the_gpu():
    # the zxh backend's run path (seed, clear, load, execute, sample_counts)
    b = zx.make_zxh_backend()
    bell = _Circuit(2, [_Inst("h", [0]), _Inst("cx", [0, 1]), _Inst("measure", [0]), _Inst("measure", [1])])
    counts = b.run(bell, shots=4000, seed_simulator=11).result().get_counts()
    assert set(counts) == {"00", "11"} and sum(counts.values()) == 4000
    assert abs(counts["00"] - 2000) < 200
    again = b.run(bell, shots=4000, seed_simulator=11).result().get_counts()
    assert again == counts
    # the same draw through the simulator directly
    s = zx.ZXH(2)
    s.set_seed(11)
    s.push_gates([(_core.H, 0, 0), (_core.CX, 0, 1)])
    s.execute()
    assert s.sample_counts(4000) == counts
    # frontend gates through the host compiler
    n = 5
    insts = [_Inst("h", [q]) for q in range(n)] + [_Inst("swap", [0, 4]), _Inst("ccx", [1, 2, 3]),
                                                   _Inst("ry", [2], [0.4]), _Inst("rzz", [0, 1], [0.3])]
    b5 = zx.make_zxh_backend(dtype="complex64")
    res = b5.run([_Circuit(n, insts)] * 2, shots=3000, seed_simulator=5, optimize_level=2).result()
    c0, c1 = res.get_counts()
    assert c0 == c1 and sum(c0.values()) == 3000 and all(len(k) == n for k in c0)
    b.close()
    b5.close()
