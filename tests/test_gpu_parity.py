"""Parity of the CUDA path with the oracle (CPU restatement of the reference
path, bit-identical to the reference's serial backend) on seeded circuits.

Tolerances: max |amp - oracle| <= 1e-12 for complex128 and <= 1e-6 for
complex64; samples fed the same seed must be identical, in the same order.
"""
import numpy as np
import pytest

import zxh_adae_b200 as zx
from oracle.bridge import Oracle
from zxh_adae_b200 import workloads as wl
from zxh_adae_b200._core import plan_stats

pytestmark = pytest.mark.gpu
TOL = {"complex128": 1e-12, "complex64": 1e-6}
DTYPES = ["complex128", "complex64"]


def run_pair(n, gates, dtype, disable_x=False, eager=False):
    o = Oracle(n, disable_x, eager)
    o.push(gates)
    o.execute()
    s = zx.ZXH(n, disable_x, eager, dtype=dtype)
    s.push_gates(gates)
    s.execute()
    return o, s


def max_err(s, o, order=0):
    return float(np.max(np.abs(s.get_state(order).astype(np.complex128) - o.get_state(order))))


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("seed", range(24))
def test_random_circuits(dtype, seed):
    n = 1 + seed % 10
    gates = wl.random_circuit(n, 80, seed)
    o, s = run_pair(n, gates, dtype)
    assert s.required_M() == o.required_M()
    assert max_err(s, o) <= TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("seed", range(8))
@pytest.mark.parametrize("flags", [(True, False), (False, True), (True, True)])
def test_ablation_flags(dtype, seed, flags):
    n = 2 + seed % 7
    gates = wl.random_circuit(n, 50, 100 + seed)
    o, s = run_pair(n, gates, dtype, *flags)
    assert max_err(s, o) <= TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("n,seed", [(13, 1), (15, 2), (17, 3)])
def test_random_circuits_multi_tile(dtype, n, seed):
    # states larger than one tile: high-qubit tiles, multi-bit deltas after CX
    gates = wl.random_circuit(n, 300, seed)
    o, s = run_pair(n, gates, dtype)
    assert max_err(s, o) <= TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
def test_plain_layers_20q(dtype):
    gates = wl.plain_layers(20, 10, seed=2024)
    o, s = run_pair(20, gates, dtype)
    assert max_err(s, o) <= TOL[dtype]
    assert max_err(s, o, order=1) <= TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
def test_diag_batch_and_cascade_16q(dtype):
    n = 16
    gates = np.concatenate([wl.h_all(n), wl.diag_batch(n, 600, 5), wl.cp_cascade(n)])
    o, s = run_pair(n, gates, dtype)
    assert max_err(s, o) <= TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("chunk_bits", [0, 1, 3, 6])
@pytest.mark.parametrize("prefetch", [0, 1])
def test_diag_pass_gray_code_chunks(dtype, chunk_bits, prefetch):
    # the diagonal pass walks chunks of 2^chunk_bits tiles in Gray-code order,
    # updating the out-of-tile coefficients one flipped bit at a time; with
    # prefetch each warp stages its next tile by a TMA bulk copy
    n = 17
    gates = np.concatenate([wl.h_all(n), wl.diag_batch(n, 900, 8), wl.cp_cascade(n)])
    o = Oracle(n)
    o.push(gates)
    o.execute()
    s = zx.ZXH(n, dtype=dtype)
    s.set_param("diag_chunk_bits", chunk_bits)
    s.set_param("diag_prefetch_c64" if dtype == "complex64" else "diag_prefetch_c128", prefetch)
    s.push_gates(gates)
    s.execute()
    assert max_err(s, o) <= TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("row_bits", [2, 3, 4])
@pytest.mark.parametrize("n", [7, 19])
def test_diag_pass_row_counts(dtype, row_bits, n):
    # warp tiles of 4, 8 or 16 rows (the default is 4 rows for complex64, 8 for
    # complex128), chunks chosen per launch; at n = 7 the state is one tile smaller
    # than a full one
    gates = np.concatenate([wl.h_all(n), wl.diag_batch(n, 700, 9 + n), wl.cp_cascade(n)])
    o = Oracle(n)
    o.push(gates)
    o.execute()
    s = zx.ZXH(n, dtype=dtype)
    s.set_param("diag_row_bits_c64" if dtype == "complex64" else "diag_row_bits_c128", row_bits)
    s.push_gates(gates)
    s.execute()
    assert max_err(s, o) <= TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("n,seed", [(6, 1), (9, 2), (12, 3), (16, 4)])
def test_general_strided_pass_after_cx_transport(dtype, n, seed):
    # CX gates make the pair deltas span several real bits; those U3 batches run as
    # general strided passes with their diagonal windows fused
    gates = wl.random_circuit(n, 400, 300 + seed)
    assert plan_stats(n, gates, dtype=dtype)["grow"] > 0
    o, s = run_pair(n, gates, dtype)
    assert max_err(s, o) <= TOL[dtype]
    s2 = zx.ZXH(n, dtype=dtype)
    s2.set_param("grow", 0)
    s2.push_gates(gates)
    s2.execute()
    assert max_err(s2, o) <= TOL[dtype]
    for staged in (0, 7):  # rows loaded straight into registers / staged one item ahead in shared memory
        s3 = zx.ZXH(n, dtype=dtype)
        s3.set_param("grow_staged", staged)
        s3.push_gates(gates)
        s3.execute()
        assert max_err(s3, o) <= TOL[dtype], staged


@pytest.mark.parametrize("seed", range(24))
def test_general_strided_pass_random(seed):
    n = 6 + seed % 9
    gates = wl.random_circuit(n, 250, 4000 + seed)
    for dtype in DTYPES:
        o, s = run_pair(n, gates, dtype)
        assert max_err(s, o) <= TOL[dtype], (n, dtype, plan_stats(n, gates, dtype=dtype))


@pytest.mark.parametrize("dtype", DTYPES)
def test_general_strided_pass_ansatz_and_hidden_string(dtype):
    from zxh_adae_b200 import adjoint as ad

    circ = ad.hardware_efficient_ansatz(12, 4)
    rec = circ.records(np.random.default_rng(5).uniform(-3.1, 3.1, circ.nparams))
    for eager in (False, True):
        o, s = run_pair(12, rec, dtype, eager=eager)
        assert max_err(s, o) <= TOL[dtype]
    recs, secret = wl.hidden_string(13, seed=8)
    o, s = run_pair(14, recs, dtype)
    assert max_err(s, o) <= TOL[dtype]
    s.set_seed(4)
    s.measure(2000)
    assert set((s.results_words() & ((1 << 13) - 1)).tolist()) == {secret}


@pytest.mark.parametrize("dtype", DTYPES)
def test_u3_matching_layers(dtype):
    gates = wl.u3_matching_layers(16, 6, seed=3)
    o, s = run_pair(16, gates, dtype)
    assert max_err(s, o) <= TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
def test_apply_continues_state(dtype):
    n = 12
    a = wl.plain_layers(n, 2, seed=9)
    b = wl.diag_batch(n, 40, seed=10)
    o, _ = run_pair(n, np.concatenate([a, b]), dtype)
    s = zx.ZXH(n, dtype=dtype)
    s.push_gates(a)
    s.execute()
    s.apply(b)
    assert max_err(s, o) <= TOL[dtype]


@pytest.mark.parametrize("n,shots,seed", [(12, 1024, 3), (16, 4096, 4), (3, 50000, 5), (1, 100, 6)])
def test_sampler_matches_reference_stream(n, shots, seed):
    gates = wl.plain_layers(n, 3, seed=seed)
    o, s = run_pair(n, gates, "complex128")
    want, _ = o.sample(seed, shots)
    s.set_seed(seed)
    s.measure(shots)
    assert s.measured_count() == shots
    assert np.array_equal(s.results_words(), want[:, 0])


def test_sampler_delta_heavy_segment():
    recs, secret = wl.hidden_string(12, seed=17)
    o, s = run_pair(13, recs, "complex128")
    s.set_seed(1)
    s.measure(40000)
    w = s.results_words()
    want, _ = o.sample(1, 40000)
    assert np.array_equal(w, want[:, 0])
    assert set((int(x) & ((1 << 12) - 1)) for x in w) == {secret}


def test_sampler_complex64_counts_identical():
    gates = wl.plain_layers(14, 4, seed=21)
    o, s = run_pair(14, gates, "complex64")
    want, _ = o.sample(77, 20000)
    s.set_seed(77)
    s.measure(20000)
    got = s.results_words()
    # complex64 masses differ from the complex128 oracle by ~1e-7 relative:
    # outcomes agree except where a uniform falls that close to a boundary
    assert np.mean(got != want[:, 0]) < 1e-3


def test_measure_api_semantics():
    n = 3
    gates = zx.as_records([(zx._core.H, 0, 0), (zx._core.CP, 0, 1, 0.37), (zx._core.H, 0, 1), (zx._core.CX, 1, 2)])
    s = zx.ZXH(n)
    s.push_gates(gates)
    s.execute()
    s.measure(0)
    assert s.measured_count() == 0 and s.get_results() == []
    s.set_seed(31415926)
    s.measure(256)
    first = s.get_results()
    assert s.get_results() == first
    s.set_seed(31415926)
    assert s.Sampling(256) == first
    s.set_seed(27182818)
    counts = s.sample_counts(64)
    s.set_seed(27182818)
    rows = s.Sampling(64)
    from collections import Counter
    assert counts == dict(Counter("".join("1" if b else "0" for b in reversed(r)) for r in rows))


def test_errors_raise_instead_of_abort():
    s = zx.ZXH(2)
    with pytest.raises(ValueError):
        s.H(2)
    with pytest.raises(ValueError):
        s.CX(0, 5)
    with pytest.raises(RuntimeError):
        s.get_state()
    with pytest.raises(ValueError):
        zx.ZXH(64)
    s.execute()
    with pytest.raises(ValueError):
        s.get_results() if False else s.results_words(5)


def _layers_with_x(n, layers, seed):
    """U3 layers with X gates and big cp cascades in between (exercises flipped
    selectors, fused and unfused windows in the fast U3 pass)."""
    rng = np.random.default_rng(seed)
    recs = [(zx._core.H, 0, q) for q in range(n)]
    for layer in range(layers):
        for q in rng.choice(n, size=n // 3, replace=False):
            recs.append((zx._core.X, 0, int(q)))
        for q in range(n):
            recs.append((zx._core.U3, 0, q, *rng.uniform(0, 2 * np.pi, 3)))
        if layer % 2:
            recs.extend((int(g["type"]), int(g["cq"]), int(g["q"]), float(g["theta"])) for g in wl.cp_cascade(n))
        else:
            for i in range(n - 1):
                recs.append((zx._core.CP, i, i + 1, rng.uniform(0, 2 * np.pi)))
        recs.append((zx._core.RZ, 0, int(rng.integers(n)), rng.uniform(0, 2 * np.pi)))
    return zx.as_records(recs)


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("n", [11, 12, 13, 18])
def test_fast_u3_pass_edges(dtype, n):
    gates = _layers_with_x(n, 4, seed=n)
    o, s = run_pair(n, gates, dtype)
    assert max_err(s, o) <= TOL[dtype]


def _run_knobs(n, gates, dtype, knobs):
    o = Oracle(n)
    o.push(gates)
    o.execute()
    s = zx.ZXH(n, dtype=dtype)
    for k, v in knobs.items():
        s.set_param(k, v)
    s.push_gates(gates)
    s.execute()
    return o, s


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("knobs", [{"low_pass": 0}, {"low_regs_c64": 0, "low_regs_c128": 0},
                                   {"low_regs_c64": 2, "low_regs_c128": 3}, {"real_split": 0}, {},
                                   {"row_wide_c64": 0}, {"row_wide_c64": 0, "real_split": 0},
                                   {"row_wide_c64": 0, "low_regs_c64": 3}, {"low_regs_c64": 5, "low_regs_c128": 4}])
@pytest.mark.parametrize("n", [10, 12, 13, 18])
def test_low_pass_forms(dtype, knobs, n):
    # TMA fast pass + strided passes, and the strided low pass (lane bits swapped
    # into registers through shared memory) with 0..4 register gates, with the
    # gates as complex matrices or as real rotations whose phases ride in the
    # windows: the same state, with X-flipped selectors and fused windows
    gates = _layers_with_x(n, 4, seed=40 + n)
    o, s = _run_knobs(n, gates, dtype, knobs)
    assert max_err(s, o) <= TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("seed", range(8))
def test_low_pass_gate_subsets(dtype, seed):
    # U3 layers on random qubit subsets: low passes with and without gates on the
    # swapped lane bits, on the unswapped lane bit, on the vector bit, with padded
    # register bits; windows between the layers fuse before and after
    n = 11 + seed % 4
    rng = np.random.default_rng(900 + seed)
    recs = [(zx._core.H, 0, q) for q in range(n)]
    for layer in range(4):
        qs = [q for q in range(n) if rng.random() < 0.5] or [0]
        for q in qs:
            recs.append((zx._core.U3, 0, q, *rng.uniform(0, 2 * np.pi, 3)))
        for i in range(n - 1):
            if rng.random() < 0.5:
                recs.append((zx._core.CP, i, i + 1, rng.uniform(0, 2 * np.pi)))
        recs.append((zx._core.P, 0, int(rng.integers(n)), rng.uniform(0, 2 * np.pi)))
    o, s = _run_knobs(n, zx.as_records(recs), dtype, {})
    assert max_err(s, o) <= TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("seed", range(3))
def test_load_circuit_through_the_host_compiler(dtype, seed):
    # frontend gates (swap, ccx, rzz, ...) lowered and scheduled by the host
    # circuit compiler at level 2, run on the GPU; the state equals the oracle's
    # run of the level-0 compile up to a global phase
    from tests.test_optimize import _Circuit, _random_frontend

    n = 9 + seed
    circ = _Circuit(_random_frontend(n, 120, 7700 + seed))
    (base, _), = zx.compile_circuit(circ, n, 0)
    o = Oracle(n)
    o.push(base)
    o.execute()
    ref = o.get_state()
    s = zx.ZXH(n, dtype=dtype)
    zx.load_circuit(s, circ, optimize_level=2)
    s.execute()
    got = s.get_state().astype(np.complex128)
    k = int(np.argmax(np.abs(ref)))
    ph = got[k] / ref[k]
    ph /= abs(ph)
    assert float(np.max(np.abs(got - ph * ref))) <= TOL[dtype] * 10


@pytest.mark.parametrize("dtype", DTYPES)
def test_empty_barrier_only_and_single_qubit_circuits(dtype):
    for n in (1, 2, 7):
        for gates in ([], [(zx._core.BARRIER, 0, 0)]):
            s = zx.ZXH(n, dtype=dtype)
            s.push_gates(zx.as_records(gates))
            s.execute()
            st = s.get_state().astype(np.complex128)
            assert st[0] == 1 and not np.any(st[1:])
            s.apply(zx.as_records([]))
            assert np.array_equal(s.get_state().astype(np.complex128), st)
    for seed in range(6):
        gates = wl.random_circuit(1, 40, 8800 + seed)
        o, s = run_pair(1, gates, dtype)
        assert max_err(s, o) <= TOL[dtype]


def _inverse_records(recs):
    """The inverse circuit: gates in reverse order, each inverted (U3(t, l, p)^-1 =
    U3(-t, -p, -l); P / CP / RZ negate the angle; H, X, CX are their own inverses)."""
    C = zx._core
    out = []
    for r in reversed(zx.as_records(recs).tolist()):
        t, cq, q, _res, th, la, ph = r
        if t == C.U3:
            out.append((t, cq, q, -th, -ph, -la))
        elif t in (C.P, C.CP, C.RZ, C.CRZ, C.RX):
            out.append((t, cq, q, -th))
        else:
            out.append((t, cq, q))
    return zx.as_records(out)


@pytest.mark.parametrize("dtype", DTYPES)
def test_large_state_round_trip(dtype):
    # size-independent check at 26 qubits: layers of U3 + cp chains, X-flipped
    # selectors and their inverse bring |+>^n back; the norm stays 1
    n = 26 if dtype == "complex64" else 25
    layers = _layers_with_x(n, 3, seed=123)
    h = len(wl.h_all(n))
    body = layers[h:]
    s = zx.ZXH(n, dtype=dtype)
    s.push_gates(layers)
    s.execute()
    st = s.get_state().astype(np.complex128)
    assert abs(np.vdot(st, st).real - 1.0) < (1e-5 if dtype == "complex64" else 1e-12)
    s.apply(_inverse_records(body))
    back = s.get_state().astype(np.complex128)
    k = int(np.argmax(np.abs(back)))
    ph = back[k] / abs(back[k])
    amp = 2.0 ** (-n / 2)
    assert np.max(np.abs(back - ph * amp)) < (1e-4 if dtype == "complex64" else 1e-10) * amp


@pytest.mark.parametrize("dtype", DTYPES)
def test_apply_async_matches_apply(dtype):
    # the same batches through zxh_apply and zxh_apply_async give the same state
    # bit for bit (same plans, same kernels); a growing program forces the pinned
    # slots and the device program to grow between steps; measure and get_state
    # settle the work in flight themselves
    n = 16
    batches = [wl.diag_batch(n, 64 << (k % 4), seed=900 + k) for k in range(6)]
    batches += [wl.u3_layer(n, seed=950 + k) for k in range(3)]
    batches += [wl.random_circuit(n, 200, 990)]
    a = zx.ZXH(n, dtype=dtype)
    b = zx.ZXH(n, dtype=dtype)
    for s in (a, b):
        s.push_gates(wl.h_all(n))
        s.execute()
    for bt in batches:
        a.apply(bt)
        b.apply_async(bt)
    b.sync()
    b.sync()  # nothing in flight: returns at once
    assert np.array_equal(a.get_state(), b.get_state())
    for bt in batches[:3]:
        b.apply_async(bt)
        a.apply(bt)
    a.set_seed(4)
    b.set_seed(4)
    a.measure(2000)
    b.measure(2000)  # settles the queued batches first
    assert np.array_equal(a.results_words(), b.results_words())
    st = b.last_stats()
    assert st[0] > 0


def _walsh_case(n, prefix, seed):
    if prefix == "cx_chain":
        pre = wl.cx_chain(n)
    elif prefix == "cx_random":  # a dense map: random CX pairs, X flips (selector betas)
        rng = np.random.default_rng(seed)
        recs = []
        for _ in range(3 * n):
            c, t = (int(v) for v in rng.choice(n, 2, replace=False))
            recs.append((zx._core.CX, c, t))
            if rng.random() < 0.3:
                recs.append((zx._core.X, 0, int(rng.integers(n))))
        pre = zx.as_records(recs)
    else:
        pre = wl.h_all(n)[:0]
    rz = zx.as_records([(zx._core.RZ, 0, q, 0.37 * q + 0.1) for q in range(0, n, 3)]
                       + [(zx._core.Z, 0, 1)])
    return np.concatenate([wl.h_all(n), pre, wl.diag_batch(n, 700, seed), rz, wl.cp_cascade(n)])


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("prefix", ["cx_chain", "cx_random", "none"])
@pytest.mark.parametrize("knobs", [{}, {"walsh_min_general": 0}, {"walsh": 0}],
                         ids=["default", "walsh_always", "walsh_off"])
@pytest.mark.parametrize("n", [10, 15])
def test_walsh_window_pass(dtype, prefix, knobs, n):
    # windows whose selectors are parities of several real bits (after CX / X
    # transport) as one Walsh-sum pass; walsh_min_general = 0 also sends windows of
    # single-bit selectors through it, walsh = 0 is the per-amplitude form
    gates = _walsh_case(n, prefix, 40 + n)
    o = Oracle(n)
    o.push(gates)
    o.execute()
    s = zx.ZXH(n, dtype=dtype)
    for k, v in knobs.items():
        s.set_param(k, v)
    s.push_gates(gates)
    s.execute()
    assert max_err(s, o) <= TOL[dtype]
    if prefix != "none" and knobs.get("walsh", 1):
        assert s.last_stats()[1] <= 3  # the window is one pass (the cascade's window may join it)


@pytest.mark.parametrize("dtype", DTYPES)
def test_walsh_window_pass_through_apply(dtype):
    n = 16
    o = Oracle(n)
    full = [wl.h_all(n), wl.cx_chain(n)]
    s = zx.ZXH(n, dtype=dtype)
    s.push_gates(np.concatenate(full))
    s.execute()
    for k in range(3):
        b = wl.diag_batch(n, 1500, 900 + k)
        s.apply(b)
        assert s.last_stats()[1] == 1
        full.append(b)
    o.push(np.concatenate(full))
    o.execute()
    assert max_err(s, o) <= TOL[dtype]


def _span_case(n, kind, seed):
    rng = np.random.default_rng(seed)
    recs = [(zx._core.H, 0, q) for q in range(n)]
    for layer in range(3):
        if kind in ("flips", "mixed"):  # X gates: selectors with beta = 1 (the partner at bit 0 leads)
            recs += [(zx._core.X, 0, int(q)) for q in rng.choice(n, n // 3, replace=False)]
        recs += [(zx._core.U3, 0, q, *rng.uniform(0, 2 * np.pi, 3)) for q in range(n)]
        if kind in ("cp", "mixed"):  # quadratic windows between the layers
            recs += [(zx._core.CP, i, i + 1, float(rng.uniform(0, 2 * np.pi))) for i in range(n - 1)]
            perm = rng.permutation(n)
            recs += [(zx._core.CP, int(perm[2 * i]), int(perm[2 * i + 1]), np.pi) for i in range(n // 2)]
    return zx.as_records(recs)


_SPAN_ORACLE = {}


def _span_oracle_state(n, kind):
    # one oracle run per circuit, shared by the dtype and plan variants
    if (n, kind) not in _SPAN_ORACLE:
        o = Oracle(n)
        o.push(_span_case(n, kind, 500 + n))
        o.execute()
        _SPAN_ORACLE[(n, kind)] = o.get_state(0)
    return _SPAN_ORACLE[(n, kind)]


@pytest.mark.parametrize("kind", ["plain", "flips", "cp", "mixed"])
@pytest.mark.parametrize("n", [12, 13, 14, 17, 21, 23])
@pytest.mark.parametrize("plan", ["span", "span_register_form", "rows"])
@pytest.mark.parametrize("dtype", DTYPES)
def test_span_passes(kind, n, plan, dtype):
    # U3 batches as span passes against the oracle, in the landing form and the
    # register form: complex64 tiles of 2^13 (13 gates on bits 0..12, up to 10
    # high-bit gates per strided pass; at 23 qubits one strided pass of 10 gates,
    # c = 3, which needs the third layout); complex128 tiles of 2^12 (12 gates on
    # bits 0..11, up to 9 per strided pass; at 21 qubits one strided pass of 9
    # gates, whose runs of 8 amplitudes need the third layout in the register
    # form); "rows" is the row-pass plan
    gates = _span_case(n, kind, 500 + n)
    want = _span_oracle_state(n, kind)
    s = zx.ZXH(n, dtype=dtype)
    s.set_param("span", int(plan != "rows"))
    s.set_param("span_land", int(plan == "span"))
    s.push_gates(gates)
    s.execute()
    assert float(np.max(np.abs(s.get_state(0).astype(np.complex128) - want))) <= TOL[dtype]


@pytest.mark.parametrize("kind", ["plain", "mixed"])
@pytest.mark.parametrize("n,min_run", [(21, 6), (23, 6), (23, 8)])
@pytest.mark.parametrize("split,order", [(1, 0), (2, 0), (0, 1), (0, 2), (2, 2)])
@pytest.mark.parametrize("dtype", DTYPES)
def test_span_passes_split_and_order(kind, n, min_run, split, order, dtype):
    # other deals of the high-bit gates to the strided span passes (knob span_split:
    # 1 round robin, every strided pass holding bits from the whole high range, none
    # of them neighbours; 2 the larger blocks on the higher bits) and other orders of
    # the strided passes (knob span_order: 1 from the lowest bits up, 2 from the
    # highest down; the window before the batch rides on the first); complex64 at 23
    # qubits and run 2^8: two passes of 5 gates; complex128: three passes of 4, 4, 3
    gates = _span_case(n, kind, 500 + n)
    want = _span_oracle_state(n, kind)
    s = zx.ZXH(n, dtype=dtype)
    s.set_param("span_min_run", min_run)
    s.set_param("span_split", split)
    s.set_param("span_order", order)
    s.push_gates(gates)
    s.execute()
    assert float(np.max(np.abs(s.get_state(0).astype(np.complex128) - want))) <= TOL[dtype]


def _mixed_case(n, seed):
    # CX gates from a few qubits first: those qubits' U3 gates then have pair
    # deltas over two real bits, the rest single-bit deltas, in the same batch
    rng = np.random.default_rng(seed)
    recs = [(zx._core.H, 0, q) for q in range(n)]
    recs += [(zx._core.CX, int(c), int(c) + 1) for c in rng.choice(n - 1, 3, replace=False)]
    for layer in range(2):
        recs += [(zx._core.U3, 0, q, *rng.uniform(0, 2 * np.pi, 3)) for q in range(n)]
        recs += [(zx._core.CP, i, i + 1, float(rng.uniform(0, 2 * np.pi))) for i in range(n - 1)]
    return zx.as_records(recs)


@pytest.mark.parametrize("n", [14, 16, 19])
@pytest.mark.parametrize("mixed", [0, 1])
@pytest.mark.parametrize("dtype", DTYPES)
def test_u3_batches_mixing_single_and_multi_bit_deltas(n, mixed, dtype):
    # knob span_mixed: the single-bit gates of a mixed batch run as span passes
    # first, the others as general strided passes after them (1), or the whole
    # batch as general strided passes (0)
    gates = _mixed_case(n, 900 + n)
    st = plan_stats(n, gates, dtype=dtype)
    assert st["span"] > 0 and st["grow"] > 0
    o = Oracle(n)
    o.push(gates)
    o.execute()
    s = zx.ZXH(n, dtype=dtype)
    s.set_param("span_mixed", mixed)
    s.push_gates(gates)
    s.execute()
    assert max_err(s, o) <= TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
def test_span_pass_through_apply_round_trip(dtype):
    # a 26-qubit U3 layer and its inverse through apply(): back to |+...+> (the
    # layer runs as three span passes each way: complex64 7 + 6 high-bit gates and
    # 13 low, complex128 7 + 7 and 12 low)
    n = 26
    rng = np.random.default_rng(9)
    ang = rng.uniform(0, 2 * np.pi, (n, 3))
    fwd = zx.as_records([(zx._core.U3, 0, q, *ang[q]) for q in range(n)])
    # U3(t, l, p)^-1 = U3(-t, -p, -l) (records carry theta, lambda, phi)
    inv = zx.as_records([(zx._core.U3, 0, q, -ang[q][0], -ang[q][2], -ang[q][1]) for q in range(n)])
    s = zx.ZXH(n, dtype=dtype)
    s.push_gates(wl.h_all(n))
    s.execute()
    s.apply(fwd)
    assert s.last_stats()[1] == 3
    s.apply(inv)
    ptr, m, eb, g = s.state_view()
    import torch

    class _CAI:
        __cuda_array_interface__ = {"shape": (1 << m,), "typestr": "<c8" if dtype == "complex64" else "<c16",
                                    "data": (ptr, False), "version": 3}
    st = torch.as_tensor(_CAI(), device="cuda").to(torch.complex128) * complex(g)
    want = 2.0 ** (-n / 2)
    assert float((st - want).abs().max()) < TOL[dtype]
