"""The allocation-free sampler entry point, zxh_sample_noalloc, through the C ABI.

Callers that cannot allocate device memory (services whose device memory is
reserved once up front, frameworks whose own allocator owns the device, latency
paths that must not take the CUDA allocator's locks) pass their own device state
and output buffers to zxh_sample_noalloc, which keeps its working memory in one
static device array. Its draws must equal those of the allocating sampler (zxh_measure)
for the same seed: same uniform stream, same output order, so the tolerance is
zero. Each case makes two calls in a row, so the second one runs on the scratch
the first one left behind.

This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

import zxh_adae_b200 as zx
from zxh_adae_b200 import workloads as wl

pytestmark = pytest.mark.gpu

ZXH_C64, ZXH_C128, ZXH_ERR_LIMIT = 1, 2, 5


def _lib():
    L = ctypes.CDLL(zx.library_path())
    L.zxh_sample_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t, ctypes.c_uint64,
                                     ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p]
    L.zxh_sample_noalloc.restype = ctypes.c_int
    L.zxh_last_error.argtypes = [ctypes.c_void_p]
    L.zxh_last_error.restype = ctypes.c_char_p
    return L


def _state(n, gates, dtype):
    s = zx.ZXH(n, dtype=dtype)
    s.push_gates(gates)
    s.execute()
    return s


CASES = [
    # H on every qubit first: the affine map is the identity, so the allocating
    # sampler's packed virtual bits equal the real indices returned here
    ("plain16", 16, lambda: wl.plain_layers(16, 3, seed=5), 20000),
    # all probability in one segment: the shared-memory resolve path
    ("delta14", 14, lambda: np.concatenate([wl.h_all(14), wl.h_all(14)]), 50000),
]


@pytest.mark.parametrize("dtype", ["complex128", "complex64"])
@pytest.mark.parametrize("name,n,make,shots", CASES, ids=[c[0] for c in CASES])
def test_noalloc_draws_equal_measure_twice(dtype, name, n, make, shots):
    import torch

    L = _lib()
    s = _state(n, make(), dtype)
    ptr, m, eb, _ = s.state_view()
    assert m == n
    out = torch.empty(shots, dtype=torch.int64, device="cuda")
    for seed in (11, 12):
        s.set_seed(seed)
        s.measure(shots)
        want = s.results_words()
        rc = L.zxh_sample_noalloc(ptr, ZXH_C64 if dtype == "complex64" else ZXH_C128, m, seed, shots,
                                  out.data_ptr(), None)
        assert rc == 0, L.zxh_last_error(None)
        got = out.cpu().numpy().view(np.uint64)
        assert np.array_equal(got, want)


def test_noalloc_rejects_states_beyond_the_static_scratch():
    L = _lib()
    rc = L.zxh_sample_noalloc(ctypes.c_void_p(256), ZXH_C64, 29, 1, 10, ctypes.c_void_p(256), None)
    assert rc == ZXH_ERR_LIMIT
    assert b"2^28" in L.zxh_last_error(None)
