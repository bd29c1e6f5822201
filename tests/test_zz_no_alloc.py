"""The allocation-free sampling entry point against the allocating one, through the C ABI.

qs_state_sampling_with_uniforms_noalloc is for callers that cannot call cudaMalloc (a host framework
that owns all device memory in its own pool, or a latency-bound loop that must not stall on an
allocation).  Its scratch is a static device array shared by every call, so this file checks two
calls in a row (the second must not see stale contents of the first) and the size limits.  It is
collected last so that a run stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import random_state
from qulacs_b200 import QuantumState
from qulacs_b200._lib import load

pytestmark = pytest.mark.gpu


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _sample(fn, state, uniforms):
    out = np.zeros(uniforms.size, dtype=np.uint64)
    rc = fn(state.data_ptr(), state.dim, _p(uniforms), uniforms.size, _p(out), None)
    assert rc == 0, load().qs_get_last_error()
    return out


def test_noalloc_sampling_matches_allocating_entry_point_twice():
    lib = load()
    rng = np.random.default_rng(4242)
    # two calls in a row with different sizes: the larger first, so stale scratch would show
    for n, shots in ((20, 4096), (13, 1000)):
        s = QuantumState(n)
        s.load(random_state(n, rng))
        u = rng.random(shots)
        u[0] = 0.0
        want = _sample(lib.qs_state_sampling_with_uniforms, s, u)
        got = _sample(lib.qs_state_sampling_with_uniforms_noalloc, s, u)
        assert np.array_equal(got, want)
        assert got[0] == np.uint64(2**64 - 1)


def test_noalloc_sampling_rejects_sizes_beyond_its_static_scratch():
    lib = load()
    u = np.zeros(4)
    out = np.zeros(4, dtype=np.uint64)
    # checked on the host before any device access (the state pointer is never read)
    assert lib.qs_state_sampling_with_uniforms_noalloc(None, 1 << 29, _p(u), 4, _p(out), None) == 5
    assert b"2^28" in lib.qs_get_last_error()
    s = QuantumState(4)
    big = np.zeros(16385)
    big_out = np.zeros(16385, dtype=np.uint64)
    assert lib.qs_state_sampling_with_uniforms_noalloc(s.data_ptr(), s.dim, _p(big), big.size, _p(big_out),
                                                       None) == 5
    assert b"16384" in lib.qs_get_last_error()
