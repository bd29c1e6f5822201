"""Reductions and sampling on the B200 against the oracle."""
import ctypes as C

import numpy as np
import pytest

from conftest import BOUNDARY_EPS, EV_TOL, mt19937_64_uniforms, random_state
from qulacs_b200 import Observable, PauliOperator, QuantumState, inner_product
from qulacs_b200 import workloads as W
from qulacs_b200._lib import call

pytestmark = pytest.mark.gpu


def dev(vec):
    s = QuantumState(int(np.log2(vec.size)))
    s.load(vec)
    return s


@pytest.mark.parametrize("n", [1, 4, 13, 20])
def test_norm_inner_probabilities(port, n):
    rng = np.random.default_rng(700 + n)
    a, b = random_state(n, rng), random_state(n, rng)
    sa, sb = dev(a), dev(b)
    assert abs(sa.get_squared_norm() - port.state_norm_squared(a)) <= 1e-13
    assert abs(inner_product(sa, sb) - port.state_inner_product(a, b)) <= 1e-13
    for t in range(0, n, max(1, n // 4)):
        assert abs(sa.get_zero_probability(t) - port.M0_prob(t, a)) <= 1e-13
    if n >= 4:
        mv = [2] * n
        mv[1], mv[3] = 1, 0
        assert abs(sa.get_marginal_probability(mv) - port.marginal_prob([1, 3], [1, 0], a)) <= 1e-13


@pytest.mark.parametrize("n", [2, 9, 18])
def test_expectation_values_single_and_batch(port, n):
    rng = np.random.default_rng(800 + n)
    a = random_state(n, rng)
    s = dev(a)
    terms = W.random_pauli_terms(n, 40, 1, min(6, n), seed=801 + n)
    obs = Observable(n)
    want = []
    for coef, tl, ids in terms:
        obs.add_operator(PauliOperator(coef=coef, targets=tl, pauli_ids=ids))
        want.append(port.expectation_value(tl, ids, a))
        single = PauliOperator(coef=1.0, targets=tl, pauli_ids=ids).get_expectation_value(s)
        assert abs(single.real - want[-1]) <= EV_TOL
    vals = obs.term_values(s)
    assert np.max(np.abs(vals - np.array(want))) <= EV_TOL
    coefs = np.array([c for c, _, _ in terms])
    assert abs(obs.get_expectation_value(s) - float(np.dot(coefs, want))) <= EV_TOL


def test_expectation_values_many_z_strings(port):
    """Z-only strings share the first tiled pass with the bit-flip strings up to the per-pass term cap
    (512); the rest go through the Z-only batch kernel."""
    n = 14
    rng = np.random.default_rng(870)
    a = random_state(n, rng)
    s = dev(a)
    terms = W.random_pauli_terms(n, 24, 1, 4, seed=871)
    for _ in range(600):
        w = int(rng.integers(1, 6))
        terms.append((float(rng.normal()), [int(x) for x in rng.choice(n, size=w, replace=False)], [3] * w))
    obs = Observable(n)
    for coef, tl, ids in terms:
        obs.add_operator(PauliOperator(coef=coef, targets=tl, pauli_ids=ids))
    want = np.array([port.expectation_value(tl, ids, a) for _, tl, ids in terms])
    assert np.max(np.abs(obs.term_values(s) - want)) <= EV_TOL


def test_transition_amplitude(port, ref):
    rng = np.random.default_rng(850)
    n = 8
    a, b = random_state(n, rng), random_state(n, rng)
    sa, sb = dev(a), dev(b)
    tl = np.array([1, 4, 6], dtype=np.uint32)
    ids = np.array([2, 1, 3], dtype=np.uint32)
    out = np.zeros(2)
    call("qs_transition_amplitude_multi_qubit_Pauli_operator_partial_list", tl.ctypes.data_as(C.c_void_p),
         ids.ctypes.data_as(C.c_void_p), 3, sa.data_ptr(), sb.data_ptr(), sa.dim, None,
         out.ctypes.data_as(C.c_void_p))
    want = np.zeros(2)
    ref.lib.ref_transition_amplitude_multi_qubit_Pauli_operator_partial_list(
        tl.ctypes.data_as(C.c_void_p), ids.ctypes.data_as(C.c_void_p), C.c_uint(3),
        a.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p), C.c_ulonglong(a.size),
        want.ctypes.data_as(C.c_void_p))
    assert np.max(np.abs(out - want)) <= 1e-13


@pytest.mark.parametrize("n", [3, 12, 21])
def test_sampling_identical_indices(port, n):
    """Same uniforms -> same indices, except draws within 1e-12 of a cumulative boundary (counted)."""
    rng = np.random.default_rng(900 + n)
    a = random_state(n, rng)
    u = rng.random(4096)
    u[0] = 0.0
    s = dev(a)
    got = s.sampling_with_uniforms(u)
    want, near = port.sampling_with_uniforms(a, u, eps=BOUNDARY_EPS)
    bad = (got != want) & ~near
    assert not bad.any(), np.nonzero(bad)[0][:10]
    assert got[0] == np.uint64(2**64 - 1)
    assert int(near.sum()) <= 8  # boundary draws are rare and reported


def test_sampling_known_answers():
    """test/cppsim/test_state.cpp:38-81."""
    s = QuantumState(10)
    s.set_computational_basis(100)
    assert set(s.sampling(1024, 7)) == {100}
    n = 5
    v = np.sqrt(2.0 ** np.arange(1 << n))
    s = dev(v / np.linalg.norm(v))
    cnt = np.bincount(np.array(s.sampling(100000, 11), dtype=np.int64), minlength=1 << n)
    assert np.all(np.diff(cnt[-8:]) > 0)


def test_sampling_past_total_gives_dim(port):
    a = 0.5 * random_state(6, np.random.default_rng(3))  # norm 1/4
    s = dev(a)
    got = s.sampling_with_uniforms([0.2, 0.9])
    want = port.sampling_with_uniforms(a, [0.2, 0.9])
    assert got[1] == 64 and np.array_equal(got, want)


def test_seeded_sampling_matches_reference_rng(port):
    """qs_state_sampling draws mt19937_64(seed) uniforms exactly as cppsim Random does."""
    a = random_state(9, np.random.default_rng(5))
    s = dev(a)
    got = np.array(s.sampling(256, 1234), dtype=np.uint64)
    want_u = mt19937_64_uniforms(1234, 256)
    want = port.sampling_with_uniforms(a, want_u)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("n", [6, 14])
def test_sampling_reports_boundary_draws(port, n):
    """The flagged sampler reports draws within eps of a cumulative boundary: uniforms planted ON the
    prefix sums (and 1e-14 beside them) are all flagged, ordinary draws agree with the oracle wherever
    neither side flags them, and the count equals the number of flags."""
    rng = np.random.default_rng(40 + n)
    a = random_state(n, rng)
    p = a.real ** 2 + a.imag ** 2
    stacked = np.cumsum(p)  # serial FP64 running sum, cppsim/state.hpp:917-922
    k = rng.choice((1 << n) - 1, size=16, replace=False)
    planted = np.concatenate([stacked[k], stacked[k] + 1e-14, stacked[k] - 1e-14])
    u = np.concatenate([planted, rng.random(512)])
    s = dev(a)
    got, flags = s.sampling_with_uniforms_flagged(u, BOUNDARY_EPS)
    assert flags[:planted.size].all()
    want, near = port.sampling_with_uniforms(a, u, eps=BOUNDARY_EPS)
    assert not ((got != want) & ~near & ~flags).any()
    assert np.array_equal(got[~flags], s.sampling_with_uniforms(u)[~flags])
    assert s.sampling_boundary_draws(256, 99) == int(
        s.sampling_with_uniforms_flagged(mt19937_64_uniforms(99, 256))[1].sum())
