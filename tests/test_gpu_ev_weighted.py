"""sum_k c_k <P_k> from the weighted passes (no per-term values) against the oracle: every kind of
term evaluation (Z-only, bit flips within a thread's registers, partner amplitudes from shared memory,
per-thread selected rows, one value each), complex coefficients, complex128 and complex64 states."""
import numpy as np
import pytest

from conftest import EV_TOL, random_state
from qulacs_b200 import Observable, PauliOperator, QuantumState, QuantumStateC64
from qulacs_b200 import workloads as W
from qulacs_b200.observable import expectation_specialized_info, set_expectation_specialized

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["generic", "generated"])
def kernels(request):
    """Every test runs with the generic pass kernel and with per-pass kernels generated at first use."""
    set_expectation_specialized(0 if request.param == "generic" else 2)
    yield request.param
    set_expectation_specialized(1)


def observable(n, terms, coefs):
    obs = Observable(n)
    for c, (_, tl, ids) in zip(coefs, terms):
        obs.add_operator(PauliOperator(coef=c, targets=tl, pauli_ids=ids))
    return obs


def oracle_sum(port, a, terms, coefs):
    return sum(c * port.expectation_value(tl, ids, a) for c, (_, tl, ids) in zip(coefs, terms))


@pytest.mark.parametrize("n", [11, 12, 15, 19])
def test_weighted_matches_oracle_every_kind(port, n, kernels):
    rng = np.random.default_rng(9100 + n)
    a = random_state(n, rng)
    s = QuantumState(n)
    s.load(a)
    terms = W.random_pauli_terms(n, 150, 1, 6, seed=9200 + n)
    terms += [(0.0, [q], [1]) for q in range(4)]  # bit flips on qubits 0..3 alone
    terms += [(0.0, [int(q) for q in rng.choice(n, 3, replace=False)], [3, 3, 3]) for _ in range(10)]  # Z-only
    coefs = rng.normal(size=len(terms)) + 1j * rng.normal(size=len(terms))
    obs = observable(n, terms, coefs)
    plan = obs.weighted_plan()
    assert plan["passes"] >= 1
    for kind in ("z_only", "in_registers", "shared_partner", "selected_rows"):
        assert plan[kind] > 0, (kind, plan)
    launches0 = expectation_specialized_info()[0]
    got = obs.get_expectation_value_complex(s)
    launched = expectation_specialized_info()[0] - launches0
    assert (launched == plan["passes"]) if kernels == "generated" else (launched == 0)
    want = oracle_sum(port, a, terms, coefs)
    tol = EV_TOL * float(np.sum(np.abs(coefs)))
    assert abs(got - want) <= tol, (got, want)
    assert abs(obs.get_expectation_value(s) - want.real) <= tol
    # the per-term path gives the same sum
    vals = obs.term_values(s)
    assert abs(got - complex(np.sum(coefs * vals))) <= tol


def test_weighted_one_value_each_paths(port, kernels):
    """Below the tile size, with fewer than four bit-flip strings, and with strings that share no span:
    every term is evaluated alone and weighted on the host."""
    rng = np.random.default_rng(9300)
    for n, terms in [(8, W.random_pauli_terms(8, 30, 1, 4, seed=9301)),
                     (14, [(1.0, [0], [1]), (0.5, [3, 9], [2, 2]), (0.2, [1, 2], [3, 3])]),
                     (26, [(1.0, [q, q + 13], [1, 2]) for q in range(4, 13)])]:
        a = random_state(n, rng)
        s = QuantumState(n)
        s.load(a)
        coefs = rng.normal(size=len(terms))
        obs = observable(n, terms, coefs)
        want = oracle_sum(port, a, terms, coefs)
        assert abs(obs.get_expectation_value(s) - want.real) <= EV_TOL * float(np.sum(np.abs(coefs)))


def test_weighted_c64(port, kernels):
    n = 16
    rng = np.random.default_rng(9400)
    a = random_state(n, rng)
    s = QuantumStateC64(n)
    ref = QuantumState(n)
    ref.load(a)
    s.load(ref)
    a64 = s.get_vector().astype(np.complex128)  # the rounded amplitudes the kernel reads
    terms = W.random_pauli_terms(n, 120, 1, 6, seed=9401)
    coefs = rng.normal(size=len(terms))
    obs = observable(n, terms, coefs)
    want = oracle_sum(port, a64, terms, coefs)
    assert abs(obs.get_expectation_value(s) - want.real) <= EV_TOL * float(np.sum(np.abs(coefs)))


def test_weighted_repeatable(kernels):
    """The same call twice gives the same bits (fixed per-thread order, per-CTA partials folded in order)."""
    n = 18
    rng = np.random.default_rng(9500)
    s = QuantumState(n)
    s.load(random_state(n, rng))
    terms = W.random_pauli_terms(n, 200, 1, 6, seed=9501)
    obs = observable(n, terms, rng.normal(size=len(terms)))
    assert obs.get_expectation_value(s) == obs.get_expectation_value(s)


def test_generated_and_generic_agree_and_coefficients_reuse_kernels(port):
    """The generated kernels and the generic kernel give the same sum to rounding; new coefficients for
    the same strings reuse the generated kernels (no compile)."""
    n = 21
    rng = np.random.default_rng(9600)
    a = random_state(n, rng)
    s = QuantumState(n)
    s.load(a)
    terms = W.random_pauli_terms(n, 160, 1, 6, seed=9601)
    obs1 = observable(n, terms, rng.normal(size=len(terms)))
    set_expectation_specialized(0)
    generic = obs1.get_expectation_value(s)
    set_expectation_specialized(2)
    try:
        gen = obs1.get_expectation_value(s)
        assert abs(gen - generic) <= 1e-12
        coefs2 = rng.normal(size=len(terms))
        obs2 = observable(n, terms, coefs2)
        l0 = expectation_specialized_info()[0]
        e2 = obs2.get_expectation_value(s)
        assert expectation_specialized_info()[0] > l0
        want = oracle_sum(port, a, terms, coefs2).real
        assert abs(e2 - want) <= EV_TOL * float(np.sum(np.abs(coefs2)))
    finally:
        set_expectation_specialized(1)


def test_default_mode_generates_on_second_use():
    """Default policy: the first evaluation of a term list on >= 20 qubits runs the generic kernel, the
    second generates the pass kernels and runs them."""
    n = 20
    rng = np.random.default_rng(9700)
    s = QuantumState(n)
    s.load(random_state(n, rng))
    terms = W.random_pauli_terms(n, 64, 1, 5, seed=9701)
    obs = observable(n, terms, rng.normal(size=len(terms)))
    set_expectation_specialized(1)
    l0 = expectation_specialized_info()[0]
    e1 = obs.get_expectation_value(s)
    assert expectation_specialized_info()[0] == l0
    e2 = obs.get_expectation_value(s)
    assert expectation_specialized_info()[0] > l0
    assert abs(e1 - e2) <= 1e-12


def test_weighted_identity_repeated_and_zero_terms(port, kernels):
    """An identity term (coef x norm), the same string twice, a zero coefficient and a Y-only string:
    the weighted sum equals the oracle's."""
    n = 13
    rng = np.random.default_rng(9800)
    a = random_state(n, rng)
    s = QuantumState(n)
    s.load(a)
    terms = W.random_pauli_terms(n, 40, 1, 5, seed=9801)
    terms += [(0.0, [], []), terms[3], terms[7], (0.0, [2, 9], [2, 2]), (0.0, [0], [2])]
    coefs = rng.normal(size=len(terms))
    coefs[5] = 0.0
    obs = observable(n, terms, coefs)
    want = oracle_sum(port, a, terms, coefs).real
    assert abs(obs.get_expectation_value(s) - want) <= EV_TOL * float(np.sum(np.abs(coefs)))
