"""Pin the oracle restatement (oracle/qs_oracle.c) to the reference csim compiled from its sources,
and to the reference's own known-answer tests.  CPU only."""
import math

import numpy as np
import pytest

from conftest import random_density_matrix, random_state, random_unitary

PIN_TOL = 1e-14


def _both(port, ref, fn_name, s0, *args):
    a, b = s0.copy(), s0.copy()
    getattr(port, fn_name)(*args, a)
    getattr(ref, fn_name)(*args, b)
    return a, b


@pytest.mark.parametrize("n", [1, 3, 7])
def test_single_qubit_gates(port, ref, n):
    rng = np.random.default_rng(n)
    s0 = random_state(n, rng)
    for t in range(n):
        m = random_unitary(1, rng)
        a, b = _both(port, ref, "single_qubit_dense_matrix_gate", s0, t, m)
        assert np.max(np.abs(a - b)) <= PIN_TOL
        d = np.exp(1j * rng.normal(size=2))
        a, b = _both(port, ref, "single_qubit_diagonal_matrix_gate", s0, t, d)
        assert np.max(np.abs(a - b)) <= PIN_TOL
        for g in ("RX_gate", "RY_gate", "RZ_gate"):
            ang = float(rng.uniform(0, 2 * math.pi))
            a, b = _both(port, ref, g, s0, t, ang)
            assert np.max(np.abs(a - b)) <= PIN_TOL, g


def test_two_qubit_named(port, ref):
    rng = np.random.default_rng(5)
    n = 6
    s0 = random_state(n, rng)
    for c in range(n):
        for t in range(n):
            if c == t:
                continue
            for g in ("CNOT_gate", "CZ_gate", "SWAP_gate"):
                a, b = _both(port, ref, g, s0, c, t)
                assert np.max(np.abs(a - b)) == 0.0, (g, c, t)


@pytest.mark.parametrize("k", [2, 3, 4, 5, 6])
def test_dense_multi(port, ref, k):
    rng = np.random.default_rng(10 + k)
    n = 8
    s0 = random_state(n, rng)
    for _ in range(3):
        tl = [int(x) for x in rng.choice(n, size=k, replace=False)]
        m = random_unitary(k, rng)
        a, b = _both(port, ref, "multi_qubit_dense_matrix_gate", s0, tl, m)
        assert np.max(np.abs(a - b)) <= PIN_TOL
    if k == 2:
        a, b = _both(port, ref, "double_qubit_dense_matrix_gate_c", s0, 5, 1, m)
        assert np.max(np.abs(a - b)) <= PIN_TOL


def test_pauli_gates_and_controls(port, ref):
    rng = np.random.default_rng(21)
    n = 7
    s0 = random_state(n, rng)
    for _ in range(5):
        w = int(rng.integers(1, 5))
        tl = [int(x) for x in rng.choice(n, size=w, replace=False)]
        ids = [int(x) for x in rng.integers(0, 4, size=w)]
        a, b = _both(port, ref, "multi_qubit_Pauli_gate_partial_list", s0, tl, ids)
        assert np.max(np.abs(a - b)) <= PIN_TOL
        a, b = _both(port, ref, "multi_qubit_Pauli_rotation_gate_partial_list", s0, tl, ids, 0.37)
        assert np.max(np.abs(a - b)) <= PIN_TOL
    m = random_unitary(1, rng)
    a, b = _both(port, ref, "multi_qubit_control_single_qubit_dense_matrix_gate", s0, [2, 5], [1, 0], 3, m)
    assert np.max(np.abs(a - b)) <= PIN_TOL
    d = np.exp(1j * rng.normal(size=8))
    a, b = _both(port, ref, "multi_qubit_diagonal_matrix_gate", s0, [4, 0, 6], d)
    assert np.max(np.abs(a - b)) <= PIN_TOL


def test_stats(port, ref):
    rng = np.random.default_rng(31)
    n = 9
    s = random_state(n, rng)
    s2 = random_state(n, rng)
    assert abs(port.state_norm_squared(s) - ref.state_norm_squared(s)) <= 1e-13
    assert abs(port.state_inner_product(s, s2) - ref.state_inner_product(s, s2)) <= 1e-13
    for t in range(n):
        assert abs(port.M0_prob(t, s) - ref.M0_prob(t, s)) <= 1e-13
        assert abs(port.M1_prob(t, s) - ref.M1_prob(t, s)) <= 1e-13
    assert abs(port.marginal_prob([1, 4], [1, 0], s) - ref.marginal_prob([1, 4], [1, 0], s)) <= 1e-13
    for _ in range(40):
        w = int(rng.integers(1, 7))
        tl = [int(x) for x in rng.choice(n, size=w, replace=False)]
        ids = [int(x) for x in rng.integers(0, 4, size=w)]
        assert abs(port.expectation_value(tl, ids, s) - ref.expectation_value(tl, ids, s)) <= 1e-13


def test_sampling_same_indices(port, ref):
    rng = np.random.default_rng(41)
    s = random_state(10, rng)
    u = rng.random(4096)
    u[0] = 0.0  # -> index -1 (2^64 - 1), state.hpp:925-927
    assert np.array_equal(port.sampling_with_uniforms(s, u), ref.sampling_with_uniforms(s, u))
    assert port.sampling_with_uniforms(s, [0.0])[0] == np.uint64(2**64 - 1)
    # sub-normalised state: r > total -> dim
    assert ref.sampling_with_uniforms(0.5 * s, [0.9])[0] == 1 << 10


def test_density_matrix_ops(port, ref):
    rng = np.random.default_rng(51)
    n = 4
    rho = random_density_matrix(n, rng)

    def cmp(fn, *args):
        a, b = rho.copy(), rho.copy()
        getattr(port, fn)(*args, a)
        getattr(ref, fn)(*args, b)
        return np.max(np.abs(a - b))

    assert cmp("dm_single_qubit_dense_matrix_gate", 2, random_unitary(1, rng)) <= PIN_TOL
    assert cmp("dm_multi_qubit_dense_matrix_gate", [3, 0], random_unitary(2, rng)) <= PIN_TOL
    assert cmp("dm_multi_qubit_dense_matrix_gate", [1, 3, 0], random_unitary(3, rng)) <= PIN_TOL
    assert cmp("dm_CNOT_gate", 3, 1) == 0.0
    assert cmp("dm_CZ_gate", 0, 2) == 0.0
    assert cmp("dm_depolarizing_noise", 2, 0.1) <= PIN_TOL
    assert cmp("dm_two_qubit_depolarizing_noise", 1, 3, 0.07) <= PIN_TOL
    for tl, ids in [([1, 2], [2, 3]), ([0], [1]), ([0, 1, 3], [3, 3, 2])]:
        assert abs(port.dm_expectation_value(tl, ids, rho) - ref.dm_expectation_value(tl, ids, rho)) <= 1e-14
    u = rng.random(256)
    assert np.array_equal(port.dm_sampling_with_uniforms(rho, u), ref.dm_sampling_with_uniforms(rho, u))


def test_state_arithmetic_and_entropy(port, ref):
    rng = np.random.default_rng(61)
    s, s2 = random_state(8, rng), random_state(8, rng)
    for fn, args in [("state_add_with_coef", (0.3 - 1.1j, s2)), ("state_multiply", (-0.2 + 0.7j,)),
                     ("normalize", (2.5,))]:
        a, b = _both(port, ref, fn, s, *args)
        assert np.max(np.abs(a - b)) <= PIN_TOL, fn
    sparse = s.copy()
    sparse[::3] = 0  # entries below the 1e-15 clamp
    for v in (s, sparse):
        assert abs(port.measurement_distribution_entropy(v) - ref.measurement_distribution_entropy(v)) <= 1e-13
    rho = random_density_matrix(4, rng)
    assert abs(port.dm_measurement_distribution_entropy(rho) - ref.dm_measurement_distribution_entropy(rho)) <= 1e-13
    a, b = rho.copy(), rho.copy()
    port.dm_normalize(1.7, a)
    ref.dm_normalize(1.7, b)
    assert np.max(np.abs(a - b)) <= PIN_TOL


def test_dm_probabilities(port, ref):
    rng = np.random.default_rng(71)
    n = 5
    rho = random_density_matrix(n, rng)
    for t in range(n):
        assert abs(port.dm_M0_prob(t, rho) - ref.dm_M0_prob(t, rho)) <= 1e-14
        assert abs(port.dm_M1_prob(t, rho) - ref.dm_M1_prob(t, rho)) <= 1e-14
        assert abs(port.dm_M0_prob(t, rho) + port.dm_M1_prob(t, rho) - 1.0) <= 1e-13
    for tl, vals in [([0, 3], [1, 0]), ([1, 2, 4], [1, 1, 0]), ([4], [1])]:
        assert abs(port.dm_marginal_prob(tl, vals, rho) - ref.dm_marginal_prob(tl, vals, rho)) <= 1e-14


# ---- known-answer tests restated from the reference's own test suite ----

def test_kat_sampling_computational_basis(port):
    """test/cppsim/test_state.cpp:38-47: basis 100 -> every sample is 100."""
    s = np.zeros(1 << 10, dtype=np.complex128)
    s[100] = 1.0
    out = port.sampling_with_uniforms(s, np.random.default_rng(0).random(1024))
    assert np.all(out == 100)


def test_kat_sampling_superposition_order(port):
    """test/cppsim/test_state.cpp:49-81: amplitudes prop. to 2^i -> counts increase with i."""
    n = 5
    s = np.array([math.sqrt(2.0 ** i) for i in range(1 << n)], dtype=np.complex128)
    s /= np.linalg.norm(s)
    out = port.sampling_with_uniforms(s, np.random.default_rng(1).random(100000))
    cnt = np.bincount(out.astype(np.int64), minlength=1 << n)
    assert np.all(np.diff(cnt[-8:]) > 0)


def test_kat_depolarizing_identity(port):
    """test/cppsim/test_noise_dm.cpp:274-309: DepolarizingNoise(0, 3p/4) = (1-p) rho + p I/2 (1 qubit)."""
    rng = np.random.default_rng(3)
    rho = random_density_matrix(1, rng)
    p = 0.2
    r = rho.copy()
    port.dm_depolarizing_noise(0, 3 * p / 4, r)
    assert np.max(np.abs(r - ((1 - p) * rho + p * np.eye(2) / 2))) <= 1e-14


def test_kat_two_qubit_depolarizing_identity(port):
    """test/cppsim/test_noise_dm.cpp:311-348: TwoQubitDepolarizingNoise(0, 1, 15p/16) = (1-p) rho + p I/4."""
    rng = np.random.default_rng(4)
    rho = random_density_matrix(2, rng)
    p = 0.3
    r = rho.copy()
    port.dm_two_qubit_depolarizing_noise(0, 1, 15 * p / 16, r)
    assert np.max(np.abs(r - ((1 - p) * rho + p * np.eye(4) / 4))) <= 1e-14


def test_kat_expectation_against_dense_matrices(port):
    """test/csim/test_stat.cpp:200-430 pattern: <psi|P|psi> against the Kronecker-expanded Pauli matrix."""
    rng = np.random.default_rng(6)
    n = 4
    P = [np.eye(2), np.array([[0, 1], [1, 0]]), np.array([[0, -1j], [1j, 0]]), np.diag([1, -1])]
    s = random_state(n, rng)
    for _ in range(20):
        ids_full = [int(x) for x in rng.integers(0, 4, size=n)]
        m = np.array([[1.0]])
        for q in reversed(range(n)):
            m = np.kron(m, P[ids_full[q]])
        want = np.real(np.vdot(s, m @ s))
        got = port.expectation_value(list(range(n)), ids_full, s)
        assert abs(got - want) <= 1e-12
        # <0|X|0> = 0 (test/cppsim/test_hamiltonian.cpp:24-40)
    z = np.zeros(1 << n, dtype=np.complex128)
    z[0] = 1
    assert port.expectation_value([0], [1], z) == 0.0


def test_kat_dense_matrix_bit_order(port):
    """test/csim/test_update_dense.cpp:100-115: matrix = kron(U_t1, U_t0) for targets (t0, t1)."""
    rng = np.random.default_rng(8)
    n = 5
    s = random_state(n, rng)
    u0, u1 = random_unitary(1, rng), random_unitary(1, rng)
    a = s.copy()
    port.multi_qubit_dense_matrix_gate([1, 3], np.kron(u1, u0), a)
    b = s.copy()
    port.single_qubit_dense_matrix_gate(1, u0, b)
    port.single_qubit_dense_matrix_gate(3, u1, b)
    assert np.max(np.abs(a - b)) <= 1e-14
