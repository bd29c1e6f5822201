"""The qulacs-name shim on the B200: whole-state arithmetic, entropy, Haar states, amplitudes, device
copies, density-matrix probabilities and arithmetic, observables applied to states, and circuits built
with the shim's adders -- against the oracle on the same inputs."""
import numpy as np
import pytest

from conftest import AMP_TOL, mt19937_64_uniforms, random_density_matrix, random_state
from qulacs_b200 import DensityMatrix, Observable, PauliOperator, QuantumCircuit, QuantumState
from qulacs_b200 import gate as G

pytestmark = pytest.mark.gpu


def dev(vec):
    s = QuantumState(int(np.log2(vec.size)))
    s.load(vec)
    return s


def dev_dm(rho):
    d = DensityMatrix(int(np.log2(rho.shape[0])))
    d.load(rho)
    return d


@pytest.mark.parametrize("n", [1, 5, 12, 20])
def test_state_arithmetic(port, n):
    rng = np.random.default_rng(900 + n)
    a, b = random_state(n, rng), random_state(n, rng)
    sa, sb = dev(a), dev(b)
    sa.add_state_with_coef(0.3 - 0.8j, sb)
    port.state_add_with_coef(0.3 - 0.8j, b, a)
    assert np.max(np.abs(sa.get_vector() - a)) <= AMP_TOL
    sa.add_state(sb)
    port.state_add_with_coef(1.0, b, a)
    assert np.max(np.abs(sa.get_vector() - a)) <= AMP_TOL
    sa.multiply_coef(-1.7 + 0.2j)
    port.state_multiply(-1.7 + 0.2j, a)
    assert np.max(np.abs(sa.get_vector() - a)) <= AMP_TOL
    nrm = sa.get_squared_norm()
    sa.normalize(nrm)
    port.normalize(port.state_norm_squared(a), a)
    assert np.max(np.abs(sa.get_vector() - a)) <= AMP_TOL
    assert abs(sa.get_squared_norm() - 1.0) <= 1e-12
    i = int(rng.integers(0, 1 << n))
    assert abs(sa.get_amplitude(i) - a[i]) <= AMP_TOL
    with pytest.raises(ValueError):
        sa.get_amplitude(1 << n)


@pytest.mark.parametrize("n", [3, 11, 18])
def test_entropy(port, n):
    rng = np.random.default_rng(950 + n)
    a = random_state(n, rng)
    a[::5] = 0  # probabilities under the 1e-15 clamp
    a /= np.linalg.norm(a)
    s = dev(a)
    assert abs(s.get_entropy() - port.measurement_distribution_entropy(a)) <= 1e-10
    rho = random_density_matrix(min(n, 8), rng)
    d = dev_dm(rho)
    assert abs(d.get_entropy() - port.dm_measurement_distribution_entropy(rho)) <= 1e-10
    basis = QuantumState(n)
    assert abs(basis.get_entropy() - port.measurement_distribution_entropy(basis.get_vector())) <= 1e-12


def test_haar_random_state():
    n = 16
    s, t, u = QuantumState(n), QuantumState(n), QuantumState(n)
    s.set_Haar_random_state(7)
    t.set_Haar_random_state(7)
    u.set_Haar_random_state(8)
    v, w = s.get_vector(), u.get_vector()
    assert np.array_equal(v, t.get_vector())
    assert abs(np.vdot(v, v).real - 1.0) <= 1e-12
    assert np.max(np.abs(v - w)) > 1e-3
    # Porter-Thomas: d |a|^2 is exponential(1) -> mean 1, variance 1; phases uniform
    p = (1 << n) * np.abs(v) ** 2
    assert abs(p.mean() - 1.0) <= 1e-9 and abs(p.var() - 1.0) < 0.05
    assert abs(np.mean(np.exp(1j * np.angle(v)))) < 0.02
    d = DensityMatrix(5)
    d.set_Haar_random_state(3)
    rho = d.get_matrix()
    assert abs(np.trace(rho) - 1.0) <= 1e-12
    assert abs(np.trace(rho @ rho) - 1.0) <= 1e-12
    assert np.max(np.abs(rho - rho.conj().T)) <= 1e-15


def test_copy_load_classical_register_and_elementwise():
    rng = np.random.default_rng(17)
    n = 10
    a = random_state(n, rng)
    s = dev(a)
    s.set_classical_value(3, 1)
    c = s.copy()
    assert np.array_equal(c.get_vector(), a) and c.get_classical_register() == [0, 0, 0, 1]
    t = s.allocate_buffer()
    assert t.get_vector()[0] == 1.0 and t.get_squared_norm() == 1.0
    t.load(s)
    assert np.array_equal(t.get_vector(), a) and t.get_classical_value(3) == 1
    with pytest.raises(TypeError):
        t.load(DensityMatrix(n))
    with pytest.raises(ValueError):
        t.add_state(QuantumState(n + 1))
    f = lambda i: np.exp(0.01j * i) * (1 + (i & 1))  # noqa: E731
    s.multiply_elementwise_function(f)
    expect = a * np.array([f(i) for i in range(1 << n)])
    assert np.max(np.abs(s.get_vector() - expect)) <= AMP_TOL
    z = dev(a)
    z.set_zero_norm_state()
    assert z.get_squared_norm() == 0.0
    assert "State vector" in QuantumState(2).to_string()


@pytest.mark.parametrize("n", [2, 6, 9])
def test_density_matrix_ops(port, n):
    rng = np.random.default_rng(1000 + n)
    rho, sig = random_density_matrix(n, rng), random_density_matrix(n, rng)
    d, e = dev_dm(rho), dev_dm(sig)
    for t in range(n):
        assert abs(d.get_zero_probability(t) - port.dm_M0_prob(t, rho)) <= 1e-13
    mv = [2] * n
    mv[0] = 1
    mv[n - 1] = 0 if n > 1 else 1
    tl = [i for i in range(n) if mv[i] != 2]
    assert abs(d.get_marginal_probability(mv) - port.dm_marginal_prob(tl, [mv[i] for i in tl], rho)) <= 1e-13
    d.add_state_with_coef(0.5j, e)
    r = rho + 0.5j * sig
    d.add_state(e)
    r = r + sig
    d.multiply_coef(0.25 - 0.1j)
    r = r * (0.25 - 0.1j)
    assert np.max(np.abs(d.get_matrix() - r)) <= AMP_TOL
    d2 = dev_dm(rho)
    d2.normalize(2.0)
    port.dm_normalize(2.0, rho)
    assert np.max(np.abs(d2.get_matrix() - rho)) <= AMP_TOL
    d3 = dev_dm(sig)
    got = d3.sampling(300, 99)
    expect = port.dm_sampling_with_uniforms(sig, mt19937_64_uniforms(99, 300))
    assert got == [int(x) for x in expect]
    b = DensityMatrix(n)
    b.set_computational_basis((1 << n) - 2)
    m = b.get_matrix()
    assert m[(1 << n) - 2, (1 << n) - 2] == 1.0 and np.count_nonzero(m) == 1
    c = b.copy()
    assert np.array_equal(c.get_matrix(), m)
    with pytest.raises(IndexError):
        b.set_computational_basis(1 << n)
    with pytest.raises(TypeError):
        b.add_state(QuantumState(n))


def _pauli_matrix(targets, ids, n):
    """Dense P on n qubits, bit j of the index <-> qubit j."""
    full = np.eye(1, dtype=np.complex128)
    d = dict(zip(targets, ids))
    for q in range(n):
        full = np.kron(G._PAULI[d.get(q, 0)], full)
    return full


@pytest.mark.parametrize("n", [3, 10])
def test_observable_transition_and_apply(n):
    rng = np.random.default_rng(1100 + n)
    a, b = random_state(n, rng), random_state(n, rng)
    o = Observable(n)
    o.add_random_operator(6, seed=n)
    o.add_operator(PauliOperator("X 0 Z 2", 0.3 + 0.2j))
    h = sum(t.get_coef() * _pauli_matrix(t.get_index_list(), t.get_pauli_id_list(), n) for t in o.terms)
    sa, sb = dev(a), dev(b)
    assert abs(o.get_transition_amplitude(sa, sb) - np.vdot(a, h @ b)) <= 1e-11
    p = o.get_term(6)
    assert abs(p.get_transition_amplitude(sa, sb)
               - (0.3 + 0.2j) * np.vdot(a, _pauli_matrix([0, 2], [1, 3], n) @ b)) <= 1e-12
    work, dst = QuantumState(n), QuantumState(n)
    o.apply_to_state(work, sb, dst)
    assert np.max(np.abs(dst.get_vector() - h @ b)) <= 1e-11
    assert np.array_equal(sb.get_vector(), b)


@pytest.mark.parametrize("mode", ["gate_by_gate", "staged", "staged_fused"])
def test_shim_circuit_against_oracle_and_inverse(port, mode):
    n = 9
    rng = np.random.default_rng(1200)
    c = QuantumCircuit(n)
    c.add_H_gate(0)
    c.add_Sdag_gate(1)
    c.add_Tdag_gate(2)
    c.add_sqrtX_gate(3)
    c.add_sqrtXdag_gate(4)
    c.add_sqrtY_gate(5)
    c.add_sqrtYdag_gate(6)
    c.add_RotInvX_gate(7, 0.3)
    c.add_RotInvY_gate(8, -0.4)
    c.add_RotInvZ_gate(0, 1.3)
    c.add_multi_Pauli_gate([1, 4, 8], [1, 2, 3])
    c.add_multi_Pauli_rotation_gate([0, 5, 6], [2, 2, 1], 0.77)
    c.add_random_unitary_gate([2, 7], 5)
    c.add_random_unitary_gate([3, 6, 1], 6)
    c.add_CNOT_gate(8, 0)
    c.add_gate(G.CZ(4, 5), 3)
    a = random_state(n, rng)
    s = dev(a)
    c.update_quantum_state(s, mode=mode)
    v = a.copy()
    for g in c.gate_list:
        k = g.kind
        if k == "PAULI":
            port.multi_qubit_Pauli_gate_partial_list(g.targets, g._pauli_ids(), v)
        elif k == "PAULI_ROTATION":
            port.multi_qubit_Pauli_rotation_gate_partial_list(g.targets, g._pauli_ids(), g.params[-1], v)
        elif k == "CNOT":
            port.CNOT_gate(g.targets[0], g.targets[1], v)
        elif k == "CZ":
            port.CZ_gate(g.targets[0], g.targets[1], v)
        elif k in ("RX", "RY", "RZ"):
            getattr(port, f"{k}_gate")(g.targets[0], g.params[0], v)
        else:
            port.multi_qubit_dense_matrix_gate(g.targets, g.get_matrix(), v)
    assert np.max(np.abs(s.get_vector() - v)) <= AMP_TOL
    c.get_inverse().update_quantum_state(s, mode=mode)
    assert np.max(np.abs(s.get_vector() - a)) <= AMP_TOL
