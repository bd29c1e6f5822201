"""Host logic: synthetic workload shapes, Pauli masks, gate matrices (CPU only)."""
import numpy as np

from qulacs_b200 import gate as G
from qulacs_b200 import observable as OB
from qulacs_b200 import workloads as W


def test_gate_counts_match_configs():
    assert len(W.layered_rotation_circuit(16, 10, 1)) == 630
    assert len(W.layered_rotation_circuit(30, 10, 1)) == 1190
    assert len(W.layered_rotation_circuit(33, 10, 1)) == 1310
    assert len(W.u3_cz_circuit(32, 20, 1)) == 960


def test_generators_deterministic():
    assert W.layered_rotation_circuit(8, 3, 7) == W.layered_rotation_circuit(8, 3, 7)
    a = W.random_pauli_terms(30, 256, 1, 6, 9)
    assert a == W.random_pauli_terms(30, 256, 1, 6, 9)
    assert all(1 <= len(t[1]) <= 6 and len(set(t[1])) == len(t[1]) for t in a)


def test_pauli_masks():
    x, z, ny = OB.masks([0, 2, 5], [1, 2, 3])
    assert x == 0b101 and z == 0b100100 and ny == 1


def test_u3_is_unitary_and_matches_ibmq():
    m = W.u3_matrix(0.3, 1.1, -0.7)
    assert np.allclose(m @ m.conj().T, np.eye(2), atol=1e-15)
    assert np.allclose(G.get_IBMQ_matrix(0.3, 1.1, -0.7), m)


def test_noise_attachment_rule():
    g = W.noisy_circuit([("RX", 1, 0.2), ("CNOT", 0, 3)], 1e-3)
    assert g[1] == ("DEPOL", (1,), 1e-3)
    assert g[3] == ("DEPOL", (3, 0), 1e-3)  # targets then controls (circuit.cpp:171-176)


def test_named_gate_matrices():
    assert np.allclose(G.H(0).get_matrix() @ G.H(0).get_matrix(), np.eye(2))
    assert np.allclose(G.sqrtX(0).get_matrix() @ G.sqrtX(0).get_matrix(), [[0, 1], [1, 0]])
    assert np.allclose(G.sqrtY(0).get_matrix() @ G.sqrtY(0).get_matrix(), [[0, -1j], [1j, 0]])


def test_reference_rng_restatement():
    """std::mt19937_64 default seed 5489: the 10000th output is 9981545732273789042 (C++ [rand.predef])."""
    from conftest import mt19937_64_uniforms
    u = mt19937_64_uniforms(5489, 10000)
    assert u[-1] == float(9981545732273789042) / 2.0 ** 64


def test_library_rng_matches_restatement(lib):
    import ctypes as C
    from conftest import mt19937_64_uniforms
    out = np.zeros(500)
    assert lib.qs_reference_uniforms(1234, 500, out.ctypes.data_as(C.c_void_p)) == 0
    assert np.array_equal(out, mt19937_64_uniforms(1234, 500))


def test_staged_planner_pass_counts():
    """Host-only scheduler: passes needed by the staged executor (one HBM read+write each)."""
    c = W.to_circuit(W.layered_rotation_circuit(30, 10, 1), 30)
    p = c.pass_count()
    assert 1 <= p <= 40  # vs 1190 gate-by-gate passes
    c = W.to_circuit(W.layered_rotation_circuit(3, 2, 1), 3)
    assert c.pass_count() == c.get_gate_count()  # below 4 qubits: gate by gate
