"""Host side of the qulacs-name shim (gate, QuantumCircuit, PauliOperator, Observable) without a GPU:
seeded constructions against the oracle's restatement of the reference's draws, gate inverses and
matrices, circuit editing, depth and text.  CPU only."""
import ctypes as C
import math

import numpy as np
import pytest

from oracle import oracle as O
from qulacs_b200 import Observable, PauliOperator, QuantumCircuit
from qulacs_b200 import gate as G
from qulacs_b200._lib import call


@pytest.mark.parametrize("k", [1, 2, 3, 4, 6])
@pytest.mark.parametrize("seed", [0, 1, 2024, 4294967295])
def test_random_unitary_matches_reference_draws(k, seed):
    g = G.RandomUnitary(list(range(k)), seed=seed)
    m = g.get_matrix()
    assert np.max(np.abs(m - O.random_unitary(k, seed))) <= 1e-12
    assert np.max(np.abs(m @ m.conj().T - np.eye(1 << k))) <= 1e-13


def test_random_unitary_unseeded_and_duplicates():
    a, b = G.RandomUnitary([0, 1]).get_matrix(), G.RandomUnitary([0, 1]).get_matrix()
    assert np.max(np.abs(a - b)) > 1e-3
    with pytest.raises(ValueError):
        G.RandomUnitary([1, 1], seed=3)


def test_std_normals_moments():
    # the restated polar method draws standard normals
    g = O.std_normals(11, 200000)
    assert abs(g.mean()) < 0.01 and abs(g.var() - 1.0) < 0.01


@pytest.mark.parametrize("n,count,seed", [(1, 5, 0), (4, 7, 99), (9, 30, 2**31 + 5)])
def test_random_operator_matches_reference_draws(n, count, seed):
    o = Observable(n)
    o.add_random_operator(count, seed=seed)
    expect = O.random_operator_terms(n, count, seed)
    assert o.get_term_count() == count
    for t, (ids, coef) in zip(o.terms, expect):
        assert t.get_index_list() == [q for q in range(n) if ids[q]]
        assert t.get_pauli_id_list() == [p for p in ids if p]
        assert t.get_coef() == coef
        assert -1.0 <= coef < 1.0


def _all_gates():
    rng = np.random.default_rng(5)
    return [G.X(0), G.Y(1), G.Z(2), G.H(0), G.S(1), G.Sdag(2), G.T(0), G.Tdag(1), G.sqrtX(2), G.sqrtXdag(0),
            G.sqrtY(1), G.sqrtYdag(2), G.Identity(0), G.RX(1, 0.3), G.RY(2, -1.1), G.RZ(0, 2.5), G.RotX(1, 0.7),
            G.U3(2, 0.1, 0.2, 0.3), G.DenseMatrix([0, 2], O.random_unitary(2, 8)),
            G.DiagonalMatrix([1, 2], np.exp(1j * rng.random(4))), G.CNOT(0, 2), G.CZ(1, 0), G.SWAP(2, 1),
            G.Pauli([0, 2], [2, 3]), G.PauliRotation([1, 0, 2], [1, 2, 3], 0.9)]


def test_inverse_is_adjoint():
    for g in _all_gates():
        inv = g.get_inverse()
        assert inv.get_target_index_list() == g.get_target_index_list(), g.get_name()
        m, mi = g.get_matrix(), inv.get_matrix()
        assert np.max(np.abs(mi - m.conj().T)) <= 1e-15, g.get_name()
    for g in (G.P0(0), G.P1(1), G.DepolarizingNoise(0, 0.1)):
        with pytest.raises(NotImplementedError):
            g.get_inverse()


def test_gate_matrices_follow_reference_conventions():
    a = 0.37
    c, s = math.cos(a / 2), math.sin(a / 2)
    # exp(+i a P / 2) for the csim rotations (update_ops_pauli_single.cpp:54-90)
    assert np.allclose(G.RX(0, a).get_matrix(), [[c, 1j * s], [1j * s, c]], atol=0)
    assert np.allclose(G.RY(0, a).get_matrix(), [[c, s], [-s, c]], atol=0)
    assert np.allclose(G.RZ(0, a).get_matrix(), np.diag([c + 1j * s, c - 1j * s]), atol=0)
    # Pauli product: bit j of the matrix index <-> targets[j]
    x = np.array([[0, 1], [1, 0]])
    z = np.diag([1, -1])
    assert np.array_equal(G.Pauli([4, 7], [1, 3]).get_matrix(), np.kron(z, x))
    assert np.allclose(G.PauliRotation([4, 7], [1, 3], a).get_matrix(),
                       c * np.eye(4) + 1j * s * np.kron(z, x), atol=1e-16)
    assert G.Z(0).is_diagonal() and G.CZ(0, 1).is_diagonal() and not G.H(0).is_diagonal()
    assert G.Pauli([0], [3]).is_diagonal() and not G.Pauli([0], [1]).is_diagonal()
    assert G.X(0).is_Pauli() and not G.S(0).is_Pauli()
    assert G.DepolarizingNoise(0, 0.1).get_name() == "Probabilistic"
    with pytest.raises(ValueError):
        G.Pauli([0, 0], [1, 2])


def test_multiply_scalar_and_controls():
    g = G.DenseMatrix([0], [[0, 1], [1, 0]])
    g.multiply_scalar(2j)
    assert np.array_equal(g.get_matrix(), [[0, 2j], [2j, 0]])
    g.add_control_qubit(3, 0)
    assert g.get_control_index_value_list() == [[3, 0]]
    with pytest.raises(ValueError):
        g.add_control_qubit(0, 1)


def _native_count(circ):
    out = C.c_uint()
    call("qs_circuit_gate_count", circ._h, C.byref(out))
    return out.value


def test_circuit_editing_keeps_native_list_in_step():
    c = QuantumCircuit(4)
    c.add_H_gate(0)
    c.add_CNOT_gate(0, 1)
    c.add_RZ_gate(1, 0.2)
    c.add_gate(G.X(3), 1)
    assert [g.get_name() for g in c.gate_list] == ["H", "X", "CNOT", "Z-rotation"]
    c.remove_gate(2)
    assert [g.get_name() for g in c.gate_list] == ["H", "X", "Z-rotation"]
    assert _native_count(c) == 3
    d = c.copy()
    d.merge_circuit(c)
    assert d.get_gate_count() == 6 and _native_count(d) == 6
    g = d.get_gate(0)
    g.name = "changed"
    assert d.gate_list[0].get_name() == "H"
    with pytest.raises(IndexError):
        c.remove_gate(5)
    with pytest.raises(IndexError):
        c.add_gate(G.X(0), 9)
    with pytest.raises(ValueError):
        c.add_X_gate(4)


def test_circuit_inverse_depth_and_text():
    c = QuantumCircuit(3)
    c.add_H_gate(0)
    c.add_CNOT_gate(0, 1)
    c.add_RX_gate(2, 0.1)
    c.add_CZ_gate(1, 2)
    c.add_S_gate(0)
    assert c.calculate_depth() == 3
    inv = c.get_inverse()
    assert [g.get_name() for g in inv.gate_list] == ["Sdag", "CZ", "X-rotation", "CNOT", "H"]
    assert inv.gate_list[2].params[0] == -0.1
    text = c.to_string()
    assert "# of qubit: 3" in text and "# of step : 3" in text and "# of 2 qubit gate: 2" in text
    assert QuantumCircuit(2).calculate_depth() == 0


def test_circuit_pauli_adders():
    c = QuantumCircuit(5)
    c.add_multi_Pauli_gate([0, 3], [1, 2])
    c.add_multi_Pauli_gate(PauliOperator("Z 1 X 4"))
    c.add_multi_Pauli_rotation_gate([2], [3], 0.5)
    c.add_multi_Pauli_rotation_gate(PauliOperator("Y 0 Y 1", 0.25))
    c.add_random_unitary_gate([1, 4], 17)
    kinds = [g.kind for g in c.gate_list]
    assert kinds == ["PAULI", "PAULI", "PAULI_ROTATION", "PAULI_ROTATION", "DENSE"]
    assert c.gate_list[3].params[-1] == 0.25
    with pytest.raises(ValueError):
        c.add_multi_Pauli_rotation_gate(PauliOperator("Y 0", 0.25j))
    assert _native_count(c) == 5


def test_pauli_operator_strings():
    p = PauliOperator("X 0 I 2 z 3", 0.5)
    assert p.get_index_list() == [0, 3] and p.get_pauli_id_list() == [1, 3]
    assert p.get_pauli_string() == "X 0 Z 3"
    p.add_single_Pauli(5, 2)
    assert p.get_pauli_string() == "X 0 Z 3 Y 5"
    q = p.copy()
    q.change_coef(-1.0)
    assert p.get_coef() == 0.5 and q.get_coef() == -1.0
    with pytest.raises(ValueError):
        PauliOperator("X 0 Y")
    with pytest.raises(ValueError):
        PauliOperator("W 0")
    o = Observable(6)
    o.add_operator(p)
    assert o.get_term(0).get_pauli_string() == "X 0 Z 3 Y 5"
    assert o.get_state_dim() == 64


def test_gate_merge_add_to_matrix_and_fused_swap():
    h, x, rz = G.H(0), G.X(0), G.RZ(0, 0.3)
    assert np.allclose(G.merge(h, x).get_matrix(), x.get_matrix() @ h.get_matrix(), atol=1e-15)
    assert np.allclose(G.add(h, rz).get_matrix(), h.get_matrix() + rz.get_matrix(), atol=1e-15)
    # union order: the first gate's qubits, then the new ones; bit j <-> union[j]
    m = G.merge(G.H(1), G.CNOT(1, 0))
    assert m.get_target_index_list() == [1, 0]
    cnot = np.eye(4)[:, [0, 3, 2, 1]]  # control = bit 0 (qubit 1), target = bit 1 (qubit 0)
    assert np.allclose(m.get_matrix(), cnot @ np.kron(np.eye(2), h.get_matrix()), atol=1e-15)
    c = G.to_matrix_gate(G.CZ(3, 1))
    assert c.get_target_index_list() == [3, 1] and np.array_equal(np.diag(c.get_matrix()), [1, 1, 1, -1])
    d = G.DenseMatrix([2], G.X(2).get_matrix())
    d.add_control_qubit(0, 0)
    t = G.to_matrix_gate(d)
    assert t.get_target_index_list() == [2, 0]
    assert np.array_equal(t.get_matrix().real, np.eye(4)[:, [1, 0, 2, 3]])  # flips bit 0 where bit 1 = 0
    f = G.FusedSWAP(0, 3, 2)
    assert f.get_target_index_list() == [0, 1, 3, 4]
    x = np.arange(16)
    assert np.array_equal(np.argmax(f.get_matrix(), axis=0), (x >> 2) | ((x & 3) << 2))
    with pytest.raises(ValueError):
        G.FusedSWAP(0, 1, 2)
    with pytest.raises(NotImplementedError):
        G.merge(G.DepolarizingNoise(0, 0.1), h)


def test_observable_copy_hermitian_and_matrix():
    o = Observable(3)
    o.add_operator(PauliOperator("X 0 Z 2", 0.5))
    o.add_operator(PauliOperator("Y 1", -0.25))
    c = o.copy()
    c.terms[0].change_coef(9.0)
    assert o.get_term(0).get_coef() == 0.5
    assert o.is_hermitian()
    x, y, z = np.array([[0, 1], [1, 0]]), np.array([[0, -1j], [1j, 0]]), np.diag([1, -1])
    want = 0.5 * np.kron(z, np.kron(np.eye(2), x)) - 0.25 * np.kron(np.eye(2), np.kron(y, np.eye(2)))
    assert np.allclose(o.get_matrix(), want, atol=0)
    o.add_operator(PauliOperator("Z 1", 0.1j))
    assert not o.is_hermitian()
    c2 = QuantumCircuit(8)
    c2.add_FusedSWAP_gate(0, 4, 2)
    assert c2.gate_list[0].get_name() == "FusedSWAP" and c2.gate_list[0].get_target_index_list() == [0, 1, 4, 5]
