"""FP64 gate fusion on the host (CPU only): the fused gate list, replayed with the oracle, gives the
same state as the gate-by-gate oracle (cppsim QuantumCircuitOptimizer / gate::merge semantics,
circuit_optimizer.cpp:113-168, gate_merge.cpp:316-356), and every fused gate fits its block size."""
import numpy as np
import pytest

from conftest import AMP_TOL, random_state, random_unitary
from qulacs_b200 import QuantumCircuit
from qulacs_b200 import gate as G
from qulacs_b200 import workloads as W
from oracle import replay as R


def replay(fused, state, port):
    for qubits, m in fused:
        port.multi_qubit_dense_matrix_gate(qubits, m, state)


@pytest.mark.parametrize("k", [0, 1, 2, 3, 4])
def test_fused_lists_reproduce_the_circuit(port, k):
    n = 9
    rng = np.random.default_rng(40 + k)
    gates = W.layered_rotation_circuit(n, 3, seed=41) + W.u3_cz_circuit(n, 3, seed=42)
    for _ in range(12):
        q = int(rng.integers(2, 4))
        tl = tuple(int(x) for x in rng.choice(n, size=q, replace=False))
        gates.append(("DENSE", tl, random_unitary(q, rng)))
    gates += W.layered_rotation_circuit(n, 2, seed=43)
    circ = W.to_circuit(gates, n)
    fused = circ.fuse(k)
    if k == 0:
        assert len(fused) == len(gates)
    s0 = random_state(n, rng)
    want = s0.copy()
    R.run_on_cpu(gates, want, port)
    got = s0.copy()
    items = [fused[i] for i in range(len(fused))]
    replay(items, got, port)
    assert np.max(np.abs(got - want)) <= AMP_TOL
    for qubits, m in items:
        assert len(qubits) <= max(k, 3)
        assert np.allclose(m @ m.conj().T, np.eye(len(m)), atol=1e-12)


def test_layered_circuit_gate_counts():
    n, depth = 10, 10
    circ = W.to_circuit(W.layered_rotation_circuit(n, depth, seed=7), n)
    assert len(circ.fuse(0)) == depth * (3 * n + n - 1)
    # k = 1: each qubit's RX RY RZ run becomes one 2x2; the CNOT ladder stays
    f1 = circ.fuse(1)
    assert len(f1) == depth * (n + n - 1)
    assert len(circ.fuse(2)) < len(f1)


def test_controls_named_and_pauli_gates(port):
    n = 7
    rng = np.random.default_rng(5)
    circ = QuantumCircuit(n)
    ref = []  # (qubits, matrix) of each original gate, built here independently
    def add(gate, qubits, m):
        circ.add_gate(gate)
        ref.append((qubits, m))
    h = np.array([[1, 1], [1, -1]]) / np.sqrt(2)
    add(G.H(0), [0], h)
    u = random_unitary(1, rng)
    cu = G.DenseMatrix(2, u)
    cu.add_control_qubit(4, 1)
    full = np.eye(4, dtype=np.complex128)  # bit0 <-> target 2, bit1 <-> control 4
    full[np.ix_([2, 3], [2, 3])] = u
    add(cu, [2, 4], full)
    add(G.SWAP(1, 5), [1, 5], np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]]))
    add(G.RZ(3, 0.7), [3], W.rotation_matrix("RZ", 0.7))
    add(G.RZ(3, -0.2), [3], W.rotation_matrix("RZ", -0.2))
    x, z = np.array([[0, 1], [1, 0]]), np.diag([1, -1])
    pxz = np.kron(z, x)  # Pauli ids (X on 0, Z on 6): bit0 <-> qubit 0
    add(G.PauliRotation([0, 6], [1, 3], 0.3), [0, 6], np.cos(0.15) * np.eye(4) + 1j * np.sin(0.15) * pxz)
    d = np.exp(1j * rng.uniform(0, 6.28, size=4))
    add(G.DiagonalMatrix([1, 3], d), [1, 3], np.diag(d))
    cu0 = G.DenseMatrix(6, u)
    cu0.add_control_qubit(5, 0)
    full0 = np.eye(4, dtype=np.complex128)
    full0[np.ix_([0, 1], [0, 1])] = u
    add(cu0, [6, 5], full0)
    add(G.CNOT(2, 3), [2, 3], np.array([[1, 0, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0], [0, 1, 0, 0]]))
    s0 = random_state(n, rng)
    want = s0.copy()
    replay(ref, want, port)
    exported = circ.fuse(0)
    for i, (qubits, m) in enumerate(ref):
        eq, em = exported[i]
        assert eq == qubits and np.max(np.abs(em - m)) <= 1e-15
    for k in (1, 2, 3):
        fused = circ.fuse(k)
        got = s0.copy()
        replay([fused[i] for i in range(len(fused))], got, port)
        assert np.max(np.abs(got - want)) <= AMP_TOL
    # the two RZ on qubit 3 merge into one diagonal 2x2 at k = 1
    f1 = circ.fuse(1)
    assert any(q == [3] and abs(m[0, 1]) == 0 and abs(m[1, 0]) == 0 for q, m in (f1[i] for i in range(len(f1))))


def test_noise_channels_stay_unfused():
    n = 4
    circ = QuantumCircuit(n)
    circ.add_gate(G.RX(0, 0.1))
    circ.add_gate(G.DepolarizingNoise(0, 0.01))
    circ.add_gate(G.RX(0, 0.2))
    f = circ.fuse(2)
    assert len(f) == 3
    with pytest.raises(NotImplementedError):
        f[1]
