"""Density-matrix circuits as 2n-qubit vector circuits (CPU only): U on the row qubits, conj(U) on the
column qubits, depolarizing channels as superoperators (gate_factory.cpp:451-500 weights,
gate_general.hpp:265-285 mixture).  Replayed with the oracle on the flattened rho, they must give
the oracle's density-matrix result."""
import numpy as np
import pytest

from conftest import AMP_TOL, random_density_matrix, random_unitary
from qulacs_b200 import QuantumCircuit
from qulacs_b200 import gate as G
from qulacs_b200 import workloads as W
from oracle import replay as R


def replay_vector(circ, rho, port):
    n = circ.qubit_count
    vec = circ.density_matrix_as_vector()
    v = rho.reshape(-1).copy()  # index = row * 2^n + col
    for i in range(len(vec)):
        qubits, m = vec[i]
        assert all(0 <= q < 2 * n for q in qubits)
        port.multi_qubit_dense_matrix_gate(qubits, m, v)
    return v.reshape(rho.shape)


@pytest.mark.parametrize("n,seed", [(3, 1), (4, 2), (5, 3)])
def test_noisy_hea_vector_matches_oracle(port, n, seed):
    gates = W.noisy_circuit(W.hea_circuit(n, 2, seed), 0.03) + W.noisy_circuit(W.u3_cz_circuit(n, 1, seed + 7), 0.05)
    rng = np.random.default_rng(seed)
    rho0 = random_density_matrix(n, rng)
    want = rho0.copy()
    R.run_on_cpu_dm(gates, want, port)
    got = replay_vector(W.to_circuit(gates, n), rho0, port)
    assert np.max(np.abs(got - want)) <= AMP_TOL


def test_pauli_controls_and_diagonals(port):
    n = 4
    rng = np.random.default_rng(9)
    circ = QuantumCircuit(n)
    gates = [G.PauliRotation([0, 2], [2, 1], 0.37),       # one Y: conj(P) = -P
             G.PauliRotation([1, 3], [2, 2], -0.9),       # two Y
             G.Pauli([0, 1, 3], [2, 3, 1]),               # one Y: global sign of P (x) conj(P)
             G.DiagonalMatrix([1, 2], np.exp(1j * rng.uniform(0, 6.28, 4))),
             G.SWAP(0, 3), G.H(2), G.RZ(1, 0.25)]
    cu = G.DenseMatrix(1, random_unitary(1, rng))
    cu.add_control_qubit(3, 0)
    gates.append(cu)
    gates.append(G.TwoQubitDepolarizingNoise(2, 0, 0.11))
    gates.append(G.DepolarizingNoise(3, 0.2))
    for g in gates:
        circ.add_gate(g)
    rho0 = random_density_matrix(n, rng)
    want = rho0.copy()
    unitary = circ.fuse(0)  # each gate's full matrix (noise channels raise)
    for i, g in enumerate(gates):
        if g.kind == "DEPOLARIZING":
            t = g.get_target_index_list()
            if len(t) == 1:
                port.dm_depolarizing_noise(t[0], float(g.params[0]), want)
            else:
                port.dm_two_qubit_depolarizing_noise(t[0], t[1], float(g.params[0]), want)
        else:
            qubits, m = unitary[i]
            port.dm_multi_qubit_dense_matrix_gate(qubits, m, want)
    got = replay_vector(circ, rho0, port)
    assert np.max(np.abs(got - want)) <= AMP_TOL
    # trace and hermiticity survive
    assert abs(np.trace(got) - np.trace(rho0)) <= 1e-12
    assert np.max(np.abs(got - got.conj().T)) <= 1e-12
