"""Density-matrix kernels on the B200 against the oracle and the reference golden fixture."""
import os

import numpy as np
import pytest

from conftest import AMP_TOL, EV_TOL, GOLDEN, random_density_matrix, random_unitary
from qulacs_b200 import DensityMatrix, QuantumState, gate as G
from qulacs_b200 import workloads as W
from oracle import replay as R

pytestmark = pytest.mark.gpu


def dev(rho):
    d = DensityMatrix(int(np.log2(rho.shape[0])))
    d.load(rho)
    return d


def test_dm_gates_and_channels(port):
    rng = np.random.default_rng(1100)
    n = 5
    rho0 = random_density_matrix(n, rng)
    cases = [
        (G.DenseMatrix(3, random_unitary(1, rng)), lambda r, g: port.dm_single_qubit_dense_matrix_gate(3, g.get_matrix(), r)),
        (G.DenseMatrix([4, 1], random_unitary(2, rng)), lambda r, g: port.dm_multi_qubit_dense_matrix_gate([4, 1], g.get_matrix(), r)),
        (G.DenseMatrix([0, 2, 4], random_unitary(3, rng)), lambda r, g: port.dm_multi_qubit_dense_matrix_gate([0, 2, 4], g.get_matrix(), r)),
        (G.DenseMatrix([0, 1, 2, 4], random_unitary(4, rng)), lambda r, g: port.dm_multi_qubit_dense_matrix_gate([0, 1, 2, 4], g.get_matrix(), r)),
        (G.CNOT(4, 0), lambda r, g: port.dm_CNOT_gate(4, 0, r)),
        (G.CZ(1, 3), lambda r, g: port.dm_CZ_gate(1, 3, r)),
        (G.RX(2, 0.4), lambda r, g: port.dm_single_qubit_dense_matrix_gate(2, W.rotation_matrix("RX", 0.4), r)),
        (G.DepolarizingNoise(1, 0.05), lambda r, g: port.dm_depolarizing_noise(1, 0.05, r)),
        (G.TwoQubitDepolarizingNoise(3, 0, 0.07), lambda r, g: port.dm_two_qubit_depolarizing_noise(3, 0, 0.07, r)),
    ]
    for gate, oracle_fn in cases:
        want = rho0.copy()
        oracle_fn(want, gate)
        d = dev(rho0)
        gate.update_quantum_state(d)
        assert np.max(np.abs(d.get_matrix() - want)) <= AMP_TOL, gate


def test_dm_dense_gate_over_seven_qubits(port):
    """A 7-target unitary on an 8-qubit density matrix: two 7-qubit dense passes (rows, then columns)."""
    rng = np.random.default_rng(1150)
    n = 8
    rho0 = random_density_matrix(n, rng)
    tl = [6, 0, 3, 1, 7, 4, 2]
    u = random_unitary(7, rng)
    want = rho0.copy()
    port.dm_multi_qubit_dense_matrix_gate(tl, u, want)
    d = dev(rho0)
    G.DenseMatrix(tl, u).update_quantum_state(d)
    assert np.max(np.abs(d.get_matrix() - want)) <= AMP_TOL


@pytest.mark.parametrize("mode", ["gate_by_gate", "staged", "staged_fused"])
def test_noisy_circuit_golden_and_stats(port, mode):
    g = np.load(os.path.join(GOLDEN, "noisy_dm_n5.npz"))
    n = int(g["n"])
    gates = W.noisy_circuit(W.hea_circuit(n, int(g["depth"]), int(g["gate_seed"])), float(g["p"]))
    d = DensityMatrix(n)
    W.to_circuit(gates, n).update_quantum_state(d, mode=mode)
    rho = d.get_matrix()
    assert np.max(np.abs(rho - g["rho"])) <= AMP_TOL
    terms = W.random_pauli_terms(n, 16, 1, 3, int(g["term_seed"]))
    obs = W.to_observable(terms, n)
    assert np.max(np.abs(obs.term_values(d) - g["term_values"])) <= EV_TOL
    assert abs(d.get_squared_norm() - 1.0) <= 1e-12
    u = np.random.default_rng(5).random(512)
    assert np.array_equal(d.sampling_with_uniforms(u), port.dm_sampling_with_uniforms(rho, u))


def test_pure_state_density_matrix_matches_state_vector(port):
    n = 6
    s = QuantumState(n)
    circ = W.to_circuit(W.hea_circuit(n, 3, seed=9), n)
    circ.update_quantum_state(s)
    d = DensityMatrix(n)
    W.to_circuit(W.hea_circuit(n, 3, seed=9), n).update_quantum_state(d)
    v = s.get_vector()
    assert np.max(np.abs(d.get_matrix() - np.outer(v, v.conj()))) <= AMP_TOL
    d2 = DensityMatrix(n)
    d2.load(s)
    assert np.max(np.abs(d2.get_matrix() - np.outer(v, v.conj()))) <= AMP_TOL


@pytest.mark.parametrize("mode", ["gate_by_gate", "staged", "staged_fused"])
@pytest.mark.parametrize("n", [3, 7, 10])
def test_noisy_circuits_every_mode_against_oracle(port, mode, n):
    rng = np.random.default_rng(1200 + n)
    gates = W.noisy_circuit(W.hea_circuit(n, 2, 50 + n), 1e-3) + W.noisy_circuit(W.u3_cz_circuit(n, 2, 60 + n), 0.02)
    rho0 = random_density_matrix(n, rng)
    want = rho0.copy()
    R.run_on_cpu_dm(gates, want, port)
    d = dev(rho0)
    W.to_circuit(gates, n).update_quantum_state(d, mode=mode)
    assert np.max(np.abs(d.get_matrix() - want)) <= AMP_TOL


def test_large_noisy_density_matrix_properties():
    """At 13 qubits (2^26 entries, beyond the oracle): the staged modes agree with the gate-by-gate
    kernels, and the trace stays 1."""
    n = 13
    gates = W.noisy_circuit(W.hea_circuit(n, 2, 71), 1e-3)
    out = {}
    for mode in ("gate_by_gate", "staged", "staged_fused"):
        d = DensityMatrix(n)
        W.to_circuit(gates, n).update_quantum_state(d, mode=mode)
        assert abs(d.get_squared_norm() - 1.0) <= 1e-12
        out[mode] = d.get_matrix()
    assert np.max(np.abs(out["staged"] - out["gate_by_gate"])) <= AMP_TOL
    assert np.max(np.abs(out["staged_fused"] - out["gate_by_gate"])) <= AMP_TOL
