"""NoiseSimulator on the B200 against the oracle restatement of noisesimulator.cpp: same trajectories,
same sampled indices (except draws within 1e-12 of a cumulative boundary), same trajectory states."""
import numpy as np
import pytest

from conftest import AMP_TOL, BOUNDARY_EPS, random_state
from oracle.oracle import noise_simulator_execute
from qulacs_b200 import NoiseSimulator, QuantumState
from qulacs_b200 import workloads as W
from oracle import replay as R

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,p,shots,seed", [(6, 0.03, 300, 11), (9, 0.002, 1000, 12), (5, 0.2, 128, 13)])
def test_samples_match_oracle(port, n, p, shots, seed):
    gates = W.noisy_circuit(W.hea_circuit(n, 3, seed) + W.u3_cz_circuit(n, 1, seed + 1), p)
    circ = W.to_circuit(gates, n)
    got = NoiseSimulator(circ, seed=seed).execute(shots)
    want, near, _ = noise_simulator_execute(gates, n, shots, seed, port, lambda g, s: R.run_on_cpu([g], s, port),
                                            eps=BOUNDARY_EPS)
    assert got.shape == want.shape
    assert np.all((got == want) | near)


def test_trajectory_states_and_initial_state(port):
    n, p, shots, seed = 7, 0.04, 200, 21
    gates = W.noisy_circuit(W.hea_circuit(n, 2, 3), p)
    circ = W.to_circuit(gates, n)
    rng = np.random.default_rng(4)
    psi0 = random_state(n, rng)
    init = QuantumState(n)
    init.load(psi0)
    sim = NoiseSimulator(circ, init, seed=seed)
    res = sim.execute_and_get_result(shots)
    _, _, requests = noise_simulator_execute(gates, n, shots, seed, port, lambda g, s: R.run_on_cpu([g], s, port),
                                             init=psi0)
    assert [c for _, c in res.result] == [m for _, m in requests]
    from oracle.oracle import depolarizing_channel, _pauli
    for (state, count), (choice, m) in zip(res.result, requests):
        want = psi0.copy()
        ci = 0
        for g in gates:
            if g[0] == "DEPOL":
                kraus, _ = depolarizing_channel(list(g[1]), g[2])
                ids = kraus[choice[ci]]
                ci += 1
                if any(ids):
                    port.multi_qubit_dense_matrix_gate(list(g[1]), _pauli(ids), want)
            else:
                R.run_on_cpu([g], want, port)
        assert np.max(np.abs(state.get_vector() - want)) <= AMP_TOL
    # the all-identity trajectory is the noise-free circuit
    clean = QuantumState(n)
    clean.load(psi0)
    W.to_circuit([g for g in gates if g[0] != "DEPOL"], n).update_quantum_state(clean)
    last_state, _ = res.result[-1]
    assert np.max(np.abs(last_state.get_vector() - clean.get_vector())) <= AMP_TOL


def test_large_state_properties():
    """20 qubits: every sample is a valid index, shot counts add up, and a noise-free circuit gives
    the noise-free sampler's indices for the same uniforms."""
    n = 20
    gates = W.noisy_circuit(W.hea_circuit(n, 2, 31), 1e-3)
    circ = W.to_circuit(gates, n)
    sim = NoiseSimulator(circ, seed=5)
    s = sim.execute(512)
    assert s.shape == (512,) and int(s.max()) < (1 << n)
    assert int(sim.trajectories(512).sum()) == 512
