"""NoiseSimulator trajectory selection on the host (CPU only): the Kraus order and cumulative
distributions follow the reference (gate_factory.cpp:451-500 reordered by optimize_ProbablisticGate,
gate_general.hpp:350-372), and the library's distinct trajectories and their shot counts equal the
oracle restatement of noisesimulator.cpp for the same seed."""
import numpy as np
import pytest

from oracle.oracle import depolarizing_channel, noise_simulator_execute
from qulacs_b200 import NoiseSimulator
from qulacs_b200 import workloads as W
from oracle import replay as R


def test_kraus_order_follows_the_reference():
    kraus, cum = depolarizing_channel([3], 0.06)
    assert kraus == [[0], [2], [3], [1]]  # I (1-p), then ties by descending index: Y, Z, X
    assert np.allclose(cum, [0, 0.94, 0.96, 0.98, 1.0])
    kraus2, cum2 = depolarizing_channel([0, 4], 0.15)
    assert kraus2[0] == [0, 0] and kraus2[1] == [15 % 4, 15 // 4] and kraus2[-1] == [1, 0]
    assert len(kraus2) == 16 and abs(cum2[-1] - 1.0) < 1e-15


@pytest.mark.parametrize("n,p,shots,seed", [(4, 0.05, 200, 7), (5, 0.01, 500, 8), (3, 0.3, 64, 9)])
def test_trajectories_match_oracle(port, n, p, shots, seed):
    gates = W.noisy_circuit(W.hea_circuit(n, 2, seed), p)
    circ = W.to_circuit(gates, n)
    got = NoiseSimulator(circ, seed=seed).trajectories(shots)
    _, _, requests = noise_simulator_execute(gates, n, shots, seed, port,
                                             lambda g, s: R.run_on_cpu([g], s, port))
    assert [c for _, c in requests] == got.tolist()
    assert int(got.sum()) == shots
