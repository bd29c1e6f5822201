"""The benchmark circuit at its full size (30 qubits, 16 GiB complex128: the layered RX/RY/RZ + CNOT
circuit, depth 10, gate seed 2124) against the REFERENCE csim's own result on the same inputs.

``tests/golden/config2_n30.npz`` holds what the reference csim computed gate by gate on the host
(``tests/golden/make_golden.py --config2``): 4096 amplitudes at seeded indices, <P_k> for 256 Pauli
strings of weight <= 6 (seed 2125) and the energy, and the indices it samples for 1024 supplied
uniforms (seed 2126), each flagged when the draw lies within 1e-12 of a cumulative boundary.  Every
execution mode of this library must give those amplitudes to 1e-12, each <P_k> and the energy to
1e-10, and the same sampled indices except flagged draws (counted and printed)."""
import gc
import os

import numpy as np
import pytest

from conftest import AMP_TOL, EV_TOL, ROOT
from qulacs_b200 import QuantumState
from qulacs_b200 import workloads as W

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(ROOT, "tests", "golden", "config2_n30.npz")


def _room_for(nbytes: int) -> bool:
    import torch
    gc.collect()
    torch.cuda.empty_cache()
    free, _ = torch.cuda.mem_get_info()
    return free >= nbytes + (2 << 30)


@pytest.fixture(scope="module")
def golden():
    if not os.path.exists(FIXTURE):
        pytest.skip("30-qubit reference fixture not generated")
    return np.load(FIXTURE)


@pytest.mark.parametrize("mode", ["staged_fused", "staged", "gate_by_gate"])
def test_30q_benchmark_circuit_matches_reference(golden, mode):
    n = int(golden["n"])
    if not _room_for(16 << n):
        pytest.skip(f"{16 << n >> 30} GiB of device memory not free")
    gates = W.layered_rotation_circuit(n, int(golden["depth"]), seed=int(golden["gate_seed"]))
    terms = W.random_pauli_terms(n, 256, 1, 6, seed=int(golden["term_seed"]))
    s = QuantumState(n)
    W.to_circuit(gates, n).update_quantum_state(s, mode=mode)

    idx, want = golden["amp_index"], golden["amps"]
    got = np.array([s.get_amplitude(int(i)) for i in idx])
    err = float(np.max(np.abs(got - want)))
    assert err <= AMP_TOL, (mode, err)
    assert abs(s.get_squared_norm() - float(golden["norm"])) <= 1e-10

    obs = W.to_observable(terms, n)
    vals = obs.term_values(s)
    assert float(np.max(np.abs(vals - golden["term_values"]))) <= EV_TOL
    assert abs(obs.get_expectation_value(s) - float(golden["energy"])) <= EV_TOL

    u = W.uniforms(1024, seed=int(golden["uniform_seed"]))
    samples = s.sampling_with_uniforms(u)
    near = golden["near_boundary"]
    differ = samples != golden["samples"]
    assert not np.any(differ & ~near), np.nonzero(differ & ~near)
    print(f"{mode}: max|d amp| = {err:.2e}, draws within 1e-12 of a boundary: {int(near.sum())}, "
          f"of which differing: {int((differ & near).sum())}")
    del s
