"""Fused complex64 tensor-core path on the B200 against the FP64 oracle.

Bar: infidelity 1 - |<psi|psi_FP64>|^2 <= 1e-6 (split-bf16 products, FP32 accumulation); the
per-term <P_k> error and the norm drift are stated and bounded loosely (single-precision state).
"""
import numpy as np
import pytest

from qulacs_b200 import QuantumState, QuantumStateC64
from qulacs_b200 import workloads as W
from oracle import replay as R

pytestmark = pytest.mark.gpu

INFIDELITY_TOL = 1e-6
EV_TOL_C64 = 1e-4


@pytest.mark.parametrize("n,kind", [(10, "u3cz"), (12, "layered"), (14, "u3cz"), (17, "mixed")])
def test_fused_against_oracle(port, n, kind):
    if kind == "u3cz":
        gates = W.u3_cz_circuit(n, 6, seed=n)
    elif kind == "layered":
        gates = W.layered_rotation_circuit(n, 4, seed=n)
    else:
        gates = W.u3_cz_circuit(n, 3, seed=n) + W.hea_circuit(n, 3, seed=n + 1)
    circ = W.to_circuit(gates, n)
    want = np.zeros(1 << n, dtype=np.complex128)
    want[0] = 1
    R.run_on_cpu(gates, want, port)
    ref = QuantumState(n)
    ref.load(want)
    s = QuantumStateC64(n)
    circ.update_quantum_state(s)
    inf = s.infidelity(ref)
    assert inf <= INFIDELITY_TOL, inf
    assert abs(s.get_squared_norm() - 1.0) <= 1e-5
    terms = W.random_pauli_terms(n, 24, 1, 4, seed=n + 7)
    obs = W.to_observable(terms, n)
    dev = obs.term_values(s)
    exact = np.array([port.expectation_value(tl, ids, want) for _, tl, ids in terms])
    assert np.max(np.abs(dev - exact)) <= EV_TOL_C64
    u = W.uniforms(512, seed=n)
    got = s.sampling_with_uniforms(u)
    ref_idx, near = port.sampling_with_uniforms(want, u, eps=1e-5)
    assert np.mean((got == ref_idx) | near) >= 0.99


def test_fused_schedule_reduces_work():
    n = 20
    circ = W.to_circuit(W.u3_cz_circuit(n, 10, seed=3), n)
    passes, blocks = circ.fused_stats()
    assert passes < 60 and blocks < 300
