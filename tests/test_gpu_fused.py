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


@pytest.mark.parametrize("executor", ["tensor", "fp64"])
@pytest.mark.parametrize("n,kind", [(10, "u3cz"), (12, "layered"), (14, "u3cz"), (17, "mixed")])
def test_fused_against_oracle(port, n, kind, executor):
    """Both complex64 executors: 6-qubit blocks on the tensor cores, and FP64 passes over the
    complex64 state (whose only error is the complex64 storage)."""
    if kind == "u3cz":
        gates = W.u3_cz_circuit(n, 6, seed=n)
    elif kind == "layered":
        gates = W.layered_rotation_circuit(n, 4, seed=n)
    else:
        gates = W.u3_cz_circuit(n, 3, seed=n) + W.hea_circuit(n, 3, seed=n + 1)
    circ = W.to_circuit(gates, n)
    circ.set_c64_executor(executor)
    want = np.zeros(1 << n, dtype=np.complex128)
    want[0] = 1
    R.run_on_cpu(gates, want, port)
    ref = QuantumState(n)
    ref.load(want)
    s = QuantumStateC64(n)
    circ.update_quantum_state(s)
    assert circ.c64_executor_info() == executor
    inf = s.infidelity(ref)
    assert inf <= (INFIDELITY_TOL if executor == "tensor" else 1e-9), inf
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


@pytest.mark.parametrize("n", [26, 31])
def test_fused_large_tile_indices(n):
    """Sizes whose tile indices reach the upper 6-bit chunks of the kernel's tile-base tables (26
    qubits: three chunks; 31: all four): the tensor-core result against the complex128 staged
    executor, which is itself checked against the reference at 30 qubits."""
    import gc

    import torch
    gc.collect()  # states of earlier tests release their device memory
    torch.cuda.empty_cache()
    if torch.cuda.mem_get_info()[0] < (24 << n) + (2 << 30):  # complex128 + complex64 state
        pytest.skip(f"{n} qubits: not enough free device memory")
    gates = W.u3_cz_circuit(n, 6, seed=900 + n)
    circ = W.to_circuit(gates, n)
    ref = QuantumState(n)
    circ.update_quantum_state(ref, mode="staged")
    circ.set_c64_executor("tensor")
    s = QuantumStateC64(n)
    circ.update_quantum_state(s)
    assert circ.c64_executor_info() == "tensor"
    inf = s.infidelity(ref)
    assert inf <= INFIDELITY_TOL, inf
    # the norm drifts by the split-bf16 rounding of every block (1.2e-5 after this circuit's ~25)
    assert abs(s.get_squared_norm() - 1.0) <= EV_TOL_C64
    del s, ref


def test_fused_schedule_reduces_work():
    n = 20
    circ = W.to_circuit(W.u3_cz_circuit(n, 10, seed=3), n)
    passes, blocks = circ.fused_stats()
    assert passes < 60 and blocks < 300


def test_c64_fp64_passes_round_only_on_store(port):
    """FP64 passes over a complex64 state equal the complex128 staged path on the same circuit (block
    size 2) up to one complex64 rounding per pass: per amplitude within a few units of FP32 rounding."""
    n = 16
    gates = W.hea_circuit(n, 8, seed=41)
    circ = W.to_circuit(gates, n)
    circ.set_c64_executor("fp64")
    s = QuantumStateC64(n)
    circ.update_quantum_state(s)
    ref = QuantumState(n)
    circ.set_fusion(2)
    circ.update_quantum_state(ref, mode="staged_fused")
    passes = circ.fusion_info()[2]
    diff = np.max(np.abs(s.get_vector().astype(np.complex128) - ref.get_vector()))
    assert diff <= passes * 2 * np.finfo(np.float32).eps * float(np.max(np.abs(ref.get_vector()))) * 4, diff


def test_c64_auto_executor_choice():
    """Default executor: the tensor cores whenever they take the circuit (>= 10 qubits, gates of <= 6
    qubits), else FP64 passes (fewer than 10 qubits)."""
    from qulacs_b200 import gate as G
    for n in (10, 14):
        c = W.to_circuit(W.hea_circuit(n, 4, seed=5), n)
        c.update_quantum_state(QuantumStateC64(n))
        assert c.c64_executor_info() == "tensor"
    c = W.to_circuit(W.hea_circuit(12, 2, seed=7), 12)
    rng = np.random.default_rng(7)
    c.add_gate(G.DenseMatrix([0, 1, 2], np.linalg.qr(rng.normal(size=(8, 8)) + 1j * rng.normal(size=(8, 8)))[0]))
    c.update_quantum_state(QuantumStateC64(12))
    assert c.c64_executor_info() == "tensor"
    small = W.to_circuit(W.hea_circuit(8, 4, seed=8), 8)
    small.update_quantum_state(QuantumStateC64(8))
    assert small.c64_executor_info() == "fp64"
