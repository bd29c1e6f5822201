"""The layered RX/RY/RZ + CNOT circuit (depth 10) at its full sizes, 30 qubits (16 GiB) and 33 qubits
(128 GiB), where the oracle cannot follow: size-independent properties only.

* circuit then its inverse returns |0...0> in every execution mode; the norm stays 1;
* at 30 qubits the three execution modes agree through device inner products (|<a|b>|^2 = 1);
* <P> of 256 strings (weight <= 6) from the many-strings-per-pass tiles equals the one-string-per-pass
  kernel on the same state, and sum c_k <P_k> equals the observable's <H> from the weighted passes
  (generic and generated kernels);
* sampling: seeded draws repeat, lie in [0, 2^n), and a basis state always yields its own index."""
import gc

import numpy as np
import pytest

from conftest import EV_TOL
from qulacs_b200 import PauliOperator, QuantumState, inner_product
from qulacs_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _room_for(nbytes: int) -> bool:
    import torch
    gc.collect()
    torch.cuda.empty_cache()
    free, _ = torch.cuda.mem_get_info()
    return free >= nbytes + (2 << 30)


def _inverse(gates):
    out = []
    for g in reversed(gates):
        out.append((g[0], g[1], -g[2]) if g[0] in ("RX", "RY", "RZ") else g)
    return out


@pytest.mark.parametrize("n", [30, 33])
def test_layered_circuit_round_trip_and_observables(n):
    states = 2 if n <= 30 else 1
    if not _room_for(states * (16 << n)):
        pytest.skip(f"{states} x {16 << n >> 30} GiB of device memory not free")
    gates = W.layered_rotation_circuit(n, 10, seed=2124)
    circ, inv = W.to_circuit(gates, n), W.to_circuit(_inverse(gates), n)
    modes = ["staged_fused", "staged"] + (["gate_by_gate"] if n <= 30 else [])
    s = QuantumState(n)
    for mode in modes:
        s.set_zero_state()
        circ.update_quantum_state(s, mode=mode)
        assert abs(s.get_squared_norm() - 1.0) <= 1e-10, mode
        inv.update_quantum_state(s, mode=mode)
        assert abs(s.get_marginal_probability([0] * n) - 1.0) <= 1e-10, mode

    s.set_zero_state()
    circ.update_quantum_state(s, mode="staged_fused")
    if states == 2:
        t = QuantumState(n)
        for mode in ("staged", "gate_by_gate"):
            t.set_zero_state()
            circ.update_quantum_state(t, mode=mode)
            assert abs(abs(inner_product(s, t)) ** 2 - 1.0) <= 1e-10, mode
        del t

    terms = W.random_pauli_terms(n, 256, 1, 6, seed=2125)
    obs = W.to_observable(terms, n)
    tiled = obs.term_values(s)
    single = np.array([PauliOperator(coef=1.0, targets=tl, pauli_ids=ids).get_expectation_value(s).real
                       for _, tl, ids in terms])
    assert np.max(np.abs(tiled - single)) <= EV_TOL
    coefs = np.array([c for c, _, _ in terms])
    assert abs(obs.get_expectation_value(s) - float(coefs @ single)) <= EV_TOL  # generic pass kernel
    from qulacs_b200.observable import set_expectation_specialized
    set_expectation_specialized(2)  # the per-pass generated kernels
    try:
        assert abs(obs.get_expectation_value(s) - float(coefs @ single)) <= EV_TOL
    finally:
        set_expectation_specialized(1)

    a, b = s.sampling(1024, 2126), s.sampling(1024, 2126)
    assert a == b and all(0 <= x < (1 << n) for x in a)
    x = (1 << n) - 3
    s.set_computational_basis(x)
    assert set(s.sampling(256, 7)) == {x}
