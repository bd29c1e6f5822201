"""Captured CUDA graphs: a circuit (three modes) or a batch recorded once and replayed equals the
direct call bit for bit (same kernels, same plans, same order), replays repeat, a replay without the
reset applies the circuit again, and work that cannot be recorded is refused with the context left
usable."""
import ctypes as C

import numpy as np
import pytest

from qulacs_b200 import QuantumState, QuantumStateC64
from qulacs_b200 import gate as G
from qulacs_b200 import workloads as W
from qulacs_b200._lib import call, load
from qulacs_b200.graph import capture_batch, capture_circuit
from oracle import replay as R

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["gate_by_gate", "staged", "staged_fused"])
def test_circuit_graph_equals_direct_call(port, mode):
    n = 14
    gates = W.layered_rotation_circuit(n, 3, seed=31) + W.u3_cz_circuit(n, 2, seed=32)
    circ = W.to_circuit(gates, n)
    if mode == "staged_fused":
        circ.set_fusion(4)  # 3..4-qubit blocks run as dense kernels whose matrices are kernel parameters
    direct = QuantumState(n)
    circ.update_quantum_state(direct, mode=mode)  # plans as the graph uses them
    direct.set_zero_state()
    circ.update_quantum_state(direct, mode=mode)
    s = QuantumState(n)
    s.set_Haar_random_state(5)  # the graph's reset makes this irrelevant
    g = capture_circuit(circ, s, mode=mode)
    assert g.kernel_count() > 0
    l0 = load().qs_launch_count()
    for _ in range(2):
        g.launch()
        assert np.array_equal(s.get_vector(), direct.get_vector())
    assert load().qs_launch_count() - l0 == 2 * g.kernel_count()
    psi = np.zeros(1 << n, dtype=np.complex128)
    psi[0] = 1
    R.run_on_cpu(gates, psi, port)
    assert np.max(np.abs(s.get_vector() - psi)) <= 1e-12
    g.close()


def test_circuit_graph_without_reset_applies_again():
    n = 12
    circ = W.to_circuit(W.hea_circuit(n, 4, seed=33), n)
    s = QuantumState(n)
    g = capture_circuit(circ, s, mode="staged", reset_state=False)  # capture records, does not run
    g.launch()
    g.launch()
    want = QuantumState(n)
    circ.update_quantum_state(want, mode="staged")
    circ.update_quantum_state(want, mode="staged")
    assert np.array_equal(s.get_vector(), want.get_vector())


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_batch_graph_equals_batch_call(precision):
    sizes = [6, 14, 11, 17, 9, 13]
    circs = [W.to_circuit(W.hea_circuit(n, 4 + i % 4, seed=3400 + i), n) for i, n in enumerate(sizes)]
    State = QuantumStateC64 if precision == "c64" else QuantumState
    direct = [State(n) for n in sizes]
    k = len(circs)
    ch = (C.c_void_p * k)(*[c._h for c in circs])
    if precision == "c64":
        call("qs_batch_update_quantum_states_c64", ch, (C.c_void_p * k)(*[s.data_ptr() for s in direct]), k, 1, None)
    else:
        call("qs_batch_update_quantum_states", ch, (C.c_void_p * k)(*[s.data_ptr() for s in direct]), k, None)
    states = [State(n) for n in sizes]
    g = capture_batch(circs, states)
    for _ in range(2):
        g.launch()
        for a, b in zip(states, direct):
            assert np.array_equal(a.get_vector(), b.get_vector())
    g.close()


def test_uncapturable_work_is_refused_and_context_stays_usable():
    n = 10
    rng = np.random.default_rng(35)
    circ = W.to_circuit(W.hea_circuit(n, 2, seed=35), n)
    u = np.linalg.qr(rng.normal(size=(64, 64)) + 1j * rng.normal(size=(64, 64)))[0]
    circ.add_gate(G.DenseMatrix([0, 2, 4, 5, 7, 9], u))  # a 6-qubit matrix is copied from host memory per run
    s = QuantumState(n)
    h = C.c_void_p()
    rc = load().qs_circuit_graph_create(circ._h, s.data_ptr(), s.dim, 0, 1, None, C.byref(h))
    assert rc == 5, load().qs_get_last_error()  # QS_ERR_NOT_SUPPORTED
    assert b"cannot be recorded" in load().qs_get_last_error()
    circ.update_quantum_state(s, mode="gate_by_gate")  # the context still works
    assert abs(s.get_squared_norm() - 1.0) <= 1e-12
