"""The remaining csim entry points (single-qubit Pauli forms, whole-list Pauli forms, controlled
multi-target dense and diagonal gates, single-qubit and whole-list <P>, whole-list transition
amplitudes, and the density-matrix named, Pauli and controlled gates) on the B200 against the oracle."""
import ctypes as C

import numpy as np
import pytest

from conftest import AMP_TOL, EV_TOL, random_density_matrix, random_state, random_unitary
from qulacs_b200 import DensityMatrix, QuantumState
from qulacs_b200 import gate as G
from qulacs_b200._lib import call

pytestmark = pytest.mark.gpu


def _p(a):
    return np.ascontiguousarray(a).ctypes.data_as(C.c_void_p)


def _u32(x):
    return np.asarray(x, dtype=np.uint32)


def dev(vec):
    s = QuantumState(int(np.log2(vec.size)))
    s.load(vec)
    return s


def dev_dm(rho):
    d = DensityMatrix(int(np.log2(rho.shape[0])))
    d.load(rho)
    return d


def test_single_qubit_and_whole_list_pauli_gates(port):
    rng = np.random.default_rng(1300)
    n = 9
    s0 = random_state(n, rng)
    for pid in range(4):
        for t in (0, 4, 8):
            s = dev(s0)
            call("qs_single_qubit_Pauli_gate", t, pid, s.data_ptr(), s.dim, None)
            want = s0.copy()
            port.multi_qubit_Pauli_gate_partial_list([t], [pid], want)
            assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL, (pid, t)
            s = dev(s0)
            call("qs_single_qubit_Pauli_rotation_gate", t, pid, 0.77, s.data_ptr(), s.dim, None)
            want = s0.copy()
            if pid:
                getattr(port, ("RX", "RY", "RZ")[pid - 1] + "_gate")(t, 0.77, want)
            assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL, (pid, t)
    with pytest.raises(ValueError):
        call("qs_single_qubit_Pauli_gate", 0, 4, s.data_ptr(), s.dim, None)
    for count in (n, 5):
        ids = rng.integers(0, 4, size=count).astype(np.uint32)
        s = dev(s0)
        call("qs_multi_qubit_Pauli_gate_whole_list", _p(ids), count, s.data_ptr(), s.dim, None)
        want = s0.copy()
        port.multi_qubit_Pauli_gate_partial_list(list(range(count)), ids, want)
        assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL
        s = dev(s0)
        call("qs_multi_qubit_Pauli_rotation_gate_whole_list", _p(ids), count, -0.4, s.data_ptr(), s.dim, None)
        want = s0.copy()
        port.multi_qubit_Pauli_rotation_gate_partial_list(list(range(count)), ids, -0.4, want)
        assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL
    with pytest.raises(ValueError):
        call("qs_multi_qubit_Pauli_gate_whole_list", _p(np.zeros(n + 1, dtype=np.uint32)), n + 1, s.data_ptr(),
             s.dim, None)


@pytest.mark.parametrize("k", [1, 3, 7])
def test_single_control_multi_target_dense(port, k):
    rng = np.random.default_rng(1310 + k)
    n = 11
    s0 = random_state(n, rng)
    q = [int(x) for x in rng.permutation(n)]
    tl, c = q[:k], q[k]
    u = random_unitary(k, rng)
    for cv in (0, 1):
        d = 1 << k
        full = np.eye(2 * d, dtype=np.complex128)
        full[cv * d:(cv + 1) * d, cv * d:(cv + 1) * d] = u  # index bit k <-> the control
        want = s0.copy()
        port.multi_qubit_dense_matrix_gate(tl + [c], full, want)
        s = dev(s0)
        call("qs_single_qubit_control_multi_qubit_dense_matrix_gate", c, cv, _p(_u32(tl)), k, _p(u), s.data_ptr(),
             s.dim, None)
        assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL, cv


def test_controlled_diagonal(port):
    rng = np.random.default_rng(1320)
    n = 10
    s0 = random_state(n, rng)
    tl, cl, cv = [7, 2, 5], [0, 9], [1, 0]
    d = np.exp(1j * rng.normal(size=8))
    full = np.ones(32, dtype=np.complex128)
    full[8:16] = d  # index bits 3, 4 <-> controls 0, 9 with values (1, 0)
    want = s0.copy()
    port.multi_qubit_diagonal_matrix_gate(tl + cl, full, want)
    s = dev(s0)
    call("qs_multi_qubit_control_multi_qubit_diagonal_matrix_gate", _p(_u32(cl)), _p(_u32(cv)), 2, _p(_u32(tl)), 3,
         _p(d), s.data_ptr(), s.dim, None)
    assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL
    with pytest.raises(ValueError):
        call("qs_multi_qubit_control_multi_qubit_diagonal_matrix_gate", _p(_u32([7])), _p(_u32([1])), 1,
             _p(_u32(tl)), 3, _p(d), s.data_ptr(), s.dim, None)


def test_single_qubit_and_whole_list_expectations(port):
    rng = np.random.default_rng(1330)
    n = 12
    a, b = random_state(n, rng), random_state(n, rng)
    a *= 1.3  # not normalised: id 0 gives <psi|psi>
    sa, sb = dev(a), dev(b)
    out = np.zeros(2)
    for t in (0, 6, 11):
        for pid in range(4):
            call("qs_expectation_value_single_qubit_Pauli_operator", t, pid, sa.data_ptr(), sa.dim, None, _p(out))
            assert abs(out[0] - port.expectation_value([t], [pid], a)) <= EV_TOL, (t, pid)
    ids = rng.integers(0, 4, size=n).astype(np.uint32)
    call("qs_expectation_value_multi_qubit_Pauli_operator_whole_list", _p(ids), n, sa.data_ptr(), sa.dim, None,
         _p(out))
    assert abs(out[0] - port.expectation_value(list(range(n)), ids, a)) <= EV_TOL
    pb = b.copy()
    port.multi_qubit_Pauli_gate_partial_list(list(range(n)), ids, pb)
    call("qs_transition_amplitude_multi_qubit_Pauli_operator_whole_list", _p(ids), n, sa.data_ptr(), sb.data_ptr(),
         sa.dim, None, _p(out))
    assert abs(complex(out[0], out[1]) - np.vdot(a, pb)) <= 1e-12


def test_density_matrix_named_pauli_and_controlled_gates(port):
    rng = np.random.default_rng(1340)
    n = 6
    rho0 = random_density_matrix(n, rng)
    for name in ("X", "Y", "Z", "H", "S", "Sdag", "T", "Tdag", "sqrtX", "sqrtXdag", "sqrtY", "sqrtYdag", "P0", "P1"):
        d = dev_dm(rho0)
        call(f"qs_dm_{name}_gate", 4, d.data_ptr(), d.dim, None)
        want = rho0.copy()
        port.dm_single_qubit_dense_matrix_gate(4, getattr(G, name)(4).get_matrix(), want)
        assert np.max(np.abs(d.get_matrix() - want)) <= AMP_TOL, name
    d = dev_dm(rho0)
    call("qs_dm_SWAP_gate", 5, 1, d.data_ptr(), d.dim, None)
    want = rho0.copy()
    port.dm_multi_qubit_dense_matrix_gate([5, 1], G.SWAP(5, 1).get_matrix(), want)
    assert np.max(np.abs(d.get_matrix() - want)) <= AMP_TOL
    tl, ids = [3, 0, 5], [2, 1, 3]
    d = dev_dm(rho0)
    call("qs_dm_multi_qubit_Pauli_gate_partial_list", _p(_u32(tl)), _p(_u32(ids)), 3, d.data_ptr(), d.dim, None)
    want = rho0.copy()
    port.dm_multi_qubit_dense_matrix_gate(tl, G.Pauli(tl, ids).get_matrix(), want)
    assert np.max(np.abs(d.get_matrix() - want)) <= AMP_TOL
    tl, ids = [1, 4, 2, 0], [1, 0, 2, 3]
    d = dev_dm(rho0)
    call("qs_dm_multi_qubit_Pauli_rotation_gate_partial_list", _p(_u32(tl)), _p(_u32(ids)), 4, 0.9, d.data_ptr(),
         d.dim, None)
    want = rho0.copy()
    port.dm_multi_qubit_dense_matrix_gate(tl, G.PauliRotation(tl, ids, 0.9).get_matrix(), want)
    assert np.max(np.abs(d.get_matrix() - want)) <= AMP_TOL
    u = random_unitary(2, rng)
    full = np.eye(16, dtype=np.complex128)
    full[4:8, 4:8] = u  # index bits 2, 3 <-> controls 5, 0 with values (1, 0)
    d = dev_dm(rho0)
    call("qs_dm_multi_qubit_control_multi_qubit_dense_matrix_gate", _p(_u32([5, 0])), _p(_u32([1, 0])), 2,
         _p(_u32([2, 3])), 2, _p(u), d.data_ptr(), d.dim, None)
    want = rho0.copy()
    port.dm_multi_qubit_dense_matrix_gate([2, 3, 5, 0], full, want)
    assert np.max(np.abs(d.get_matrix() - want)) <= AMP_TOL
    m1 = random_unitary(1, rng)
    full = np.eye(4, dtype=np.complex128)
    full[0:2, 0:2] = m1  # index bit 1 <-> control 3 with value 0
    d = dev_dm(rho0)
    call("qs_dm_multi_qubit_control_single_qubit_dense_matrix_gate", _p(_u32([3])), _p(_u32([0])), 1, 1, _p(m1),
         d.data_ptr(), d.dim, None)
    want = rho0.copy()
    port.dm_multi_qubit_dense_matrix_gate([1, 3], full, want)
    assert np.max(np.abs(d.get_matrix() - want)) <= AMP_TOL
