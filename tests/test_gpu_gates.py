"""Gate kernels on the B200 against the oracle, per gate, every target (complex128, max |d amp| <= 1e-12)."""
import ctypes as C
import math

import numpy as np
import pytest

from conftest import AMP_TOL, random_state, random_unitary
from qulacs_b200 import QuantumState, gate as G
from qulacs_b200._lib import call

pytestmark = pytest.mark.gpu


def _p(a):
    return np.ascontiguousarray(a).ctypes.data_as(C.c_void_p)


def dev(vec):
    n = int(np.log2(vec.size))
    s = QuantumState(n)
    s.load(vec)
    return s


@pytest.mark.parametrize("n", [1, 2, 5, 6, 11])
def test_single_qubit_dense_every_target(port, n):
    rng = np.random.default_rng(100 + n)
    s0 = random_state(n, rng)
    for t in range(n):
        m = random_unitary(1, rng)
        want = s0.copy()
        port.single_qubit_dense_matrix_gate(t, m, want)
        s = dev(s0)
        mm = np.ascontiguousarray(m, dtype=np.complex128)
        call("qs_single_qubit_dense_matrix_gate", t, _p(mm), s.data_ptr(), s.dim, None)
        assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL, t


@pytest.mark.parametrize("n", [3, 12])
def test_rotations_diagonal_named(port, n):
    rng = np.random.default_rng(200 + n)
    s0 = random_state(n, rng)
    for t in range(n):
        a = float(rng.uniform(0, 2 * math.pi))
        for kind in ("RX", "RY", "RZ"):
            want = s0.copy()
            getattr(port, kind + "_gate")(t, a, want)
            s = dev(s0)
            call(f"qs_{kind}_gate", t, a, s.data_ptr(), s.dim, None)
            assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL, (kind, t)
        d = np.exp(1j * rng.normal(size=2))
        want = s0.copy()
        port.single_qubit_diagonal_matrix_gate(t, d, want)
        s = dev(s0)
        call("qs_single_qubit_diagonal_matrix_gate", t, _p(d), s.data_ptr(), s.dim, None)
        assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL
    # named gates against their reference matrices
    for name, mat in [("X", [[0, 1], [1, 0]]), ("Y", [[0, -1j], [1j, 0]]), ("Z", [[1, 0], [0, -1]]),
                      ("H", G.H(0).get_matrix()), ("S", [[1, 0], [0, 1j]]), ("Sdag", [[1, 0], [0, -1j]]),
                      ("T", G.T(0).get_matrix()), ("Tdag", G.Tdag(0).get_matrix()),
                      ("sqrtX", G.sqrtX(0).get_matrix()), ("sqrtXdag", G.sqrtXdag(0).get_matrix()),
                      ("sqrtY", G.sqrtY(0).get_matrix()), ("sqrtYdag", G.sqrtYdag(0).get_matrix()),
                      ("P0", [[1, 0], [0, 0]]), ("P1", [[0, 0], [0, 1]])]:
        t = n - 1
        want = s0.copy()
        port.single_qubit_dense_matrix_gate(t, np.asarray(mat, dtype=np.complex128), want)
        s = dev(s0)
        call(f"qs_{name}_gate", t, s.data_ptr(), s.dim, None)
        assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL, name


def test_two_qubit_named_all_pairs(port):
    rng = np.random.default_rng(300)
    n = 7
    s0 = random_state(n, rng)
    for c in range(n):
        for t in range(n):
            if c == t:
                continue
            for name in ("CNOT", "CZ", "SWAP"):
                want = s0.copy()
                getattr(port, name + "_gate")(c, t, want)
                s = dev(s0)
                call(f"qs_{name}_gate", c, t, s.data_ptr(), s.dim, None)
                assert np.max(np.abs(s.get_vector() - want)) == 0.0, (name, c, t)


@pytest.mark.parametrize("n", [10, 13])
def test_low_qubit_permutations_tile_kernel(port, n):
    """CNOT and SWAP with a qubit below 5 on states of >= 2^10 amplitudes run the shared-memory tile
    kernel (full-sector accesses): every pair with a low qubit, including partners 9 and n - 1."""
    rng = np.random.default_rng(310 + n)
    s0 = random_state(n, rng)
    pairs = [(c, t) for c in range(n) for t in range(n) if c != t and min(c, t) < 5]
    for c, t in pairs:
        for name in ("CNOT", "SWAP"):
            want = s0.copy()
            getattr(port, name + "_gate")(c, t, want)
            s = dev(s0)
            call(f"qs_{name}_gate", c, t, s.data_ptr(), s.dim, None)
            assert np.max(np.abs(s.get_vector() - want)) == 0.0, (name, c, t)


@pytest.mark.parametrize("k", [2, 3, 4, 5, 6])
def test_multi_qubit_dense(port, k):
    rng = np.random.default_rng(400 + k)
    n = 10
    s0 = random_state(n, rng)
    for trial in range(4):
        tl = [int(x) for x in rng.choice(n, size=k, replace=False)]
        if trial == 0:
            tl = list(range(k))  # lowest qubits
        m = random_unitary(k, rng)
        want = s0.copy()
        port.multi_qubit_dense_matrix_gate(tl, m, want)
        s = dev(s0)
        tla = np.asarray(tl, dtype=np.uint32)
        call("qs_multi_qubit_dense_matrix_gate", _p(tla), k, _p(m.astype(np.complex128)), s.data_ptr(), s.dim, None)
        assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL, tl


def _dense(k, rng):
    """A random complex 2^k x 2^k matrix of unit-scale rows (the gate does not need a unitary)."""
    d = 1 << k
    return (rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))) / np.sqrt(2 * d)


@pytest.mark.parametrize("k,n", [(7, 10), (8, 12), (10, 13), (12, 12)])
def test_multi_qubit_dense_beyond_six(port, k, n):
    """7..12 targets: the matrix streams from L2 (the reference takes any target count)."""
    rng = np.random.default_rng(450 + k)
    s0 = random_state(n, rng)
    for trial in range(2):
        tl = list(range(n - k, n)) if trial == 0 else [int(x) for x in rng.choice(n, size=k, replace=False)]
        m = _dense(k, rng)
        want = s0.copy()
        port.multi_qubit_dense_matrix_gate(tl, m, want)
        s = dev(s0)
        call("qs_multi_qubit_dense_matrix_gate", _p(np.asarray(tl, dtype=np.uint32)), k, _p(m), s.data_ptr(),
             s.dim, None)
        assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL, tl
    # 7 targets under 2 controls (values 1, 0), against the full 9-qubit matrix: index bits 0..6 <-> the
    # targets, bit 7 <-> cl[0], bit 8 <-> cl[1]; the block acts where bit 7 = 1 and bit 8 = 0
    u = _dense(7, rng)
    full = np.eye(512, dtype=np.complex128)
    full[128:256, 128:256] = u
    q = [int(x) for x in rng.permutation(n)]
    tl, cl = q[:7], q[7:9]
    want = s0.copy()
    port.multi_qubit_dense_matrix_gate(tl + cl, full, want)
    s = dev(s0)
    call("qs_multi_qubit_control_multi_qubit_dense_matrix_gate", _p(np.asarray(cl, dtype=np.uint32)),
         _p(np.asarray([1, 0], dtype=np.uint32)), 2, _p(np.asarray(tl, dtype=np.uint32)), 7, _p(u),
         s.data_ptr(), s.dim, None)
    assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL
    with pytest.raises(NotImplementedError):
        call("qs_multi_qubit_dense_matrix_gate", _p(np.arange(13, dtype=np.uint32)), 13,
             _p(np.zeros(2, dtype=np.complex128)), s.data_ptr(), s.dim, None)


@pytest.mark.parametrize("mode", ["gate_by_gate", "staged", "staged_fused"])
def test_circuit_with_a_nine_qubit_dense_gate(port, mode):
    from qulacs_b200 import QuantumCircuit
    rng = np.random.default_rng(470)
    n = 12
    s0 = random_state(n, rng)
    c = QuantumCircuit(n)
    c.add_H_gate(0)
    c.add_CNOT_gate(0, 11)
    tl = [int(x) for x in rng.choice(n, size=9, replace=False)]
    m = _dense(9, rng)
    c.add_dense_matrix_gate(tl, m)
    c.add_RX_gate(3, 0.4)
    s = dev(s0)
    c.update_quantum_state(s, mode=mode)
    want = s0.copy()
    port.single_qubit_dense_matrix_gate(0, G.H(0).get_matrix(), want)
    port.CNOT_gate(0, 11, want)
    port.multi_qubit_dense_matrix_gate(tl, m, want)
    port.RX_gate(3, 0.4, want)
    assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL


def test_controlled_and_diagonal_and_pauli(port):
    rng = np.random.default_rng(500)
    n = 9
    s0 = random_state(n, rng)
    m = random_unitary(1, rng)
    want = s0.copy()
    port.multi_qubit_control_single_qubit_dense_matrix_gate([2, 7], [1, 0], 4, m, want)
    s = dev(s0)
    cl, cv = np.array([2, 7], dtype=np.uint32), np.array([1, 0], dtype=np.uint32)
    call("qs_multi_qubit_control_single_qubit_dense_matrix_gate", _p(cl), _p(cv), 2, 4, _p(m), s.data_ptr(),
         s.dim, None)
    assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL
    # controlled 2-target against a full-matrix oracle application
    u = random_unitary(2, rng)
    full = np.eye(8, dtype=np.complex128)
    full[4:, 4:] = u  # control = bit 2 of the 3-qubit index (targets 0, 5 ; control 3)
    want = s0.copy()
    port.multi_qubit_dense_matrix_gate([0, 5, 3], full, want)
    s = dev(s0)
    tl, cl, cv = (np.array(x, dtype=np.uint32) for x in ([0, 5], [3], [1]))
    call("qs_multi_qubit_control_multi_qubit_dense_matrix_gate", _p(cl), _p(cv), 1, _p(tl), 2, _p(u),
         s.data_ptr(), s.dim, None)
    assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL
    d = np.exp(1j * rng.normal(size=8))
    want = s0.copy()
    port.multi_qubit_diagonal_matrix_gate([4, 0, 6], d, want)
    s = dev(s0)
    tl = np.array([4, 0, 6], dtype=np.uint32)
    call("qs_multi_qubit_diagonal_matrix_gate", _p(tl), 3, _p(d), s.data_ptr(), s.dim, None)
    assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL
    for _ in range(6):
        w = int(rng.integers(1, 5))
        tl = np.asarray(rng.choice(n, size=w, replace=False), dtype=np.uint32)
        ids = np.asarray(rng.integers(0, 4, size=w), dtype=np.uint32)
        want = s0.copy()
        port.multi_qubit_Pauli_gate_partial_list(tl, ids, want)
        s = dev(s0)
        call("qs_multi_qubit_Pauli_gate_partial_list", _p(tl), _p(ids), w, s.data_ptr(), s.dim, None)
        assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL
        want = s0.copy()
        port.multi_qubit_Pauli_rotation_gate_partial_list(tl, ids, 0.61, want)
        s = dev(s0)
        call("qs_multi_qubit_Pauli_rotation_gate_partial_list", _p(tl), _p(ids), w, 0.61, s.data_ptr(), s.dim, None)
        assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL


def test_gate_objects_update_quantum_state(port):
    rng = np.random.default_rng(600)
    n = 6
    s0 = random_state(n, rng)
    s = dev(s0)
    want = s0.copy()
    G.U3(2, 0.3, 0.4, 0.5).update_quantum_state(s)
    port.single_qubit_dense_matrix_gate(2, G.get_IBMQ_matrix(0.3, 0.4, 0.5), want)
    G.RotX(1, 0.7).update_quantum_state(s)
    port.RX_gate(1, -0.7, want)
    G.CNOT(5, 0).update_quantum_state(s)
    port.CNOT_gate(5, 0, want)
    assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL


def test_invalid_arguments_raise():
    s = QuantumState(3)
    with pytest.raises(ValueError):
        G.CNOT(0, 5).update_quantum_state(s)
    with pytest.raises(ValueError):
        call("qs_RX_gate", 3, 0.1, s.data_ptr(), s.dim, None)


def test_out_of_memory_is_reported():
    from qulacs_b200._lib import load
    p = C.c_void_p()
    rc = load().qs_allocate_quantum_state(1 << 40, C.byref(p))  # 16 TiB
    assert rc == 2  # QS_ERR_OUT_OF_MEMORY
    s = QuantumState(4)  # the context is still usable
    assert abs(s.get_squared_norm() - 1.0) < 1e-15
