"""The C-ABI library loads, exports every declared symbol, and validates arguments on the host
(these checks return before any CUDA call, so they run without a GPU)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from qulacs_b200 import _lib


def declared_symbols():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names += re.findall(r"QS_API\s+[\w\s\*]+?\b(qs_\w+)\s*\(", txt)
    return names


def test_library_exports_every_declared_symbol(lib):
    names = declared_symbols()
    assert len(names) > 60
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    names = set(declared_symbols())
    assert names <= set(_lib.SIGNATURES), sorted(names - set(_lib.SIGNATURES))


def test_version(lib):
    assert b"sm_100a" in lib.qs_version()


def test_invalid_dim_rejected_on_host(lib):
    m = np.eye(2, dtype=np.complex128)
    rc = lib.qs_single_qubit_dense_matrix_gate(0, m.ctypes.data_as(C.c_void_p), None, 3, None)
    assert rc == 1  # QS_ERR_INVALID_ARGUMENT
    assert b"power of two" in lib.qs_get_last_error()


def test_target_out_of_range_rejected(lib):
    m = np.eye(2, dtype=np.complex128)
    rc = lib.qs_single_qubit_dense_matrix_gate(7, m.ctypes.data_as(C.c_void_p), None, 1 << 4, None)
    assert rc == 1
    assert b"qubit index 7" in lib.qs_get_last_error()


def test_duplicate_targets_rejected(lib):
    tl = np.array([1, 1], dtype=np.uint32)
    m = np.eye(4, dtype=np.complex128)
    rc = lib.qs_multi_qubit_dense_matrix_gate(tl.ctypes.data_as(C.c_void_p), 2, m.ctypes.data_as(C.c_void_p),
                                              None, 1 << 4, None)
    assert rc == 1
    assert b"duplicated" in lib.qs_get_last_error()


def test_dense_k_limit(lib):
    """Dense gates take 1..12 targets; 13 is refused before any device work (the matrix is not read)."""
    tl = np.arange(13, dtype=np.uint32)
    m = np.eye(2, dtype=np.complex128)
    rc = lib.qs_multi_qubit_dense_matrix_gate(tl.ctypes.data_as(C.c_void_p), 13, m.ctypes.data_as(C.c_void_p),
                                              None, 1 << 14, None)
    assert rc == 5  # QS_ERR_NOT_SUPPORTED


def test_circuit_host_validation(lib):
    h = C.c_void_p()
    assert lib.qs_circuit_create(4, C.byref(h)) == 0
    t = np.array([0, 9], dtype=np.uint32)
    rc = lib.qs_circuit_add_gate(h, 5, t.ctypes.data_as(C.c_void_p), 2, None, None, 0, None, 0)
    assert rc == 1
    t = np.array([0, 1], dtype=np.uint32)
    assert lib.qs_circuit_add_gate(h, 5, t.ctypes.data_as(C.c_void_p), 2, None, None, 0, None, 0) == 0
    cnt = C.c_uint()
    assert lib.qs_circuit_gate_count(h, C.byref(cnt)) == 0 and cnt.value == 1
    # wrong state dimension is refused before touching the device
    assert lib.qs_circuit_update_quantum_state(h, None, 1 << 5, 0, None) == 1
    assert lib.qs_circuit_destroy(h) == 0


def test_python_errors_map_to_exceptions():
    with pytest.raises(ValueError):
        _lib.check(1, "x")
    with pytest.raises(MemoryError):
        _lib.check(2, "x")
    with pytest.raises(NotImplementedError):
        _lib.check(5, "x")


def _u32p(x):
    a = np.ascontiguousarray(np.asarray(x, dtype=np.uint32))
    return a, a.ctypes.data_as(C.c_void_p)


def test_added_entry_points_validate_on_host(lib):
    """The csim forms, state manipulation and density-matrix gates refuse bad arguments before any
    device work (status 1 = invalid argument, 5 = not supported)."""
    dim = 1 << 6
    keep = []

    def u(x):
        a, p = _u32p(x)
        keep.append(a)
        return p

    assert lib.qs_single_qubit_Pauli_gate(0, 4, None, dim, None) == 1          # Pauli id 4
    assert lib.qs_single_qubit_Pauli_rotation_gate(6, 1, C.c_double(0.1), None, dim, None) == 1  # qubit 6 of 6
    assert lib.qs_multi_qubit_Pauli_gate_whole_list(u([1] * 7), 7, None, dim, None) == 1  # more ids than qubits
    assert lib.qs_multi_qubit_control_multi_qubit_diagonal_matrix_gate(
        u([2]), u([1]), 1, u([2, 3]), 2, None, None, dim, None) == 1          # control is a target
    assert lib.qs_multi_qubit_control_multi_qubit_diagonal_matrix_gate(
        u([0]), u([2]), 1, u([1]), 1, None, None, dim, None) == 1             # control value 2
    assert lib.qs_single_qubit_control_multi_qubit_dense_matrix_gate(1, 0, u([1, 2]), 2, None, None, dim,
                                                                     None) == 1  # control is a target
    assert lib.qs_state_permutate_qubit(u([0, 1, 2]), None, None, 3, dim, None) == 1      # not every qubit
    assert lib.qs_state_permutate_qubit(u([0, 1, 2, 3, 4, 4]), None, None, 6, dim, None) == 1  # repeated
    assert lib.qs_state_drop_qubits(u([1]), u([2]), 1, None, None, dim, None) == 1        # projection 2
    assert lib.qs_state_drop_qubits(u(range(6)), u([0] * 6), 6, None, None, dim, None) == 1  # nothing left
    assert lib.qs_dm_state_partial_trace_from_state_vector(u([0, 0]), 2, None, None, dim, None) == 1
    assert lib.qs_FusedSWAP_gate(0, 2, 3, None, dim, None) == 1                           # blocks overlap
    assert lib.qs_FusedSWAP_gate(0, 4, 3, None, dim, None) == 1                           # past qubit 5
    assert lib.qs_dm_multi_qubit_Pauli_gate_partial_list(u([0, 1]), u([1, 5]), 2, None, 1 << 3, None) == 1
    assert lib.qs_dm_multi_qubit_Pauli_rotation_gate_partial_list(u(range(13)), u([1] * 13), 13,
                                                                  C.c_double(0.2), None, 1 << 14, None) == 5
    assert lib.qs_dm_multi_qubit_control_multi_qubit_dense_matrix_gate(u([0]), u([1]), 1, u([0]), 1, None, None,
                                                                       1 << 3, None) == 1
    assert lib.qs_state_tensor_product(None, 1 << 30, None, 1 << 11, None, None) == 5      # 41 qubits


def test_new_entry_points_validate_on_host(lib):
    """Executor choices, specialisation modes and graph creation reject bad arguments before any CUDA
    call; a weighted expectation with a mask beyond the qubit count is refused."""
    from qulacs_b200 import workloads as W
    circ = W.to_circuit(W.hea_circuit(6, 2, seed=1), 6)
    assert lib.qs_circuit_set_c64_executor(circ._h, 2) == 1
    assert lib.qs_circuit_set_c64_executor(None, 0) == 1
    assert lib.qs_set_expectation_specialized(3) == 1
    assert lib.qs_set_expectation_specialized(1) == 0
    h = C.c_void_p()
    assert lib.qs_circuit_graph_create(None, None, 1 << 6, 1, 1, None, C.byref(h)) == 1
    assert lib.qs_circuit_graph_create(circ._h, C.c_void_p(16), 1 << 5, 1, 1, None, C.byref(h)) == 1
    assert b"dim differs" in lib.qs_get_last_error()
    assert lib.qs_circuit_graph_create(circ._h, C.c_void_p(16), 1 << 6, 7, 1, None, C.byref(h)) == 1
    assert lib.qs_graph_launch(None, None) == 1
    assert lib.qs_graph_destroy(None) == 0
    ch = (C.c_void_p * 1)(circ._h)
    st = (C.c_void_p * 1)(16)
    assert lib.qs_batch_update_quantum_states_c64(ch, st, 1, 5, None) == 1
    assert lib.qs_batch_graph_create(None, None, 0, 0, 1, None, C.byref(h)) == 1
    x = np.array([1 << 7], dtype=np.uint64)
    z = np.zeros(1, dtype=np.uint64)
    y = np.zeros(1, dtype=np.uint32)
    cf = np.array([1.0, 0.0])
    out = np.zeros(2)
    rc = lib.qs_expectation_value_pauli_weighted(x.ctypes.data_as(C.c_void_p), z.ctypes.data_as(C.c_void_p),
                                                 y.ctypes.data_as(C.c_void_p), cf.ctypes.data_as(C.c_void_p), 1,
                                                 C.c_void_p(16), 1 << 6, None, out.ctypes.data_as(C.c_void_p))
    assert rc == 1
    assert b"mask beyond qubit count" in lib.qs_get_last_error()
