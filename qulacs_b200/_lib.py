"""ctypes binding of the C ABI declared in include/qulacs_b200.h.

The shared object is the in-tree ``qulacs_b200/libqulacs_b200.so`` built by ``qulacs_b200/build.py``.
There is no fallback: if it is missing, importing the API raises.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libqulacs_b200.so")

U = C.c_uint
IT = C.c_ulonglong
D = C.c_double
P = C.c_void_p
I = C.c_int

# name -> argtypes (every function returns int status unless listed in _RESTYPES)
_STATE = [P, IT, P]  # state, dim, stream
SIGNATURES = {
    "qs_get_last_error": [],
    "qs_version": [],
    "qs_launch_count": [],
    "qs_device_synchronize": [],
    "qs_stream_synchronize": [P],
    "qs_stream_create": [C.POINTER(P)],
    "qs_stream_create_with_priority": [I, C.POINTER(P)],
    "qs_stream_destroy": [P],
    "qs_allocate_quantum_state": [IT, C.POINTER(P)],
    "qs_allocate_quantum_state_c64": [IT, C.POINTER(P)],
    "qs_release_quantum_state": [P],
    "qs_allocate_bytes": [IT, C.POINTER(P)],
    "qs_initialize_quantum_state": _STATE,
    "qs_initialize_quantum_state_c64": _STATE,
    "qs_set_computational_basis": [IT] + _STATE,
    "qs_load_state": [P] + _STATE,
    "qs_get_state": [P, P, IT, P],
    "qs_state_to_c64": [P, P, IT, P],
    "qs_state_to_c128": [P, P, IT, P],
    "qs_single_qubit_dense_matrix_gate": [U, P] + _STATE,
    "qs_single_qubit_diagonal_matrix_gate": [U, P] + _STATE,
    "qs_single_qubit_phase_gate": [U, P] + _STATE,
    "qs_RX_gate": [U, D] + _STATE,
    "qs_RY_gate": [U, D] + _STATE,
    "qs_RZ_gate": [U, D] + _STATE,
    "qs_CNOT_gate": [U, U] + _STATE,
    "qs_CZ_gate": [U, U] + _STATE,
    "qs_SWAP_gate": [U, U] + _STATE,
    "qs_double_qubit_dense_matrix_gate_c": [U, U, P] + _STATE,
    "qs_multi_qubit_dense_matrix_gate": [P, U, P] + _STATE,
    "qs_multi_qubit_diagonal_matrix_gate": [P, U, P] + _STATE,
    "qs_single_qubit_control_single_qubit_dense_matrix_gate": [U, U, U, P] + _STATE,
    "qs_multi_qubit_control_single_qubit_dense_matrix_gate": [P, P, U, U, P] + _STATE,
    "qs_multi_qubit_control_multi_qubit_dense_matrix_gate": [P, P, U, P, U, P] + _STATE,
    "qs_multi_qubit_Pauli_gate_partial_list": [P, P, U] + _STATE,
    "qs_multi_qubit_Pauli_rotation_gate_partial_list": [P, P, U, D] + _STATE,
    "qs_multi_qubit_Pauli_gate_whole_list": [P, U] + _STATE,
    "qs_multi_qubit_Pauli_rotation_gate_whole_list": [P, U, D] + _STATE,
    "qs_single_qubit_Pauli_gate": [U, U] + _STATE,
    "qs_single_qubit_Pauli_rotation_gate": [U, U, D] + _STATE,
    "qs_single_qubit_control_multi_qubit_dense_matrix_gate": [U, U, P, U, P] + _STATE,
    "qs_multi_qubit_control_multi_qubit_diagonal_matrix_gate": [P, P, U, P, U, P] + _STATE,
    "qs_state_norm_squared": [P, IT, P, P],
    "qs_measurement_distribution_entropy": [P, IT, P, P],
    "qs_dm_measurement_distribution_entropy": [P, IT, P, P],
    "qs_state_add": [P, P, IT, P],
    "qs_state_add_with_coef": [P, P, P, IT, P],
    "qs_state_multiply": [P, P, IT, P],
    "qs_normalize": [D, P, IT, P],
    "qs_dm_state_add": [P, P, IT, P],
    "qs_dm_state_add_with_coef": [P, P, P, IT, P],
    "qs_dm_state_multiply": [P, P, IT, P],
    "qs_initialize_Haar_random_state_with_seed": [P, IT, U, P],
    "qs_get_amplitude": [P, IT, IT, P, P],
    "qs_copy_state": [P, P, IT, P],
    "qs_batch_update_quantum_states_fused_c64": [P, P, U, P],
    "qs_random_unitary_matrix": [U, U, P],
    "qs_random_operator_terms": [U, U, U, P, P],
    "qs_state_multiply_elementwise": [P, P, IT, P],
    "qs_dm_normalize": [D, P, IT, P],
    "qs_dm_M0_prob": [U, P, IT, P, P],
    "qs_dm_M1_prob": [U, P, IT, P, P],
    "qs_dm_marginal_prob": [P, P, U, P, IT, P, P],
    "qs_state_inner_product": [P, P, IT, P, P],
    "qs_M0_prob": [U, P, IT, P, P],
    "qs_M1_prob": [U, P, IT, P, P],
    "qs_marginal_prob": [P, P, U, P, IT, P, P],
    "qs_expectation_value_multi_qubit_Pauli_operator_partial_list": [P, P, U, P, IT, P, P],
    "qs_transition_amplitude_multi_qubit_Pauli_operator_partial_list": [P, P, U, P, P, IT, P, P],
    "qs_expectation_value_single_qubit_Pauli_operator": [U, U, P, IT, P, P],
    "qs_expectation_value_multi_qubit_Pauli_operator_whole_list": [P, U, P, IT, P, P],
    "qs_transition_amplitude_multi_qubit_Pauli_operator_whole_list": [P, U, P, P, IT, P, P],
    "qs_expectation_value_pauli_batch": [P, P, P, U, P, IT, P, P],
    "qs_expectation_value_pauli_weighted": [P, P, P, P, U, P, IT, P, P],
    "qs_expectation_value_pauli_weighted_c64": [P, P, P, P, U, P, IT, P, P],
    "qs_expectation_value_pauli_weighted_plan": [P, P, P, U, IT, P, P],
    "qs_set_expectation_specialized": [C.c_int],
    "qs_expectation_specialized_info": [P, P],
    "qs_expectation_pass_source": [P, P, P, U, IT, U, C.c_int, P, IT, P],
    "qs_state_sampling_with_uniforms": [P, IT, P, U, P, P],
    "qs_state_sampling": [P, IT, U, U, P, P],
    "qs_state_sampling_with_uniforms_flagged": [P, IT, P, U, D, P, P, P, P],
    "qs_reference_uniforms": [U, U, P],
    "qs_state_sampling_with_uniforms_noalloc": [P, IT, P, U, P, P],
    "qs_dm_allocate": [IT, C.POINTER(P)],
    "qs_dm_initialize_quantum_state": _STATE,
    "qs_dm_initialize_with_pure_state": [P, P, IT, P],
    "qs_dm_single_qubit_dense_matrix_gate": [U, P] + _STATE,
    "qs_dm_multi_qubit_dense_matrix_gate": [P, U, P] + _STATE,
    "qs_dm_CNOT_gate": [U, U] + _STATE,
    "qs_dm_CZ_gate": [U, U] + _STATE,
    "qs_dm_RX_gate": [U, D] + _STATE,
    "qs_dm_RY_gate": [U, D] + _STATE,
    "qs_dm_RZ_gate": [U, D] + _STATE,
    **{f"qs_dm_{g}_gate": [U] + _STATE for g in ("X", "Y", "Z", "H", "S", "Sdag", "T", "Tdag", "sqrtX", "sqrtXdag",
                                                 "sqrtY", "sqrtYdag", "P0", "P1")},
    "qs_dm_SWAP_gate": [U, U] + _STATE,
    "qs_reflection_gate": [P, P, IT, P],
    "qs_FusedSWAP_gate": [U, U, U] + _STATE,
    "qs_initialize_Haar_random_state": [P, IT, P],
    "qs_state_tensor_product": [P, IT, P, IT, P, P],
    "qs_state_permutate_qubit": [P, P, P, U, IT, P],
    "qs_state_drop_qubits": [P, P, U, P, P, IT, P],
    "qs_dm_state_tensor_product": [P, IT, P, IT, P, P],
    "qs_dm_state_permutate_qubit": [P, P, P, U, IT, P],
    "qs_dm_state_partial_trace_from_density_matrix": [P, U, P, P, IT, P],
    "qs_dm_state_partial_trace_from_state_vector": [P, U, P, P, IT, P],
    "qs_dm_multi_qubit_Pauli_gate_partial_list": [P, P, U] + _STATE,
    "qs_dm_multi_qubit_Pauli_rotation_gate_partial_list": [P, P, U, D] + _STATE,
    "qs_dm_multi_qubit_control_single_qubit_dense_matrix_gate": [P, P, U, U, P] + _STATE,
    "qs_dm_multi_qubit_control_multi_qubit_dense_matrix_gate": [P, P, U, P, U, P] + _STATE,
    "qs_dm_depolarizing_noise": [U, D] + _STATE,
    "qs_dm_two_qubit_depolarizing_noise": [U, U, D] + _STATE,
    "qs_dm_expectation_value_multi_qubit_Pauli_operator_partial_list": [P, P, U, P, IT, P, P],
    "qs_dm_sampling_with_uniforms": [P, IT, P, U, P, P],
    "qs_dm_state_norm_squared": [P, IT, P, P],
    "qs_circuit_create": [U, C.POINTER(P)],
    "qs_circuit_destroy": [P],
    "qs_circuit_add_gate": [P, I, P, U, P, P, U, P, U],
    "qs_circuit_gate_count": [P, C.POINTER(U)],
    "qs_circuit_update_quantum_state": [P, P, IT, I, P],
    "qs_circuit_pass_count": [P, IT, C.POINTER(U)],
    "qs_circuit_staged_stats": [P, C.POINTER(U), C.POINTER(U), C.POINTER(U), C.POINTER(U)],
    "qs_circuit_update_density_matrix": [P, P, IT, I, P],
    "qs_circuit_fuse": [P, I, C.POINTER(P)],
    "qs_noise_simulator_trajectories": [P, U, U, C.POINTER(U), P],
    "qs_noise_simulator_execute": [P, P, IT, U, U, P, P, P],
    "qs_circuit_density_matrix_as_vector": [P, C.POINTER(P)],
    "qs_circuit_gate_matrix": [P, U, P, C.POINTER(U), P],
    "qs_circuit_set_fusion": [P, I],
    "qs_circuit_fusion_info": [P, C.POINTER(I), C.POINTER(U), C.POINTER(U), P],
    "qs_circuit_update_quantum_state_fused_c64": [P, P, IT, P],
    "qs_circuit_update_quantum_state_c64": [P, P, IT, P],
    "qs_circuit_set_c64_executor": [P, C.c_int],
    "qs_circuit_c64_executor_info": [P, P],
    "qs_batch_update_quantum_states_c64": [P, P, U, C.c_int, P],
    "qs_batch_update_quantum_states": [P, P, U, P],
    "qs_circuit_graph_create": [P, P, IT, C.c_int, C.c_int, P, P],
    "qs_batch_graph_create": [P, P, U, C.c_int, C.c_int, P, P],
    "qs_graph_launch": [P, P],
    "qs_graph_kernel_count": [P, P],
    "qs_graph_destroy": [P],
    "qs_debug_batch_wait_expiry": [P, P, U, P],
    "qs_debug_batch_wait_expiry_fused_c64": [P, P, U, P],
    "qs_circuit_set_specialized": [P, I],
    "qs_circuit_specialized_info": [P, C.POINTER(I), C.POINTER(I), C.POINTER(D)],
    "qs_circuit_specialized_source": [P, IT, U, C.c_char_p, C.POINTER(IT)],
    "qs_batch_expectation_values": [P, P, U, P, P, P, P, P, P],
    "qs_batch_expectation_weighted": [P, P, U, P, P, P, P, P, C.c_int, P, P],
    "qs_batch_expectation_values_c64": [P, P, U, P, P, P, P, P, P],
    "qs_state_norm_squared_c64": [P, IT, P, P],
    "qs_state_inner_product_c128_c64": [P, P, IT, P, P],
    "qs_expectation_value_pauli_batch_c64": [P, P, P, U, P, IT, P, P],
    "qs_state_sampling_with_uniforms_c64": [P, IT, P, U, P, P],
    "qs_circuit_fused_stats": [P, C.POINTER(U), C.POINTER(U)],
    "qs_circuit_fused_block_export": [P, U, P, C.POINTER(I), P, P, P],
    "qs_circuit_fused_block_layout": [P, U, P, P, P, P],
}
for _n in ("X", "Y", "Z", "H", "S", "Sdag", "T", "Tdag", "sqrtX", "sqrtXdag", "sqrtY", "sqrtYdag", "P0", "P1"):
    SIGNATURES[f"qs_{_n}_gate"] = [U] + _STATE

_RESTYPES = {"qs_get_last_error": C.c_char_p, "qs_version": C.c_char_p, "qs_launch_count": C.c_ulonglong}

ERRORS = {
    1: ValueError,       # QS_ERR_INVALID_ARGUMENT
    2: MemoryError,      # QS_ERR_OUT_OF_MEMORY
    3: RuntimeError,     # QS_ERR_CUDA
    4: TimeoutError,     # QS_ERR_TIMEOUT
    5: NotImplementedError,  # QS_ERR_NOT_SUPPORTED
    6: RuntimeError,     # QS_ERR_NO_DEVICE
    7: RuntimeError,     # QS_ERR_REJECTED
}

GATE_KINDS = {
    "DENSE": 0, "DIAGONAL": 1, "RX": 2, "RY": 3, "RZ": 4, "CNOT": 5, "CZ": 6, "SWAP": 7,
    "PAULI": 8, "PAULI_ROTATION": 9, "DEPOLARIZING": 10,
}
EXEC_GATE_BY_GATE = 0
EXEC_STAGED = 1
EXEC_STAGED_FUSED = 2


class QsError(RuntimeError):
    pass


_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"qulacs_b200 CUDA library not found at {path}; build it with `python qulacs_b200/build.py` "
            "or __graft_entry__.build()")
    lib = C.CDLL(path)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, C.c_int)
    _lib = lib
    return lib


def check(rc: int, what: str = "") -> None:
    """Raise the Python exception matching a non-zero status code."""
    if rc == 0:
        return
    msg = load().qs_get_last_error().decode(errors="replace")
    exc = ERRORS.get(rc, QsError)
    raise exc(f"{what}: {msg} (status {rc})" if what else f"{msg} (status {rc})")


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args), name)
