// csim_compat.hpp -- the reference's csim operator signatures over device memory (libcsim_b200.so).
//
// A program written against csim's headers (src/csim/update_ops.hpp, stat_ops.hpp, init_ops.hpp,
// memory_ops.hpp, update_ops_dm.hpp, stat_ops_dm.hpp, memory_ops_dm.hpp) links against libcsim_b200.so
// unchanged: the functions below have csim's names, C++ linkage and argument lists, with csim's types
// UINT = unsigned int, ITYPE = unsigned long long, CTYPE = std::complex<double> (csim/type.hpp:15-30),
// so the mangled symbols are the ones such a program references.
//
// Differences from csim, by design:
//  * `state` (and every CTYPE* state-like argument) is a DEVICE pointer of dim complex128 amplitudes in
//    csim's layout; allocate_quantum_state / dm_allocate_quantum_state return device memory.  Matrices,
//    diagonals and index lists are host arrays, as in csim.
//  * Each call runs on the legacy default stream and returns when its work is complete (csim is
//    synchronous; so are the reference GPU backend's host wrappers, gpusim update_ops_cuda.h).
//  * Invalid input throws std::runtime_error carrying the library's message, where csim asserts or calls
//    exit(1) (csim/utility.cpp:38-40, memory_ops.cpp:21-25).
// The MPI variants, the QFT helpers and H_gate_unnormalized are not provided.
#pragma once

#include <complex>

using UINT = unsigned int;
using ITYPE = unsigned long long;
using CTYPE = std::complex<double>;

// memory / initialisation (memory_ops.hpp, init_ops.hpp, memory_ops_dm.hpp)
CTYPE* allocate_quantum_state(ITYPE dim);
void release_quantum_state(CTYPE* state);
void initialize_quantum_state(CTYPE* state, ITYPE dim);
void initialize_Haar_random_state(CTYPE* state, ITYPE dim);
void initialize_Haar_random_state_with_seed(CTYPE* state, ITYPE dim, UINT seed);
CTYPE* dm_allocate_quantum_state(ITYPE dim);
void dm_release_quantum_state(CTYPE* state);
void dm_initialize_quantum_state(CTYPE* state, ITYPE dim);
void dm_initialize_with_pure_state(CTYPE* state, const CTYPE* pure_state, ITYPE dim);

// one-qubit gates (update_ops.hpp)
void X_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void Y_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void Z_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void S_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void Sdag_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void T_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void Tdag_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void sqrtX_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void sqrtXdag_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void sqrtY_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void sqrtYdag_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void H_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void P0_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void P1_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void RX_gate(UINT target_qubit_index, double angle, CTYPE* state, ITYPE dim);
void RY_gate(UINT target_qubit_index, double angle, CTYPE* state, ITYPE dim);
void RZ_gate(UINT target_qubit_index, double angle, CTYPE* state, ITYPE dim);
void single_qubit_Pauli_gate(UINT target_qubit_index, UINT Pauli_operator_type, CTYPE* state, ITYPE dim);
void single_qubit_Pauli_rotation_gate(
    UINT target_qubit_index, UINT Pauli_operator_index, double angle, CTYPE* state, ITYPE dim);
void single_qubit_dense_matrix_gate(UINT target_qubit_index, const CTYPE matrix[4], CTYPE* state, ITYPE dim);
void single_qubit_diagonal_matrix_gate(
    UINT target_qubit_index, const CTYPE diagonal_matrix[2], CTYPE* state, ITYPE dim);
void single_qubit_phase_gate(UINT target_qubit_index, CTYPE phase, CTYPE* state, ITYPE dim);
void single_qubit_control_single_qubit_dense_matrix_gate(UINT control_qubit_index, UINT control_value,
    UINT target_qubit_index, const CTYPE matrix[4], CTYPE* state, ITYPE dim);
void multi_qubit_control_single_qubit_dense_matrix_gate(const UINT* control_qubit_index_list,
    const UINT* control_value_list, UINT control_qubit_index_count, UINT target_qubit_index, const CTYPE matrix[4],
    CTYPE* state, ITYPE dim);

// two- and multi-qubit gates (update_ops.hpp)
void CNOT_gate(UINT control_qubit_index, UINT target_qubit_index, CTYPE* state, ITYPE dim);
void CZ_gate(UINT control_qubit_index, UINT target_qubit_index, CTYPE* state, ITYPE dim);
void SWAP_gate(UINT target_qubit_index_0, UINT target_qubit_index_1, CTYPE* state, ITYPE dim);
void FusedSWAP_gate(
    UINT target_qubit_index_0, UINT target_qubit_index_1, UINT block_size, CTYPE* state, ITYPE dim);
void double_qubit_dense_matrix_gate_c(
    UINT target_qubit_index1, UINT target_qubit_index2, const CTYPE matrix[16], CTYPE* state, ITYPE dim);
void multi_qubit_dense_matrix_gate(const UINT* target_qubit_index_list, UINT target_qubit_index_count,
    const CTYPE* matrix, CTYPE* state, ITYPE dim);
void single_qubit_control_multi_qubit_dense_matrix_gate(UINT control_qubit_index, UINT control_value,
    const UINT* target_qubit_index_list, UINT target_qubit_index_count, const CTYPE* matrix, CTYPE* state,
    ITYPE dim);
void multi_qubit_control_multi_qubit_dense_matrix_gate(const UINT* control_qubit_index_list,
    const UINT* control_value_list, UINT control_qubit_index_count, const UINT* target_qubit_index_list,
    UINT target_qubit_index_count, const CTYPE* matrix, CTYPE* state, ITYPE dim);
void multi_qubit_diagonal_matrix_gate(const UINT* target_qubit_index_list, UINT target_qubit_index_count,
    const CTYPE* diagonal_element, CTYPE* state, ITYPE dim);
void multi_qubit_control_multi_qubit_diagonal_matrix_gate(const UINT* control_qubit_index_list,
    const UINT* control_value_list, UINT control_qubit_index_count, const UINT* target_qubit_index_list,
    UINT target_qubit_index_count, const CTYPE* diagonal_element, CTYPE* state, ITYPE dim);
void multi_qubit_Pauli_gate_whole_list(const UINT* Pauli_operator_type_list, UINT qubit_count, CTYPE* state,
    ITYPE dim_);
void multi_qubit_Pauli_gate_whole_list_single_thread(const UINT* Pauli_operator_type_list, UINT qubit_count,
    CTYPE* state, ITYPE dim_);
void multi_qubit_Pauli_gate_partial_list(const UINT* target_qubit_index_list, const UINT* Pauli_operator_type_list,
    UINT target_qubit_index_count, CTYPE* state, ITYPE dim);
void multi_qubit_Pauli_gate_partial_list_single_thread(const UINT* target_qubit_index_list,
    const UINT* Pauli_operator_type_list, UINT target_qubit_index_count, CTYPE* state, ITYPE dim);
void multi_qubit_Pauli_rotation_gate_whole_list(const UINT* Pauli_operator_type_list, UINT qubit_count,
    double angle, CTYPE* state, ITYPE dim_);
void multi_qubit_Pauli_rotation_gate_whole_list_single_thread(const UINT* Pauli_operator_type_list,
    UINT qubit_count, double angle, CTYPE* state, ITYPE dim_);
void multi_qubit_Pauli_rotation_gate_partial_list(const UINT* target_qubit_index_list,
    const UINT* Pauli_operator_type_list, UINT target_qubit_index_count, double angle, CTYPE* state, ITYPE dim);
void multi_qubit_Pauli_rotation_gate_partial_list_single_thread(const UINT* target_qubit_index_list,
    const UINT* Pauli_operator_type_list, UINT target_qubit_index_count, double angle, CTYPE* state, ITYPE dim);
void reflection_gate(const CTYPE* reflection_state, CTYPE* state, ITYPE dim);

// state arithmetic (update_ops.hpp)
void normalize(double squared_norm, CTYPE* state, ITYPE dim);
void normalize_single_thread(double squared_norm, CTYPE* state, ITYPE dim);
void state_add(const CTYPE* state_added, CTYPE* state, ITYPE dim);
void state_add_with_coef(CTYPE coef, const CTYPE* state_added, CTYPE* state, ITYPE dim);
void state_add_with_coef_single_thread(CTYPE coef, const CTYPE* state_added, CTYPE* state, ITYPE dim);
void state_multiply(CTYPE coef, CTYPE* state, ITYPE dim);

// statistics (stat_ops.hpp)
double state_norm_squared(const CTYPE* state, ITYPE dim);
double state_norm_squared_single_thread(const CTYPE* state, ITYPE dim);
double measurement_distribution_entropy(const CTYPE* state, ITYPE dim);
CTYPE state_inner_product(const CTYPE* state_bra, const CTYPE* state_ket, ITYPE dim);
void state_tensor_product(
    const CTYPE* state_left, ITYPE dim_left, const CTYPE* state_right, ITYPE dim_right, CTYPE* state_dst);
void state_permutate_qubit(
    const UINT* qubit_order, const CTYPE* state_src, CTYPE* state_dst, UINT qubit_count, ITYPE dim);
void state_drop_qubits(const UINT* target, const UINT* projection, UINT target_count, const CTYPE* state_src,
    CTYPE* state_dst, ITYPE dim);
double M0_prob(UINT target_qubit_index, const CTYPE* state, ITYPE dim);
double M1_prob(UINT target_qubit_index, const CTYPE* state, ITYPE dim);
double marginal_prob(const UINT* sorted_target_qubit_index_list, const UINT* measured_value_list,
    UINT target_qubit_index_count, const CTYPE* state, ITYPE dim);
double expectation_value_single_qubit_Pauli_operator(
    UINT target_qubit_index, UINT Pauli_operator_type, const CTYPE* state, ITYPE dim);
double expectation_value_multi_qubit_Pauli_operator_whole_list(
    const UINT* Pauli_operator_type_list, UINT qubit_count, const CTYPE* state, ITYPE dim);
double expectation_value_multi_qubit_Pauli_operator_partial_list(const UINT* target_qubit_index_list,
    const UINT* Pauli_operator_type_list, UINT target_qubit_index_count, const CTYPE* state, ITYPE dim);
double expectation_value_multi_qubit_Pauli_operator_partial_list_single_thread(const UINT* target_qubit_index_list,
    const UINT* Pauli_operator_type_list, UINT target_qubit_index_count, const CTYPE* state, ITYPE dim);
CTYPE transition_amplitude_multi_qubit_Pauli_operator_whole_list(const UINT* Pauli_operator_type_list,
    UINT qubit_count, const CTYPE* state_bra, const CTYPE* state_ket, ITYPE dim);
CTYPE transition_amplitude_multi_qubit_Pauli_operator_partial_list(const UINT* target_qubit_index_list,
    const UINT* Pauli_operator_type_list, UINT target_qubit_index_count, const CTYPE* state_bra,
    const CTYPE* state_ket, ITYPE dim);

// density matrices (update_ops_dm.hpp, stat_ops_dm.hpp); `state` is the dim x dim row-major rho
void dm_normalize(double squared_norm, CTYPE* state, ITYPE dim);
void dm_single_qubit_dense_matrix_gate(UINT target_qubit_index, const CTYPE matrix[4], CTYPE* state, ITYPE dim);
void dm_multi_qubit_control_single_qubit_dense_matrix_gate(const UINT* control_qubit_index_list,
    const UINT* control_value_list, UINT control_qubit_index_count, UINT target_qubit_index, const CTYPE matrix[4],
    CTYPE* state, ITYPE dim);
void dm_multi_qubit_dense_matrix_gate(const UINT* target_qubit_index_list, UINT target_qubit_index_count,
    const CTYPE* matrix, CTYPE* state, ITYPE dim);
void dm_multi_qubit_control_multi_qubit_dense_matrix_gate(const UINT* control_qubit_index_list,
    const UINT* control_value_list, UINT control_qubit_index_count, const UINT* target_qubit_index_list,
    UINT target_qubit_index_count, const CTYPE* matrix, CTYPE* state, ITYPE dim);
void dm_X_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void dm_Y_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void dm_Z_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void dm_S_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void dm_Sdag_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void dm_T_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void dm_Tdag_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void dm_sqrtX_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void dm_sqrtXdag_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void dm_sqrtY_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void dm_sqrtYdag_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void dm_H_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void dm_CNOT_gate(UINT control_qubit_index, UINT target_qubit_index, CTYPE* state, ITYPE dim);
void dm_CZ_gate(UINT control_qubit_index, UINT target_qubit_index, CTYPE* state, ITYPE dim);
void dm_SWAP_gate(UINT target_qubit_index_0, UINT target_qubit_index_1, CTYPE* state, ITYPE dim);
void dm_P0_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void dm_P1_gate(UINT target_qubit_index, CTYPE* state, ITYPE dim);
void dm_RX_gate(UINT target_qubit_index, double angle, CTYPE* state, ITYPE dim);
void dm_RY_gate(UINT target_qubit_index, double angle, CTYPE* state, ITYPE dim);
void dm_RZ_gate(UINT target_qubit_index, double angle, CTYPE* state, ITYPE dim);
void dm_multi_qubit_Pauli_gate_partial_list(const UINT* target_qubit_index_list,
    const UINT* Pauli_operator_type_list, UINT target_qubit_index_count, CTYPE* state, ITYPE dim);
void dm_multi_qubit_Pauli_rotation_gate_partial_list(const UINT* target_qubit_index_list,
    const UINT* Pauli_operator_type_list, UINT target_qubit_index_count, double angle, CTYPE* state, ITYPE dim);
double dm_state_norm_squared(const CTYPE* state, ITYPE dim);
double dm_measurement_distribution_entropy(const CTYPE* state, ITYPE dim);
void dm_state_add(const CTYPE* state_added, CTYPE* state, ITYPE dim);
void dm_state_add_with_coef(CTYPE coef, const CTYPE* state_added, CTYPE* state, ITYPE dim);
void dm_state_multiply(CTYPE coef, CTYPE* state, ITYPE dim);
void dm_state_tensor_product(
    const CTYPE* state_left, ITYPE dim_left, const CTYPE* state_right, ITYPE dim_right, CTYPE* state_dst);
void dm_state_permutate_qubit(
    const UINT* qubit_order, const CTYPE* state_src, CTYPE* state_dst, UINT qubit_count, ITYPE dim);
void dm_state_partial_trace_from_density_matrix(
    const UINT* target, UINT target_count, const CTYPE* state_src, CTYPE* state_dst, ITYPE dim);
void dm_state_partial_trace_from_state_vector(
    const UINT* target, UINT target_count, const CTYPE* state_src, CTYPE* state_dst, ITYPE dim);
double dm_M0_prob(UINT target_qubit_index, const CTYPE* state, ITYPE dim);
double dm_M1_prob(UINT target_qubit_index, const CTYPE* state, ITYPE dim);
double dm_marginal_prob(const UINT* sorted_target_qubit_index_list, const UINT* measured_value_list,
    UINT target_qubit_index_count, const CTYPE* state, ITYPE dim);
double dm_expectation_value_multi_qubit_Pauli_operator_partial_list(const UINT* target_qubit_index_list,
    const UINT* Pauli_operator_type_list, UINT target_qubit_index_count, const CTYPE* state, ITYPE dim);
