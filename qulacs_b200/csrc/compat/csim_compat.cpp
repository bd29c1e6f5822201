// libcsim_b200.so: csim's operator functions (C++ linkage, csim's exact argument lists) over device
// memory, each forwarding to the qulacs_b200 C ABI on the legacy default stream and returning when its
// work is complete.  Declarations: include/qulacs_b200/csim_compat.hpp.  A failing call throws
// std::runtime_error with the library's message (csim asserts or exits instead).
#include "qulacs_b200/csim_compat.hpp"

#include <stdexcept>
#include <string>

#include "qulacs_b200.h"

#define CSIM_API __attribute__((visibility("default")))

namespace {

void ok(int rc, const char* fn) {
    if (rc != QS_OK) throw std::runtime_error(std::string(fn) + ": " + qs_get_last_error());
}
// gates: launch, then wait for the default stream (csim returns with the state updated)
void done(int rc, const char* fn) {
    ok(rc, fn);
    ok(qs_stream_synchronize(nullptr), fn);
}
const double* d(const CTYPE* p) { return reinterpret_cast<const double*>(p); }
CTYPE cx(const double v[2]) { return CTYPE(v[0], v[1]); }

}  // namespace

#define G1(name)                                                 \
    CSIM_API void name(UINT target_qubit_index, CTYPE* state, ITYPE dim) { \
        done(qs_##name(target_qubit_index, state, dim, nullptr), #name);   \
    }

// ---------------------------------------------------------------- memory / initialisation
CSIM_API CTYPE* allocate_quantum_state(ITYPE dim) {
    void* p = nullptr;
    ok(qs_allocate_quantum_state(dim, &p), "allocate_quantum_state");
    return static_cast<CTYPE*>(p);
}
CSIM_API void release_quantum_state(CTYPE* state) { ok(qs_release_quantum_state(state), "release_quantum_state"); }
CSIM_API void initialize_quantum_state(CTYPE* state, ITYPE dim) {
    done(qs_initialize_quantum_state(state, dim, nullptr), "initialize_quantum_state");
}
CSIM_API void initialize_Haar_random_state(CTYPE* state, ITYPE dim) {
    done(qs_initialize_Haar_random_state(state, dim, nullptr), "initialize_Haar_random_state");
}
CSIM_API void initialize_Haar_random_state_with_seed(CTYPE* state, ITYPE dim, UINT seed) {
    done(qs_initialize_Haar_random_state_with_seed(state, dim, seed, nullptr), "initialize_Haar_random_state_with_seed");
}
CSIM_API CTYPE* dm_allocate_quantum_state(ITYPE dim) {
    void* p = nullptr;
    ok(qs_dm_allocate(dim, &p), "dm_allocate_quantum_state");
    return static_cast<CTYPE*>(p);
}
CSIM_API void dm_release_quantum_state(CTYPE* state) { ok(qs_release_quantum_state(state), "dm_release_quantum_state"); }
CSIM_API void dm_initialize_quantum_state(CTYPE* state, ITYPE dim) {
    done(qs_dm_initialize_quantum_state(state, dim, nullptr), "dm_initialize_quantum_state");
}
CSIM_API void dm_initialize_with_pure_state(CTYPE* state, const CTYPE* pure_state, ITYPE dim) {
    done(qs_dm_initialize_with_pure_state(state, pure_state, dim, nullptr), "dm_initialize_with_pure_state");
}

// ---------------------------------------------------------------- one-qubit gates
G1(X_gate) G1(Y_gate) G1(Z_gate) G1(S_gate) G1(Sdag_gate) G1(T_gate) G1(Tdag_gate) G1(sqrtX_gate) G1(sqrtXdag_gate)
G1(sqrtY_gate) G1(sqrtYdag_gate) G1(H_gate) G1(P0_gate) G1(P1_gate)

CSIM_API void RX_gate(UINT target_qubit_index, double angle, CTYPE* state, ITYPE dim) {
    done(qs_RX_gate(target_qubit_index, angle, state, dim, nullptr), "RX_gate");
}
CSIM_API void RY_gate(UINT target_qubit_index, double angle, CTYPE* state, ITYPE dim) {
    done(qs_RY_gate(target_qubit_index, angle, state, dim, nullptr), "RY_gate");
}
CSIM_API void RZ_gate(UINT target_qubit_index, double angle, CTYPE* state, ITYPE dim) {
    done(qs_RZ_gate(target_qubit_index, angle, state, dim, nullptr), "RZ_gate");
}
CSIM_API void single_qubit_Pauli_gate(UINT target_qubit_index, UINT Pauli_operator_type, CTYPE* state, ITYPE dim) {
    done(qs_single_qubit_Pauli_gate(target_qubit_index, Pauli_operator_type, state, dim, nullptr),
        "single_qubit_Pauli_gate");
}
CSIM_API void single_qubit_Pauli_rotation_gate(
    UINT target_qubit_index, UINT Pauli_operator_index, double angle, CTYPE* state, ITYPE dim) {
    done(qs_single_qubit_Pauli_rotation_gate(target_qubit_index, Pauli_operator_index, angle, state, dim, nullptr),
        "single_qubit_Pauli_rotation_gate");
}
CSIM_API void single_qubit_dense_matrix_gate(UINT target_qubit_index, const CTYPE matrix[4], CTYPE* state, ITYPE dim) {
    done(qs_single_qubit_dense_matrix_gate(target_qubit_index, d(matrix), state, dim, nullptr),
        "single_qubit_dense_matrix_gate");
}
CSIM_API void single_qubit_diagonal_matrix_gate(
    UINT target_qubit_index, const CTYPE diagonal_matrix[2], CTYPE* state, ITYPE dim) {
    done(qs_single_qubit_diagonal_matrix_gate(target_qubit_index, d(diagonal_matrix), state, dim, nullptr),
        "single_qubit_diagonal_matrix_gate");
}
CSIM_API void single_qubit_phase_gate(UINT target_qubit_index, CTYPE phase, CTYPE* state, ITYPE dim) {
    const double p[2] = {phase.real(), phase.imag()};
    done(qs_single_qubit_phase_gate(target_qubit_index, p, state, dim, nullptr), "single_qubit_phase_gate");
}
CSIM_API void single_qubit_control_single_qubit_dense_matrix_gate(UINT control_qubit_index, UINT control_value,
    UINT target_qubit_index, const CTYPE matrix[4], CTYPE* state, ITYPE dim) {
    done(qs_single_qubit_control_single_qubit_dense_matrix_gate(
             control_qubit_index, control_value, target_qubit_index, d(matrix), state, dim, nullptr),
        "single_qubit_control_single_qubit_dense_matrix_gate");
}
CSIM_API void multi_qubit_control_single_qubit_dense_matrix_gate(const UINT* control_qubit_index_list,
    const UINT* control_value_list, UINT control_qubit_index_count, UINT target_qubit_index, const CTYPE matrix[4],
    CTYPE* state, ITYPE dim) {
    done(qs_multi_qubit_control_single_qubit_dense_matrix_gate(control_qubit_index_list, control_value_list,
             control_qubit_index_count, target_qubit_index, d(matrix), state, dim, nullptr),
        "multi_qubit_control_single_qubit_dense_matrix_gate");
}

// ---------------------------------------------------------------- two- and multi-qubit gates
CSIM_API void CNOT_gate(UINT control_qubit_index, UINT target_qubit_index, CTYPE* state, ITYPE dim) {
    done(qs_CNOT_gate(control_qubit_index, target_qubit_index, state, dim, nullptr), "CNOT_gate");
}
CSIM_API void CZ_gate(UINT control_qubit_index, UINT target_qubit_index, CTYPE* state, ITYPE dim) {
    done(qs_CZ_gate(control_qubit_index, target_qubit_index, state, dim, nullptr), "CZ_gate");
}
CSIM_API void SWAP_gate(UINT target_qubit_index_0, UINT target_qubit_index_1, CTYPE* state, ITYPE dim) {
    done(qs_SWAP_gate(target_qubit_index_0, target_qubit_index_1, state, dim, nullptr), "SWAP_gate");
}
CSIM_API void FusedSWAP_gate(
    UINT target_qubit_index_0, UINT target_qubit_index_1, UINT block_size, CTYPE* state, ITYPE dim) {
    done(qs_FusedSWAP_gate(target_qubit_index_0, target_qubit_index_1, block_size, state, dim, nullptr),
        "FusedSWAP_gate");
}
CSIM_API void double_qubit_dense_matrix_gate_c(
    UINT target_qubit_index1, UINT target_qubit_index2, const CTYPE matrix[16], CTYPE* state, ITYPE dim) {
    done(qs_double_qubit_dense_matrix_gate_c(target_qubit_index1, target_qubit_index2, d(matrix), state, dim, nullptr),
        "double_qubit_dense_matrix_gate_c");
}
CSIM_API void multi_qubit_dense_matrix_gate(const UINT* target_qubit_index_list, UINT target_qubit_index_count,
    const CTYPE* matrix, CTYPE* state, ITYPE dim) {
    done(qs_multi_qubit_dense_matrix_gate(target_qubit_index_list, target_qubit_index_count, d(matrix), state, dim,
             nullptr),
        "multi_qubit_dense_matrix_gate");
}
CSIM_API void single_qubit_control_multi_qubit_dense_matrix_gate(UINT control_qubit_index, UINT control_value,
    const UINT* target_qubit_index_list, UINT target_qubit_index_count, const CTYPE* matrix, CTYPE* state,
    ITYPE dim) {
    done(qs_single_qubit_control_multi_qubit_dense_matrix_gate(control_qubit_index, control_value,
             target_qubit_index_list, target_qubit_index_count, d(matrix), state, dim, nullptr),
        "single_qubit_control_multi_qubit_dense_matrix_gate");
}
CSIM_API void multi_qubit_control_multi_qubit_dense_matrix_gate(const UINT* control_qubit_index_list,
    const UINT* control_value_list, UINT control_qubit_index_count, const UINT* target_qubit_index_list,
    UINT target_qubit_index_count, const CTYPE* matrix, CTYPE* state, ITYPE dim) {
    done(qs_multi_qubit_control_multi_qubit_dense_matrix_gate(control_qubit_index_list, control_value_list,
             control_qubit_index_count, target_qubit_index_list, target_qubit_index_count, d(matrix), state, dim,
             nullptr),
        "multi_qubit_control_multi_qubit_dense_matrix_gate");
}
CSIM_API void multi_qubit_diagonal_matrix_gate(const UINT* target_qubit_index_list, UINT target_qubit_index_count,
    const CTYPE* diagonal_element, CTYPE* state, ITYPE dim) {
    done(qs_multi_qubit_diagonal_matrix_gate(target_qubit_index_list, target_qubit_index_count, d(diagonal_element),
             state, dim, nullptr),
        "multi_qubit_diagonal_matrix_gate");
}
CSIM_API void multi_qubit_control_multi_qubit_diagonal_matrix_gate(const UINT* control_qubit_index_list,
    const UINT* control_value_list, UINT control_qubit_index_count, const UINT* target_qubit_index_list,
    UINT target_qubit_index_count, const CTYPE* diagonal_element, CTYPE* state, ITYPE dim) {
    done(qs_multi_qubit_control_multi_qubit_diagonal_matrix_gate(control_qubit_index_list, control_value_list,
             control_qubit_index_count, target_qubit_index_list, target_qubit_index_count, d(diagonal_element), state,
             dim, nullptr),
        "multi_qubit_control_multi_qubit_diagonal_matrix_gate");
}
CSIM_API void multi_qubit_Pauli_gate_whole_list(
    const UINT* Pauli_operator_type_list, UINT qubit_count, CTYPE* state, ITYPE dim_) {
    done(qs_multi_qubit_Pauli_gate_whole_list(Pauli_operator_type_list, qubit_count, state, dim_, nullptr),
        "multi_qubit_Pauli_gate_whole_list");
}
CSIM_API void multi_qubit_Pauli_gate_whole_list_single_thread(
    const UINT* Pauli_operator_type_list, UINT qubit_count, CTYPE* state, ITYPE dim_) {
    multi_qubit_Pauli_gate_whole_list(Pauli_operator_type_list, qubit_count, state, dim_);
}
CSIM_API void multi_qubit_Pauli_gate_partial_list(const UINT* target_qubit_index_list,
    const UINT* Pauli_operator_type_list, UINT target_qubit_index_count, CTYPE* state, ITYPE dim) {
    done(qs_multi_qubit_Pauli_gate_partial_list(target_qubit_index_list, Pauli_operator_type_list,
             target_qubit_index_count, state, dim, nullptr),
        "multi_qubit_Pauli_gate_partial_list");
}
CSIM_API void multi_qubit_Pauli_gate_partial_list_single_thread(const UINT* target_qubit_index_list,
    const UINT* Pauli_operator_type_list, UINT target_qubit_index_count, CTYPE* state, ITYPE dim) {
    multi_qubit_Pauli_gate_partial_list(target_qubit_index_list, Pauli_operator_type_list, target_qubit_index_count,
        state, dim);
}
CSIM_API void multi_qubit_Pauli_rotation_gate_whole_list(
    const UINT* Pauli_operator_type_list, UINT qubit_count, double angle, CTYPE* state, ITYPE dim_) {
    done(qs_multi_qubit_Pauli_rotation_gate_whole_list(Pauli_operator_type_list, qubit_count, angle, state, dim_,
             nullptr),
        "multi_qubit_Pauli_rotation_gate_whole_list");
}
CSIM_API void multi_qubit_Pauli_rotation_gate_whole_list_single_thread(
    const UINT* Pauli_operator_type_list, UINT qubit_count, double angle, CTYPE* state, ITYPE dim_) {
    multi_qubit_Pauli_rotation_gate_whole_list(Pauli_operator_type_list, qubit_count, angle, state, dim_);
}
CSIM_API void multi_qubit_Pauli_rotation_gate_partial_list(const UINT* target_qubit_index_list,
    const UINT* Pauli_operator_type_list, UINT target_qubit_index_count, double angle, CTYPE* state, ITYPE dim) {
    done(qs_multi_qubit_Pauli_rotation_gate_partial_list(target_qubit_index_list, Pauli_operator_type_list,
             target_qubit_index_count, angle, state, dim, nullptr),
        "multi_qubit_Pauli_rotation_gate_partial_list");
}
CSIM_API void multi_qubit_Pauli_rotation_gate_partial_list_single_thread(const UINT* target_qubit_index_list,
    const UINT* Pauli_operator_type_list, UINT target_qubit_index_count, double angle, CTYPE* state, ITYPE dim) {
    multi_qubit_Pauli_rotation_gate_partial_list(target_qubit_index_list, Pauli_operator_type_list,
        target_qubit_index_count, angle, state, dim);
}
CSIM_API void reflection_gate(const CTYPE* reflection_state, CTYPE* state, ITYPE dim) {
    done(qs_reflection_gate(reflection_state, state, dim, nullptr), "reflection_gate");
}

// ---------------------------------------------------------------- state arithmetic
CSIM_API void normalize(double squared_norm, CTYPE* state, ITYPE dim) {
    done(qs_normalize(squared_norm, state, dim, nullptr), "normalize");
}
CSIM_API void normalize_single_thread(double squared_norm, CTYPE* state, ITYPE dim) { normalize(squared_norm, state, dim); }
CSIM_API void state_add(const CTYPE* state_added, CTYPE* state, ITYPE dim) {
    done(qs_state_add(state_added, state, dim, nullptr), "state_add");
}
CSIM_API void state_add_with_coef(CTYPE coef, const CTYPE* state_added, CTYPE* state, ITYPE dim) {
    const double c[2] = {coef.real(), coef.imag()};
    done(qs_state_add_with_coef(c, state_added, state, dim, nullptr), "state_add_with_coef");
}
CSIM_API void state_add_with_coef_single_thread(CTYPE coef, const CTYPE* state_added, CTYPE* state, ITYPE dim) {
    state_add_with_coef(coef, state_added, state, dim);
}
CSIM_API void state_multiply(CTYPE coef, CTYPE* state, ITYPE dim) {
    const double c[2] = {coef.real(), coef.imag()};
    done(qs_state_multiply(c, state, dim, nullptr), "state_multiply");
}

// ---------------------------------------------------------------- statistics
CSIM_API double state_norm_squared(const CTYPE* state, ITYPE dim) {
    double v = 0;
    ok(qs_state_norm_squared(state, dim, nullptr, &v), "state_norm_squared");
    return v;
}
CSIM_API double state_norm_squared_single_thread(const CTYPE* state, ITYPE dim) { return state_norm_squared(state, dim); }
CSIM_API double measurement_distribution_entropy(const CTYPE* state, ITYPE dim) {
    double v = 0;
    ok(qs_measurement_distribution_entropy(state, dim, nullptr, &v), "measurement_distribution_entropy");
    return v;
}
CSIM_API CTYPE state_inner_product(const CTYPE* state_bra, const CTYPE* state_ket, ITYPE dim) {
    double v[2];
    ok(qs_state_inner_product(state_bra, state_ket, dim, nullptr, v), "state_inner_product");
    return cx(v);
}
CSIM_API void state_tensor_product(
    const CTYPE* state_left, ITYPE dim_left, const CTYPE* state_right, ITYPE dim_right, CTYPE* state_dst) {
    done(qs_state_tensor_product(state_left, dim_left, state_right, dim_right, state_dst, nullptr),
        "state_tensor_product");
}
CSIM_API void state_permutate_qubit(
    const UINT* qubit_order, const CTYPE* state_src, CTYPE* state_dst, UINT qubit_count, ITYPE dim) {
    done(qs_state_permutate_qubit(qubit_order, state_src, state_dst, qubit_count, dim, nullptr), "state_permutate_qubit");
}
CSIM_API void state_drop_qubits(const UINT* target, const UINT* projection, UINT target_count, const CTYPE* state_src,
    CTYPE* state_dst, ITYPE dim) {
    done(qs_state_drop_qubits(target, projection, target_count, state_src, state_dst, dim, nullptr),
        "state_drop_qubits");
}
CSIM_API double M0_prob(UINT target_qubit_index, const CTYPE* state, ITYPE dim) {
    double v = 0;
    ok(qs_M0_prob(target_qubit_index, state, dim, nullptr, &v), "M0_prob");
    return v;
}
CSIM_API double M1_prob(UINT target_qubit_index, const CTYPE* state, ITYPE dim) {
    double v = 0;
    ok(qs_M1_prob(target_qubit_index, state, dim, nullptr, &v), "M1_prob");
    return v;
}
CSIM_API double marginal_prob(const UINT* sorted_target_qubit_index_list, const UINT* measured_value_list,
    UINT target_qubit_index_count, const CTYPE* state, ITYPE dim) {
    double v = 0;
    ok(qs_marginal_prob(sorted_target_qubit_index_list, measured_value_list, target_qubit_index_count, state, dim,
           nullptr, &v),
        "marginal_prob");
    return v;
}
CSIM_API double expectation_value_single_qubit_Pauli_operator(
    UINT target_qubit_index, UINT Pauli_operator_type, const CTYPE* state, ITYPE dim) {
    double v = 0;
    ok(qs_expectation_value_single_qubit_Pauli_operator(target_qubit_index, Pauli_operator_type, state, dim, nullptr,
           &v),
        "expectation_value_single_qubit_Pauli_operator");
    return v;
}
CSIM_API double expectation_value_multi_qubit_Pauli_operator_whole_list(
    const UINT* Pauli_operator_type_list, UINT qubit_count, const CTYPE* state, ITYPE dim) {
    double v = 0;
    ok(qs_expectation_value_multi_qubit_Pauli_operator_whole_list(Pauli_operator_type_list, qubit_count, state, dim,
           nullptr, &v),
        "expectation_value_multi_qubit_Pauli_operator_whole_list");
    return v;
}
CSIM_API double expectation_value_multi_qubit_Pauli_operator_partial_list(const UINT* target_qubit_index_list,
    const UINT* Pauli_operator_type_list, UINT target_qubit_index_count, const CTYPE* state, ITYPE dim) {
    double v = 0;
    ok(qs_expectation_value_multi_qubit_Pauli_operator_partial_list(target_qubit_index_list, Pauli_operator_type_list,
           target_qubit_index_count, state, dim, nullptr, &v),
        "expectation_value_multi_qubit_Pauli_operator_partial_list");
    return v;
}
CSIM_API double expectation_value_multi_qubit_Pauli_operator_partial_list_single_thread(
    const UINT* target_qubit_index_list, const UINT* Pauli_operator_type_list, UINT target_qubit_index_count,
    const CTYPE* state, ITYPE dim) {
    return expectation_value_multi_qubit_Pauli_operator_partial_list(
        target_qubit_index_list, Pauli_operator_type_list, target_qubit_index_count, state, dim);
}
CSIM_API CTYPE transition_amplitude_multi_qubit_Pauli_operator_whole_list(const UINT* Pauli_operator_type_list,
    UINT qubit_count, const CTYPE* state_bra, const CTYPE* state_ket, ITYPE dim) {
    double v[2];
    ok(qs_transition_amplitude_multi_qubit_Pauli_operator_whole_list(Pauli_operator_type_list, qubit_count, state_bra,
           state_ket, dim, nullptr, v),
        "transition_amplitude_multi_qubit_Pauli_operator_whole_list");
    return cx(v);
}
CSIM_API CTYPE transition_amplitude_multi_qubit_Pauli_operator_partial_list(const UINT* target_qubit_index_list,
    const UINT* Pauli_operator_type_list, UINT target_qubit_index_count, const CTYPE* state_bra,
    const CTYPE* state_ket, ITYPE dim) {
    double v[2];
    ok(qs_transition_amplitude_multi_qubit_Pauli_operator_partial_list(target_qubit_index_list,
           Pauli_operator_type_list, target_qubit_index_count, state_bra, state_ket, dim, nullptr, v),
        "transition_amplitude_multi_qubit_Pauli_operator_partial_list");
    return cx(v);
}

// ---------------------------------------------------------------- density matrices
#define DMG1(name)                                                            \
    CSIM_API void dm_##name(UINT target_qubit_index, CTYPE* state, ITYPE dim) { \
        done(qs_dm_##name(target_qubit_index, state, dim, nullptr), "dm_" #name); \
    }
DMG1(X_gate) DMG1(Y_gate) DMG1(Z_gate) DMG1(S_gate) DMG1(Sdag_gate) DMG1(T_gate) DMG1(Tdag_gate) DMG1(sqrtX_gate)
DMG1(sqrtXdag_gate) DMG1(sqrtY_gate) DMG1(sqrtYdag_gate) DMG1(H_gate) DMG1(P0_gate) DMG1(P1_gate)

CSIM_API void dm_normalize(double squared_norm, CTYPE* state, ITYPE dim) {
    done(qs_dm_normalize(squared_norm, state, dim, nullptr), "dm_normalize");
}
CSIM_API void dm_single_qubit_dense_matrix_gate(UINT target_qubit_index, const CTYPE matrix[4], CTYPE* state, ITYPE dim) {
    done(qs_dm_single_qubit_dense_matrix_gate(target_qubit_index, d(matrix), state, dim, nullptr),
        "dm_single_qubit_dense_matrix_gate");
}
CSIM_API void dm_multi_qubit_control_single_qubit_dense_matrix_gate(const UINT* control_qubit_index_list,
    const UINT* control_value_list, UINT control_qubit_index_count, UINT target_qubit_index, const CTYPE matrix[4],
    CTYPE* state, ITYPE dim) {
    done(qs_dm_multi_qubit_control_single_qubit_dense_matrix_gate(control_qubit_index_list, control_value_list,
             control_qubit_index_count, target_qubit_index, d(matrix), state, dim, nullptr),
        "dm_multi_qubit_control_single_qubit_dense_matrix_gate");
}
CSIM_API void dm_multi_qubit_dense_matrix_gate(const UINT* target_qubit_index_list, UINT target_qubit_index_count,
    const CTYPE* matrix, CTYPE* state, ITYPE dim) {
    done(qs_dm_multi_qubit_dense_matrix_gate(target_qubit_index_list, target_qubit_index_count, d(matrix), state, dim,
             nullptr),
        "dm_multi_qubit_dense_matrix_gate");
}
CSIM_API void dm_multi_qubit_control_multi_qubit_dense_matrix_gate(const UINT* control_qubit_index_list,
    const UINT* control_value_list, UINT control_qubit_index_count, const UINT* target_qubit_index_list,
    UINT target_qubit_index_count, const CTYPE* matrix, CTYPE* state, ITYPE dim) {
    done(qs_dm_multi_qubit_control_multi_qubit_dense_matrix_gate(control_qubit_index_list, control_value_list,
             control_qubit_index_count, target_qubit_index_list, target_qubit_index_count, d(matrix), state, dim,
             nullptr),
        "dm_multi_qubit_control_multi_qubit_dense_matrix_gate");
}
CSIM_API void dm_CNOT_gate(UINT control_qubit_index, UINT target_qubit_index, CTYPE* state, ITYPE dim) {
    done(qs_dm_CNOT_gate(control_qubit_index, target_qubit_index, state, dim, nullptr), "dm_CNOT_gate");
}
CSIM_API void dm_CZ_gate(UINT control_qubit_index, UINT target_qubit_index, CTYPE* state, ITYPE dim) {
    done(qs_dm_CZ_gate(control_qubit_index, target_qubit_index, state, dim, nullptr), "dm_CZ_gate");
}
CSIM_API void dm_SWAP_gate(UINT target_qubit_index_0, UINT target_qubit_index_1, CTYPE* state, ITYPE dim) {
    done(qs_dm_SWAP_gate(target_qubit_index_0, target_qubit_index_1, state, dim, nullptr), "dm_SWAP_gate");
}
CSIM_API void dm_RX_gate(UINT target_qubit_index, double angle, CTYPE* state, ITYPE dim) {
    done(qs_dm_RX_gate(target_qubit_index, angle, state, dim, nullptr), "dm_RX_gate");
}
CSIM_API void dm_RY_gate(UINT target_qubit_index, double angle, CTYPE* state, ITYPE dim) {
    done(qs_dm_RY_gate(target_qubit_index, angle, state, dim, nullptr), "dm_RY_gate");
}
CSIM_API void dm_RZ_gate(UINT target_qubit_index, double angle, CTYPE* state, ITYPE dim) {
    done(qs_dm_RZ_gate(target_qubit_index, angle, state, dim, nullptr), "dm_RZ_gate");
}
CSIM_API void dm_multi_qubit_Pauli_gate_partial_list(const UINT* target_qubit_index_list,
    const UINT* Pauli_operator_type_list, UINT target_qubit_index_count, CTYPE* state, ITYPE dim) {
    done(qs_dm_multi_qubit_Pauli_gate_partial_list(target_qubit_index_list, Pauli_operator_type_list,
             target_qubit_index_count, state, dim, nullptr),
        "dm_multi_qubit_Pauli_gate_partial_list");
}
CSIM_API void dm_multi_qubit_Pauli_rotation_gate_partial_list(const UINT* target_qubit_index_list,
    const UINT* Pauli_operator_type_list, UINT target_qubit_index_count, double angle, CTYPE* state, ITYPE dim) {
    done(qs_dm_multi_qubit_Pauli_rotation_gate_partial_list(target_qubit_index_list, Pauli_operator_type_list,
             target_qubit_index_count, angle, state, dim, nullptr),
        "dm_multi_qubit_Pauli_rotation_gate_partial_list");
}
CSIM_API double dm_state_norm_squared(const CTYPE* state, ITYPE dim) {
    double v = 0;
    ok(qs_dm_state_norm_squared(state, dim, nullptr, &v), "dm_state_norm_squared");
    return v;
}
CSIM_API double dm_measurement_distribution_entropy(const CTYPE* state, ITYPE dim) {
    double v = 0;
    ok(qs_dm_measurement_distribution_entropy(state, dim, nullptr, &v), "dm_measurement_distribution_entropy");
    return v;
}
CSIM_API void dm_state_add(const CTYPE* state_added, CTYPE* state, ITYPE dim) {
    done(qs_dm_state_add(state_added, state, dim, nullptr), "dm_state_add");
}
CSIM_API void dm_state_add_with_coef(CTYPE coef, const CTYPE* state_added, CTYPE* state, ITYPE dim) {
    const double c[2] = {coef.real(), coef.imag()};
    done(qs_dm_state_add_with_coef(c, state_added, state, dim, nullptr), "dm_state_add_with_coef");
}
CSIM_API void dm_state_multiply(CTYPE coef, CTYPE* state, ITYPE dim) {
    const double c[2] = {coef.real(), coef.imag()};
    done(qs_dm_state_multiply(c, state, dim, nullptr), "dm_state_multiply");
}
CSIM_API void dm_state_tensor_product(
    const CTYPE* state_left, ITYPE dim_left, const CTYPE* state_right, ITYPE dim_right, CTYPE* state_dst) {
    done(qs_dm_state_tensor_product(state_left, dim_left, state_right, dim_right, state_dst, nullptr),
        "dm_state_tensor_product");
}
CSIM_API void dm_state_permutate_qubit(
    const UINT* qubit_order, const CTYPE* state_src, CTYPE* state_dst, UINT qubit_count, ITYPE dim) {
    done(qs_dm_state_permutate_qubit(qubit_order, state_src, state_dst, qubit_count, dim, nullptr),
        "dm_state_permutate_qubit");
}
CSIM_API void dm_state_partial_trace_from_density_matrix(
    const UINT* target, UINT target_count, const CTYPE* state_src, CTYPE* state_dst, ITYPE dim) {
    done(qs_dm_state_partial_trace_from_density_matrix(target, target_count, state_src, state_dst, dim, nullptr),
        "dm_state_partial_trace_from_density_matrix");
}
CSIM_API void dm_state_partial_trace_from_state_vector(
    const UINT* target, UINT target_count, const CTYPE* state_src, CTYPE* state_dst, ITYPE dim) {
    done(qs_dm_state_partial_trace_from_state_vector(target, target_count, state_src, state_dst, dim, nullptr),
        "dm_state_partial_trace_from_state_vector");
}
CSIM_API double dm_M0_prob(UINT target_qubit_index, const CTYPE* state, ITYPE dim) {
    double v = 0;
    ok(qs_dm_M0_prob(target_qubit_index, state, dim, nullptr, &v), "dm_M0_prob");
    return v;
}
CSIM_API double dm_M1_prob(UINT target_qubit_index, const CTYPE* state, ITYPE dim) {
    double v = 0;
    ok(qs_dm_M1_prob(target_qubit_index, state, dim, nullptr, &v), "dm_M1_prob");
    return v;
}
CSIM_API double dm_marginal_prob(const UINT* sorted_target_qubit_index_list, const UINT* measured_value_list,
    UINT target_qubit_index_count, const CTYPE* state, ITYPE dim) {
    double v = 0;
    ok(qs_dm_marginal_prob(sorted_target_qubit_index_list, measured_value_list, target_qubit_index_count, state, dim,
           nullptr, &v),
        "dm_marginal_prob");
    return v;
}
CSIM_API double dm_expectation_value_multi_qubit_Pauli_operator_partial_list(const UINT* target_qubit_index_list,
    const UINT* Pauli_operator_type_list, UINT target_qubit_index_count, const CTYPE* state, ITYPE dim) {
    double v = 0;
    ok(qs_dm_expectation_value_multi_qubit_Pauli_operator_partial_list(target_qubit_index_list,
           Pauli_operator_type_list, target_qubit_index_count, state, dim, nullptr, &v),
        "dm_expectation_value_multi_qubit_Pauli_operator_partial_list");
    return v;
}
