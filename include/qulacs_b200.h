/*
 * qulacs_b200.h -- C ABI of the B200 (sm_100a) state-update library.
 *
 * Drop-in boundary for the reference's csim / gpusim operator layer.  Every entry point keeps the
 * csim name and argument order (src/csim/update_ops.hpp, src/csim/stat_ops.hpp,
 * src/csim/update_ops_dm.hpp, src/csim/stat_ops_dm.hpp), prefixed `qs_`, and differs in three ways:
 *   - `state` is a DEVICE pointer to `dim` complex128 amplitudes ((re, im) doubles, the layout of
 *     csim's CTYPE = std::complex<double>), as gpusim's `void* state` (src/gpusim/update_ops_cuda.h);
 *   - a trailing `void* stream` (a cudaStream_t; NULL = the legacy default stream) replaces gpusim's
 *     `(void* stream, UINT device_number)`: the device is the current device of the calling thread;
 *   - every function returns an int status (QS_OK or a QS_ERR_* code, message in
 *     qs_get_last_error()) instead of void / exit(1) (src/gpusim/util.cuh:28-42).
 * Matrices and index lists are HOST pointers, read before the call returns.  Gate calls are
 * asynchronous on `stream`; calls that return a value to the host synchronise `stream`.
 * Complex matrices are row-major arrays of interleaved doubles; for a k-target matrix, bit j of the
 * row/column index refers to target_qubit_index_list[j] (src/csim/utility.cpp:77-93).
 */
#ifndef QULACS_B200_H_
#define QULACS_B200_H_

#ifdef __cplusplus
extern "C" {
#endif

#define QS_API __attribute__((visibility("default")))

typedef unsigned int QS_UINT;       /* csim UINT  (src/csim/type.hpp:14) */
typedef unsigned long long QS_ITYPE; /* csim ITYPE (src/csim/type.hpp:29) */

/* ---- status codes ---- */
#define QS_OK 0
#define QS_ERR_INVALID_ARGUMENT 1 /* bad qubit index, duplicate targets, dim not 2^n, k out of range */
#define QS_ERR_OUT_OF_MEMORY 2    /* cudaMalloc failed (the reference calls exit(1), memory_ops.cpp:21-25) */
#define QS_ERR_CUDA 3             /* any other CUDA runtime error */
#define QS_ERR_TIMEOUT 4          /* a bounded device wait expired (persistent executor) */
#define QS_ERR_NOT_SUPPORTED 5    /* valid request outside this library's limits */
#define QS_ERR_NO_DEVICE 6        /* no CUDA device visible */
#define QS_ERR_REJECTED 7         /* admission control refused a request (serving loop) */

QS_API const char* qs_get_last_error(void);
QS_API const char* qs_version(void);
/* Number of kernels this library has launched in this process (diagnostic; no reference counterpart). */
QS_API unsigned long long qs_launch_count(void);
QS_API int qs_device_synchronize(void);
QS_API int qs_stream_synchronize(void* stream);
/* Non-blocking CUDA stream for concurrent work (serving workers); no reference counterpart. */
QS_API int qs_stream_create(void** stream_out);
/* Same with the device's highest (high != 0) or lowest scheduling priority: pending CTAs of kernels on
 * a higher-priority stream are scheduled before those of lower-priority streams (serving: small
 * requests are not held behind a large one). */
QS_API int qs_stream_create_with_priority(int high, void** stream_out);
QS_API int qs_stream_destroy(void* stream);

/* ---- memory and initialisation (src/csim/memory_ops.hpp, src/csim/init_ops.hpp) ---- */
/* allocate_quantum_state (memory_ops.cpp:17-27): device buffer of dim complex128 amplitudes. */
QS_API int qs_allocate_quantum_state(QS_ITYPE dim, void** state_out);
/* complex64 variant for the reduced-precision (fused) path: dim (re, im) floats. */
QS_API int qs_allocate_quantum_state_c64(QS_ITYPE dim, void** state_out);
/* Device buffer of `bytes` bytes (e.g. an arena that several states are carved from); release with
 * qs_release_quantum_state.  No reference counterpart. */
QS_API int qs_allocate_bytes(QS_ITYPE bytes, void** out);
/* release_quantum_state (memory_ops.cpp:29-31). */
QS_API int qs_release_quantum_state(void* state);
/* initialize_quantum_state (init_ops_fill.cpp:10-23): |0...0>. */
QS_API int qs_initialize_quantum_state(void* state, QS_ITYPE dim, void* stream);
QS_API int qs_initialize_quantum_state_c64(void* state, QS_ITYPE dim, void* stream);
/* set_computational_basis-style fill: |basis>. */
QS_API int qs_set_computational_basis(QS_ITYPE basis, void* state, QS_ITYPE dim, void* stream);
/* Host <-> device copies of a whole state (cppsim QuantumStateGpu::load / duplicate_data_cpp). */
QS_API int qs_load_state(const void* host_src, void* state, QS_ITYPE dim, void* stream);
QS_API int qs_get_state(const void* state, void* host_dst, QS_ITYPE dim, void* stream);
/* complex128 -> complex64 and back (rounding to nearest). */
QS_API int qs_state_to_c64(const void* state_c128, void* state_c64, QS_ITYPE dim, void* stream);
QS_API int qs_state_to_c128(const void* state_c64, void* state_c128, QS_ITYPE dim, void* stream);

/* ---- whole-state arithmetic (src/csim/update_ops.hpp:510, 1500-1505; update_ops_named_state.cpp) ---- */
/* state_add (:1500): state += state_added */
QS_API int qs_state_add(const void* state_added, void* state, QS_ITYPE dim, void* stream);
/* state_add_with_coef (:1501): state += coef * state_added (coef interleaved complex) */
QS_API int qs_state_add_with_coef(const double coef[2], const void* state_added, void* state, QS_ITYPE dim,
    void* stream);
/* state_multiply (:1505): state *= coef */
QS_API int qs_state_multiply(const double coef[2], void* state, QS_ITYPE dim, void* stream);
/* normalize (:510): state *= sqrt(1 / squared_norm) */
QS_API int qs_normalize(double squared_norm, void* state, QS_ITYPE dim, void* stream);
/* Haar-random pure state: amplitudes g1 + i g2 of independent standard normals, normalised.  The
 * reference (init_ops_random.cpp:21-80) draws from per-OpenMP-thread xorshift streams, so its values
 * depend on the host's thread count; this draws from a counter-based generator (splitmix64 per
 * amplitude index and seed), the same distribution, reproducible for a seed on any device. */
QS_API int qs_initialize_Haar_random_state_with_seed(void* state, QS_ITYPE dim, QS_UINT seed, void* stream);
/* state[i] *= factors[i], `factors` a device array of dim complex128 (cppsim
 * QuantumStateCpu::multiply_elementwise_function, cppsim/state.hpp:885-891, with func(i) tabulated). */
QS_API int qs_state_multiply_elementwise(const void* factors, void* state, QS_ITYPE dim, void* stream);
/* cppsim gate::RandomUnitary(targets, seed) (gate_factory.cpp:351-380) on the host: the same
 * mt19937_64 / std::normal_distribution draws in the same order, and the Q of their QR factorisation
 * with a positive real R diagonal.  `matrix_out`: 4^qubit_count complex128, row-major; 1..10 qubits. */
QS_API int qs_random_unitary_matrix(QS_UINT qubit_count, QS_UINT seed, double* matrix_out);
/* GeneralQuantumOperator::add_random_operator(count, seed) (general_quantum_operator.cpp:179-202) on
 * the host: for each term t, pauli_ids_out[t * qubit_count + q] is qubit q's Pauli id (0..3) and
 * coefs_out[t] its real coefficient in [-1, 1), from the reference's mt19937_64 draws. */
QS_API int qs_random_operator_terms(QS_UINT qubit_count, QS_UINT operator_count, QS_UINT seed,
    QS_UINT* pauli_ids_out, double* coefs_out);
/* Device-to-device copy of `count` complex128 entries (cppsim QuantumStateGpu::load(state)). */
QS_API int qs_copy_state(const void* src, void* dst, QS_ITYPE count, void* stream);
/* One amplitude to the host (cppsim QuantumState::data_cpp()[index]).  Synchronises `stream`. */
QS_API int qs_get_amplitude(const void* state, QS_ITYPE dim, QS_ITYPE index, double out[2], void* stream);

/* ---- single-qubit gates (src/csim/update_ops.hpp) ---- */
/* update_ops.hpp:720 single_qubit_dense_matrix_gate(UINT, const CTYPE[4], CTYPE*, ITYPE) */
QS_API int qs_single_qubit_dense_matrix_gate(
    QS_UINT target_qubit_index, const double matrix[8], void* state, QS_ITYPE dim, void* stream);
/* update_ops.hpp:758 single_qubit_diagonal_matrix_gate */
QS_API int qs_single_qubit_diagonal_matrix_gate(
    QS_UINT target_qubit_index, const double diagonal_matrix[4], void* state, QS_ITYPE dim, void* stream);
/* update_ops.hpp:793 single_qubit_phase_gate */
QS_API int qs_single_qubit_phase_gate(
    QS_UINT target_qubit_index, const double phase[2], void* state, QS_ITYPE dim, void* stream);
/* update_ops.hpp:559/589/619 RX_gate / RY_gate / RZ_gate: exp(+i angle P / 2) */
QS_API int qs_RX_gate(QS_UINT target_qubit_index, double angle, void* state, QS_ITYPE dim, void* stream);
QS_API int qs_RY_gate(QS_UINT target_qubit_index, double angle, void* state, QS_ITYPE dim, void* stream);
QS_API int qs_RZ_gate(QS_UINT target_qubit_index, double angle, void* state, QS_ITYPE dim, void* stream);
/* update_ops.hpp:42-330 named one-qubit gates */
QS_API int qs_X_gate(QS_UINT target_qubit_index, void* state, QS_ITYPE dim, void* stream);
QS_API int qs_Y_gate(QS_UINT target_qubit_index, void* state, QS_ITYPE dim, void* stream);
QS_API int qs_Z_gate(QS_UINT target_qubit_index, void* state, QS_ITYPE dim, void* stream);
QS_API int qs_H_gate(QS_UINT target_qubit_index, void* state, QS_ITYPE dim, void* stream);
QS_API int qs_S_gate(QS_UINT target_qubit_index, void* state, QS_ITYPE dim, void* stream);
QS_API int qs_Sdag_gate(QS_UINT target_qubit_index, void* state, QS_ITYPE dim, void* stream);
QS_API int qs_T_gate(QS_UINT target_qubit_index, void* state, QS_ITYPE dim, void* stream);
QS_API int qs_Tdag_gate(QS_UINT target_qubit_index, void* state, QS_ITYPE dim, void* stream);
QS_API int qs_sqrtX_gate(QS_UINT target_qubit_index, void* state, QS_ITYPE dim, void* stream);
QS_API int qs_sqrtXdag_gate(QS_UINT target_qubit_index, void* state, QS_ITYPE dim, void* stream);
QS_API int qs_sqrtY_gate(QS_UINT target_qubit_index, void* state, QS_ITYPE dim, void* stream);
QS_API int qs_sqrtYdag_gate(QS_UINT target_qubit_index, void* state, QS_ITYPE dim, void* stream);
QS_API int qs_P0_gate(QS_UINT target_qubit_index, void* state, QS_ITYPE dim, void* stream);
QS_API int qs_P1_gate(QS_UINT target_qubit_index, void* state, QS_ITYPE dim, void* stream);

/* ---- two-qubit and multi-qubit gates ---- */
/* update_ops.hpp:343 CNOT_gate(UINT control, UINT target, CTYPE*, ITYPE) */
QS_API int qs_CNOT_gate(QS_UINT control_qubit_index, QS_UINT target_qubit_index, void* state,
    QS_ITYPE dim, void* stream);
/* update_ops.hpp:373 CZ_gate */
QS_API int qs_CZ_gate(QS_UINT control_qubit_index, QS_UINT target_qubit_index, void* state,
    QS_ITYPE dim, void* stream);
/* update_ops.hpp:403 SWAP_gate */
QS_API int qs_SWAP_gate(QS_UINT target_qubit_index_0, QS_UINT target_qubit_index_1, void* state,
    QS_ITYPE dim, void* stream);
/* update_ops.hpp:1277 double_qubit_dense_matrix_gate_c (matrix bit 0 <-> t1, bit 1 <-> t2) */
QS_API int qs_double_qubit_dense_matrix_gate_c(QS_UINT target_qubit_index1,
    QS_UINT target_qubit_index2, const double matrix[32], void* state, QS_ITYPE dim, void* stream);
/* update_ops.hpp:1330 multi_qubit_dense_matrix_gate; this library supports 1 <= count <= 12. */
QS_API int qs_multi_qubit_dense_matrix_gate(const QS_UINT* target_qubit_index_list,
    QS_UINT target_qubit_index_count, const double* matrix, void* state, QS_ITYPE dim, void* stream);
/* update_ops.hpp:1459 multi_qubit_diagonal_matrix_gate; 1 <= count <= 20. */
QS_API int qs_multi_qubit_diagonal_matrix_gate(const QS_UINT* target_qubit_index_list,
    QS_UINT target_qubit_index_count, const double* diagonal_element, void* state, QS_ITYPE dim,
    void* stream);
/* update_ops.hpp:832 single_qubit_control_single_qubit_dense_matrix_gate */
QS_API int qs_single_qubit_control_single_qubit_dense_matrix_gate(QS_UINT control_qubit_index,
    QS_UINT control_value, QS_UINT target_qubit_index, const double matrix[8], void* state,
    QS_ITYPE dim, void* stream);
/* update_ops.hpp:880 multi_qubit_control_single_qubit_dense_matrix_gate */
QS_API int qs_multi_qubit_control_single_qubit_dense_matrix_gate(
    const QS_UINT* control_qubit_index_list, const QS_UINT* control_value_list,
    QS_UINT control_qubit_index_count, QS_UINT target_qubit_index, const double matrix[8],
    void* state, QS_ITYPE dim, void* stream);
/* update_ops.hpp:1445 multi_qubit_control_multi_qubit_dense_matrix_gate; targets <= 12. */
QS_API int qs_multi_qubit_control_multi_qubit_dense_matrix_gate(
    const QS_UINT* control_qubit_index_list, const QS_UINT* control_value_list,
    QS_UINT control_qubit_index_count, const QS_UINT* target_qubit_index_list,
    QS_UINT target_qubit_index_count, const double* matrix, void* state, QS_ITYPE dim, void* stream);
/* update_ops.hpp:1003 multi_qubit_Pauli_gate_partial_list (ids: 0=I 1=X 2=Y 3=Z) */
QS_API int qs_multi_qubit_Pauli_gate_partial_list(const QS_UINT* target_qubit_index_list,
    const QS_UINT* Pauli_operator_type_list, QS_UINT target_qubit_index_count, void* state,
    QS_ITYPE dim, void* stream);
/* update_ops.hpp:1191 multi_qubit_Pauli_rotation_gate_partial_list: exp(i angle P / 2) */
QS_API int qs_multi_qubit_Pauli_rotation_gate_partial_list(const QS_UINT* target_qubit_index_list,
    const QS_UINT* Pauli_operator_type_list, QS_UINT target_qubit_index_count, double angle,
    void* state, QS_ITYPE dim, void* stream);
/* update_ops.hpp:927 / :1097 multi_qubit_Pauli(_rotation)_gate_whole_list: id j acts on qubit j,
 * j < qubit_count (<= the state's qubit count). */
QS_API int qs_multi_qubit_Pauli_gate_whole_list(const QS_UINT* Pauli_operator_type_list, QS_UINT qubit_count,
    void* state, QS_ITYPE dim, void* stream);
QS_API int qs_multi_qubit_Pauli_rotation_gate_whole_list(const QS_UINT* Pauli_operator_type_list,
    QS_UINT qubit_count, double angle, void* state, QS_ITYPE dim, void* stream);
/* update_ops_pauli_single.cpp:14-52 single_qubit_Pauli_gate / single_qubit_Pauli_rotation_gate:
 * id 0 leaves the state unchanged, 1/2/3 apply X/Y/Z or RX/RY/RZ(angle); other ids are invalid. */
QS_API int qs_single_qubit_Pauli_gate(QS_UINT target_qubit_index, QS_UINT Pauli_operator_type, void* state,
    QS_ITYPE dim, void* stream);
QS_API int qs_single_qubit_Pauli_rotation_gate(QS_UINT target_qubit_index, QS_UINT Pauli_operator_index,
    double angle, void* state, QS_ITYPE dim, void* stream);
/* update_ops.hpp:1387 single_qubit_control_multi_qubit_dense_matrix_gate; targets <= 12. */
QS_API int qs_single_qubit_control_multi_qubit_dense_matrix_gate(QS_UINT control_qubit_index,
    QS_UINT control_value, const QS_UINT* target_qubit_index_list, QS_UINT target_qubit_index_count,
    const double* matrix, void* state, QS_ITYPE dim, void* stream);
/* update_ops.hpp:1464 multi_qubit_control_multi_qubit_diagonal_matrix_gate
 * (update_ops_matrix_diagonal_multi.cpp:60-112): diagonal_element[y] multiplies the amplitudes whose
 * target bits spell y and whose control bits equal the control values; targets + controls <= 20. */
QS_API int qs_multi_qubit_control_multi_qubit_diagonal_matrix_gate(const QS_UINT* control_qubit_index_list,
    const QS_UINT* control_value_list, QS_UINT control_qubit_index_count, const QS_UINT* target_qubit_index_list,
    QS_UINT target_qubit_index_count, const double* diagonal_element, void* state, QS_ITYPE dim, void* stream);

/* update_ops.hpp:1495 reflection_gate: state <- 2 <r|state> r - state (synchronises `stream`) */
QS_API int qs_reflection_gate(const void* reflection_state, void* state, QS_ITYPE dim, void* stream);
/* update_ops.hpp:435 FusedSWAP_gate: qubits [t0, t0 + block_size) swapped with [t1, t1 + block_size);
 * the blocks must not overlap and must lie inside the state. */
QS_API int qs_FusedSWAP_gate(QS_UINT target_qubit_index_0, QS_UINT target_qubit_index_1, QS_UINT block_size,
    void* state, QS_ITYPE dim, void* stream);
/* init_ops.hpp:20 initialize_Haar_random_state: the seeded form with a seed from std::random_device */
QS_API int qs_initialize_Haar_random_state(void* state, QS_ITYPE dim, void* stream);

/* ---- state manipulation (src/csim/stat_ops.hpp:17-22, stat_ops_dm.hpp:13-20); `dst` is a separate,
 * caller-allocated device buffer of the result's size ---- */
/* dst[l * dim_right + r] = left[l] right[r] (the right state on the low qubits) */
QS_API int qs_state_tensor_product(const void* state_left, QS_ITYPE dim_left, const void* state_right,
    QS_ITYPE dim_right, void* state_dst, void* stream);
/* dst[i] = src[sum over set bits q of i of 2^qubit_order[q]]; qubit_order lists every qubit once */
QS_API int qs_state_permutate_qubit(const QS_UINT* qubit_order, const void* state_src, void* state_dst,
    QS_UINT qubit_count, QS_ITYPE dim, void* stream);
/* dst (dim >> target_count amplitudes) = src restricted to target[j] = projection[j] */
QS_API int qs_state_drop_qubits(const QS_UINT* target, const QS_UINT* projection, QS_UINT target_count,
    const void* state_src, void* state_dst, QS_ITYPE dim, void* stream);
QS_API int qs_dm_state_tensor_product(const void* state_left, QS_ITYPE dim_left, const void* state_right,
    QS_ITYPE dim_right, void* state_dst, void* stream);
QS_API int qs_dm_state_permutate_qubit(const QS_UINT* qubit_order, const void* state_src, void* state_dst,
    QS_UINT qubit_count, QS_ITYPE dim, void* stream);
/* partial trace over the targets; dim is the source's 2^n, dst holds (dim >> target_count)^2 entries */
QS_API int qs_dm_state_partial_trace_from_density_matrix(const QS_UINT* target, QS_UINT target_count,
    const void* state_src, void* state_dst, QS_ITYPE dim, void* stream);
QS_API int qs_dm_state_partial_trace_from_state_vector(const QS_UINT* target, QS_UINT target_count,
    const void* state_src, void* state_dst, QS_ITYPE dim, void* stream);

/* ---- statistics (src/csim/stat_ops.hpp); results to host, stream synchronised ---- */
/* stat_ops.hpp:5 state_norm_squared */
/* measurement_distribution_entropy (stat_ops.hpp:10, stat_ops_probability.cpp:83-99): sum of -p log p
 * over p = |a_i|^2 clamped below at 1e-15.  Synchronises `stream`. */
QS_API int qs_measurement_distribution_entropy(const void* state, QS_ITYPE dim, void* stream, double* out);
QS_API int qs_state_norm_squared(const void* state, QS_ITYPE dim, void* stream, double* out);
/* stat_ops.hpp:12 state_inner_product: sum conj(bra_i) ket_i -> out[0] + i out[1] */
QS_API int qs_state_inner_product(const void* state_bra, const void* state_ket, QS_ITYPE dim,
    void* stream, double out[2]);
/* stat_ops.hpp:24/26/28 M0_prob, M1_prob, marginal_prob */
QS_API int qs_M0_prob(QS_UINT target_qubit_index, const void* state, QS_ITYPE dim, void* stream, double* out);
QS_API int qs_M1_prob(QS_UINT target_qubit_index, const void* state, QS_ITYPE dim, void* stream, double* out);
QS_API int qs_marginal_prob(const QS_UINT* sorted_target_qubit_index_list, const QS_UINT* measured_value_list,
    QS_UINT target_qubit_index_count, const void* state, QS_ITYPE dim, void* stream, double* out);
/* stat_ops.hpp:38 expectation_value_multi_qubit_Pauli_operator_partial_list */
QS_API int qs_expectation_value_multi_qubit_Pauli_operator_partial_list(
    const QS_UINT* target_qubit_index_list, const QS_UINT* Pauli_operator_type_list,
    QS_UINT target_qubit_index_count, const void* state, QS_ITYPE dim, void* stream, double* out);
/* stat_ops.hpp:32 expectation_value_single_qubit_Pauli_operator (id 0 gives <psi|psi>) */
QS_API int qs_expectation_value_single_qubit_Pauli_operator(QS_UINT target_qubit_index,
    QS_UINT Pauli_operator_type, const void* state, QS_ITYPE dim, void* stream, double* out);
/* stat_ops.hpp:35 expectation_value_multi_qubit_Pauli_operator_whole_list: id j on qubit j */
QS_API int qs_expectation_value_multi_qubit_Pauli_operator_whole_list(const QS_UINT* Pauli_operator_type_list,
    QS_UINT qubit_count, const void* state, QS_ITYPE dim, void* stream, double* out);
/* stat_ops.hpp:42 transition_amplitude_multi_qubit_Pauli_operator_whole_list: <bra|P|ket> */
QS_API int qs_transition_amplitude_multi_qubit_Pauli_operator_whole_list(const QS_UINT* Pauli_operator_type_list,
    QS_UINT qubit_count, const void* state_bra, const void* state_ket, QS_ITYPE dim, void* stream, double out[2]);
/* stat_ops.hpp:45 transition_amplitude_multi_qubit_Pauli_operator_partial_list: <bra|P|ket> */
QS_API int qs_transition_amplitude_multi_qubit_Pauli_operator_partial_list(
    const QS_UINT* target_qubit_index_list, const QS_UINT* Pauli_operator_type_list,
    QS_UINT target_qubit_index_count, const void* state_bra, const void* state_ket, QS_ITYPE dim,
    void* stream, double out[2]);
/*
 * Batched <P_k> for many Pauli strings in one call (GeneralQuantumOperator::get_expectation_value,
 * cppsim/general_quantum_operator.cpp:105-141, without the coefficient).  Term k is given by its
 * bit-flip mask x_masks[k], phase-flip mask z_masks[k] and Y count (src/csim/utility.cpp:12-43).
 * Writes values[k] = <psi|P_k|psi> (real) for k < term_count.
 */
QS_API int qs_expectation_value_pauli_batch(const QS_ITYPE* x_masks, const QS_ITYPE* z_masks,
    const QS_UINT* y_counts, QS_UINT term_count, const void* state, QS_ITYPE dim, void* stream,
    double* values);
/*
 * sum_k coef_k <P_k> (GeneralQuantumOperator::get_expectation_value,
 * cppsim/general_quantum_operator.cpp:105-141) with the terms as qs_expectation_value_pauli_batch and
 * coefs[2k], coefs[2k+1] the real and imaginary parts of coef_k; out[0], out[1] receive the real and
 * imaginary parts of the sum.  No per-term values are formed: each pass over the state folds every
 * term it covers into one FP64 sum per thread.  Synchronises `stream` before returning.
 */
QS_API int qs_expectation_value_pauli_weighted(const QS_ITYPE* x_masks, const QS_ITYPE* z_masks,
    const QS_UINT* y_counts, const double* coefs, QS_UINT term_count, const void* state, QS_ITYPE dim,
    void* stream, double out[2]);
/* The plan qs_expectation_value_pauli_weighted follows for these terms on a state of dim amplitudes,
 * host only (diagnostic; no reference counterpart): *passes_out = passes over the state;
 * kind_counts = terms evaluated {Z-only, bit flips within a thread's registers, partner amplitudes
 * from shared memory, partner rows selected per thread, one value each outside the passes}. */
QS_API int qs_expectation_value_pauli_weighted_plan(const QS_ITYPE* x_masks, const QS_ITYPE* z_masks,
    const QS_UINT* y_counts, QS_UINT term_count, QS_ITYPE dim, QS_UINT* passes_out, QS_UINT kind_counts[5]);
/* Generated per-pass kernels for qs_expectation_value_pauli_weighted (no reference counterpart): each
 * pass's term masks compiled into a kernel with NVRTC (sm_100a), the coefficients read from device
 * memory, so one compile serves every coefficient set of the same strings.  mode 0: generic kernel
 * only; 1 (default): generate when the same terms are evaluated a second time on >= 20 qubits;
 * 2: generate at the first evaluation, any size.  Plans and kernels are cached for the process. */
QS_API int qs_set_expectation_specialized(int mode);
/* Launches of generated expectation kernels so far, and the total compile time of the last plan
 * whose kernels were generated (ms). */
QS_API int qs_expectation_specialized_info(unsigned long long* launches, double* compile_ms_last);
/* CUDA C source of pass `pass` of the weighted plan for these terms (complex64 state when c64 != 0):
 * at most out_bytes - 1 characters and a terminating 0 into `out` (may be NULL); *needed receives the
 * full size including the 0. */
QS_API int qs_expectation_pass_source(const QS_ITYPE* x_masks, const QS_ITYPE* z_masks, const QS_UINT* y_counts,
    QS_UINT term_count, QS_ITYPE dim, QS_UINT pass, int c64, char* out, QS_ITYPE out_bytes, QS_ITYPE* needed);
/*
 * cppsim QuantumStateCpu::sampling (cppsim/state.hpp:909-929) with caller-supplied uniforms in
 * [0, 1): out[c] = lower_bound(stacked_prob, uniforms[c]) - 1 over the FP64 prefix sums of |a_i|^2
 * (so 0 -> 2^64 - 1 and r > norm -> dim, as in the reference).
 */
QS_API int qs_state_sampling_with_uniforms(const void* state, QS_ITYPE dim, const double* uniforms,
    QS_UINT sampling_count, QS_ITYPE* out, void* stream);
/* qs_state_sampling_with_uniforms that also reports which draws lie within `eps` of a cumulative
 * boundary of the FP64 prefix sums (near_boundary[i] = 1; may be NULL) and how many (near_count; may
 * be NULL).  Such a draw is the one whose index may differ from the reference's serial prefix sum
 * (cppsim/state.hpp:909-929) by rounding; parity with the reference excepts exactly these draws. */
QS_API int qs_state_sampling_with_uniforms_flagged(const void* state, QS_ITYPE dim, const double* uniforms,
    QS_UINT sampling_count, double eps, QS_ITYPE* out, unsigned char* near_boundary, QS_UINT* near_count,
    void* stream);
/* qs_state_sampling_with_uniforms drawing the uniforms as the reference's Random does
 * (cppsim/utility.hpp:54-80): std::mt19937_64 seeded with `random_seed`,
 * std::uniform_real_distribution<double>(0, 1). */
QS_API int qs_state_sampling(const void* state, QS_ITYPE dim, QS_UINT sampling_count,
    QS_UINT random_seed, QS_ITYPE* out, void* stream);
/*
 * qs_state_sampling_with_uniforms without any device allocation.  No counterpart in the reference:
 * it exists for callers that cannot call cudaMalloc -- a host framework that owns all device memory
 * through its own pool and forbids foreign allocations, or a latency-bound loop where cudaMalloc /
 * cudaFree would stall (they can synchronise the whole device).  Its scratch is a statically
 * reserved 2.25 MiB array in the library's device image, held by every GPU that loads the library
 * until the process exits.  Limits: dim <= 2^28 and sampling_count <= 16384, else
 * QS_ERR_NOT_SUPPORTED.  Same results as qs_state_sampling_with_uniforms.  The first call on a
 * device looks up the array's device address, so make it before any stream capture.  That address
 * is kept for the life of the process: after a cudaDeviceReset the library's device image is loaded
 * again and the kept address is stale, so do not call this entry point after resetting a device.
 * All calls share the array: calls that overlap on the GPU race.
 */
QS_API int qs_state_sampling_with_uniforms_noalloc(const void* state, QS_ITYPE dim, const double* uniforms,
    QS_UINT sampling_count, QS_ITYPE* out, void* stream);
/* The uniforms qs_state_sampling draws for a seed (host only; cppsim/utility.hpp:54-80). */
QS_API int qs_reference_uniforms(QS_UINT random_seed, QS_UINT count, double* out);

/* ---- density matrix (src/csim/update_ops_dm.hpp, src/csim/stat_ops_dm.hpp) ----
 * `rho` is a device pointer to dim*dim complex128 entries, row-major; dim = 2^n. */
QS_API int qs_dm_allocate(QS_ITYPE dim, void** rho_out);
QS_API int qs_dm_initialize_quantum_state(void* rho, QS_ITYPE dim, void* stream); /* |0><0| */
QS_API int qs_dm_initialize_with_pure_state(void* rho, const void* pure_state, QS_ITYPE dim, void* stream);
QS_API int qs_dm_single_qubit_dense_matrix_gate(
    QS_UINT target_qubit_index, const double matrix[8], void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_multi_qubit_dense_matrix_gate(const QS_UINT* target_qubit_index_list,
    QS_UINT target_qubit_index_count, const double* matrix, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_CNOT_gate(QS_UINT control_qubit_index, QS_UINT target_qubit_index, void* rho,
    QS_ITYPE dim, void* stream);
QS_API int qs_dm_CZ_gate(QS_UINT control_qubit_index, QS_UINT target_qubit_index, void* rho,
    QS_ITYPE dim, void* stream);
QS_API int qs_dm_RX_gate(QS_UINT target_qubit_index, double angle, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_RY_gate(QS_UINT target_qubit_index, double angle, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_RZ_gate(QS_UINT target_qubit_index, double angle, void* rho, QS_ITYPE dim, void* stream);
/* update_ops_dm.hpp:37-58 named gates on rho (U rho U^dagger with csim's constant.cpp matrices; P0/P1
 * project: P rho P) */
QS_API int qs_dm_X_gate(QS_UINT target_qubit_index, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_Y_gate(QS_UINT target_qubit_index, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_Z_gate(QS_UINT target_qubit_index, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_H_gate(QS_UINT target_qubit_index, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_S_gate(QS_UINT target_qubit_index, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_Sdag_gate(QS_UINT target_qubit_index, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_T_gate(QS_UINT target_qubit_index, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_Tdag_gate(QS_UINT target_qubit_index, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_sqrtX_gate(QS_UINT target_qubit_index, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_sqrtXdag_gate(QS_UINT target_qubit_index, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_sqrtY_gate(QS_UINT target_qubit_index, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_sqrtYdag_gate(QS_UINT target_qubit_index, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_P0_gate(QS_UINT target_qubit_index, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_P1_gate(QS_UINT target_qubit_index, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_SWAP_gate(QS_UINT target_qubit_index_0, QS_UINT target_qubit_index_1, void* rho, QS_ITYPE dim,
    void* stream);
/* update_ops_dm.hpp:65-70 Pauli product and exp(i angle P / 2) on rho; ids 0=I 1=X 2=Y 3=Z, count <= 12 */
QS_API int qs_dm_multi_qubit_Pauli_gate_partial_list(const QS_UINT* target_qubit_index_list,
    const QS_UINT* Pauli_operator_type_list, QS_UINT target_qubit_index_count, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_multi_qubit_Pauli_rotation_gate_partial_list(const QS_UINT* target_qubit_index_list,
    const QS_UINT* Pauli_operator_type_list, QS_UINT target_qubit_index_count, double angle, void* rho,
    QS_ITYPE dim, void* stream);
/* update_ops_dm.hpp:24-34 controlled dense gates on rho; targets + controls <= 12 */
QS_API int qs_dm_multi_qubit_control_single_qubit_dense_matrix_gate(const QS_UINT* control_qubit_index_list,
    const QS_UINT* control_value_list, QS_UINT control_qubit_index_count, QS_UINT target_qubit_index,
    const double matrix[8], void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_multi_qubit_control_multi_qubit_dense_matrix_gate(const QS_UINT* control_qubit_index_list,
    const QS_UINT* control_value_list, QS_UINT control_qubit_index_count, const QS_UINT* target_qubit_index_list,
    QS_UINT target_qubit_index_count, const double* matrix, void* rho, QS_ITYPE dim, void* stream);
/* DepolarizingNoise(t, p) on a density matrix (cppsim/gate_factory.cpp:456-466 through the exact
 * branch of cppsim/gate_general.hpp:265-285), in one pass. */
QS_API int qs_dm_depolarizing_noise(QS_UINT target_qubit_index, double probability, void* rho,
    QS_ITYPE dim, void* stream);
/* TwoQubitDepolarizingNoise(t1, t2, p) (cppsim/gate_factory.cpp:471-500), in one pass. */
QS_API int qs_dm_two_qubit_depolarizing_noise(QS_UINT target_qubit_index1,
    QS_UINT target_qubit_index2, double probability, void* rho, QS_ITYPE dim, void* stream);
/* stat_ops_dm.hpp dm_expectation_value_multi_qubit_Pauli_operator_partial_list (stat_ops_dm.cpp:164-191) */
QS_API int qs_dm_expectation_value_multi_qubit_Pauli_operator_partial_list(
    const QS_UINT* target_qubit_index_list, const QS_UINT* Pauli_operator_type_list,
    QS_UINT target_qubit_index_count, const void* rho, QS_ITYPE dim, void* stream, double* out);
/* DensityMatrixCpu::sampling (cppsim/state_dm.hpp:383-401) with supplied uniforms. */
QS_API int qs_dm_sampling_with_uniforms(const void* rho, QS_ITYPE dim, const double* uniforms,
    QS_UINT sampling_count, QS_ITYPE* out, void* stream);
/* stat_ops_dm.hpp dm_state_norm_squared (trace) */
/* stat_ops_dm.hpp:6-11: dm_measurement_distribution_entropy (diagonal p = Re rho_ii, p <= 1e-15
 * skipped), dm_state_add, dm_state_add_with_coef, dm_state_multiply (over all dim x dim entries). */
QS_API int qs_dm_measurement_distribution_entropy(const void* rho, QS_ITYPE dim, void* stream, double* out);
QS_API int qs_dm_state_add(const void* rho_added, void* rho, QS_ITYPE dim, void* stream);
QS_API int qs_dm_state_add_with_coef(const double coef[2], const void* rho_added, void* rho, QS_ITYPE dim,
    void* stream);
QS_API int qs_dm_state_multiply(const double coef[2], void* rho, QS_ITYPE dim, void* stream);
/* update_ops_dm.cpp:14-28 dm_normalize: rho *= 1 / squared_norm (the trace, not its square root). */
QS_API int qs_dm_normalize(double squared_norm, void* rho, QS_ITYPE dim, void* stream);
/* stat_ops_dm.cpp:50-120 dm_M0_prob, dm_M1_prob, dm_marginal_prob: sums of Re rho_ii over the
 * matching diagonal indices.  Synchronise `stream`. */
QS_API int qs_dm_M0_prob(QS_UINT target, const void* rho, QS_ITYPE dim, void* stream, double* out);
QS_API int qs_dm_M1_prob(QS_UINT target, const void* rho, QS_ITYPE dim, void* stream, double* out);
QS_API int qs_dm_marginal_prob(const QS_UINT* targets, const QS_UINT* values, QS_UINT count, const void* rho,
    QS_ITYPE dim, void* stream, double* out);
QS_API int qs_dm_state_norm_squared(const void* rho, QS_ITYPE dim, void* stream, double* out);

/* ---- circuits (cppsim QuantumCircuit, src/cppsim/circuit.hpp) ----
 * A circuit is a host-side gate list plus its device-resident schedule.  update_quantum_state
 * applies it to a complex128 state (or density matrix) in place, like
 * QuantumCircuit::update_quantum_state (circuit.cpp:46-57). */
typedef struct qs_circuit_s* qs_circuit_t;

/* Gate kinds accepted by qs_circuit_add_gate. */
#define QS_GATE_DENSE 0          /* matrix on targets (row-major 2^k x 2^k), optional controls */
#define QS_GATE_DIAGONAL 1       /* diagonal entries on targets */
#define QS_GATE_RX 2             /* params[0] = angle; csim RX_gate convention */
#define QS_GATE_RY 3
#define QS_GATE_RZ 4
#define QS_GATE_CNOT 5           /* targets[0] = control, targets[1] = target */
#define QS_GATE_CZ 6             /* targets[0] = control, targets[1] = target */
#define QS_GATE_SWAP 7
#define QS_GATE_PAULI 8          /* targets + pauli ids in params (as doubles) */
#define QS_GATE_PAULI_ROTATION 9 /* targets + ids; angle in params[count] */
#define QS_GATE_DEPOLARIZING 10  /* 1 or 2 targets, params[0] = probability (density matrix only) */

/* Execution modes of qs_circuit_update_quantum_state. */
#define QS_EXEC_GATE_BY_GATE 0 /* one kernel per gate: the reference's method */
#define QS_EXEC_STAGED 1       /* several gates per HBM pass, identical arithmetic per gate */
#define QS_EXEC_STAGED_FUSED 2 /* runs of gates composed in FP64 into k-qubit dense blocks (k chosen per
                                  circuit by measurement, or forced by qs_circuit_set_fusion), then staged */

QS_API int qs_circuit_create(QS_UINT qubit_count, qs_circuit_t* out);
QS_API int qs_circuit_destroy(qs_circuit_t circuit);
QS_API int qs_circuit_add_gate(qs_circuit_t circuit, int kind, const QS_UINT* targets,
    QS_UINT target_count, const QS_UINT* controls, const QS_UINT* control_values,
    QS_UINT control_count, const double* params, QS_UINT param_count);
QS_API int qs_circuit_gate_count(qs_circuit_t circuit, QS_UINT* out);
QS_API int qs_circuit_update_quantum_state(
    qs_circuit_t circuit, void* state, QS_ITYPE dim, int exec_mode, void* stream);
/* Number of HBM passes (kernel launches over the whole state) the staged schedule uses. */
QS_API int qs_circuit_pass_count(qs_circuit_t circuit, QS_ITYPE dim, QS_UINT* out);
/* Host-only statistics of the staged schedule (no reference counterpart): HBM passes, register
 * phases, operations inside phases, gates run by the gate-by-gate kernels between passes. */
QS_API int qs_circuit_staged_stats(qs_circuit_t circuit, QS_UINT* passes, QS_UINT* phases, QS_UINT* ops,
    QS_UINT* single_gates);
/* ---- FP64 gate fusion (the reference's counterpart: QuantumCircuitOptimizer::optimize(circuit, k),
 * cppsim/circuit_optimizer.cpp:113-168, composing with gate::merge, cppsim/gate_merge.cpp:316-356) ----
 * New circuit whose gates are the greedy k-qubit fusion of `circuit` (0 <= k <= 6): each run of
 * gates whose qubits fit in k qubits becomes one dense gate on them (ascending qubit order; a
 * one-qubit diagonal product stays diagonal; a run of one gate is kept as it is).  Host only. */
QS_API int qs_circuit_fuse(qs_circuit_t circuit, int k, qs_circuit_t* out);
/* Dense matrix of gate `index` over its qubits (targets then controls, controls expanded; matrix
 * index bit j <-> qubits[j]): qubits[<=6], matrix[2 * 4^count] interleaved complex.  Host only. */
QS_API int qs_circuit_gate_matrix(qs_circuit_t circuit, QS_UINT index, QS_UINT* qubits, QS_UINT* qubit_count,
    double* matrix);
/* QS_EXEC_STAGED_FUSED: force the block size k (0..6; 0 = no fusion), or -1 (default) to let the
 * autotuner choose on the next run: it times each candidate k = 0..6's staged passes (the specialised
 * kernels when the circuit uses them) with 2^12-amplitude tiles, then the best k with 2^11-amplitude
 * tiles, and keeps the fastest schedule. */
QS_API int qs_circuit_set_fusion(qs_circuit_t circuit, int k);
/* Specialised pass kernels (no reference counterpart): the single-state staged modes can run each HBM
 * pass as its own kernel, generated from the pass's schedule with every tile qubit, phase bit and gate
 * matrix entry a compile-time constant, compiled for sm_100a with NVRTC when the plan is built and
 * cached for the process.  mode 1 = always, 0 = never (the generic pass kernel), -1 = for states of at
 * least 2^22 amplitudes (default).  Changing the mode drops the circuit's cached schedules. */
QS_API int qs_circuit_set_specialized(qs_circuit_t circuit, int mode);
/* Whether the last-built QS_EXEC_STAGED / QS_EXEC_STAGED_FUSED schedules run specialised kernels, and the
 * wall time of compiling them (ms; 0 when every kernel came from the cache; may be NULL). */
QS_API int qs_circuit_specialized_info(qs_circuit_t circuit, int* staged, int* staged_fused, double* compile_ms);
/* CUDA C source of the specialised kernel of pass `pass` of the QS_EXEC_STAGED schedule at dim
 * amplitudes (host only; dim = 2^qubit_count >= 2^7).  buf == NULL: *size receives length + 1. */
QS_API int qs_circuit_specialized_source(qs_circuit_t circuit, QS_ITYPE dim, QS_UINT pass, char* buf,
    QS_ITYPE* size);
/* The schedule last built for QS_EXEC_STAGED_FUSED: block size (-1 before the first run), gate count
 * after fusion, HBM passes, and the autotuner's estimates in ms (estimates_ms[8], may be NULL; < 0
 * where not tried): [k] for k = 0..6 with 2^12-amplitude tiles, [7] for the best k with 2^11-amplitude
 * tiles, the tile shape the schedule uses when [7] is the smallest. */
QS_API int qs_circuit_fusion_info(qs_circuit_t circuit, int* k, QS_UINT* gate_count, QS_UINT* passes,
    double* estimates_ms);
/* The circuit acting on a density matrix of n qubits, as a circuit on the 2n-qubit vector
 * rho[row * 2^n + col] (column = qubits 0..n-1, row = n..2n-1): each gate U becomes U on the row
 * qubits and conj(U) on the column qubits, each depolarizing channel its superoperator
 * sum_k p_k K_k (x) conj(K_k) as a dense gate on (column qubits, row qubits).  Host only; this is
 * what the staged modes of qs_circuit_update_density_matrix execute. */
QS_API int qs_circuit_density_matrix_as_vector(qs_circuit_t circuit, qs_circuit_t* out);
/* Apply to a density matrix (gates as U rho U^dagger, depolarizing channels exact).
 * QS_EXEC_GATE_BY_GATE: one density-matrix kernel per gate or channel (the reference's method);
 * QS_EXEC_STAGED / QS_EXEC_STAGED_FUSED: the vector circuit above through the staged executors, so
 * a gate and the noise after it share passes (and, fused, one superoperator block). */
QS_API int qs_circuit_update_density_matrix(
    qs_circuit_t circuit, void* rho, QS_ITYPE dim, int exec_mode, void* stream);

/* ---- batched execution of many circuits (no reference counterpart: the reference runs one
 * QuantumCircuit::update_quantum_state at a time) ----
 * Applies circuits[i] to states[i] (complex128, 2^n_i amplitudes, n_i >= 4, every gate stageable:
 * <= 2 targets, no controls) for all i in ONE persistent kernel launch.  Each circuit's gates are
 * FP64-fused at block size 2 (or its qs_circuit_set_fusion size when that is 0, 1 or 2), so each
 * state's result is the same as running its circuit alone with QS_EXEC_STAGED_FUSED at that size.
 * Synchronises `stream`. */
QS_API int qs_batch_update_quantum_states(const qs_circuit_t* circuits, void* const* states, QS_UINT count,
    void* stream);
/* ---- captured CUDA graphs (no reference counterpart; the reference launches and synchronises every
 * gate, gpusim/update_ops_single.cu:126-131) ----
 * A circuit applied to one device state (mode as qs_circuit_update_quantum_state), or a batch of
 * circuits applied to their states in one persistent launch (as qs_batch_update_quantum_states, or as
 * qs_batch_update_quantum_states_c64 with FP64 passes when c64 != 0), recorded once as a CUDA graph
 * and replayed by qs_graph_launch: host planning, parameter uploads and launches are paid at creation.
 * With reset_state(s) != 0 the graph first sets each state to |0...0>.  The graph is bound to the
 * state pointers and to the circuits' gates and parameters at creation (later changes to a circuit
 * are not seen).  Creation builds plans (and autotunes, and compiles specialised kernels) first and
 * synchronises `stream`; work that copies from host memory during a run cannot be recorded, since a
 * replay would read that memory again after the call returned: a dense gate of >= 6 qubits outside the
 * staged passes (gate by gate, or a QS_EXEC_STAGED_FUSED block of 6 qubits: force a smaller block size
 * with qs_circuit_set_fusion) or a multi-qubit diagonal -> QS_ERR_NOT_SUPPORTED.  (Dense gates of 3..5
 * qubits carry their matrices as kernel parameters, which a graph keeps.)
 * A NULL stream is fine (capture then runs on a private stream). */
typedef struct qs_graph_s* qs_graph_t;
QS_API int qs_circuit_graph_create(qs_circuit_t circuit, void* state, QS_ITYPE dim, int mode, int reset_state,
    void* stream, qs_graph_t* out);
QS_API int qs_batch_graph_create(const qs_circuit_t* circuits, void* const* states, QS_UINT count, int c64,
    int reset_states, void* stream, qs_graph_t* out);
/* Replays the graph on `stream`: asynchronous for a circuit graph; a batch graph synchronises `stream`
 * and returns QS_ERR_TIMEOUT when a bounded dependency wait expired. */
QS_API int qs_graph_launch(qs_graph_t graph, void* stream);
/* Kernel launches one replay performs (they are added to qs_launch_count at each replay). */
QS_API int qs_graph_kernel_count(qs_graph_t graph, QS_ITYPE* kernels);
QS_API int qs_graph_destroy(qs_graph_t graph);
/* Failure-path check of the batch executor (no reference counterpart; the reference's GPU backend
 * exits the process on a device error, gpusim/util.cuh:28-42): runs `circuit` on `state` as a
 * one-circuit batch whose last pass waits on a completion counter that never completes, with the
 * dependency wait bounded by `wait_limit_us` (1 us .. 2 s; ordinary batches use 2 s).  Returns
 * QS_ERR_TIMEOUT, leaves the CUDA context usable, and leaves `state` with every pass but the last
 * applied.  Synchronises `stream`. */
QS_API int qs_debug_batch_wait_expiry(qs_circuit_t circuit, void* state, QS_UINT wait_limit_us, void* stream);
/* The same check for the complex64 batch kernel (qs_batch_update_quantum_states_fused_c64): its last
 * pass waits on its own counter, bounded by wait_limit_us; returns QS_ERR_TIMEOUT, context usable. */
QS_API int qs_debug_batch_wait_expiry_fused_c64(qs_circuit_t circuit, void* state_c64, QS_UINT wait_limit_us,
    void* stream);
/* The same on the fused complex64 tensor-core path: states_c64[i] holds circuits[i]'s 2^n complex64
 * amplitudes (n >= 10).  Missing plans are built on host threads in parallel; then every circuit's
 * passes run in ONE persistent launch (work items: tile pairs of (circuit, pass), a circuit's pass
 * waiting, bounded, for its previous pass).  Synchronises `stream`. */
QS_API int qs_batch_update_quantum_states_fused_c64(qs_circuit_t const* circuits, void* const* states_c64,
    QS_UINT count, void* stream);
/* Many circuits on complex64 states in one persistent launch with a chosen executor: exec 0 = tensor-core
 * blocks (qs_batch_update_quantum_states_fused_c64), 1 = FP64 passes over the complex64 tiles (the
 * kernel of qs_batch_update_quantum_states, widening on load and rounding on store; gates of <= 2
 * qubits, n >= 4), -1 = FP64 passes when every circuit's gates are stageable, else tensor cores.
 * Synchronises `stream`. */
QS_API int qs_batch_update_quantum_states_c64(qs_circuit_t const* circuits, void* const* states_c64, QS_UINT count,
    int exec, void* stream);
/* <P_k> for the Pauli terms of many complex128 states.  Terms of state i are term_offsets[i] ..
 * term_offsets[i+1]-1 (masks as qs_expectation_value_pauli_batch); values[k] receives <P_k>.  States
 * of fewer than 18 qubits share one launch (jobs of 16 Z-only strings or one bit-flip string);
 * larger states are evaluated as qs_expectation_value_pauli_batch does (bit-flip strings from
 * shared-memory span tiles).  Synchronises `stream`. */
QS_API int qs_batch_expectation_values(void* const* states, const QS_UINT* qubit_counts, QS_UINT count,
    const QS_UINT* term_offsets, const QS_ITYPE* x_masks, const QS_ITYPE* z_masks, const QS_UINT* y_counts,
    double* values, void* stream);
/* sum_k coef_k <P_k> per state (GeneralQuantumOperator::get_expectation_value for many states): terms as
 * qs_batch_expectation_values, coefs[2k], coefs[2k+1] = Re, Im of coef_k; energies[2i], energies[2i+1]
 * receive state i's sum.  Small states share one launch as above; each state of >= 18 qubits takes
 * the weighted passes of qs_expectation_value_pauli_weighted.  c64 != 0: complex64 states.
 * Synchronises `stream`. */
QS_API int qs_batch_expectation_weighted(void* const* states, const QS_UINT* qubit_counts, QS_UINT count,
    const QS_UINT* term_offsets, const QS_ITYPE* x_masks, const QS_ITYPE* z_masks, const QS_UINT* y_counts,
    const double* coefs, int c64, double* energies, void* stream);
/* Same for complex64 states (FP64 accumulation). */
QS_API int qs_batch_expectation_values_c64(void* const* states, const QS_UINT* qubit_counts, QS_UINT count,
    const QS_UINT* term_offsets, const QS_ITYPE* x_masks, const QS_ITYPE* z_masks, const QS_UINT* y_counts,
    double* values, void* stream);

/* ---- noisy sampling by trajectories (cppsim NoiseSimulator, noisesimulator.cpp:18-198) ----
 * Each of `sample_count` samples replaces every depolarizing channel of `circuit` by one Kraus operator
 * drawn as the reference draws it: the channel's operators in descending (probability, index) order
 * (QuantumGate_Probabilistic::optimize_ProbablisticGate, gate_general.hpp:350-372), one uniform u per
 * channel, operator lower_bound(cumulative, u) - 1 (noisesimulator.cpp:167-185).  Identical
 * trajectories are merged and visited in descending lexicographic order of their choices; each is
 * simulated once (from a shared device prefix state) and sampled as many times as it was drawn.  The
 * reference seeds its generator from std::random_device; here one mt19937_64(seed) stream gives all
 * selection uniforms (sample-major, channels in circuit order) and then each trajectory's sampling
 * uniforms, so a run is reproducible.
 * Host only: the number of distinct trajectories and, if `shots` is not NULL, each one's sample count. */
QS_API int qs_noise_simulator_trajectories(qs_circuit_t circuit, QS_UINT sample_count, QS_UINT seed,
    QS_UINT* trajectory_count, QS_UINT* shots);
/* Run it: `samples` (may be NULL) receives sample_count basis indices grouped by trajectory in that
 * order (Result::sampling, noisesimulator.cpp:57-65); `trajectory_states` (may be NULL, else
 * trajectory_count device complex128 buffers of dim amplitudes, NULL entries skipped) receives each
 * trajectory's final state (execute_and_get_result).  `initial_state` is a device state or NULL for
 * |0...0>.  Synchronises `stream`. */
QS_API int qs_noise_simulator_execute(qs_circuit_t circuit, const void* initial_state, QS_ITYPE dim,
    QS_UINT sample_count, QS_UINT seed, QS_ITYPE* samples, void* const* trajectory_states, void* stream);

/* ---- fused reduced-precision execution (no reference counterpart; its comparison point is the
 * reference's gate merging, QuantumCircuitOptimizer::optimize, cppsim/circuit_optimizer.cpp:113-168,
 * and gate::merge, cppsim/gate_merge.cpp:316-356) ----
 * Applies the circuit to a complex64 state (dim (re, im) floats): gates are fused into 6-qubit blocks
 * composed in FP64 and applied on the tensor cores as split-bf16 products (hi*hi + hi*lo + lo*hi)
 * with FP32 accumulation.  Needs >= 10 qubits and gates of <= 6 qubits (no noise channels). */
QS_API int qs_circuit_update_quantum_state_fused_c64(qs_circuit_t circuit, void* state_c64, QS_ITYPE dim, void* stream);
/* Applies the circuit to a complex64 state with the circuit's complex64 executor (see
 * qs_circuit_set_c64_executor): the tensor-core blocks above, or FP64 passes over the complex64 state
 * (each tile widened to FP64 in shared memory, gates fused into blocks of <= 2 qubits, rounded back
 * on the store; >= 4 qubits). */
QS_API int qs_circuit_update_quantum_state_c64(qs_circuit_t circuit, void* state_c64, QS_ITYPE dim, void* stream);
/* Complex64 executor of qs_circuit_update_quantum_state_c64: 0 = tensor-core blocks, 1 = FP64 passes,
 * -1 (default) = the tensor-core blocks when they take the circuit (>= 10 qubits, gates of <= 6
 * qubits), else the FP64 passes. */
QS_API int qs_circuit_set_c64_executor(qs_circuit_t circuit, int mode);
/* The executor of the last complex64 run on this circuit (0 tensor cores, 1 FP64 passes, -1 none). */
QS_API int qs_circuit_c64_executor_info(qs_circuit_t circuit, int* chosen);
/* Statistics of a complex64 state with FP64 accumulation (the fused path's reductions): norm, the
 * inner product <bra_c128|ket_c64> (for the infidelity 1 - |<psi|psi_FP64>|^2), batched <P_k>
 * (masks as qs_expectation_value_pauli_batch), sum_k coef_k <P_k> and sampling with supplied uniforms. */
QS_API int qs_state_norm_squared_c64(const void* state_c64, QS_ITYPE dim, void* stream, double* out);
QS_API int qs_state_inner_product_c128_c64(const void* bra_c128, const void* ket_c64, QS_ITYPE dim,
    void* stream, double out[2]);
QS_API int qs_expectation_value_pauli_batch_c64(const QS_ITYPE* x_masks, const QS_ITYPE* z_masks,
    const QS_UINT* y_counts, QS_UINT term_count, const void* state_c64, QS_ITYPE dim, void* stream,
    double* values);
/* qs_expectation_value_pauli_weighted over a complex64 state (FP64 arithmetic). */
QS_API int qs_expectation_value_pauli_weighted_c64(const QS_ITYPE* x_masks, const QS_ITYPE* z_masks,
    const QS_UINT* y_counts, const double* coefs, QS_UINT term_count, const void* state_c64, QS_ITYPE dim,
    void* stream, double out[2]);
QS_API int qs_state_sampling_with_uniforms_c64(const void* state_c64, QS_ITYPE dim, const double* uniforms,
    QS_UINT sampling_count, QS_ITYPE* out, void* stream);
/* Number of tile passes and fused blocks of the fused schedule (host only). */
QS_API int qs_circuit_fused_stats(qs_circuit_t circuit, QS_UINT* passes, QS_UINT* blocks);
/* Host-only export of fused block `index` (application order): the pass's tile qubits (<= 13),
 * the block's 6 tile-local bits, its FP64 64x64 matrix (row-major interleaved complex, may be NULL)
 * and its bf16 operand image (hi then lo, 2 x 128 x 128, may be NULL) in the UMMA K-major layout
 * with the 128-byte swizzle: 8-row x 64-element atoms of 1 KiB, atom (r / 8, k / 64) at
 * ((r / 8) * 2 + k / 64) KiB, row r % 8 at 128 (r % 8) bytes, 16-byte chunk (k / 8) % 8 stored at
 * chunk ((k / 8) % 8) ^ (r % 8); rows and columns in the order qs_circuit_fused_block_layout reports. */
QS_API int qs_circuit_fused_block_export(qs_circuit_t circuit, QS_UINT index, QS_UINT* tile_qubits,
    int* tile_qubit_count, QS_UINT* block_bits, double* matrix, unsigned short* operand_image);
/* Host-only export of fused block `index`'s operand orders and device index tables:
 * row_source[7]  source of accumulator (A) row bit i: block-local bit 0..5, or 6 = real/imaginary part;
 * k_source[6]    block-local bit at K bit 1 + i of both operands (K bit 0 = real/imaginary part);
 * coset_bits[m-6] tile bit at bit i of the coset (MMA N) index;
 * tables[640]    32-bit words rowtab[128] | coltab[128] | gn[128] (64-bit) | gj[64] (64-bit) as the
 *                kernel reads them (may be NULL): accumulator element (y, n) goes to byte
 *                rowtab[y] ^ coltab[n] of the next block's B operand (float rowtab[y] ^ coltab[n] of
 *                the swizzled output tile after the last block); the first block's B[n][2j + part] is
 *                complex64 amplitude tile_base | gn[n] | gj[j] of the state. */
QS_API int qs_circuit_fused_block_layout(qs_circuit_t circuit, QS_UINT index, int* row_source, int* k_source,
    QS_UINT* coset_bits, unsigned int* tables);

#ifdef __cplusplus
}
#endif

#endif /* QULACS_B200_H_ */
