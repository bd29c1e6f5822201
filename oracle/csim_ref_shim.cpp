// C-linkage shim over the reference csim (test infrastructure only).
//
// csim exports C++-linkage functions over std::complex<double> arrays (csim/type.hpp:15-30);
// this file gives them flat extern "C" names so that Python tests can call the reference
// itself through ctypes.  It is compiled together with the reference's own csim sources by
// oracle/Makefile into oracle/_ref/libcsim_ref.so.  Where the state-update path needs a piece of
// cppsim (which needs Eigen and Boost and cannot be built here), the few lines of cppsim control
// flow are restated below on top of the compiled csim kernels, each citing the cppsim lines.
#include <algorithm>
#include <complex>
#include <vector>

#include "csim/init_ops.hpp"
#include "csim/stat_ops.hpp"
#include "csim/stat_ops_dm.hpp"
#include "csim/update_ops.hpp"
#include "csim/update_ops_dm.hpp"

#define REF_API extern "C" __attribute__((visibility("default")))

static inline CTYPE* C(double* p) { return reinterpret_cast<CTYPE*>(p); }
static inline const CTYPE* CC(const double* p) { return reinterpret_cast<const CTYPE*>(p); }

// ---- state-vector gates (csim/update_ops.hpp) ----
REF_API void ref_single_qubit_dense_matrix_gate(UINT t, const double* m, double* s, ITYPE dim) {
    single_qubit_dense_matrix_gate(t, CC(m), C(s), dim);
}
REF_API void ref_single_qubit_diagonal_matrix_gate(UINT t, const double* d, double* s, ITYPE dim) {
    single_qubit_diagonal_matrix_gate(t, CC(d), C(s), dim);
}
REF_API void ref_single_qubit_phase_gate(UINT t, const double* ph, double* s, ITYPE dim) {
    single_qubit_phase_gate(t, *CC(ph), C(s), dim);
}
REF_API void ref_RX_gate(UINT t, double a, double* s, ITYPE dim) { RX_gate(t, a, C(s), dim); }
REF_API void ref_RY_gate(UINT t, double a, double* s, ITYPE dim) { RY_gate(t, a, C(s), dim); }
REF_API void ref_RZ_gate(UINT t, double a, double* s, ITYPE dim) { RZ_gate(t, a, C(s), dim); }
REF_API void ref_X_gate(UINT t, double* s, ITYPE dim) { X_gate(t, C(s), dim); }
REF_API void ref_Y_gate(UINT t, double* s, ITYPE dim) { Y_gate(t, C(s), dim); }
REF_API void ref_Z_gate(UINT t, double* s, ITYPE dim) { Z_gate(t, C(s), dim); }
REF_API void ref_H_gate(UINT t, double* s, ITYPE dim) { H_gate(t, C(s), dim); }
REF_API void ref_S_gate(UINT t, double* s, ITYPE dim) { S_gate(t, C(s), dim); }
REF_API void ref_Sdag_gate(UINT t, double* s, ITYPE dim) { Sdag_gate(t, C(s), dim); }
REF_API void ref_T_gate(UINT t, double* s, ITYPE dim) { T_gate(t, C(s), dim); }
REF_API void ref_Tdag_gate(UINT t, double* s, ITYPE dim) { Tdag_gate(t, C(s), dim); }
REF_API void ref_sqrtX_gate(UINT t, double* s, ITYPE dim) { sqrtX_gate(t, C(s), dim); }
REF_API void ref_sqrtXdag_gate(UINT t, double* s, ITYPE dim) { sqrtXdag_gate(t, C(s), dim); }
REF_API void ref_sqrtY_gate(UINT t, double* s, ITYPE dim) { sqrtY_gate(t, C(s), dim); }
REF_API void ref_sqrtYdag_gate(UINT t, double* s, ITYPE dim) { sqrtYdag_gate(t, C(s), dim); }
REF_API void ref_P0_gate(UINT t, double* s, ITYPE dim) { P0_gate(t, C(s), dim); }
REF_API void ref_P1_gate(UINT t, double* s, ITYPE dim) { P1_gate(t, C(s), dim); }
REF_API void ref_CNOT_gate(UINT c, UINT t, double* s, ITYPE dim) { CNOT_gate(c, t, C(s), dim); }
REF_API void ref_CZ_gate(UINT c, UINT t, double* s, ITYPE dim) { CZ_gate(c, t, C(s), dim); }
REF_API void ref_SWAP_gate(UINT a, UINT b, double* s, ITYPE dim) { SWAP_gate(a, b, C(s), dim); }
REF_API void ref_double_qubit_dense_matrix_gate_c(
    UINT t1, UINT t2, const double* m, double* s, ITYPE dim) {
    double_qubit_dense_matrix_gate_c(t1, t2, CC(m), C(s), dim);
}
REF_API void ref_multi_qubit_dense_matrix_gate(
    const UINT* tl, UINT k, const double* m, double* s, ITYPE dim) {
    multi_qubit_dense_matrix_gate(tl, k, CC(m), C(s), dim);
}
REF_API void ref_multi_qubit_diagonal_matrix_gate(
    const UINT* tl, UINT k, const double* d, double* s, ITYPE dim) {
    multi_qubit_diagonal_matrix_gate(tl, k, CC(d), C(s), dim);
}
REF_API void ref_single_qubit_control_single_qubit_dense_matrix_gate(
    UINT c, UINT cv, UINT t, const double* m, double* s, ITYPE dim) {
    single_qubit_control_single_qubit_dense_matrix_gate(c, cv, t, CC(m), C(s), dim);
}
REF_API void ref_multi_qubit_control_single_qubit_dense_matrix_gate(const UINT* cl,
    const UINT* cv, UINT nc, UINT t, const double* m, double* s, ITYPE dim) {
    multi_qubit_control_single_qubit_dense_matrix_gate(cl, cv, nc, t, CC(m), C(s), dim);
}
REF_API void ref_multi_qubit_control_multi_qubit_dense_matrix_gate(const UINT* cl,
    const UINT* cv, UINT nc, const UINT* tl, UINT nt, const double* m, double* s, ITYPE dim) {
    multi_qubit_control_multi_qubit_dense_matrix_gate(cl, cv, nc, tl, nt, CC(m), C(s), dim);
}
REF_API void ref_multi_qubit_Pauli_gate_partial_list(
    const UINT* tl, const UINT* ids, UINT cnt, double* s, ITYPE dim) {
    multi_qubit_Pauli_gate_partial_list(tl, ids, cnt, C(s), dim);
}
REF_API void ref_multi_qubit_Pauli_rotation_gate_partial_list(
    const UINT* tl, const UINT* ids, UINT cnt, double angle, double* s, ITYPE dim) {
    multi_qubit_Pauli_rotation_gate_partial_list(tl, ids, cnt, angle, C(s), dim);
}

// ---- statistics (csim/stat_ops.hpp) ----
REF_API void ref_state_add_with_coef(const double* coef, const double* added, double* s, ITYPE dim) {
    state_add_with_coef(CTYPE(coef[0], coef[1]), CC(added), C(s), dim);
}
REF_API void ref_state_multiply(const double* coef, double* s, ITYPE dim) {
    state_multiply(CTYPE(coef[0], coef[1]), C(s), dim);
}
REF_API void ref_normalize(double squared_norm, double* s, ITYPE dim) { normalize(squared_norm, C(s), dim); }
REF_API double ref_measurement_distribution_entropy(const double* s, ITYPE dim) {
    return measurement_distribution_entropy(CC(s), dim);
}
REF_API double ref_dm_measurement_distribution_entropy(const double* r, ITYPE dim) {
    return dm_measurement_distribution_entropy(CC(r), dim);
}
REF_API double ref_dm_M0_prob(UINT t, const double* r, ITYPE dim) { return dm_M0_prob(t, CC(r), dim); }
REF_API double ref_dm_M1_prob(UINT t, const double* r, ITYPE dim) { return dm_M1_prob(t, CC(r), dim); }
REF_API double ref_dm_marginal_prob(
    const UINT* sorted_tl, const UINT* vals, UINT cnt, const double* r, ITYPE dim) {
    return dm_marginal_prob(sorted_tl, vals, cnt, CC(r), dim);
}
REF_API void ref_dm_normalize(double squared_norm, double* r, ITYPE dim) { dm_normalize(squared_norm, C(r), dim); }
REF_API double ref_state_norm_squared(const double* s, ITYPE dim) {
    return state_norm_squared(CC(s), dim);
}
REF_API void ref_state_inner_product(const double* a, const double* b, ITYPE dim, double* out) {
    CTYPE r = state_inner_product(CC(a), CC(b), dim);
    out[0] = r.real();
    out[1] = r.imag();
}
REF_API double ref_expectation_value_multi_qubit_Pauli_operator_partial_list(
    const UINT* tl, const UINT* ids, UINT cnt, const double* s, ITYPE dim) {
    return expectation_value_multi_qubit_Pauli_operator_partial_list(tl, ids, cnt, CC(s), dim);
}
REF_API double ref_M0_prob(UINT t, const double* s, ITYPE dim) { return M0_prob(t, CC(s), dim); }
REF_API double ref_M1_prob(UINT t, const double* s, ITYPE dim) { return M1_prob(t, CC(s), dim); }
REF_API double ref_marginal_prob(
    const UINT* sorted_tl, const UINT* vals, UINT cnt, const double* s, ITYPE dim) {
    return marginal_prob(sorted_tl, vals, cnt, CC(s), dim);
}
REF_API void ref_transition_amplitude_multi_qubit_Pauli_operator_partial_list(const UINT* tl,
    const UINT* ids, UINT cnt, const double* bra, const double* ket, ITYPE dim, double* out) {
    CTYPE r = transition_amplitude_multi_qubit_Pauli_operator_partial_list(
        tl, ids, cnt, CC(bra), CC(ket), dim);
    out[0] = r.real();
    out[1] = r.imag();
}

// cppsim QuantumStateCpu::sampling (cppsim/state.hpp:909-929): serial FP64 running sum of
// norm(a_i) into stacked_prob[0..dim], then lower_bound(r) - 1 for each supplied uniform r.
REF_API void ref_sampling_with_uniforms(
    const double* s, ITYPE dim, const double* uniforms, UINT count, ITYPE* out) {
    const CTYPE* ptr = CC(s);
    std::vector<double> stacked_prob(dim + 1);
    double sum = 0.;
    stacked_prob[0] = 0.;
    for (ITYPE i = 0; i < dim; ++i) {
        sum += std::norm(ptr[i]);
        stacked_prob[i + 1] = sum;
    }
    for (UINT c = 0; c < count; ++c) {
        auto ite = std::lower_bound(stacked_prob.begin(), stacked_prob.end(), uniforms[c]);
        out[c] = (ITYPE)(std::distance(stacked_prob.begin(), ite) - 1);
    }
}

// ---- density matrix (csim/update_ops_dm.hpp, csim/stat_ops_dm.hpp) ----
REF_API void ref_dm_single_qubit_dense_matrix_gate(UINT t, const double* m, double* r, ITYPE dim) {
    dm_single_qubit_dense_matrix_gate(t, CC(m), C(r), dim);
}
REF_API void ref_dm_multi_qubit_dense_matrix_gate(
    const UINT* tl, UINT k, const double* m, double* r, ITYPE dim) {
    dm_multi_qubit_dense_matrix_gate(tl, k, CC(m), C(r), dim);
}
REF_API void ref_dm_CNOT_gate(UINT c, UINT t, double* r, ITYPE dim) { dm_CNOT_gate(c, t, C(r), dim); }
REF_API void ref_dm_CZ_gate(UINT c, UINT t, double* r, ITYPE dim) { dm_CZ_gate(c, t, C(r), dim); }
REF_API void ref_dm_RX_gate(UINT t, double a, double* r, ITYPE dim) { dm_RX_gate(t, a, C(r), dim); }
REF_API void ref_dm_RY_gate(UINT t, double a, double* r, ITYPE dim) { dm_RY_gate(t, a, C(r), dim); }
REF_API void ref_dm_RZ_gate(UINT t, double a, double* r, ITYPE dim) { dm_RZ_gate(t, a, C(r), dim); }
REF_API void ref_dm_X_gate(UINT t, double* r, ITYPE dim) { dm_X_gate(t, C(r), dim); }
REF_API void ref_dm_Y_gate(UINT t, double* r, ITYPE dim) { dm_Y_gate(t, C(r), dim); }
REF_API void ref_dm_Z_gate(UINT t, double* r, ITYPE dim) { dm_Z_gate(t, C(r), dim); }
REF_API double ref_dm_expectation_value_multi_qubit_Pauli_operator_partial_list(
    const UINT* tl, const UINT* ids, UINT cnt, const double* r, ITYPE dim) {
    return dm_expectation_value_multi_qubit_Pauli_operator_partial_list(tl, ids, cnt, CC(r), dim);
}

// cppsim QuantumGate_Probabilistic::update_quantum_state, density-matrix branch
// (cppsim/gate_general.hpp:265-285): copy rho twice, scale rho by (1 - sum(p)), and for every branch
// load the copy, apply the branch gate, scale by p_k, add.  The branch lists are those of
// DepolarizingNoise (cppsim/gate_factory.cpp:456-466: {X, Z, Y, I} with {p/3, p/3, p/3, 1-p}) and
// TwoQubitDepolarizingNoise (:471-500: I then the 15 two-qubit Paulis i%4 on t1, i/4 on t2, each
// p/15, applied as dense 4x4 matrices).
static void apply_pauli_dm(UINT t, int pid, CTYPE* r, ITYPE dim) {
    if (pid == 1) dm_X_gate(t, r, dim);
    else if (pid == 2) dm_Y_gate(t, r, dim);
    else if (pid == 3) dm_Z_gate(t, r, dim);
}
static void probabilistic_mixture_dm(const std::vector<double>& dist,
    const std::vector<int>& branch, UINT t1, UINT t2, bool two_qubit, CTYPE* r, ITYPE dim) {
    const ITYPE n = dim * dim;
    std::vector<CTYPE> org(r, r + n), tmp(n);
    double cum = 0.;
    for (double p : dist) cum += p;
    dm_state_multiply(1.0 - cum, r, dim);
    for (size_t g = 0; g < dist.size(); ++g) {
        CTYPE* target = org.data();
        if (g + 1 < dist.size()) {
            std::copy(org.begin(), org.end(), tmp.begin());
            target = tmp.data();
        }
        int code = branch[g];
        if (!two_qubit) {
            apply_pauli_dm(t1, code, target, dim);
        } else if (code != 0) {
            // dense 4x4 matrix of (Pauli code%4 on t1) x (Pauli code/4 on t2); matrix bit0 <-> t1
            static const CTYPE P[4][4] = {{1, 0, 0, 1}, {0, 1, 1, 0},
                {0, CTYPE(0, -1), CTYPE(0, 1), 0}, {1, 0, 0, -1}};
            const CTYPE* a = P[code % 4];
            const CTYPE* b = P[code / 4];
            CTYPE m[16];
            for (int y = 0; y < 4; ++y)
                for (int x = 0; x < 4; ++x)
                    m[y * 4 + x] = b[(y >> 1) * 2 + (x >> 1)] * a[(y & 1) * 2 + (x & 1)];
            UINT tl[2] = {t1, t2};
            dm_multi_qubit_dense_matrix_gate(tl, 2, m, target, dim);
        }
        dm_state_multiply(dist[g], target, dim);
        dm_state_add(target, r, dim);
    }
}
REF_API void ref_dm_depolarizing_noise(UINT t, double p, double* r, ITYPE dim) {
    probabilistic_mixture_dm({p / 3, p / 3, p / 3, 1 - p}, {1, 3, 2, 0}, t, 0, false, C(r), dim);
}
REF_API void ref_dm_two_qubit_depolarizing_noise(UINT t1, UINT t2, double p, double* r, ITYPE dim) {
    std::vector<double> dist(16, p / 15);
    dist[0] = 1 - p;
    std::vector<int> br(16);
    for (int i = 0; i < 16; ++i) br[i] = i;
    probabilistic_mixture_dm(dist, br, t1, t2, true, C(r), dim);
}

// DensityMatrixCpu::sampling (cppsim/state_dm.hpp:383-401): prefix of abs(rho_ii).
REF_API void ref_dm_sampling_with_uniforms(
    const double* r, ITYPE dim, const double* uniforms, UINT count, ITYPE* out) {
    const CTYPE* ptr = CC(r);
    std::vector<double> stacked_prob(dim + 1);
    double sum = 0.;
    stacked_prob[0] = 0.;
    for (ITYPE i = 0; i < dim; ++i) {
        sum += std::abs(ptr[i * dim + i]);
        stacked_prob[i + 1] = sum;
    }
    for (UINT c = 0; c < count; ++c) {
        auto ite = std::lower_bound(stacked_prob.begin(), stacked_prob.end(), uniforms[c]);
        out[c] = (ITYPE)(std::distance(stacked_prob.begin(), ite) - 1);
    }
}
