// A program written against csim's operator API (names, argument lists, CTYPE = std::complex<double>),
// linked against libcsim_b200.so and run on device memory.  It applies a fixed gate sequence and writes
// the final state and a few statistics to the file named by argv[1]; tests/test_csim_compat.py replays
// the same sequence with the oracle and compares.
#include <cmath>
#include <complex>
#include <cstdio>
#include <stdexcept>
#include <vector>

#include "qulacs_b200.h"
#include "qulacs_b200/csim_compat.hpp"

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    const UINT n = 10;
    const ITYPE dim = ITYPE(1) << n;
    CTYPE* state = allocate_quantum_state(dim);
    initialize_quantum_state(state, dim);
    for (UINT q = 0; q < n; ++q) {
        RX_gate(q, 0.3 + 0.1 * q, state, dim);
        RY_gate(q, -0.7 + 0.05 * q, state, dim);
        RZ_gate(q, 1.1 - 0.2 * q, state, dim);
    }
    for (UINT q = 0; q + 1 < n; ++q) CNOT_gate(q, q + 1, state, dim);
    const double h = 1.0 / std::sqrt(2.0);
    const CTYPE u[4] = {CTYPE(h, 0), CTYPE(0, h), CTYPE(0, h), CTYPE(h, 0)};
    single_qubit_dense_matrix_gate(4, u, state, dim);
    CTYPE m2[16];
    for (int i = 0; i < 16; ++i) m2[i] = (i % 5 == 0) ? CTYPE(std::cos(0.4), std::sin(0.4)) : CTYPE(0, 0);
    double_qubit_dense_matrix_gate_c(2, 7, m2, state, dim);
    CZ_gate(1, 8, state, dim);
    SWAP_gate(0, 9, state, dim);
    H_gate(3, state, dim);
    T_gate(5, state, dim);
    const UINT tl[3] = {6, 2, 8};
    std::vector<CTYPE> m3(64, CTYPE(0, 0));
    for (int i = 0; i < 8; ++i) m3[i * 8 + (7 - i)] = CTYPE(0, 1);  // i * reversal permutation
    multi_qubit_dense_matrix_gate(tl, 3, m3.data(), state, dim);
    const UINT pt[3] = {1, 4, 7}, pid[3] = {1, 2, 3};
    multi_qubit_Pauli_rotation_gate_partial_list(pt, pid, 3, 0.9, state, dim);
    const UINT ct[1] = {3}, cv[1] = {1};
    multi_qubit_control_single_qubit_dense_matrix_gate(ct, cv, 1, 6, u, state, dim);

    const double ev = expectation_value_multi_qubit_Pauli_operator_partial_list(pt, pid, 3, state, dim);
    const double norm = state_norm_squared(state, dim);
    const double p0 = M0_prob(2, state, dim);
    const CTYPE ip = state_inner_product(state, state, dim);
    std::vector<CTYPE> host(dim);
    if (qs_get_state(state, host.data(), dim, nullptr) != QS_OK) return 3;
    release_quantum_state(state);
    // an invalid call throws instead of exiting
    bool threw = false;
    try {
        CTYPE* s2 = allocate_quantum_state(dim);
        RX_gate(n + 3, 0.1, s2, dim);
    } catch (const std::runtime_error&) {
        threw = true;
    }
    FILE* f = std::fopen(argv[1], "wb");
    if (!f) return 4;
    const double stats[5] = {ev, norm, p0, ip.real(), threw ? 1.0 : 0.0};
    std::fwrite(stats, sizeof(double), 5, f);
    std::fwrite(host.data(), sizeof(CTYPE), dim, f);
    std::fclose(f);
    std::printf("OK\n");
    return 0;
}
