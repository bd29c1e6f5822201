// Host routines that reproduce the reference's seeded random constructions: gate::RandomUnitary and
// GeneralQuantumOperator::add_random_operator.
//
// RandomUnitary(targets, seed) (gate_factory.cpp:351-380):
// The reference fills a 2^k x 2^k matrix row by row with (normal() + i normal()) / sqrt(2) from
// Random (cppsim/utility.hpp:53-100: std::mt19937_64 seeded with `seed`, std::normal_distribution
// <double>(0, 1)), takes a QR factorisation and multiplies column c of Q by R_cc / |R_cc|.  That
// product is the unique Q whose R has a positive real diagonal, so it is computed here by
// Gram-Schmidt (two projection sweeps per column), which yields that Q directly.  With g++ the
// operands of `normal() + 1.i * normal()` are evaluated right to left: the imaginary part is drawn
// first; the same order is kept so that a seed gives the reference's matrix.
#include <cmath>
#include <complex>
#include <random>
#include <string>
#include <vector>

#include "../../include/qulacs_b200.h"

namespace qs {
int set_error(int code, const std::string& msg);
}

extern "C" {

QS_API int qs_random_unitary_matrix(QS_UINT qubit_count, QS_UINT seed, double* matrix_out) {
    using cd = std::complex<double>;
    if (!matrix_out) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null output matrix");
    if (qubit_count < 1 || qubit_count > 10)
        return qs::set_error(QS_ERR_INVALID_ARGUMENT, "random unitary: 1..10 qubits");
    const size_t d = size_t(1) << qubit_count;
    std::mt19937_64 mt(seed);
    std::normal_distribution<double> normal(0., 1.);
    std::vector<cd> a(d * d);  // row-major
    const double inv_sqrt2 = 1. / std::sqrt(2.);
    for (size_t i = 0; i < d; ++i)
        for (size_t j = 0; j < d; ++j) {
            const double im = normal(mt);
            const double re = normal(mt);
            a[i * d + j] = cd(re, im) * inv_sqrt2;
        }
    std::vector<cd> q(d * d);  // column c at q[c * d .. c * d + d)
    for (size_t c = 0; c < d; ++c) {
        cd* v = &q[c * d];
        for (size_t r = 0; r < d; ++r) v[r] = a[r * d + c];
        for (int sweep = 0; sweep < 2; ++sweep)
            for (size_t p = 0; p < c; ++p) {
                const cd* u = &q[p * d];
                cd dot = 0.;
                for (size_t r = 0; r < d; ++r) dot += std::conj(u[r]) * v[r];
                for (size_t r = 0; r < d; ++r) v[r] -= dot * u[r];
            }
        double nrm = 0.;
        for (size_t r = 0; r < d; ++r) nrm += std::norm(v[r]);
        nrm = std::sqrt(nrm);
        for (size_t r = 0; r < d; ++r) v[r] /= nrm;
    }
    for (size_t r = 0; r < d; ++r)
        for (size_t c = 0; c < d; ++c) {
            matrix_out[2 * (r * d + c)] = q[c * d + r].real();
            matrix_out[2 * (r * d + c) + 1] = q[c * d + r].imag();
        }
    return QS_OK;
}

// GeneralQuantumOperator::add_random_operator(count, seed) (general_quantum_operator.cpp:179-202): per
// term, one Pauli id per qubit 0..n-1 from Random::int32() % 4 (int32 is mt() % ULONG_MAX), then the
// coefficient uniform() * 2 - 1, all from one mt19937_64(seed) stream.
QS_API int qs_random_operator_terms(QS_UINT qubit_count, QS_UINT operator_count, QS_UINT seed,
    QS_UINT* pauli_ids_out, double* coefs_out) {
    if ((operator_count && qubit_count && !pauli_ids_out) || (operator_count && !coefs_out))
        return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null output array");
    std::mt19937_64 mt(seed);
    std::uniform_real_distribution<double> uniform(0., 1.);
    for (QS_UINT t = 0; t < operator_count; ++t) {
        for (QS_UINT q = 0; q < qubit_count; ++q)
            pauli_ids_out[(size_t)t * qubit_count + q] = (QS_UINT)((mt() % 0xFFFFFFFFFFFFFFFFULL) % 4);
        coefs_out[t] = uniform(mt) * 2 - 1.0;
    }
    return QS_OK;
}

}  // extern "C"
