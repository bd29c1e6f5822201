/*
 * qs_oracle.c -- CPU restatement of the reference's state-update path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load this file's shared object, and only as the checker; the product (qulacs_b200) never links,
 * imports or calls it.
 *
 * Every function restates one reference function in plain scalar C over an interleaved
 * (re, im) double array of `dim` amplitudes, the memory layout of std::complex<double> used by
 * csim (csim/type.hpp:15-30).  Paths are relative to the reference project root (src/...).
 * Parity of this restatement is pinned against the reference csim itself, compiled from its own
 * sources into oracle/_ref/libcsim_ref.so (tests/test_oracle_pin.py).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double _Complex cplx;
typedef unsigned int UINT;
typedef unsigned long long ITYPE;

#define OR_API __attribute__((visibility("default")))

/* src/csim/utility.hpp:14-19 insert_zero_to_basis_index */
static inline ITYPE insert_zero(ITYPE basis, UINT q) {
    ITYPE low = basis & ((1ULL << q) - 1ULL);
    return ((basis >> q) << (q + 1)) | low;
}

static inline UINT popcount64(ITYPE x) { return (UINT)__builtin_popcountll(x); }

/* src/csim/update_ops_matrix_dense_single.cpp:50-68 (pairs b0 = insert0(i, t), b1 = b0 | 2^t) */
OR_API void or_single_qubit_dense_matrix_gate(UINT t, const double* m, double* s, ITYPE dim) {
    cplx* st = (cplx*)s;
    const cplx* mm = (const cplx*)m;
    const ITYPE mask = 1ULL << t;
    for (ITYPE i = 0; i < dim / 2; ++i) {
        ITYPE b0 = insert_zero(i, t), b1 = b0 | mask;
        cplx v0 = st[b0], v1 = st[b1];
        st[b0] = mm[0] * v0 + mm[1] * v1;
        st[b1] = mm[2] * v0 + mm[3] * v1;
    }
}

/* src/csim/update_ops_matrix_diagonal_single.cpp:22-68 */
OR_API void or_single_qubit_diagonal_matrix_gate(UINT t, const double* d, double* s, ITYPE dim) {
    cplx* st = (cplx*)s;
    const cplx* dd = (const cplx*)d;
    for (ITYPE i = 0; i < dim; ++i) st[i] *= dd[(i >> t) & 1ULL];
}

/* src/csim/update_ops_matrix_phase_single.cpp: a[i] *= phase when bit t of i is 1 */
OR_API void or_single_qubit_phase_gate(UINT t, const double* ph, double* s, ITYPE dim) {
    cplx* st = (cplx*)s;
    cplx p = *(const cplx*)ph;
    for (ITYPE i = 0; i < dim; ++i)
        if ((i >> t) & 1ULL) st[i] *= p;
}

/* src/csim/update_ops_pauli_single.cpp:54-66 RX: {c, i s; i s, c}, c = cos(a/2), s = sin(a/2) */
OR_API void or_RX_gate(UINT t, double a, double* s, ITYPE dim) {
    double c = cos(a / 2), sn = sin(a / 2);
    double m[8] = {c, 0, 0, sn, 0, sn, c, 0};
    or_single_qubit_dense_matrix_gate(t, m, s, dim);
}
/* src/csim/update_ops_pauli_single.cpp:81-94 RY: {c, s; -s, c} */
OR_API void or_RY_gate(UINT t, double a, double* s, ITYPE dim) {
    double c = cos(a / 2), sn = sin(a / 2);
    double m[8] = {c, 0, sn, 0, -sn, 0, c, 0};
    or_single_qubit_dense_matrix_gate(t, m, s, dim);
}
/* src/csim/update_ops_pauli_single.cpp:108-120 RZ: diag(c + i s, c - i s) */
OR_API void or_RZ_gate(UINT t, double a, double* s, ITYPE dim) {
    double c = cos(a / 2), sn = sin(a / 2);
    double d[4] = {c, sn, c, -sn};
    or_single_qubit_diagonal_matrix_gate(t, d, s, dim);
}

/* src/csim/update_ops_named_CNOT.cpp:21-104: swap a[b|2^c] <-> a[b|2^c|2^t] */
OR_API void or_CNOT_gate(UINT c, UINT t, double* s, ITYPE dim) {
    cplx* st = (cplx*)s;
    UINT lo = c < t ? c : t, hi = c < t ? t : c;
    for (ITYPE i = 0; i < dim / 4; ++i) {
        ITYPE b = insert_zero(insert_zero(i, lo), hi) | (1ULL << c);
        ITYPE b1 = b | (1ULL << t);
        cplx tmp = st[b];
        st[b] = st[b1];
        st[b1] = tmp;
    }
}

/* src/csim/update_ops_named_CZ.cpp:14-75: negate a[b|2^c|2^t] */
OR_API void or_CZ_gate(UINT c, UINT t, double* s, ITYPE dim) {
    cplx* st = (cplx*)s;
    UINT lo = c < t ? c : t, hi = c < t ? t : c;
    for (ITYPE i = 0; i < dim / 4; ++i) {
        ITYPE b = insert_zero(insert_zero(i, lo), hi) | (1ULL << c) | (1ULL << t);
        st[b] = -st[b];
    }
}

/* src/csim/update_ops_named_SWAP.cpp: swap a[b|2^t0] <-> a[b|2^t1] */
OR_API void or_SWAP_gate(UINT t0, UINT t1, double* s, ITYPE dim) {
    cplx* st = (cplx*)s;
    UINT lo = t0 < t1 ? t0 : t1, hi = t0 < t1 ? t1 : t0;
    for (ITYPE i = 0; i < dim / 4; ++i) {
        ITYPE b = insert_zero(insert_zero(i, lo), hi);
        ITYPE x = b | (1ULL << t0), y = b | (1ULL << t1);
        cplx tmp = st[x];
        st[x] = st[y];
        st[y] = tmp;
    }
}

/*
 * src/csim/update_ops_matrix_dense_multi.cpp:59-128 multi_qubit_dense_matrix_gate_parallel:
 * for every coset base b (zeros inserted at the sorted target positions) gather the 2^k amplitudes
 * b ^ mask[x], where mask[x] sets target_list[j] iff bit j of x is set
 * (src/csim/utility.cpp:77-93 create_matrix_mask_list), multiply by the row-major matrix, scatter.
 * double_qubit_dense_matrix_gate_c (src/csim/update_ops_matrix_dense_double.cpp:42-113) uses the
 * same convention with k = 2 (matrix-index bit 0 <-> t1, bit 1 <-> t2).
 */
OR_API void or_multi_qubit_dense_matrix_gate(
    const UINT* tl, UINT k, const double* m, double* s, ITYPE dim) {
    cplx* st = (cplx*)s;
    const cplx* mm = (const cplx*)m;
    const ITYPE md = 1ULL << k;
    UINT sorted[64];
    memcpy(sorted, tl, sizeof(UINT) * k);
    for (UINT i = 0; i < k; ++i)
        for (UINT j = i + 1; j < k; ++j)
            if (sorted[j] < sorted[i]) {
                UINT tmp = sorted[i];
                sorted[i] = sorted[j];
                sorted[j] = tmp;
            }
    ITYPE* mask = (ITYPE*)calloc(md, sizeof(ITYPE));
    cplx* buf = (cplx*)malloc(sizeof(cplx) * md);
    for (ITYPE x = 0; x < md; ++x)
        for (UINT j = 0; j < k; ++j)
            if ((x >> j) & 1ULL) mask[x] |= 1ULL << tl[j];
    for (ITYPE i = 0; i < (dim >> k); ++i) {
        ITYPE b = i;
        for (UINT j = 0; j < k; ++j) b = insert_zero(b, sorted[j]);
        for (ITYPE y = 0; y < md; ++y) {
            cplx acc = 0;
            for (ITYPE x = 0; x < md; ++x) acc += mm[y * md + x] * st[b ^ mask[x]];
            buf[y] = acc;
        }
        for (ITYPE y = 0; y < md; ++y) st[b ^ mask[y]] = buf[y];
    }
    free(mask);
    free(buf);
}

OR_API void or_double_qubit_dense_matrix_gate_c(
    UINT t1, UINT t2, const double* m, double* s, ITYPE dim) {
    UINT tl[2] = {t1, t2};
    or_multi_qubit_dense_matrix_gate(tl, 2, m, s, dim);
}

/* src/csim/update_ops_matrix_diagonal_multi.cpp:22-112: a[i] *= diag[index of i's target bits] */
OR_API void or_multi_qubit_diagonal_matrix_gate(
    const UINT* tl, UINT k, const double* d, double* s, ITYPE dim) {
    cplx* st = (cplx*)s;
    const cplx* dd = (const cplx*)d;
    for (ITYPE i = 0; i < dim; ++i) {
        ITYPE x = 0;
        for (UINT j = 0; j < k; ++j) x |= ((i >> tl[j]) & 1ULL) << j;
        st[i] *= dd[x];
    }
}

/*
 * src/csim/update_ops_control_multi_target_single.cpp: apply the 2x2 matrix on target t to the
 * pairs whose control bits equal the control values.
 */
OR_API void or_multi_qubit_control_single_qubit_dense_matrix_gate(const UINT* cl, const UINT* cv,
    UINT nc, UINT t, const double* m, double* s, ITYPE dim) {
    cplx* st = (cplx*)s;
    const cplx* mm = (const cplx*)m;
    for (ITYPE b0 = 0; b0 < dim; ++b0) {
        if ((b0 >> t) & 1ULL) continue;
        int ok = 1;
        for (UINT j = 0; j < nc; ++j)
            if (((b0 >> cl[j]) & 1ULL) != cv[j]) ok = 0;
        if (!ok) continue;
        ITYPE b1 = b0 | (1ULL << t);
        cplx v0 = st[b0], v1 = st[b1];
        st[b0] = mm[0] * v0 + mm[1] * v1;
        st[b1] = mm[2] * v0 + mm[3] * v1;
    }
}

/*
 * src/csim/utility.cpp:12-43 get_Pauli_masks_partial_list: X -> bit flip, Y -> bit and phase flip
 * plus one 90-degree rotation, Z -> phase flip; the pivot is the last X/Y qubit.
 */
static void pauli_masks(const UINT* tl, const UINT* ids, UINT cnt, ITYPE* xm, ITYPE* zm,
    UINT* nrot, UINT* pivot) {
    *xm = 0;
    *zm = 0;
    *nrot = 0;
    *pivot = 0;
    for (UINT i = 0; i < cnt; ++i) {
        ITYPE b = 1ULL << tl[i];
        if (ids[i] == 1) {
            *xm ^= b;
            *pivot = tl[i];
        } else if (ids[i] == 2) {
            *xm ^= b;
            *zm ^= b;
            (*nrot)++;
            *pivot = tl[i];
        } else if (ids[i] == 3) {
            *zm ^= b;
        }
    }
}

/* src/csim/constant.cpp:36 PHASE_90ROT = {1, i, -1, -i} */
static const cplx PHASE_90ROT[4] = {1.0, I, -1.0, -I};

/*
 * src/csim/stat_ops_expectation_value.cpp:539-587 (partial list), with the two kernels
 * _XZ_mask (:352-373): sum over pivot-0 indices b0 of 2 Re(a[b0] conj(a[b0^X]) PHASE_90ROT[(nY +
 * 2 popcount(b0 & Z)) % 4]), and _Z_mask (:467-482): sum |a_i|^2 (-1)^popcount(i & Z).
 */
OR_API double or_expectation_value_multi_qubit_Pauli_operator_partial_list(
    const UINT* tl, const UINT* ids, UINT cnt, const double* s, ITYPE dim) {
    const cplx* st = (const cplx*)s;
    ITYPE xm, zm;
    UINT nrot, pivot;
    pauli_masks(tl, ids, cnt, &xm, &zm, &nrot, &pivot);
    double sum = 0.;
    if (xm == 0) {
        for (ITYPE i = 0; i < dim; ++i) {
            double p = creal(st[i]) * creal(st[i]) + cimag(st[i]) * cimag(st[i]);
            sum += (popcount64(i & zm) & 1) ? -p : p;
        }
    } else {
        for (ITYPE i = 0; i < dim / 2; ++i) {
            ITYPE b0 = insert_zero(i, pivot), b1 = b0 ^ xm;
            UINT sgn = popcount64(b0 & zm) & 1;
            sum += creal(st[b0] * conj(st[b1]) * PHASE_90ROT[(nrot + sgn * 2) % 4] * 2.0);
        }
    }
    return sum;
}

/* src/csim/update_ops_pauli_multi.cpp:29-120 multi-qubit Pauli gate: a'[i ^ X] = phase(i) a[i] */
OR_API void or_multi_qubit_Pauli_gate_partial_list(
    const UINT* tl, const UINT* ids, UINT cnt, double* s, ITYPE dim) {
    cplx* st = (cplx*)s;
    ITYPE xm, zm;
    UINT nrot, pivot;
    pauli_masks(tl, ids, cnt, &xm, &zm, &nrot, &pivot);
    cplx* out = (cplx*)malloc(sizeof(cplx) * dim);
    for (ITYPE i = 0; i < dim; ++i) {
        /* P|i> = i^{nY} (-1)^{popcount(i & Z)} |i ^ X>, with Y = i X Z */
        UINT sgn = popcount64(i & zm) & 1;
        out[i ^ xm] = st[i] * PHASE_90ROT[(nrot + 2 * sgn) % 4];
    }
    memcpy(st, out, sizeof(cplx) * dim);
    free(out);
}

/* src/csim/update_ops_pauli_multi.cpp:200-460: exp(i a/2 P) = cos(a/2) I + i sin(a/2) P */
OR_API void or_multi_qubit_Pauli_rotation_gate_partial_list(
    const UINT* tl, const UINT* ids, UINT cnt, double angle, double* s, ITYPE dim) {
    cplx* st = (cplx*)s;
    cplx* p = (cplx*)malloc(sizeof(cplx) * dim);
    memcpy(p, st, sizeof(cplx) * dim);
    or_multi_qubit_Pauli_gate_partial_list(tl, ids, cnt, (double*)p, dim);
    double c = cos(angle / 2), sn = sin(angle / 2);
    for (ITYPE i = 0; i < dim; ++i) st[i] = c * st[i] + I * sn * p[i];
    free(p);
}

/* src/csim/stat_ops.cpp:13-29 */
OR_API double or_state_norm_squared(const double* s, ITYPE dim) {
    double sum = 0.;
    for (ITYPE i = 0; i < 2 * dim; ++i) sum += s[i] * s[i];
    return sum;
}

/* src/csim/stat_ops.cpp:65-86: sum conj(bra_i) ket_i */
OR_API void or_state_inner_product(const double* a, const double* b, ITYPE dim, double* out) {
    const cplx* x = (const cplx*)a;
    const cplx* y = (const cplx*)b;
    cplx acc = 0;
    for (ITYPE i = 0; i < dim; ++i) acc += conj(x[i]) * y[i];
    out[0] = creal(acc);
    out[1] = cimag(acc);
}

/* src/csim/stat_ops_probability.cpp:11-56 M0_prob / M1_prob */
OR_API double or_M0_prob(UINT t, const double* s, ITYPE dim) {
    double sum = 0.;
    for (ITYPE i = 0; i < dim; ++i)
        if (!((i >> t) & 1ULL)) sum += s[2 * i] * s[2 * i] + s[2 * i + 1] * s[2 * i + 1];
    return sum;
}
OR_API double or_M1_prob(UINT t, const double* s, ITYPE dim) {
    double sum = 0.;
    for (ITYPE i = 0; i < dim; ++i)
        if ((i >> t) & 1ULL) sum += s[2 * i] * s[2 * i] + s[2 * i + 1] * s[2 * i + 1];
    return sum;
}
/* src/csim/stat_ops_probability.cpp:58-100 marginal_prob */
OR_API double or_marginal_prob(
    const UINT* tl, const UINT* vals, UINT cnt, const double* s, ITYPE dim) {
    double sum = 0.;
    for (ITYPE i = 0; i < dim; ++i) {
        int ok = 1;
        for (UINT j = 0; j < cnt; ++j)
            if (((i >> tl[j]) & 1ULL) != vals[j]) ok = 0;
        if (ok) sum += s[2 * i] * s[2 * i] + s[2 * i + 1] * s[2 * i + 1];
    }
    return sum;
}

/*
 * src/cppsim/state.hpp:909-929 QuantumStateCpu::sampling: serial FP64 running sum of |a_i|^2 into
 * stacked[0..dim] (stacked[0] = 0), then index = lower_bound(stacked, r) - 1 for each uniform r.
 * r == 0 gives -1 (2^64 - 1); r > stacked[dim] gives dim.  `near_boundary` (optional) receives 1
 * for a draw within `eps` of stacked[index] or stacked[index + 1].
 */
OR_API void or_sampling_with_uniforms(const double* s, ITYPE dim, const double* uniforms, UINT count,
    ITYPE* out, double eps, unsigned char* near_boundary) {
    double* stacked = (double*)malloc(sizeof(double) * (dim + 1));
    double sum = 0.;
    stacked[0] = 0.;
    for (ITYPE i = 0; i < dim; ++i) {
        sum += s[2 * i] * s[2 * i] + s[2 * i + 1] * s[2 * i + 1];
        stacked[i + 1] = sum;
    }
    for (UINT c = 0; c < count; ++c) {
        double r = uniforms[c];
        ITYPE lo = 0, hi = dim + 1; /* first k in [0, dim+1) with stacked[k] >= r */
        while (lo < hi) {
            ITYPE mid = lo + (hi - lo) / 2;
            if (stacked[mid] < r) lo = mid + 1;
            else hi = mid;
        }
        ITYPE idx = lo - 1ULL;
        out[c] = idx;
        if (near_boundary) {
            int nb = 0;
            if (lo <= dim && fabs(stacked[lo] - r) <= eps) nb = 1;
            if (lo >= 1 && fabs(stacked[lo - 1] - r) <= eps) nb = 1;
            near_boundary[c] = (unsigned char)nb;
        }
    }
    free(stacked);
}

/* ---------------- density matrix (row-major rho[y * dim + x]) ---------------- */

/*
 * src/csim/update_ops_dm.cpp:33-102 dm_single_qubit_dense_matrix_gate: rho <- U rho U^dagger on the
 * quads (y0|y1) x (x0|x1) via the 4x4 extended matrix ext[y][x] = U[y1][x1] conj(U[y2][x2]).
 */
OR_API void or_dm_multi_qubit_dense_matrix_gate(
    const UINT* tl, UINT k, const double* m, double* r, ITYPE dim) {
    /* rho' = U rho U^dagger: apply U to every column, then conj(U) to every row (rho U^dagger =
     * (conj(U) rho^T)^T), restated directly over the index sets. */
    cplx* rho = (cplx*)r;
    const cplx* u = (const cplx*)m;
    const ITYPE md = 1ULL << k;
    ITYPE* mask = (ITYPE*)calloc(md, sizeof(ITYPE));
    for (ITYPE x = 0; x < md; ++x)
        for (UINT j = 0; j < k; ++j)
            if ((x >> j) & 1ULL) mask[x] |= 1ULL << tl[j];
    ITYPE all = mask[md - 1];
    cplx* buf = (cplx*)malloc(sizeof(cplx) * md);
    /* left multiply: for each column x, each row coset */
    for (ITYPE col = 0; col < dim; ++col)
        for (ITYPE b = 0; b < dim; ++b) {
            if (b & all) continue;
            for (ITYPE y = 0; y < md; ++y) {
                cplx acc = 0;
                for (ITYPE x = 0; x < md; ++x) acc += u[y * md + x] * rho[(b ^ mask[x]) * dim + col];
                buf[y] = acc;
            }
            for (ITYPE y = 0; y < md; ++y) rho[(b ^ mask[y]) * dim + col] = buf[y];
        }
    /* right multiply by U^dagger: rho[row][c'] = sum_c rho[row][c] conj(U[c'][c]) */
    for (ITYPE row = 0; row < dim; ++row)
        for (ITYPE b = 0; b < dim; ++b) {
            if (b & all) continue;
            for (ITYPE y = 0; y < md; ++y) {
                cplx acc = 0;
                for (ITYPE x = 0; x < md; ++x)
                    acc += conj(u[y * md + x]) * rho[row * dim + (b ^ mask[x])];
                buf[y] = acc;
            }
            for (ITYPE y = 0; y < md; ++y) rho[row * dim + (b ^ mask[y])] = buf[y];
        }
    free(buf);
    free(mask);
}

OR_API void or_dm_single_qubit_dense_matrix_gate(UINT t, const double* m, double* r, ITYPE dim) {
    or_dm_multi_qubit_dense_matrix_gate(&t, 1, m, r, dim);
}

/* src/csim/update_ops_dm.cpp:745-762: CNOT and CZ as controlled Pauli-X / Pauli-Z */
OR_API void or_dm_CNOT_gate(UINT c, UINT t, double* r, ITYPE dim) {
    /* matrix over (bit0 <-> c, bit1 <-> t): |c=1> flips t */
    double m[32] = {0};
    cplx* mm = (cplx*)m;
    mm[0 * 4 + 0] = 1; /* c=0,t=0 */
    mm[2 * 4 + 2] = 1; /* c=0,t=1 */
    mm[1 * 4 + 3] = 1; /* c=1,t=0 <- c=1,t=1 */
    mm[3 * 4 + 1] = 1;
    UINT tl[2] = {c, t};
    or_dm_multi_qubit_dense_matrix_gate(tl, 2, m, r, dim);
}
OR_API void or_dm_CZ_gate(UINT c, UINT t, double* r, ITYPE dim) {
    double m[32] = {0};
    cplx* mm = (cplx*)m;
    mm[0] = 1;
    mm[5] = 1;
    mm[10] = 1;
    mm[15] = -1;
    UINT tl[2] = {c, t};
    or_dm_multi_qubit_dense_matrix_gate(tl, 2, m, r, dim);
}

/*
 * Depolarizing channels, exact density-matrix branch of QuantumGate_Probabilistic
 * (src/cppsim/gate_general.hpp:265-285) with the distributions of DepolarizingNoise
 * (src/cppsim/gate_factory.cpp:456-466) and TwoQubitDepolarizingNoise (:471-500).  The mixture
 * sum_k p_k P_k rho P_k over the single-qubit Paulis {X, Z, Y} (p/3 each) and I (1 - p) equals,
 * per 2x2 block B over the target's row and column bit, (1 - 4p/3) B + (2p/3) Tr(B) I; over the 15
 * two-qubit Paulis (p/15 each) and I (1 - p) it equals (1 - 16p/15) B + (4p/15) Tr(B) I per 4x4 block.
 * The restatement below evaluates the branch sum literally (as the reference does) so that it
 * checks the closed form used by the device kernel.
 */
static void dm_apply_pauli_literal(const UINT* tl, const UINT* ids, UINT cnt, cplx* rho, ITYPE dim,
    cplx* out) {
    /* out = P rho P^dagger with P the Pauli string; P|i> = ph(i)|i^X>, so
     * out[i^X][j^X] = ph(i) conj(ph(j)) rho[i][j] */
    ITYPE xm, zm;
    UINT nrot, pivot;
    pauli_masks(tl, ids, cnt, &xm, &zm, &nrot, &pivot);
    for (ITYPE i = 0; i < dim; ++i) {
        cplx pi = PHASE_90ROT[(nrot + 2 * (popcount64(i & zm) & 1)) % 4];
        for (ITYPE j = 0; j < dim; ++j) {
            cplx pj = PHASE_90ROT[(nrot + 2 * (popcount64(j & zm) & 1)) % 4];
            out[(i ^ xm) * dim + (j ^ xm)] = pi * conj(pj) * rho[i * dim + j];
        }
    }
}

OR_API void or_dm_depolarizing_noise(UINT t, double p, double* r, ITYPE dim) {
    cplx* rho = (cplx*)r;
    const ITYPE n = dim * dim;
    cplx* acc = (cplx*)calloc(n, sizeof(cplx));
    cplx* tmp = (cplx*)malloc(sizeof(cplx) * n);
    const UINT ids[3] = {1, 3, 2};
    for (int g = 0; g < 3; ++g) {
        dm_apply_pauli_literal(&t, &ids[g], 1, rho, dim, tmp);
        for (ITYPE i = 0; i < n; ++i) acc[i] += (p / 3) * tmp[i];
    }
    for (ITYPE i = 0; i < n; ++i) rho[i] = acc[i] + (1 - p) * rho[i];
    free(acc);
    free(tmp);
}

OR_API void or_dm_two_qubit_depolarizing_noise(UINT t1, UINT t2, double p, double* r, ITYPE dim) {
    cplx* rho = (cplx*)r;
    const ITYPE n = dim * dim;
    cplx* acc = (cplx*)calloc(n, sizeof(cplx));
    cplx* tmp = (cplx*)malloc(sizeof(cplx) * n);
    const UINT tl[2] = {t1, t2};
    for (int g = 1; g < 16; ++g) {
        UINT ids[2] = {(UINT)(g % 4), (UINT)(g / 4)};
        dm_apply_pauli_literal(tl, ids, 2, rho, dim, tmp);
        for (ITYPE i = 0; i < n; ++i) acc[i] += (p / 15) * tmp[i];
    }
    for (ITYPE i = 0; i < n; ++i) rho[i] = acc[i] + (1 - p) * rho[i];
    free(acc);
    free(tmp);
}

/* src/csim/stat_ops_dm.cpp:164-191: Re sum_i coef(i) rho[i][i ^ X] */
OR_API double or_dm_expectation_value_multi_qubit_Pauli_operator_partial_list(
    const UINT* tl, const UINT* ids, UINT cnt, const double* r, ITYPE dim) {
    const cplx* rho = (const cplx*)r;
    cplx sum = 0;
    for (ITYPE i = 0; i < dim; ++i) {
        cplx coef = 1.0;
        ITYPE sub = i;
        for (UINT j = 0; j < cnt; ++j) {
            ITYPE b = 1ULL << tl[j];
            if (ids[j] == 1) {
                sub ^= b;
            } else if (ids[j] == 2) {
                coef *= I;
                if (sub & b) coef *= -1.;
                sub ^= b;
            } else if (ids[j] == 3) {
                if (sub & b) coef *= -1.;
            }
        }
        sum += coef * rho[i * dim + sub];
    }
    return creal(sum);
}

/* src/cppsim/state_dm.hpp:383-401 DensityMatrixCpu::sampling: prefix of abs(rho_ii), then the
 * same lower_bound rule as QuantumStateCpu::sampling. */
OR_API void or_dm_sampling_with_uniforms(const double* r, ITYPE dim, const double* uniforms,
    UINT count, ITYPE* out) {
    const cplx* rho = (const cplx*)r;
    double* stacked = (double*)malloc(sizeof(double) * (dim + 1));
    double sum = 0.;
    stacked[0] = 0.;
    for (ITYPE i = 0; i < dim; ++i) {
        sum += cabs(rho[i * dim + i]);
        stacked[i + 1] = sum;
    }
    for (UINT c = 0; c < count; ++c) {
        ITYPE lo = 0, hi = dim + 1;
        while (lo < hi) {
            ITYPE mid = lo + (hi - lo) / 2;
            if (stacked[mid] < uniforms[c]) lo = mid + 1;
            else hi = mid;
        }
        out[c] = lo - 1ULL;
    }
    free(stacked);
}

/* ---- whole-state arithmetic and entropy ---- */

/* update_ops_named_state.cpp:62-75 state_add_with_coef: state[i] += coef * added[i]
 * (state_add, :47-60, is coef = 1). */
OR_API void or_state_add_with_coef(const double* coef, const double* added, double* s, ITYPE dim) {
    const cplx c = coef[0] + I * coef[1];
    for (ITYPE i = 0; i < dim; ++i) {
        cplx v = s[2 * i] + I * s[2 * i + 1];
        v += c * (added[2 * i] + I * added[2 * i + 1]);
        s[2 * i] = creal(v);
        s[2 * i + 1] = cimag(v);
    }
}

/* update_ops_named_state.cpp:86-95 state_multiply: state[i] *= coef. */
OR_API void or_state_multiply(const double* coef, double* s, ITYPE dim) {
    const cplx c = coef[0] + I * coef[1];
    for (ITYPE i = 0; i < dim; ++i) {
        const cplx v = c * (s[2 * i] + I * s[2 * i + 1]);
        s[2 * i] = creal(v);
        s[2 * i + 1] = cimag(v);
    }
}

/* update_ops_named_state.cpp:21-30 normalize: state[i] *= sqrt(1 / squared_norm). */
OR_API void or_normalize(double squared_norm, double* s, ITYPE dim) {
    const double f = sqrt(1. / squared_norm);
    for (ITYPE i = 0; i < 2 * dim; ++i) s[i] *= f;
}

/* stat_ops_probability.cpp:83-99 measurement_distribution_entropy: sum of -p log p over
 * p = |amplitude|^2 clamped below at 1e-15. */
OR_API double or_measurement_distribution_entropy(const double* s, ITYPE dim) {
    const double eps = 1e-15;
    double ent = 0;
    for (ITYPE i = 0; i < dim; ++i) {
        double p = pow(cabs(s[2 * i] + I * s[2 * i + 1]), 2);
        p = (p > eps) ? p : eps;
        ent += -1.0 * p * log(p);
    }
    return ent;
}

/* stat_ops_dm.cpp:29-46 dm_measurement_distribution_entropy: sum of -p log p over the diagonal
 * p = Re rho[i][i], terms with p <= 1e-15 skipped. */
OR_API double or_dm_measurement_distribution_entropy(const double* r, ITYPE dim) {
    const double eps = 1e-15;
    double ent = 0;
    for (ITYPE i = 0; i < dim; ++i) {
        const double p = r[2 * (i * dim + i)];
        if (p > eps) ent += -1.0 * p * log(p);
    }
    return ent;
}

/* ---- density-matrix probabilities and normalisation ---- */

/* stat_ops_dm.cpp:95-120 dm_marginal_prob: sum of Re rho[b][b] over the basis indices b whose
 * bits at the (sorted) targets equal the measured values; dm_M0_prob (:50-67) and dm_M1_prob
 * (:70-89) are the one-target cases. */
OR_API double or_dm_marginal_prob(const UINT* sorted_targets, const UINT* values, UINT count,
    const double* r, ITYPE dim) {
    const ITYPE loop_dim = dim >> count;
    double sum = 0.;
    for (ITYPE k = 0; k < loop_dim; ++k) {
        ITYPE b = k;
        for (UINT c = 0; c < count; ++c) {
            const ITYPE low = b & ((1ULL << sorted_targets[c]) - 1);
            b = ((b - low) << 1) | low | ((ITYPE)values[c] << sorted_targets[c]);
        }
        sum += r[2 * (b * dim + b)];
    }
    return sum;
}
OR_API double or_dm_M0_prob(UINT t, const double* r, ITYPE dim) {
    const UINT v = 0;
    return or_dm_marginal_prob(&t, &v, 1, r, dim);
}
OR_API double or_dm_M1_prob(UINT t, const double* r, ITYPE dim) {
    const UINT v = 1;
    return or_dm_marginal_prob(&t, &v, 1, r, dim);
}

/* update_ops_dm.cpp:14-28 dm_normalize: rho *= 1 / squared_norm. */
OR_API void or_dm_normalize(double squared_norm, double* r, ITYPE dim) {
    const double f = 1. / squared_norm;
    for (ITYPE i = 0; i < 2 * dim * dim; ++i) r[i] *= f;
}
