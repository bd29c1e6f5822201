// Density-matrix operations (csim/update_ops_dm.cpp, csim/stat_ops_dm.cpp) on the B200.
//
// rho (dim x dim, row-major) is treated as a 2n-qubit vector: column bits 0..n-1, row bits n..2n-1.
// rho <- U rho U^dagger is then U on the row bits and conj(U) on the column bits, applied by the
// state-vector kernels in ONE pass over rho as the 2k-qubit matrix U (x) conj(U) (the reference
// builds the same "extended matrix", update_ops_dm.cpp:37-49, and loops over index quads).
// Depolarizing channels, which the reference applies as copy / apply / scale / add over 4 or 16
// Pauli branches (cppsim/gate_general.hpp:265-285, about 12-48 passes over rho), are one pass of
// their closed form per 2x2 or 4x4 block B:  (1 - 4p/3) B + (2p/3) Tr(B) I  for one qubit and
// (1 - 16p/15) B + (4p/15) Tr(B) I  for two.
#include <cmath>
#include <complex>
#include <vector>

#include "qs_internal.cuh"

namespace qs {

typedef std::complex<double> cd;

static int dm_dims(ITYPE dim, UINT* n) {
    QS_TRY(check_dim(dim, n));
    if (*n > 20) return set_error(QS_ERR_NOT_SUPPORTED, "density matrix: more than 20 qubits");
    return QS_OK;
}

// Apply a k-target unitary (k <= 3) to rho as U (x) conj(U) on 2k vector qubits in one pass.
int dm_apply_unitary(const UINT* tl, UINT k, const cd* u, double2* rho, ITYPE dim, UINT n, cudaStream_t st) {
    const UINT md = 1u << k;
    if (k > 3) {
        // rows: U on bits tl + n ; columns: conj(U) on bits tl
        std::vector<cd> uc(md * md);
        for (UINT i = 0; i < md * md; ++i) uc[i] = std::conj(u[i]);
        std::vector<UINT> rows(k);
        for (UINT j = 0; j < k; ++j) rows[j] = tl[j] + n;
        QS_TRY(launch_denseK(rows.data(), k, (const double*)u, rho, dim * dim, nullptr, nullptr, 0, st));
        return launch_denseK(tl, k, (const double*)uc.data(), rho, dim * dim, nullptr, nullptr, 0, st);
    }
    // extended matrix over targets [tl (columns, low bits of the index), tl + n (rows, high bits)]
    const UINT ed = md * md;
    std::vector<cd> ext((size_t)ed * ed);
    for (UINT Y = 0; Y < md; ++Y)
        for (UINT y = 0; y < md; ++y)
            for (UINT X = 0; X < md; ++X)
                for (UINT x = 0; x < md; ++x)
                    ext[(size_t)(Y * md + y) * ed + (X * md + x)] = u[Y * md + X] * std::conj(u[y * md + x]);
    std::vector<UINT> targets(2 * k);
    for (UINT j = 0; j < k; ++j) {
        targets[j] = tl[j];
        targets[k + j] = tl[j] + n;
    }
    if (k == 1) {
        Mat4 m;
        for (int i = 0; i < 16; ++i) m.m[i] = make_double2(ext[i].real(), ext[i].imag());
        return launch_dense2(targets[0], targets[1], m, rho, dim * dim, nullptr, nullptr, 0, st);
    }
    return launch_denseK(targets.data(), 2 * k, (const double*)ext.data(), rho, dim * dim, nullptr, nullptr, 0, st);
}

int dm_depolarizing(const UINT* tl, UINT k, double p, double2* rho, ITYPE dim, UINT n, cudaStream_t st) {
    const UINT md = 1u << k;  // block side
    const UINT ed = md * md;
    const double keep = k == 1 ? 1. - 4. * p / 3. : 1. - 16. * p / 15.;
    const double tr = k == 1 ? 2. * p / 3. : 4. * p / 15.;
    // superoperator on vector index (R << k) | C, R = row bits, C = column bits
    std::vector<cd> sop((size_t)ed * ed, cd(0., 0.));
    for (UINT R = 0; R < md; ++R)
        for (UINT Cc = 0; Cc < md; ++Cc) {
            const UINT o = (R << k) | Cc;
            sop[(size_t)o * ed + o] += keep;
            if (R == Cc)
                for (UINT j = 0; j < md; ++j) sop[(size_t)o * ed + ((j << k) | j)] += tr;
        }
    std::vector<UINT> targets(2 * k);
    for (UINT j = 0; j < k; ++j) {
        targets[j] = tl[j];
        targets[k + j] = tl[j] + n;
    }
    if (k == 1) {
        Mat4 m;
        for (int i = 0; i < 16; ++i) m.m[i] = make_double2(sop[i].real(), sop[i].imag());
        return launch_dense2(targets[0], targets[1], m, rho, dim * dim, nullptr, nullptr, 0, st);
    }
    return launch_denseK(targets.data(), 2 * k, (const double*)sop.data(), rho, dim * dim, nullptr, nullptr, 0, st);
}

// Re sum_i i^{nY} (-1)^{popcount(i & z)} rho[i][i ^ x]   (stat_ops_dm.cpp:164-191)
__global__ void k_dm_ev(const double2* __restrict__ rho, ITYPE dim, ITYPE xm, ITYPE zm, UINT nrot,
    double* __restrict__ part) {
    __shared__ double sm[32];
    double acc = 0.;
    const ITYPE stride = (ITYPE)gridDim.x * blockDim.x;
    for (ITYPE i = (ITYPE)blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += stride) {
        const double2 v = rho[i * dim + (i ^ xm)];
        const UINT r = (nrot + 2u * (UINT)(__popcll(i & zm) & 1)) & 3u;
        acc += r == 0 ? v.x : (r == 1 ? -v.y : (r == 2 ? -v.x : v.y));
    }
    acc = block_sum(acc, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}
__global__ void k_dm_trace(const double2* __restrict__ rho, ITYPE dim, double* __restrict__ part) {
    __shared__ double sm[32];
    double acc = 0.;
    const ITYPE stride = (ITYPE)gridDim.x * blockDim.x;
    for (ITYPE i = (ITYPE)blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += stride) acc += rho[i * dim + i].x;
    acc = block_sum(acc, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}
__global__ void k_fold(const double* __restrict__ part, int count, double* __restrict__ out) {
    __shared__ double sm[32];
    double v = 0.;
    for (int p = threadIdx.x; p < count; p += blockDim.x) v += part[p];
    v = block_sum(v, sm);
    if (threadIdx.x == 0) *out = v;
}
__global__ void k_dm_outer(const double2* __restrict__ psi, double2* __restrict__ rho, ITYPE dim) {
    const ITYPE total = dim * dim;
    const ITYPE stride = (ITYPE)gridDim.x * blockDim.x;
    for (ITYPE k = (ITYPE)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += stride) {
        const ITYPE y = k / dim, x = k % dim;
        rho[k] = cmul(psi[y], cconj(psi[x]));
    }
}

static int dm_reduce(void (*launch)(double*, unsigned, cudaStream_t, const void*), const void* ctx, ITYPE dim,
    cudaStream_t st, double* out) {
    unsigned blocks = (unsigned)std::min<ITYPE>((dim + 255) / 256, 1024);
    void* buf;
    QS_TRY(scratch(st, sizeof(double) * (blocks + 1), &buf));
    launch((double*)buf, blocks, st, ctx);
    QS_TRY(check_launch("dm reduction"));
    k_fold<<<1, 256, 0, st>>>((double*)buf, (int)blocks, (double*)buf + blocks);
    QS_TRY(check_launch("k_fold"));
    QS_CUDA_CHECK(cudaMemcpyAsync(out, (double*)buf + blocks, sizeof(double), cudaMemcpyDeviceToHost, st));
    QS_CUDA_CHECK(cudaStreamSynchronize(st));
    return QS_OK;
}

}  // namespace qs

using namespace qs;

#define DM_ARGS void *rho, QS_ITYPE dim, void *stream
#define R2 ((double2*)rho)
#define ST ((cudaStream_t)stream)

extern "C" {

QS_API int qs_dm_allocate(QS_ITYPE dim, void** rho_out) {
    UINT n;
    QS_TRY(dm_dims(dim, &n));
    return qs_allocate_quantum_state(dim * dim, rho_out);
}
QS_API int qs_dm_initialize_quantum_state(DM_ARGS) {
    UINT n;
    QS_TRY(dm_dims(dim, &n));
    return qs_set_computational_basis(0, rho, dim * dim, stream);
}
QS_API int qs_dm_initialize_with_pure_state(void* rho, const void* psi, QS_ITYPE dim, void* stream) {
    UINT n;
    QS_TRY(dm_dims(dim, &n));
    k_dm_outer<<<(unsigned)std::min<ITYPE>((dim * dim + 255) / 256, 65535), 256, 0, ST>>>(
        (const double2*)psi, R2, dim);
    return check_launch("k_dm_outer");
}

QS_API int qs_dm_single_qubit_dense_matrix_gate(QS_UINT t, const double matrix[8], DM_ARGS) {
    UINT n;
    QS_TRY(dm_dims(dim, &n));
    QS_TRY(check_target(t, n, "dm_single_qubit_dense_matrix_gate"));
    return dm_apply_unitary(&t, 1, (const cd*)matrix, R2, dim, n, ST);
}
QS_API int qs_dm_multi_qubit_dense_matrix_gate(const QS_UINT* tl, QS_UINT k, const double* matrix, DM_ARGS) {
    UINT n;
    QS_TRY(dm_dims(dim, &n));
    if (k < 1 || k > (UINT)kMaxDenseTargets)
        return set_error(QS_ERR_NOT_SUPPORTED, "dm_multi_qubit_dense_matrix_gate: 1..12 targets");
    QS_TRY(check_distinct(tl, k, n, "dm_multi_qubit_dense_matrix_gate"));
    return dm_apply_unitary(tl, k, (const cd*)matrix, R2, dim, n, ST);
}
QS_API int qs_dm_CNOT_gate(QS_UINT c, QS_UINT t, DM_ARGS) {
    UINT n;
    QS_TRY(dm_dims(dim, &n));
    const UINT l[2] = {c, t};
    QS_TRY(check_distinct(l, 2, n, "dm_CNOT_gate"));
    // X is real: the row and column permutations are both CNOTs.
    QS_TRY(qs_CNOT_gate(c + n, t + n, rho, dim * dim, stream));
    return qs_CNOT_gate(c, t, rho, dim * dim, stream);
}
QS_API int qs_dm_CZ_gate(QS_UINT c, QS_UINT t, DM_ARGS) {
    UINT n;
    QS_TRY(dm_dims(dim, &n));
    const UINT l[2] = {c, t};
    QS_TRY(check_distinct(l, 2, n, "dm_CZ_gate"));
    QS_TRY(qs_CZ_gate(c + n, t + n, rho, dim * dim, stream));
    return qs_CZ_gate(c, t, rho, dim * dim, stream);
}
// update_ops_dm.cpp:775-810: cos(a/2) I + i sin(a/2) P
static int dm_rot(UINT t, double a, int pauli, void* rho, ITYPE dim, void* stream) {
    const double c = std::cos(a / 2), s = std::sin(a / 2);
    cd m[4];
    if (pauli == 1) { m[0] = c; m[1] = cd(0, s); m[2] = cd(0, s); m[3] = c; }
    else if (pauli == 2) { m[0] = c; m[1] = s; m[2] = -s; m[3] = c; }
    else { m[0] = cd(c, s); m[1] = 0; m[2] = 0; m[3] = cd(c, -s); }
    return qs_dm_single_qubit_dense_matrix_gate(t, (const double*)m, rho, dim, stream);
}
QS_API int qs_dm_RX_gate(QS_UINT t, double a, DM_ARGS) { return dm_rot(t, a, 1, rho, dim, stream); }
QS_API int qs_dm_RY_gate(QS_UINT t, double a, DM_ARGS) { return dm_rot(t, a, 2, rho, dim, stream); }
QS_API int qs_dm_RZ_gate(QS_UINT t, double a, DM_ARGS) { return dm_rot(t, a, 3, rho, dim, stream); }

// Named gates: U rho U^dagger with csim's matrices (constant.cpp:4-30), row-major interleaved re, im.
#define QS_DM_NAMED(NAME, ...)                                                      \
    QS_API int qs_dm_##NAME##_gate(QS_UINT t, DM_ARGS) {                            \
        static const double m[8] = {__VA_ARGS__};                                   \
        return qs_dm_single_qubit_dense_matrix_gate(t, m, rho, dim, stream);        \
    }
#define QS_H 0.70710678118654752440
QS_DM_NAMED(X, 0, 0, 1, 0, 1, 0, 0, 0)
QS_DM_NAMED(Y, 0, 0, 0, -1, 0, 1, 0, 0)
QS_DM_NAMED(Z, 1, 0, 0, 0, 0, 0, -1, 0)
QS_DM_NAMED(H, QS_H, 0, QS_H, 0, QS_H, 0, -QS_H, 0)
QS_DM_NAMED(S, 1, 0, 0, 0, 0, 0, 0, 1)
QS_DM_NAMED(Sdag, 1, 0, 0, 0, 0, 0, 0, -1)
QS_DM_NAMED(T, 1, 0, 0, 0, 0, 0, QS_H, QS_H)
QS_DM_NAMED(Tdag, 1, 0, 0, 0, 0, 0, QS_H, -QS_H)
QS_DM_NAMED(sqrtX, 0.5, 0.5, 0.5, -0.5, 0.5, -0.5, 0.5, 0.5)
QS_DM_NAMED(sqrtXdag, 0.5, -0.5, 0.5, 0.5, 0.5, 0.5, 0.5, -0.5)
QS_DM_NAMED(sqrtY, 0.5, 0.5, -0.5, -0.5, 0.5, 0.5, 0.5, 0.5)
QS_DM_NAMED(sqrtYdag, 0.5, -0.5, 0.5, -0.5, -0.5, 0.5, 0.5, -0.5)
QS_DM_NAMED(P0, 1, 0, 0, 0, 0, 0, 0, 0)
QS_DM_NAMED(P1, 0, 0, 0, 0, 0, 0, 1, 0)
#undef QS_H
#undef QS_DM_NAMED

QS_API int qs_dm_SWAP_gate(QS_UINT t0, QS_UINT t1, DM_ARGS) {
    // matrix bit 0 <-> t0, bit 1 <-> t1: |01> <-> |10>
    static const double m[32] = {1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0,
                                 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0};
    const UINT tl[2] = {t0, t1};
    return qs_dm_multi_qubit_dense_matrix_gate(tl, 2, m, rho, dim, stream);
}

static int dm_pauli_checks(const UINT* tl, const UINT* ids, UINT cnt, ITYPE dim, const char* what) {
    UINT n;
    QS_TRY(dm_dims(dim, &n));
    if (cnt > (UINT)kMaxDenseTargets) return set_error(QS_ERR_NOT_SUPPORTED, std::string(what) + ": at most 12 qubits");
    for (UINT j = 0; j < cnt; ++j)
        if (ids[j] > 3) return set_error(QS_ERR_INVALID_ARGUMENT, std::string(what) + ": Pauli id must be 0..3");
    return check_distinct(tl, cnt, n, what);
}
// P rho P^dagger for P a product over distinct qubits: one single-qubit Pauli at a time.
QS_API int qs_dm_multi_qubit_Pauli_gate_partial_list(const QS_UINT* tl, const QS_UINT* ids, QS_UINT cnt, DM_ARGS) {
    QS_TRY(dm_pauli_checks(tl, ids, cnt, dim, "dm_multi_qubit_Pauli_gate_partial_list"));
    for (UINT j = 0; j < cnt; ++j) {
        if (ids[j] == 1) QS_TRY(qs_dm_X_gate(tl[j], rho, dim, stream));
        else if (ids[j] == 2) QS_TRY(qs_dm_Y_gate(tl[j], rho, dim, stream));
        else if (ids[j] == 3) QS_TRY(qs_dm_Z_gate(tl[j], rho, dim, stream));
    }
    return QS_OK;
}
// exp(i angle P / 2) = cos(angle/2) I + i sin(angle/2) P as a dense matrix over the listed qubits
// (bit j <-> tl[j]); P[x ^ xmask][x] = prod_j sigma_{id_j}[y_j][x_j].
QS_API int qs_dm_multi_qubit_Pauli_rotation_gate_partial_list(const QS_UINT* tl, const QS_UINT* ids, QS_UINT cnt,
    double angle, DM_ARGS) {
    QS_TRY(dm_pauli_checks(tl, ids, cnt, dim, "dm_multi_qubit_Pauli_rotation_gate_partial_list"));
    if (cnt == 0) return QS_OK;  // a global phase: rho is unchanged
    const size_t md = size_t(1) << cnt;
    size_t xmask = 0;
    for (UINT j = 0; j < cnt; ++j)
        if (ids[j] == 1 || ids[j] == 2) xmask |= size_t(1) << j;
    const double c = std::cos(angle / 2), sn = std::sin(angle / 2);
    std::vector<cd> m(md * md, 0.);
    for (size_t x = 0; x < md; ++x) {
        const size_t y = x ^ xmask;
        cd v = 1.;
        for (UINT j = 0; j < cnt; ++j) {
            const bool xb = (x >> j) & 1;
            if (ids[j] == 2) v *= xb ? cd(0, -1) : cd(0, 1);  // sigma_Y[y][x]: [[0, -i], [i, 0]]
            else if (ids[j] == 3 && xb) v = -v;
        }
        m[y * md + x] += cd(0, sn) * v;
        m[x * md + x] += c;
    }
    return qs_dm_multi_qubit_dense_matrix_gate(tl, cnt, (const double*)m.data(), rho, dim, stream);
}

// Controlled dense on rho: the matrix over (targets, controls), targets on the low bits, identity where
// the control bits differ from the control values.
static int dm_controlled(const UINT* ctl, const UINT* cval, UINT nc, const UINT* tl, UINT k, const cd* u,
    void* rho, ITYPE dim, void* stream, const char* what) {
    UINT n;
    QS_TRY(dm_dims(dim, &n));
    if (k < 1 || k + nc > (UINT)kMaxDenseTargets)
        return set_error(QS_ERR_NOT_SUPPORTED, std::string(what) + ": targets + controls must be 1..12");
    std::vector<UINT> all(tl, tl + k);
    size_t cbits = 0;
    for (UINT j = 0; j < nc; ++j) {
        if (cval[j] > 1) return set_error(QS_ERR_INVALID_ARGUMENT, "control value must be 0 or 1");
        if (cval[j]) cbits |= size_t(1) << j;
        all.push_back(ctl[j]);
    }
    QS_TRY(check_distinct(all.data(), k + nc, n, what));
    const size_t md = size_t(1) << (k + nc), mt = size_t(1) << k;
    std::vector<cd> full(md * md, 0.);
    for (size_t y = 0; y < md; ++y) {
        if ((y >> k) != cbits) {
            full[y * md + y] = 1.;
            continue;
        }
        for (size_t x = 0; x < mt; ++x) full[y * md + ((y >> k) << k) + x] = u[(y & (mt - 1)) * mt + x];
    }
    return qs_dm_multi_qubit_dense_matrix_gate(all.data(), k + nc, (const double*)full.data(), rho, dim, stream);
}
QS_API int qs_dm_multi_qubit_control_single_qubit_dense_matrix_gate(const QS_UINT* ctl, const QS_UINT* cval,
    QS_UINT nc, QS_UINT t, const double matrix[8], DM_ARGS) {
    return dm_controlled(ctl, cval, nc, &t, 1, (const cd*)matrix, rho, dim, stream,
        "dm_multi_qubit_control_single_qubit_dense_matrix_gate");
}
QS_API int qs_dm_multi_qubit_control_multi_qubit_dense_matrix_gate(const QS_UINT* ctl, const QS_UINT* cval,
    QS_UINT nc, const QS_UINT* tl, QS_UINT k, const double* matrix, DM_ARGS) {
    return dm_controlled(ctl, cval, nc, tl, k, (const cd*)matrix, rho, dim, stream,
        "dm_multi_qubit_control_multi_qubit_dense_matrix_gate");
}

QS_API int qs_dm_depolarizing_noise(QS_UINT t, double p, DM_ARGS) {
    UINT n;
    QS_TRY(dm_dims(dim, &n));
    QS_TRY(check_target(t, n, "dm_depolarizing_noise"));
    if (!(p >= 0. && p <= 1.)) return set_error(QS_ERR_INVALID_ARGUMENT, "probability outside [0, 1]");
    return dm_depolarizing(&t, 1, p, R2, dim, n, ST);
}
QS_API int qs_dm_two_qubit_depolarizing_noise(QS_UINT t1, QS_UINT t2, double p, DM_ARGS) {
    UINT n;
    QS_TRY(dm_dims(dim, &n));
    const UINT l[2] = {t1, t2};
    QS_TRY(check_distinct(l, 2, n, "dm_two_qubit_depolarizing_noise"));
    if (!(p >= 0. && p <= 1.)) return set_error(QS_ERR_INVALID_ARGUMENT, "probability outside [0, 1]");
    return dm_depolarizing(l, 2, p, R2, dim, n, ST);
}

struct EvCtx {
    const double2* rho;
    ITYPE dim, x, z;
    UINT nrot;
};
static void launch_ev(double* part, unsigned blocks, cudaStream_t st, const void* c) {
    const EvCtx* e = (const EvCtx*)c;
    k_dm_ev<<<blocks, 256, 0, st>>>(e->rho, e->dim, e->x, e->z, e->nrot, part);
}
static void launch_trace(double* part, unsigned blocks, cudaStream_t st, const void* c) {
    const EvCtx* e = (const EvCtx*)c;
    k_dm_trace<<<blocks, 256, 0, st>>>(e->rho, e->dim, part);
}

QS_API int qs_dm_expectation_value_multi_qubit_Pauli_operator_partial_list(const QS_UINT* tl, const QS_UINT* ids,
    QS_UINT cnt, const void* rho, QS_ITYPE dim, void* stream, double* out) {
    UINT n;
    QS_TRY(dm_dims(dim, &n));
    QS_TRY(check_distinct(tl, cnt, n, "dm_expectation_value"));
    EvCtx e{(const double2*)rho, dim, 0, 0, 0};
    for (UINT i = 0; i < cnt; ++i) {
        const ITYPE b = 1ULL << tl[i];
        if (ids[i] == 1) e.x ^= b;
        else if (ids[i] == 2) { e.x ^= b; e.z ^= b; e.nrot++; }
        else if (ids[i] == 3) e.z ^= b;
        else if (ids[i] != 0) return set_error(QS_ERR_INVALID_ARGUMENT, "Pauli id must be 0..3");
    }
    return dm_reduce(launch_ev, &e, dim, ST, out);
}
QS_API int qs_dm_state_norm_squared(const void* rho, QS_ITYPE dim, void* stream, double* out) {
    UINT n;
    QS_TRY(dm_dims(dim, &n));
    EvCtx e{(const double2*)rho, dim, 0, 0, 0};
    return dm_reduce(launch_trace, &e, dim, ST, out);
}
QS_API int qs_dm_sampling_with_uniforms(const void* rho, QS_ITYPE dim, const double* uniforms, QS_UINT count,
    QS_ITYPE* out, void* stream) {
    UINT n;
    QS_TRY(dm_dims(dim, &n));
    return sample_with_uniforms((const double2*)rho, dim, dim + 1, uniforms, count, out, ST);
}

}  // extern "C"
