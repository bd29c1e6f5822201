// State manipulation of csim stat_ops.cpp:111-158 (tensor product, qubit permutation, dropping
// projected qubits) and stat_ops_dm.cpp:193-296 (the density-matrix forms and partial traces), the
// reflection gate (update_ops_reflection.cpp:14-27) and FusedSWAP (update_ops_named_FusedSWAP.cpp:19-
// 60): gather kernels over 64-bit indices, one output element per thread-iteration.
#include <algorithm>
#include <random>
#include <string>
#include <vector>

#include "qs_internal.cuh"

namespace qs {

constexpr int kManThreads = 256;

static unsigned man_grid(ITYPE n) {
    const ITYPE b = (n + kManThreads - 1) / kManThreads;
    const ITYPE cap = (ITYPE)sm_count() * 16;
    return (unsigned)(b < cap ? (b > 0 ? b : 1) : cap);
}

struct QubitList {
    int count;
    UINT q[kMaxQubits];
};

// bits of i scattered to the listed positions: bit j of i -> position q[j]
__device__ __forceinline__ ITYPE scatter_bits(ITYPE i, const QubitList& l) {
    ITYPE r = 0;
    for (int j = 0; j < l.count; ++j)
        if ((i >> j) & 1) r |= 1ULL << l.q[j];
    return r;
}
// zeros inserted at the ascending positions q[0] < q[1] < ...
__device__ __forceinline__ ITYPE insert_zeros(ITYPE i, const QubitList& sorted) {
    for (int j = 0; j < sorted.count; ++j) i = insert0(i, sorted.q[j]);
    return i;
}

// dst[l * dim_right + r] = left[l] right[r]  (stat_ops.cpp:111-121)
__global__ void k_tensor(const double2* __restrict__ left, const double2* __restrict__ right, UINT right_bits,
    double2* __restrict__ dst, ITYPE n) {
    const ITYPE stride = (ITYPE)gridDim.x * kManThreads, rmask = (1ULL << right_bits) - 1;
    for (ITYPE i = (ITYPE)blockIdx.x * kManThreads + threadIdx.x; i < n; i += stride)
        dst[i] = cmul(left[i >> right_bits], right[i & rmask]);
}
// rho_dst[(yl dr + yr) D + (xl dr + xr)] = right[yr][xr] left[yl][xl]  (stat_ops_dm.cpp:193-211)
__global__ void k_dm_tensor(const double2* __restrict__ left, UINT left_bits, const double2* __restrict__ right,
    UINT right_bits, double2* __restrict__ dst) {
    const UINT nb = left_bits + right_bits;
    const ITYPE n = 1ULL << (2 * nb), stride = (ITYPE)gridDim.x * kManThreads;
    const ITYPE rmask = (1ULL << right_bits) - 1, dmask = (1ULL << nb) - 1;
    for (ITYPE e = (ITYPE)blockIdx.x * kManThreads + threadIdx.x; e < n; e += stride) {
        const ITYPE y = e >> nb, x = e & dmask;
        const ITYPE l = ((y >> right_bits) << left_bits) | (x >> right_bits);
        const ITYPE r = ((y & rmask) << right_bits) | (x & rmask);
        dst[e] = cmul(right[r], left[l]);
    }
}
// dst[i] = src[sum over set bits q of i of 2^order[q]]  (stat_ops.cpp:122-134)
__global__ void k_permutate(const double2* __restrict__ src, double2* __restrict__ dst, const __grid_constant__ QubitList order,
    ITYPE n) {
    const ITYPE stride = (ITYPE)gridDim.x * kManThreads;
    for (ITYPE i = (ITYPE)blockIdx.x * kManThreads + threadIdx.x; i < n; i += stride) dst[i] = src[scatter_bits(i, order)];
}
// rho_dst[y][x] = rho_src[perm(y)][perm(x)]  (stat_ops_dm.cpp:213-231)
__global__ void k_dm_permutate(const double2* __restrict__ src, double2* __restrict__ dst,
    const __grid_constant__ QubitList order, UINT nbits) {
    const ITYPE n = 1ULL << (2 * nbits), stride = (ITYPE)gridDim.x * kManThreads, m = (1ULL << nbits) - 1;
    for (ITYPE e = (ITYPE)blockIdx.x * kManThreads + threadIdx.x; e < n; e += stride)
        dst[e] = src[(scatter_bits(e >> nbits, order) << nbits) | scatter_bits(e & m, order)];
}
// dst[i] = src[insert zeros at the targets into i, then the projection bits]  (stat_ops.cpp:136-158)
__global__ void k_drop(const double2* __restrict__ src, double2* __restrict__ dst, const __grid_constant__ QubitList sorted,
    ITYPE projection, ITYPE n) {
    const ITYPE stride = (ITYPE)gridDim.x * kManThreads;
    for (ITYPE i = (ITYPE)blockIdx.x * kManThreads + threadIdx.x; i < n; i += stride)
        dst[i] = src[insert_zeros(i, sorted) ^ projection];
}
// rho_dst[y][x] = sum_t rho[by ^ m_t][bx ^ m_t] (from_dm) or psi[by ^ m_t] conj(psi[bx ^ m_t]) (from a
// state vector), m_t = the traced qubits' bits spelling t  (stat_ops_dm.cpp:233-296)
template <bool FROM_DM>
__global__ void k_partial_trace(const double2* __restrict__ src, double2* __restrict__ dst,
    const __grid_constant__ QubitList sorted, const __grid_constant__ QubitList listed, UINT dst_bits, ITYPE dim) {
    const ITYPE n = 1ULL << (2 * dst_bits), stride = (ITYPE)gridDim.x * kManThreads, m = (1ULL << dst_bits) - 1;
    const ITYPE trace = 1ULL << listed.count;
    for (ITYPE e = (ITYPE)blockIdx.x * kManThreads + threadIdx.x; e < n; e += stride) {
        const ITYPE by = insert_zeros(e >> dst_bits, sorted), bx = insert_zeros(e & m, sorted);
        double2 acc = make_double2(0., 0.);
        for (ITYPE t = 0; t < trace; ++t) {
            const ITYPE mt = scatter_bits(t, listed);
            if (FROM_DM) {
                const double2 v = src[(by ^ mt) * dim + (bx ^ mt)];
                acc.x += v.x;
                acc.y += v.y;
            } else {
                acc = cfma(src[by ^ mt], cconj(src[bx ^ mt]), acc);
            }
        }
        dst[e] = acc;
    }
}
// state = 2 coef r - state  (update_ops_reflection.cpp:14-27, coef = <r|state>)
__global__ void k_reflect(const double2* __restrict__ r, double2* __restrict__ s, double2 two_coef, ITYPE n) {
    const ITYPE stride = (ITYPE)gridDim.x * kManThreads;
    for (ITYPE i = (ITYPE)blockIdx.x * kManThreads + threadIdx.x; i < n; i += stride) {
        const double2 a = s[i];
        s[i] = cfma(two_coef, r[i], make_double2(-a.x, -a.y));
    }
}

static int qubit_count_of(ITYPE dim, UINT* n) { return check_dim(dim, n); }

static QubitList make_list(const UINT* q, UINT count, bool sort) {
    QubitList l{};
    l.count = (int)count;
    std::vector<UINT> v(q, q + count);
    if (sort) std::sort(v.begin(), v.end());
    for (UINT j = 0; j < count; ++j) l.q[j] = v[j];
    return l;
}

static int check_permutation(const UINT* order, UINT count, UINT n, const char* what) {
    if (count != n) return set_error(QS_ERR_INVALID_ARGUMENT, std::string(what) + ": the order must list every qubit");
    return check_distinct(order, count, n, what);
}

}  // namespace qs

using namespace qs;

extern "C" {

QS_API int qs_state_tensor_product(const void* left, QS_ITYPE dim_left, const void* right, QS_ITYPE dim_right,
    void* dst, void* stream) {
    UINT nl, nr;
    QS_TRY(qubit_count_of(dim_left, &nl));
    QS_TRY(qubit_count_of(dim_right, &nr));
    if (nl + nr > (UINT)kMaxQubits) return set_error(QS_ERR_NOT_SUPPORTED, "state_tensor_product: more than 40 qubits");
    if (!left || !right || !dst) return set_error(QS_ERR_INVALID_ARGUMENT, "null state");
    const ITYPE n = dim_left * dim_right;
    cudaStream_t st = (cudaStream_t)stream;
    k_tensor<<<man_grid(n), kManThreads, 0, st>>>((const double2*)left, (const double2*)right, nr, (double2*)dst, n);
    return check_launch("k_tensor");
}

QS_API int qs_state_permutate_qubit(const QS_UINT* qubit_order, const void* src, void* dst, QS_UINT qubit_count,
    QS_ITYPE dim, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    QS_TRY(check_permutation(qubit_order, qubit_count, n, "state_permutate_qubit"));
    if (!src || !dst) return set_error(QS_ERR_INVALID_ARGUMENT, "null state");
    cudaStream_t st = (cudaStream_t)stream;
    k_permutate<<<man_grid(dim), kManThreads, 0, st>>>((const double2*)src, (double2*)dst,
        make_list(qubit_order, qubit_count, false), dim);
    return check_launch("k_permutate");
}

QS_API int qs_state_drop_qubits(const QS_UINT* target, const QS_UINT* projection, QS_UINT target_count, const void* src,
    void* dst, QS_ITYPE dim, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (target_count >= n) return set_error(QS_ERR_INVALID_ARGUMENT, "state_drop_qubits: at least one qubit must stay");
    QS_TRY(check_distinct(target, target_count, n, "state_drop_qubits"));
    ITYPE proj = 0;
    for (UINT j = 0; j < target_count; ++j) {
        if (projection[j] > 1) return set_error(QS_ERR_INVALID_ARGUMENT, "state_drop_qubits: projection must be 0 or 1");
        if (projection[j]) proj |= 1ULL << target[j];
    }
    if (!src || !dst) return set_error(QS_ERR_INVALID_ARGUMENT, "null state");
    const ITYPE out = dim >> target_count;
    cudaStream_t st = (cudaStream_t)stream;
    k_drop<<<man_grid(out), kManThreads, 0, st>>>((const double2*)src, (double2*)dst,
        make_list(target, target_count, true), proj, out);
    return check_launch("k_drop");
}

QS_API int qs_dm_state_tensor_product(const void* left, QS_ITYPE dim_left, const void* right, QS_ITYPE dim_right,
    void* dst, void* stream) {
    UINT nl, nr;
    QS_TRY(qubit_count_of(dim_left, &nl));
    QS_TRY(qubit_count_of(dim_right, &nr));
    if (nl + nr > 20) return set_error(QS_ERR_NOT_SUPPORTED, "dm_state_tensor_product: more than 20 qubits");
    if (!left || !right || !dst) return set_error(QS_ERR_INVALID_ARGUMENT, "null state");
    cudaStream_t st = (cudaStream_t)stream;
    k_dm_tensor<<<man_grid(1ULL << (2 * (nl + nr))), kManThreads, 0, st>>>((const double2*)left, nl,
        (const double2*)right, nr, (double2*)dst);
    return check_launch("k_dm_tensor");
}

QS_API int qs_dm_state_permutate_qubit(const QS_UINT* qubit_order, const void* src, void* dst, QS_UINT qubit_count,
    QS_ITYPE dim, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (n > 20) return set_error(QS_ERR_NOT_SUPPORTED, "density matrix: more than 20 qubits");
    QS_TRY(check_permutation(qubit_order, qubit_count, n, "dm_state_permutate_qubit"));
    if (!src || !dst) return set_error(QS_ERR_INVALID_ARGUMENT, "null state");
    cudaStream_t st = (cudaStream_t)stream;
    k_dm_permutate<<<man_grid(dim * dim), kManThreads, 0, st>>>((const double2*)src, (double2*)dst,
        make_list(qubit_order, qubit_count, false), n);
    return check_launch("k_dm_permutate");
}

static int partial_trace(bool from_dm, const UINT* target, UINT count, const void* src, void* dst, ITYPE dim,
    void* stream, const char* what) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (from_dm && n > 20) return set_error(QS_ERR_NOT_SUPPORTED, "density matrix: more than 20 qubits");
    if (count >= n) return set_error(QS_ERR_INVALID_ARGUMENT, std::string(what) + ": at least one qubit must stay");
    if (n - count > 20) return set_error(QS_ERR_NOT_SUPPORTED, std::string(what) + ": result over 20 qubits");
    QS_TRY(check_distinct(target, count, n, what));
    if (!src || !dst) return set_error(QS_ERR_INVALID_ARGUMENT, "null state");
    const UINT db = n - count;
    const QubitList sorted = make_list(target, count, true), listed = make_list(target, count, false);
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned grid = man_grid(1ULL << (2 * db));
    if (from_dm)
        k_partial_trace<true><<<grid, kManThreads, 0, st>>>((const double2*)src, (double2*)dst, sorted, listed, db, dim);
    else
        k_partial_trace<false><<<grid, kManThreads, 0, st>>>((const double2*)src, (double2*)dst, sorted, listed, db, dim);
    return check_launch("k_partial_trace");
}
QS_API int qs_dm_state_partial_trace_from_density_matrix(const QS_UINT* target, QS_UINT target_count, const void* src,
    void* dst, QS_ITYPE dim, void* stream) {
    return partial_trace(true, target, target_count, src, dst, dim, stream, "dm_state_partial_trace_from_density_matrix");
}
QS_API int qs_dm_state_partial_trace_from_state_vector(const QS_UINT* target, QS_UINT target_count, const void* src,
    void* dst, QS_ITYPE dim, void* stream) {
    return partial_trace(false, target, target_count, src, dst, dim, stream, "dm_state_partial_trace_from_state_vector");
}

QS_API int qs_reflection_gate(const void* reflection_state, void* state, QS_ITYPE dim, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (!reflection_state || !state) return set_error(QS_ERR_INVALID_ARGUMENT, "null state");
    double c[2];
    QS_TRY(qs_state_inner_product(reflection_state, state, dim, stream, c));
    cudaStream_t st = (cudaStream_t)stream;
    k_reflect<<<man_grid(dim), kManThreads, 0, st>>>((const double2*)reflection_state, (double2*)state,
        make_double2(2. * c[0], 2. * c[1]), dim);
    return check_launch("k_reflect");
}

// The block [t0, t0 + block) swapped with [t1, t1 + block), qubit by qubit (the reference's own
// single-process form, update_ops_named_FusedSWAP.cpp:21-25; its preconditions at :36-37).
QS_API int qs_FusedSWAP_gate(QS_UINT t0, QS_UINT t1, QS_UINT block_size, void* state, QS_ITYPE dim, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    const UINT lo = t0 < t1 ? t0 : t1, hi = t0 < t1 ? t1 : t0;
    if (block_size == 0 || hi <= lo + block_size - 1 || hi + block_size - 1 >= n)
        return set_error(QS_ERR_INVALID_ARGUMENT, "FusedSWAP_gate: blocks overlap or leave the state");
    for (UINT i = 0; i < block_size; ++i) QS_TRY(qs_SWAP_gate(t0 + i, t1 + i, state, dim, stream));
    return QS_OK;
}

// Unseeded Haar-random state (init_ops.hpp:20): the seeded form with a seed from std::random_device.
QS_API int qs_initialize_Haar_random_state(void* state, QS_ITYPE dim, void* stream) {
    std::random_device rd;
    return qs_initialize_Haar_random_state_with_seed(state, dim, (QS_UINT)rd(), stream);
}

}  // extern "C"
