// Whole-state arithmetic (csim update_ops_named_state.cpp, stat_ops_dm.cpp:121-162) and state
// initialisation / element access that cppsim's QuantumState and DensityMatrix expose.
#include <cmath>

#include "qs_internal.cuh"

namespace qs {

constexpr int kOpThreads = 256;

static unsigned elem_grid(ITYPE n) {
    const ITYPE b = (n + kOpThreads - 1) / kOpThreads;
    const ITYPE cap = (ITYPE)sm_count() * 16;
    return (unsigned)(b < cap ? (b > 0 ? b : 1) : cap);
}

// state[i] += coef * added[i]  (update_ops_named_state.cpp:47-75; coef = 1 is state_add)
__global__ void k_axpy(double2* __restrict__ s, const double2* __restrict__ added, double2 coef, ITYPE n) {
    const ITYPE stride = (ITYPE)gridDim.x * kOpThreads;
    for (ITYPE i = (ITYPE)blockIdx.x * kOpThreads + threadIdx.x; i < n; i += stride)
        st_stream(s + i, cfma(coef, ld_stream(added + i), ld_stream(s + i)));
}

// state[i] *= coef  (update_ops_named_state.cpp:86-95; normalize, :21-30, is coef = sqrt(1 / |psi|^2))
__global__ void k_scale(double2* __restrict__ s, double2 coef, ITYPE n) {
    const ITYPE stride = (ITYPE)gridDim.x * kOpThreads;
    for (ITYPE i = (ITYPE)blockIdx.x * kOpThreads + threadIdx.x; i < n; i += stride)
        st_stream(s + i, cmul(coef, ld_stream(s + i)));
}

// state[i] *= factors[i]  (QuantumStateCpu::multiply_elementwise_function, cppsim/state.hpp:885-891,
// with the function's values tabulated on the host)
__global__ void k_mul_elementwise(double2* __restrict__ s, const double2* __restrict__ f, ITYPE n) {
    const ITYPE stride = (ITYPE)gridDim.x * kOpThreads;
    for (ITYPE i = (ITYPE)blockIdx.x * kOpThreads + threadIdx.x; i < n; i += stride)
        st_stream(s + i, cmul(ld_stream(f + i), ld_stream(s + i)));
}

// splitmix64 (Steele, Lea & Flood 2014): a counter-based generator, so amplitude i's value does not
// depend on the launch shape.
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// a_i = g1 + i g2 with independent standard normals (Box-Muller from two uniforms in (0, 1]);
// normalised afterwards, this is a Haar-random pure state.
__global__ void k_gaussian_state(double2* __restrict__ s, unsigned long long seed, ITYPE n) {
    const ITYPE stride = (ITYPE)gridDim.x * kOpThreads;
    const unsigned long long key = splitmix64(seed ^ 0x5DEECE66DULL);
    for (ITYPE i = (ITYPE)blockIdx.x * kOpThreads + threadIdx.x; i < n; i += stride) {
        const unsigned long long r1 = splitmix64(key + 2 * i), r2 = splitmix64(key + 2 * i + 1);
        const double u1 = (double)((r1 >> 11) + 1) * (1.0 / 9007199254740992.0);
        const double u2 = (double)(r2 >> 11) * (1.0 / 9007199254740992.0);
        const double r = sqrt(-2.0 * log(u1));
        double sn, cs;
        sincospi(2.0 * u2, &sn, &cs);
        s[i] = make_double2(r * cs, r * sn);
    }
}

static int axpy(void* state, const void* added, double2 coef, ITYPE n, cudaStream_t st) {
    if (!state || !added) return set_error(QS_ERR_INVALID_ARGUMENT, "null state");
    k_axpy<<<elem_grid(n), kOpThreads, 0, st>>>((double2*)state, (const double2*)added, coef, n);
    return check_launch("k_axpy");
}
static int scale(void* state, double2 coef, ITYPE n, cudaStream_t st) {
    if (!state) return set_error(QS_ERR_INVALID_ARGUMENT, "null state");
    k_scale<<<elem_grid(n), kOpThreads, 0, st>>>((double2*)state, coef, n);
    return check_launch("k_scale");
}
static int dm_entries(ITYPE dim, ITYPE* n) {
    UINT q;
    QS_TRY(check_dim(dim, &q));
    if (q > 20) return set_error(QS_ERR_NOT_SUPPORTED, "density matrix: at most 20 qubits");
    *n = dim * dim;
    return QS_OK;
}

}  // namespace qs

using namespace qs;

extern "C" {

QS_API int qs_state_add(const void* state_added, void* state, QS_ITYPE dim, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    return axpy(state, state_added, make_double2(1., 0.), dim, (cudaStream_t)stream);
}
QS_API int qs_state_add_with_coef(const double coef[2], const void* state_added, void* state, QS_ITYPE dim,
    void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (!coef) return set_error(QS_ERR_INVALID_ARGUMENT, "null coefficient");
    return axpy(state, state_added, make_double2(coef[0], coef[1]), dim, (cudaStream_t)stream);
}
QS_API int qs_state_multiply(const double coef[2], void* state, QS_ITYPE dim, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (!coef) return set_error(QS_ERR_INVALID_ARGUMENT, "null coefficient");
    return scale(state, make_double2(coef[0], coef[1]), dim, (cudaStream_t)stream);
}
QS_API int qs_normalize(double squared_norm, void* state, QS_ITYPE dim, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (!(squared_norm > 0.)) return set_error(QS_ERR_INVALID_ARGUMENT, "normalize: squared norm must be positive");
    return scale(state, make_double2(std::sqrt(1. / squared_norm), 0.), dim, (cudaStream_t)stream);
}
QS_API int qs_state_multiply_elementwise(const void* factors, void* state, QS_ITYPE dim, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (!state || !factors) return set_error(QS_ERR_INVALID_ARGUMENT, "null state");
    k_mul_elementwise<<<elem_grid(dim), kOpThreads, 0, (cudaStream_t)stream>>>((double2*)state,
        (const double2*)factors, dim);
    return check_launch("k_mul_elementwise");
}
QS_API int qs_dm_state_add(const void* rho_added, void* rho, QS_ITYPE dim, void* stream) {
    ITYPE n;
    QS_TRY(dm_entries(dim, &n));
    return axpy(rho, rho_added, make_double2(1., 0.), n, (cudaStream_t)stream);
}
QS_API int qs_dm_state_add_with_coef(const double coef[2], const void* rho_added, void* rho, QS_ITYPE dim,
    void* stream) {
    ITYPE n;
    QS_TRY(dm_entries(dim, &n));
    if (!coef) return set_error(QS_ERR_INVALID_ARGUMENT, "null coefficient");
    return axpy(rho, rho_added, make_double2(coef[0], coef[1]), n, (cudaStream_t)stream);
}
QS_API int qs_dm_state_multiply(const double coef[2], void* rho, QS_ITYPE dim, void* stream) {
    ITYPE n;
    QS_TRY(dm_entries(dim, &n));
    if (!coef) return set_error(QS_ERR_INVALID_ARGUMENT, "null coefficient");
    return scale(rho, make_double2(coef[0], coef[1]), n, (cudaStream_t)stream);
}
QS_API int qs_dm_normalize(double squared_norm, void* rho, QS_ITYPE dim, void* stream) {
    ITYPE n;
    QS_TRY(dm_entries(dim, &n));
    if (!(squared_norm > 0.)) return set_error(QS_ERR_INVALID_ARGUMENT, "dm_normalize: squared norm must be positive");
    return scale(rho, make_double2(1. / squared_norm, 0.), n, (cudaStream_t)stream);
}
QS_API int qs_copy_state(const void* src, void* dst, QS_ITYPE count, void* stream) {
    if (!src || !dst) return set_error(QS_ERR_INVALID_ARGUMENT, "null state");
    QS_CUDA_CHECK(cudaMemcpyAsync(dst, src, count * sizeof(double2), cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
    return QS_OK;
}
QS_API int qs_initialize_Haar_random_state_with_seed(void* state, QS_ITYPE dim, QS_UINT seed, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (!state) return set_error(QS_ERR_INVALID_ARGUMENT, "null state");
    k_gaussian_state<<<elem_grid(dim), kOpThreads, 0, (cudaStream_t)stream>>>((double2*)state, seed, dim);
    QS_TRY(check_launch("k_gaussian_state"));
    double nrm = 0.;
    QS_TRY(qs_state_norm_squared(state, dim, stream, &nrm));
    return qs_normalize(nrm, state, dim, stream);
}
QS_API int qs_get_amplitude(const void* state, QS_ITYPE dim, QS_ITYPE index, double out[2], void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (!state || !out) return set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    if (index >= dim) return set_error(QS_ERR_INVALID_ARGUMENT, "amplitude index out of range");
    QS_CUDA_CHECK(cudaMemcpyAsync(out, (const double2*)state + index, sizeof(double2), cudaMemcpyDeviceToHost,
        (cudaStream_t)stream));
    QS_CUDA_CHECK(cudaStreamSynchronize((cudaStream_t)stream));
    return QS_OK;
}

}  // extern "C"
