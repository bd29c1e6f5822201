// Internal definitions shared by the qulacs_b200 CUDA translation units.
//
// State layout in HBM: a state vector of n qubits is 2^n amplitudes, contiguous, amplitude i at
// byte offset 16*i as (re, im) doubles -- the layout of csim's CTYPE array (csim/type.hpp:15-30),
// so a device buffer is a drop-in for the reference's `CTYPE* state` / gpusim's `void* state`.
// Bit q of an amplitude index is qubit q.  A density matrix rho of n qubits is dim x dim
// amplitudes, row-major rho[y * dim + x] (cppsim/state_dm.hpp), i.e. a 2n-qubit vector whose
// bits 0..n-1 are the column index and bits n..2n-1 the row index.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/qulacs_b200.h"
#include "circuit.hpp"  // kMaxQubits, kMaxDenseTargets

typedef unsigned long long ITYPE;
typedef unsigned int UINT;

namespace qs {

// ---------------------------------------------------------------- errors
// Records the message of the last failing call of this host thread and returns its code.
int set_error(int code, const std::string& msg);
int check_cuda(cudaError_t e, const char* what);
#define QS_CUDA_CHECK(expr)                                   \
    do {                                                      \
        cudaError_t _e = (expr);                              \
        if (_e != cudaSuccess) return qs::check_cuda(_e, #expr); \
    } while (0)
#define QS_TRY(expr)                 \
    do {                             \
        int _rc = (expr);            \
        if (_rc != QS_OK) return _rc; \
    } while (0)

// Checks common to every state-vector entry point: dim a power of two >= 2.
int check_dim(ITYPE dim, UINT* n_out);
int check_target(UINT target, UINT n, const char* what);
int check_distinct(const UINT* list, UINT count, UINT n, const char* what);

// After a launch: returns QS_ERR_CUDA with the launch error, if any.
int check_launch(const char* kernel);
// Adjusts the launch counter (graph replays: the kernels a captured graph holds; capture itself: minus
// the launches it recorded, which did not run).
void count_launches(long long delta);
// Graph capture (this thread): calls whose run copies from host memory refuse to be recorded, since a
// replay would read that host memory again after the call has returned.
void set_capturing(bool on);
int refuse_if_capturing(const char* what);

// Per (device, stream) scratch buffer for reduction partials and uploaded matrices.  Grows on
// demand with cudaMalloc; stream order makes reuse by the next call on the same stream safe.
int scratch(cudaStream_t stream, size_t bytes, void** out);

// Number of SMs of the current device (cached).
int sm_count();

// ---------------------------------------------------------------- device helpers
__host__ __device__ __forceinline__ ITYPE insert0(ITYPE i, UINT q) {
    const ITYPE low = i & ((1ULL << q) - 1ULL);
    return ((i >> q) << (q + 1)) | low;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// acc + a * b
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 acc) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
    return acc;
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double norm2(double2 a) { return fma(a.x, a.x, a.y * a.y); }

// Streaming 128-bit global accesses: every amplitude is touched once per pass, so loads bypass
// L1 allocation and stores are marked evict-first in L2.
__device__ __forceinline__ double2 ld_stream(const double2* p) {
    double2 v;
    asm volatile("ld.global.cs.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
}
__device__ __forceinline__ void st_stream(double2* p, double2 v) {
    asm volatile("st.global.cs.v2.f64 [%0], {%1, %2};" ::"l"(p), "d"(v.x), "d"(v.y) : "memory");
}
// An amplitude of a complex128 or complex64 state as FP64, and back (complex64: rounded to nearest).
__device__ __forceinline__ double2 ld_amp(const double2* p) { return ld_stream(p); }
__device__ __forceinline__ double2 ld_amp(const float2* p) {
    const float2 v = __ldcs(p);
    return make_double2((double)v.x, (double)v.y);
}
__device__ __forceinline__ void st_amp(double2* p, double2 v) { st_stream(p, v); }
__device__ __forceinline__ void st_amp(float2* p, double2 v) {
    __stcs(p, make_float2(__double2float_rn(v.x), __double2float_rn(v.y)));
}

struct Mat2 {
    double2 m[4];  // row-major
};
struct Mat4 {
    double2 m[16];  // row-major, matrix-index bit j <-> target j
};

// Launchers shared between translation units (gates_c128.cu, stats_c128.cu).
int launch_dense1(UINT t, const Mat2& m, double2* s, ITYPE dim, const UINT* ctl, const UINT* cval,
    UINT nc, cudaStream_t st);
int launch_diag1(UINT t, double2 d0, double2 d1, double2* s, ITYPE dim, cudaStream_t st);
int launch_dense2(UINT t1, UINT t2, const Mat4& m, double2* s, ITYPE dim, const UINT* ctl,
    const UINT* cval, UINT nc, cudaStream_t st);
// matrix: host pointer, row-major 2^k x 2^k interleaved doubles, 3 <= k <= kMaxDenseTargets
int launch_denseK(const UINT* tl, UINT k, const double* matrix, double2* s, ITYPE dim,
    const UINT* ctl, const UINT* cval, UINT nc, cudaStream_t st);
int prob_sum(const double2* s, ITYPE dim, ITYPE mask, ITYPE value, cudaStream_t st, double* out);
// diag_stride 0: state vector; dim + 1: density matrix diagonal (|rho_ii|).
int sample_with_uniforms(const double2* s, ITYPE dim, ITYPE diag_stride, const double* uniforms,
    UINT count, ITYPE* out, cudaStream_t st);

// Block-wide FP64 sum of one value per thread (blockDim.x a multiple of 32, <= 1024), fixed order:
// a warp shuffle tree, then warp 0 folds the per-warp sums.  Result valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* smem32) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) smem32[warp] = v;
    __syncthreads();
    double r = 0.;
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        r = lane < nw ? smem32[lane] : 0.;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;
}

}  // namespace qs
