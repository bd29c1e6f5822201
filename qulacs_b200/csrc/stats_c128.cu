// Reductions over a complex128 state: norm, inner product, probabilities, Pauli expectation values
// and sampling.  All sums are FP64 and deterministic: a fixed per-thread order, a warp shuffle tree,
// one partial per CTA written to scratch, then one CTA folds the partials in index order (no
// floating-point atomics).
#include <algorithm>
#include <cstring>
#include <mutex>
#include <random>
#include <unordered_map>
#include <atomic>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <vector>

#include "ev_spec.hpp"
#include "qs_internal.cuh"

namespace qs {

constexpr int kRThreads = 256;

// FP64 view of one amplitude of a complex128 or complex64 state.
__device__ __forceinline__ double2 amp(const double2* p) { return ld_stream(p); }
__device__ __forceinline__ double2 amp(const float2* p) {
    const float2 v = __ldcs(p);
    return make_double2((double)v.x, (double)v.y);
}
constexpr int kMaxPartials = 4096;

static unsigned reduce_blocks(ITYPE items) {
    ITYPE b = (items + kRThreads - 1) / kRThreads;
    ITYPE cap = std::min<ITYPE>((ITYPE)sm_count() * 8, kMaxPartials);
    return (unsigned)std::max<ITYPE>(1, std::min(b, cap));
}

// Folds `count` partial vectors (each `width` doubles, partial p of value w at p * width + w)
// into out[w], one CTA per value.
__global__ void k_fold_partials(const double* __restrict__ part, int count, int width, double* __restrict__ out) {
    __shared__ double sm[32];
    const int w = blockIdx.x;
    double v = 0.;
    for (int p = threadIdx.x; p < count; p += blockDim.x) v += part[(size_t)p * width + w];
    v = block_sum(v, sm);
    if (threadIdx.x == 0) out[w] = v;
}

// ---------------------------------------------------------------- norm / probabilities
// mode 0: sum |a|^2 ; mode 1: sum over bit t == 0 ; mode 2: bit t == 1 ;
// mode 3: marginal (mask/value pair)
template <class T>
__global__ void __launch_bounds__(kRThreads) k_prob_sum(
    const T* __restrict__ s, ITYPE dim, ITYPE mask, ITYPE value, double* __restrict__ part) {
    __shared__ double sm[32];
    double acc = 0.;
    const ITYPE stride = (ITYPE)gridDim.x * kRThreads;
    for (ITYPE i = (ITYPE)blockIdx.x * kRThreads + threadIdx.x; i < dim; i += stride)
        if ((i & mask) == value) acc += norm2(amp(s + i));
    acc = block_sum(acc, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

__global__ void __launch_bounds__(kRThreads) k_inner(const double2* __restrict__ a, const double2* __restrict__ b,
    ITYPE dim, double* __restrict__ part) {
    __shared__ double sm[32];
    double re = 0., im = 0.;
    const ITYPE stride = (ITYPE)gridDim.x * kRThreads;
    for (ITYPE i = (ITYPE)blockIdx.x * kRThreads + threadIdx.x; i < dim; i += stride) {
        const double2 x = ld_stream(a + i), y = ld_stream(b + i);
        re = fma(x.x, y.x, fma(x.y, y.y, re));
        im = fma(x.x, y.y, fma(-x.y, y.x, im));
    }
    re = block_sum(re, sm);
    im = block_sum(im, sm);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = re;
        part[2 * blockIdx.x + 1] = im;
    }
}

static int finish_reduce(double* part, unsigned blocks, int width, cudaStream_t st, double* host_out) {
    double* fin = part + (size_t)blocks * width;
    k_fold_partials<<<width, 256, 0, st>>>(part, (int)blocks, width, fin);
    QS_TRY(check_launch("k_fold_partials"));
    QS_CUDA_CHECK(cudaMemcpyAsync(host_out, fin, sizeof(double) * width, cudaMemcpyDeviceToHost, st));
    QS_CUDA_CHECK(cudaStreamSynchronize(st));
    return QS_OK;
}

template <class T>
int prob_sum_t(const T* s, ITYPE dim, ITYPE mask, ITYPE value, cudaStream_t st, double* out) {
    const unsigned blocks = reduce_blocks(dim);
    void* buf;
    QS_TRY(scratch(st, sizeof(double) * (blocks + 1), &buf));
    k_prob_sum<T><<<blocks, kRThreads, 0, st>>>(s, dim, mask, value, (double*)buf);
    QS_TRY(check_launch("k_prob_sum"));
    return finish_reduce((double*)buf, blocks, 1, st, out);
}
int prob_sum(const double2* s, ITYPE dim, ITYPE mask, ITYPE value, cudaStream_t st, double* out) {
    return prob_sum_t<double2>(s, dim, mask, value, st, out);
}

// Shannon entropy of the measurement distribution (stat_ops_probability.cpp:83-99): sum of -p log p,
// p = |a_i|^2 clamped below at 1e-15.  Density matrix (stat_ops_dm.cpp:29-46): p = Re rho_ii taken at
// stride dim + 1, terms with p <= 1e-15 skipped.
template <bool DM>
__global__ void __launch_bounds__(kRThreads) k_entropy(const double2* __restrict__ s, ITYPE count, ITYPE stride_elems,
    double* __restrict__ part) {
    __shared__ double sm[32];
    const double eps = 1e-15;
    double acc = 0.;
    const ITYPE stride = (ITYPE)gridDim.x * kRThreads;
    for (ITYPE i = (ITYPE)blockIdx.x * kRThreads + threadIdx.x; i < count; i += stride) {
        const double2 v = s[i * stride_elems];
        if (DM) {
            const double p = v.x;
            if (p > eps) acc += -1.0 * p * log(p);
        } else {
            double p = v.x * v.x + v.y * v.y;
            p = (p > eps) ? p : eps;
            acc += -1.0 * p * log(p);
        }
    }
    acc = block_sum(acc, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// Sum of Re rho_ii over the diagonal indices i with (i & mask) == value (stat_ops_dm.cpp:50-120:
// dm_M0_prob, dm_M1_prob, dm_marginal_prob).
__global__ void __launch_bounds__(kRThreads) k_dm_diag_sum(const double2* __restrict__ rho, ITYPE dim, ITYPE mask,
    ITYPE value, double* __restrict__ part) {
    __shared__ double sm[32];
    double acc = 0.;
    const ITYPE stride = (ITYPE)gridDim.x * kRThreads;
    for (ITYPE i = (ITYPE)blockIdx.x * kRThreads + threadIdx.x; i < dim; i += stride)
        if ((i & mask) == value) acc += rho[i * (dim + 1)].x;
    acc = block_sum(acc, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

static int dm_diag_sum(const double2* rho, ITYPE dim, ITYPE mask, ITYPE value, cudaStream_t st, double* out) {
    const unsigned blocks = reduce_blocks(dim);
    void* buf;
    QS_TRY(scratch(st, sizeof(double) * (blocks + 1), &buf));
    k_dm_diag_sum<<<blocks, kRThreads, 0, st>>>(rho, dim, mask, value, (double*)buf);
    QS_TRY(check_launch("k_dm_diag_sum"));
    return finish_reduce((double*)buf, blocks, 1, st, out);
}

template <bool DM>
static int entropy(const double2* s, ITYPE count, ITYPE stride_elems, cudaStream_t st, double* out) {
    const unsigned blocks = reduce_blocks(count);
    void* buf;
    QS_TRY(scratch(st, sizeof(double) * (blocks + 1), &buf));
    k_entropy<DM><<<blocks, kRThreads, 0, st>>>(s, count, stride_elems, (double*)buf);
    QS_TRY(check_launch("k_entropy"));
    return finish_reduce((double*)buf, blocks, 1, st, out);
}

// sum conj(bra_i) ket_i with a complex128 bra and a complex64 ket, FP64 accumulation
__global__ void __launch_bounds__(kRThreads) k_inner_mixed(const double2* __restrict__ a, const float2* __restrict__ b,
    ITYPE dim, double* __restrict__ part) {
    __shared__ double sm[32];
    double re = 0., im = 0.;
    const ITYPE stride = (ITYPE)gridDim.x * kRThreads;
    for (ITYPE i = (ITYPE)blockIdx.x * kRThreads + threadIdx.x; i < dim; i += stride) {
        const double2 x = ld_stream(a + i), y = amp(b + i);
        re = fma(x.x, y.x, fma(x.y, y.y, re));
        im = fma(x.x, y.y, fma(-x.y, y.x, im));
    }
    re = block_sum(re, sm);
    im = block_sum(im, sm);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = re;
        part[2 * blockIdx.x + 1] = im;
    }
}

// ---------------------------------------------------------------- Pauli expectation values
struct PauliTerm {
    ITYPE x, z;
    UINT nrot, pivot;
};

__device__ __forceinline__ double phase_re_part(double2 v, UINT r) {
    // Re(v * i^r)
    switch (r & 3u) {
        case 0: return v.x;
        case 1: return -v.y;
        case 2: return -v.x;
        default: return v.y;
    }
}

// One term with a bit flip: sum over pivot-0 indices b0 of 2 Re(a[b0] conj(a[b0 ^ x]) i^{nY + 2 par}),
// stat_ops_expectation_value.cpp:352-373.
template <class T>
__global__ void __launch_bounds__(kRThreads) k_ev_xz(const T* __restrict__ s, ITYPE half, PauliTerm t,
    double* __restrict__ part) {
    __shared__ double sm[32];
    double acc = 0.;
    const ITYPE stride = (ITYPE)gridDim.x * kRThreads;
    for (ITYPE p = (ITYPE)blockIdx.x * kRThreads + threadIdx.x; p < half; p += stride) {
        const ITYPE b0 = insert0(p, t.pivot), b1 = b0 ^ t.x;
        const double2 a0 = amp(s + b0), a1 = amp(s + b1);
        const double2 v = cmul(a0, cconj(a1));
        const UINT r = t.nrot + 2u * (UINT)(__popcll(b0 & t.z) & 1);
        acc += 2.0 * phase_re_part(v, r);
    }
    acc = block_sum(acc, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// All Z-only terms in one pass: values[w] = sum |a_i|^2 (-1)^{popcount(i & z_w)}
// (stat_ops_expectation_value.cpp:467-482).  Partial p of term w at part[p * nz + w].
template <int MAXZ, class T>
__global__ void __launch_bounds__(kRThreads) k_ev_z_batch(const T* __restrict__ s, ITYPE dim,
    const ITYPE* __restrict__ zmasks, int nz, double* __restrict__ part) {
    __shared__ double sm[32];
    __shared__ ITYPE zs[MAXZ];
    for (int w = threadIdx.x; w < nz; w += kRThreads) zs[w] = zmasks[w];
    __syncthreads();
    double acc[MAXZ];
#pragma unroll
    for (int w = 0; w < MAXZ; ++w) acc[w] = 0.;
    const ITYPE stride = (ITYPE)gridDim.x * kRThreads;
    for (ITYPE i = (ITYPE)blockIdx.x * kRThreads + threadIdx.x; i < dim; i += stride) {
        const double p = norm2(amp(s + i));
#pragma unroll
        for (int w = 0; w < MAXZ; ++w)
            if (w < nz) acc[w] += (__popcll(i & zs[w]) & 1) ? -p : p;
    }
    for (int w = 0; w < nz; ++w) {
        const double v = block_sum(acc[w], sm);
        if (threadIdx.x == 0) part[(size_t)blockIdx.x * nz + w] = v;
    }
}

// Transition amplitude <bra|P|ket> = sum_i conj(bra[i ^ x]) ph(i) ket[i]  (stat_ops_transition_amplitude.cpp)
__global__ void __launch_bounds__(kRThreads) k_transition(const double2* __restrict__ bra,
    const double2* __restrict__ ket, ITYPE dim, PauliTerm t, double* __restrict__ part) {
    __shared__ double sm[32];
    double re = 0., im = 0.;
    const ITYPE stride = (ITYPE)gridDim.x * kRThreads;
    for (ITYPE i = (ITYPE)blockIdx.x * kRThreads + threadIdx.x; i < dim; i += stride) {
        const UINT r = (t.nrot + 2u * (UINT)(__popcll(i & t.z) & 1)) & 3u;
        const double2 ph = make_double2(r == 0 ? 1. : (r == 2 ? -1. : 0.), r == 1 ? 1. : (r == 3 ? -1. : 0.));
        const double2 v = cmul(cconj(ld_stream(bra + (i ^ t.x))), cmul(ph, ld_stream(ket + i)));
        re += v.x;
        im += v.y;
    }
    re = block_sum(re, sm);
    im = block_sum(im, sm);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = re;
        part[2 * blockIdx.x + 1] = im;
    }
}

static int pauli_term(const UINT* tl, const UINT* ids, UINT cnt, UINT n, PauliTerm* t) {
    t->x = t->z = 0;
    t->nrot = t->pivot = 0;
    ITYPE seen = 0;
    for (UINT i = 0; i < cnt; ++i) {
        QS_TRY(check_target(tl[i], n, "Pauli operator"));
        if (seen & (1ULL << tl[i])) return set_error(QS_ERR_INVALID_ARGUMENT, "Pauli operator: duplicated qubit");
        seen |= 1ULL << tl[i];
        const ITYPE b = 1ULL << tl[i];
        switch (ids[i]) {
            case 0: break;
            case 1: t->x ^= b; t->pivot = tl[i]; break;
            case 2: t->x ^= b; t->z ^= b; t->nrot++; t->pivot = tl[i]; break;
            case 3: t->z ^= b; break;
            default: return set_error(QS_ERR_INVALID_ARGUMENT, "Pauli id must be 0..3");
        }
    }
    return QS_OK;
}

constexpr int kEvTileBitsDecl = 11;  // tile qubits of the many-terms-per-pass kernel below
template <class T>
int ev_tiled(const PauliTerm* terms, const std::vector<int>& xidx, UINT n, const T* s, ITYPE dim, cudaStream_t st,
    double* values, std::vector<int>* rest, std::vector<int>* zidx);

template <class T>
int ev_batch(const PauliTerm* terms, UINT count, const T* s, ITYPE dim, cudaStream_t st, double* values) {
    std::vector<int> zidx, xidx;
    for (UINT k = 0; k < count; ++k) (terms[k].x == 0 ? zidx : xidx).push_back((int)k);
    const unsigned blocks = reduce_blocks(dim);
    constexpr int kZChunk = 16;
    const size_t part_doubles = (size_t)blocks * std::max<size_t>(kZChunk, 1) + kZChunk + 64;
    void* buf;
    QS_TRY(scratch(st, sizeof(double) * part_doubles + sizeof(ITYPE) * kZChunk + 1024, &buf));
    double* part = (double*)buf;
    ITYPE* dz = (ITYPE*)((char*)buf + sizeof(double) * part_doubles);
    // many terms with a bit flip: evaluate them from shared-memory tiles, several terms per pass; the
    // Z-only terms ride along in the first tiled pass
    UINT n = 0;
    while ((1ULL << n) < dim) ++n;
    if (n >= (UINT)kEvTileBitsDecl && xidx.size() >= 4) {
        std::vector<int> rest;
        QS_TRY(ev_tiled<T>(terms, xidx, n, s, dim, st, values, &rest, &zidx));
        xidx.swap(rest);
        // the tiled passes may have grown (and so moved) this stream's scratch buffer
        QS_TRY(scratch(st, sizeof(double) * part_doubles + sizeof(ITYPE) * kZChunk + 1024, &buf));
        part = (double*)buf;
        dz = (ITYPE*)((char*)buf + sizeof(double) * part_doubles);
    }
    // Z-only terms left: kZChunk per pass.
    for (size_t c0 = 0; c0 < zidx.size(); c0 += kZChunk) {
        const int nz = (int)std::min<size_t>(kZChunk, zidx.size() - c0);
        ITYPE hz[kZChunk];
        for (int w = 0; w < nz; ++w) hz[w] = terms[zidx[c0 + w]].z;
        QS_CUDA_CHECK(cudaMemcpyAsync(dz, hz, sizeof(ITYPE) * nz, cudaMemcpyHostToDevice, st));
        k_ev_z_batch<kZChunk, T><<<blocks, kRThreads, 0, st>>>(s, dim, dz, nz, part);
        QS_TRY(check_launch("k_ev_z_batch"));
        double out[kZChunk];
        QS_TRY(finish_reduce(part, blocks, nz, st, out));
        for (int w = 0; w < nz; ++w) values[zidx[c0 + w]] = out[w];
    }
    const unsigned xblocks = reduce_blocks(dim / 2);
    for (int k : xidx) {
        k_ev_xz<T><<<xblocks, kRThreads, 0, st>>>(s, dim / 2, terms[k], part);
        QS_TRY(check_launch("k_ev_xz"));
        QS_TRY(finish_reduce(part, xblocks, 1, st, &values[k]));
    }
    return QS_OK;
}

// ---------------------------------------------------------------- sampling
// Prefix structure: chunks of kChunk amplitudes; chunk sums (FP64, fixed order), then an inclusive
// scan of the chunk sums by one CTA.  Per shot one warp binary-searches the chunk scan and re-scans
// its chunk serially from the chunk's exclusive prefix, mirroring the reference's serial running
// sum (cppsim/state.hpp:917-922) inside the chunk.
constexpr int kChunk = 2048;

// diag_stride: 0 = state vector (p_i = |a_i|^2); otherwise density matrix with p_i = |rho[i*(dim+1)]|.
__device__ __forceinline__ double prob_at(const double2* s, ITYPE i, ITYPE diag_stride) {
    if (diag_stride == 0) return norm2(s[i]);
    const double2 v = s[i * diag_stride];
    return sqrt(norm2(v));
}
__device__ __forceinline__ double prob_at(const float2* s, ITYPE i, ITYPE) {
    const float2 v = s[i];
    return norm2(make_double2((double)v.x, (double)v.y));
}

template <class T>
__global__ void __launch_bounds__(256) k_chunk_sums(const T* __restrict__ s, ITYPE dim, ITYPE diag_stride,
    double* __restrict__ sums) {
    __shared__ double sm[32];
    const ITYPE c0 = (ITYPE)blockIdx.x * kChunk;
    double acc = 0.;
    for (int j = threadIdx.x; j < kChunk; j += 256)
        if (c0 + j < dim) acc += prob_at(s, c0 + j, diag_stride);
    acc = block_sum(acc, sm);
    if (threadIdx.x == 0) sums[blockIdx.x] = acc;
}

// Inclusive scan of n values by one CTA of 1024 threads: thread t owns a contiguous range.
__global__ void __launch_bounds__(1024) k_scan_sums(const double* __restrict__ sums, ITYPE n, double* __restrict__ incl) {
    __shared__ double part[1024];
    const ITYPE per = (n + 1023) / 1024;
    const ITYPE lo = (ITYPE)threadIdx.x * per, hi = min(n, lo + per);
    double acc = 0.;
    for (ITYPE i = lo; i < hi; ++i) acc += sums[i];
    part[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double run = 0.;
        for (int t = 0; t < 1024; ++t) {
            const double v = part[t];
            part[t] = run;  // exclusive offset of thread t
            run += v;
        }
    }
    __syncthreads();
    double run = part[threadIdx.x];
    for (ITYPE i = lo; i < hi; ++i) {
        run += sums[i];
        incl[i] = run;
    }
}

// One warp per shot.  With `near` set, near[shot] = 1 when the draw lies within `eps` of one of the two
// cumulative sums that bracket it (prefix before the sampled index, prefix through it): a draw whose
// index could differ under another summation order of the same probabilities.
template <class T>
__global__ void k_sample(const T* __restrict__ s, ITYPE dim, ITYPE diag_stride, const double* __restrict__ incl,
    ITYPE nchunks, const double* __restrict__ uniforms, UINT count, ITYPE* __restrict__ out, double eps = 0.,
    unsigned char* __restrict__ near = nullptr) {
    const int lane = threadIdx.x & 31;
    const UINT shot = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (shot >= count) return;
    const double r = uniforms[shot];
    if (!(r > 0.)) {  // lower_bound hits stacked_prob[0] = 0 -> index -1
        if (lane == 0) {
            out[shot] = ~0ULL;
            if (near) near[shot] = r >= -eps;
        }
        return;
    }
    if (r > incl[nchunks - 1]) {  // past the total -> index dim
        if (lane == 0) {
            out[shot] = dim;
            if (near) near[shot] = r - incl[nchunks - 1] <= eps;
        }
        return;
    }
    // first chunk c with incl[c] >= r
    ITYPE lo = 0, hi = nchunks - 1;
    while (lo < hi) {
        const ITYPE mid = lo + (hi - lo) / 2;
        if (incl[mid] < r) lo = mid + 1;
        else hi = mid;
    }
    const ITYPE c = lo;
    const double base = c ? incl[c - 1] : 0.;
    // lane-local sums of 64 consecutive probabilities, exclusive warp scan in lane order
    const ITYPE c0 = c * kChunk + (ITYPE)lane * (kChunk / 32);
    double lsum = 0.;
    for (int j = 0; j < kChunk / 32; ++j)
        if (c0 + j < dim) lsum += prob_at(s, c0 + j, diag_stride);
    double excl = 0.;
    for (int l = 0; l < 32; ++l) {
        const double v = __shfl_sync(0xffffffffu, lsum, l);
        if (l < lane) excl += v;
    }
    const double start = base + excl;
    const double end = start + lsum;
    // the first lane whose running end reaches r owns the answer
    const unsigned ball = __ballot_sync(0xffffffffu, end >= r);
    const int owner = ball ? __ffs(ball) - 1 : 31;
    if (lane == owner) {
        double run = start, prev = start;
        ITYPE idx = c0 + kChunk / 32 - 1;
        for (int j = 0; j < kChunk / 32; ++j) {
            if (c0 + j >= dim) break;
            prev = run;
            run += prob_at(s, c0 + j, diag_stride);
            if (run >= r) {
                idx = c0 + j;
                break;
            }
        }
        out[shot] = idx < dim ? idx : dim - 1;
        if (near) near[shot] = (r - prev <= eps) || (run - r <= eps);
    }
}

// near_host (may be null): per draw, 1 when it lies within eps of a bracketing cumulative sum.
template <class T>
int sample_with_uniforms_t(const T* s, ITYPE dim, ITYPE diag_stride, const double* uniforms, UINT count,
    ITYPE* out, cudaStream_t st, double eps = 0., unsigned char* near_host = nullptr) {
    if (count == 0) return QS_OK;
    const ITYPE nchunks = (dim + kChunk - 1) / kChunk;
    const size_t bytes = sizeof(double) * (2 * nchunks + count) + sizeof(ITYPE) * count + count + 1024;
    void* buf;
    QS_TRY(scratch(st, bytes, &buf));
    double* sums = (double*)buf;
    double* incl = sums + nchunks;
    double* du = incl + nchunks;
    ITYPE* dout = (ITYPE*)(du + count);
    unsigned char* dnear = near_host ? (unsigned char*)(dout + count) : nullptr;
    QS_CUDA_CHECK(cudaMemcpyAsync(du, uniforms, sizeof(double) * count, cudaMemcpyHostToDevice, st));
    k_chunk_sums<T><<<(unsigned)nchunks, 256, 0, st>>>(s, dim, diag_stride, sums);
    QS_TRY(check_launch("k_chunk_sums"));
    k_scan_sums<<<1, 1024, 0, st>>>(sums, nchunks, incl);
    QS_TRY(check_launch("k_scan_sums"));
    const unsigned threads = 256;
    const unsigned blocks = (unsigned)(((ITYPE)count * 32 + threads - 1) / threads);
    k_sample<T><<<blocks, threads, 0, st>>>(s, dim, diag_stride, incl, nchunks, du, count, dout, eps, dnear);
    QS_TRY(check_launch("k_sample"));
    QS_CUDA_CHECK(cudaMemcpyAsync(out, dout, sizeof(ITYPE) * count, cudaMemcpyDeviceToHost, st));
    if (dnear) QS_CUDA_CHECK(cudaMemcpyAsync(near_host, dnear, count, cudaMemcpyDeviceToHost, st));
    QS_CUDA_CHECK(cudaStreamSynchronize(st));
    return QS_OK;
}
int sample_with_uniforms(const double2* s, ITYPE dim, ITYPE diag_stride, const double* uniforms, UINT count,
    ITYPE* out, cudaStream_t st) {
    return sample_with_uniforms_t<double2>(s, dim, diag_stride, uniforms, count, out, st);
}

// ---------------------------------------------------------------- sampling without allocation
// Scratch for qs_state_sampling_with_uniforms_noalloc, reserved statically in this module so that
// the call never allocates: chunk sums | inclusive scan | uniforms | sampled indices.  Every GPU
// that loads the library holds it (2.25 MiB) until the process exits.  Nothing in it has to start
// at zero: each element a call reads was written earlier in the same call.  Calls share it, so
// calls that overlap on the GPU (other streams, other host threads) race.
constexpr ITYPE kNoAllocMaxDim = 1ULL << 28;   // states of up to 28 qubits
constexpr UINT kNoAllocMaxShots = 16384;
constexpr size_t kNoAllocChunks = kNoAllocMaxDim / kChunk;
constexpr size_t kNoAllocDoubles = 2 * kNoAllocChunks + 2 * (size_t)kNoAllocMaxShots;
static __device__ __align__(256) double g_noalloc_sampling_scratch[kNoAllocDoubles];

static std::mutex g_noalloc_mu;
static double* g_noalloc_ptr[64] = {nullptr};

// Device address of the static scratch on the current device.  In host code the array's name is
// only a host-side stand-in, so the address is looked up once per device (with that device
// current) and cached.
static int noalloc_scratch(double** out) {
    int dev = 0;
    QS_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(QS_ERR_NOT_SUPPORTED, "device ordinal beyond 63");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_sampling_scratch);
        if (e != cudaSuccess) return check_cuda(e, "cudaGetSymbolAddress(g_noalloc_sampling_scratch)");
        g_noalloc_ptr[dev] = (double*)p;
    }
    *out = g_noalloc_ptr[dev];
    return QS_OK;
}

// Reference RNG (cppsim/utility.hpp:54-80): mt19937_64 seeded with the seed, uniform_real_distribution(0, 1).
void reference_uniforms(UINT seed, UINT count, std::vector<double>* u) {
    std::mt19937_64 mt;
    mt.seed(seed);
    std::uniform_real_distribution<double> dist(0, 1);
    u->resize(count);
    for (UINT c = 0; c < count; ++c) (*u)[c] = dist(mt);
}

}  // namespace qs

using namespace qs;

extern "C" {

QS_API int qs_measurement_distribution_entropy(const void* state, QS_ITYPE dim, void* stream, double* out) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (!out) return set_error(QS_ERR_INVALID_ARGUMENT, "null output pointer");
    return entropy<false>((const double2*)state, dim, 1, (cudaStream_t)stream, out);
}
QS_API int qs_dm_measurement_distribution_entropy(const void* rho, QS_ITYPE dim, void* stream, double* out) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (n > 20) return set_error(QS_ERR_NOT_SUPPORTED, "density matrix: at most 20 qubits");
    if (!out) return set_error(QS_ERR_INVALID_ARGUMENT, "null output pointer");
    return entropy<true>((const double2*)rho, dim, dim + 1, (cudaStream_t)stream, out);
}
QS_API int qs_dm_M0_prob(QS_UINT t, const void* rho, QS_ITYPE dim, void* stream, double* out) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    QS_TRY(check_target(t, n, "dm_M0_prob"));
    if (!out) return set_error(QS_ERR_INVALID_ARGUMENT, "null output pointer");
    return dm_diag_sum((const double2*)rho, dim, 1ULL << t, 0, (cudaStream_t)stream, out);
}
QS_API int qs_dm_M1_prob(QS_UINT t, const void* rho, QS_ITYPE dim, void* stream, double* out) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    QS_TRY(check_target(t, n, "dm_M1_prob"));
    if (!out) return set_error(QS_ERR_INVALID_ARGUMENT, "null output pointer");
    return dm_diag_sum((const double2*)rho, dim, 1ULL << t, 1ULL << t, (cudaStream_t)stream, out);
}
QS_API int qs_dm_marginal_prob(const QS_UINT* targets, const QS_UINT* values, QS_UINT count, const void* rho,
    QS_ITYPE dim, void* stream, double* out) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    QS_TRY(check_distinct(targets, count, n, "dm_marginal_prob"));
    if (!out || (count && !values)) return set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    ITYPE mask = 0, value = 0;
    for (UINT i = 0; i < count; ++i) {
        mask |= 1ULL << targets[i];
        if (values[i] > 1) return set_error(QS_ERR_INVALID_ARGUMENT, "dm_marginal_prob: measured value must be 0 or 1");
        if (values[i]) value |= 1ULL << targets[i];
    }
    return dm_diag_sum((const double2*)rho, dim, mask, value, (cudaStream_t)stream, out);
}
QS_API int qs_state_norm_squared(const void* state, QS_ITYPE dim, void* stream, double* out) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    return prob_sum((const double2*)state, dim, 0, 0, (cudaStream_t)stream, out);
}
QS_API int qs_M0_prob(QS_UINT t, const void* state, QS_ITYPE dim, void* stream, double* out) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    QS_TRY(check_target(t, n, "M0_prob"));
    return prob_sum((const double2*)state, dim, 1ULL << t, 0, (cudaStream_t)stream, out);
}
QS_API int qs_M1_prob(QS_UINT t, const void* state, QS_ITYPE dim, void* stream, double* out) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    QS_TRY(check_target(t, n, "M1_prob"));
    return prob_sum((const double2*)state, dim, 1ULL << t, 1ULL << t, (cudaStream_t)stream, out);
}
QS_API int qs_marginal_prob(const QS_UINT* tl, const QS_UINT* vals, QS_UINT cnt, const void* state,
    QS_ITYPE dim, void* stream, double* out) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    QS_TRY(check_distinct(tl, cnt, n, "marginal_prob"));
    ITYPE mask = 0, value = 0;
    for (UINT i = 0; i < cnt; ++i) {
        if (vals[i] > 1) return set_error(QS_ERR_INVALID_ARGUMENT, "marginal_prob: value must be 0 or 1");
        mask |= 1ULL << tl[i];
        if (vals[i]) value |= 1ULL << tl[i];
    }
    return prob_sum((const double2*)state, dim, mask, value, (cudaStream_t)stream, out);
}

QS_API int qs_state_inner_product(const void* bra, const void* ket, QS_ITYPE dim, void* stream, double out[2]) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned blocks = reduce_blocks(dim);
    void* buf;
    QS_TRY(scratch(st, sizeof(double) * (2 * blocks + 2), &buf));
    k_inner<<<blocks, kRThreads, 0, st>>>((const double2*)bra, (const double2*)ket, dim, (double*)buf);
    QS_TRY(check_launch("k_inner"));
    return finish_reduce((double*)buf, blocks, 2, st, out);
}

QS_API int qs_expectation_value_multi_qubit_Pauli_operator_partial_list(const QS_UINT* tl, const QS_UINT* ids,
    QS_UINT cnt, const void* state, QS_ITYPE dim, void* stream, double* out) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    PauliTerm t;
    QS_TRY(pauli_term(tl, ids, cnt, n, &t));
    return ev_batch<double2>(&t, 1, (const double2*)state, dim, (cudaStream_t)stream, out);
}

QS_API int qs_expectation_value_pauli_batch(const QS_ITYPE* x_masks, const QS_ITYPE* z_masks, const QS_UINT* y_counts,
    QS_UINT term_count, const void* state, QS_ITYPE dim, void* stream, double* values) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    std::vector<PauliTerm> terms(term_count);
    for (UINT k = 0; k < term_count; ++k) {
        if ((x_masks[k] | z_masks[k]) >> n)
            return set_error(QS_ERR_INVALID_ARGUMENT, "expectation_value_pauli_batch: mask beyond qubit count");
        terms[k].x = x_masks[k];
        terms[k].z = z_masks[k];
        terms[k].nrot = y_counts[k];
        terms[k].pivot = x_masks[k] ? (UINT)(63 - __builtin_clzll(x_masks[k])) : 0;
    }
    return ev_batch<double2>(terms.data(), term_count, (const double2*)state, dim, (cudaStream_t)stream, values);
}

QS_API int qs_transition_amplitude_multi_qubit_Pauli_operator_partial_list(const QS_UINT* tl, const QS_UINT* ids,
    QS_UINT cnt, const void* bra, const void* ket, QS_ITYPE dim, void* stream, double out[2]) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    PauliTerm t;
    QS_TRY(pauli_term(tl, ids, cnt, n, &t));
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned blocks = reduce_blocks(dim);
    void* buf;
    QS_TRY(scratch(st, sizeof(double) * (2 * blocks + 2), &buf));
    k_transition<<<blocks, kRThreads, 0, st>>>((const double2*)bra, (const double2*)ket, dim, t, (double*)buf);
    QS_TRY(check_launch("k_transition"));
    return finish_reduce((double*)buf, blocks, 2, st, out);
}

QS_API int qs_expectation_value_single_qubit_Pauli_operator(QS_UINT t, QS_UINT id, const void* state, QS_ITYPE dim,
    void* stream, double* out) {
    return qs_expectation_value_multi_qubit_Pauli_operator_partial_list(&t, &id, 1, state, dim, stream, out);
}

// Whole-list forms (stat_ops_expectation_value.cpp, stat_ops_transition_amplitude.cpp): id j on qubit j.
static int whole_list(QS_UINT count, QS_ITYPE dim, const char* what, std::vector<UINT>* tl) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (count > n) return set_error(QS_ERR_INVALID_ARGUMENT, std::string(what) + ": more Pauli ids than qubits");
    tl->resize(count);
    for (UINT j = 0; j < count; ++j) (*tl)[j] = j;
    return QS_OK;
}
QS_API int qs_expectation_value_multi_qubit_Pauli_operator_whole_list(const QS_UINT* ids, QS_UINT count,
    const void* state, QS_ITYPE dim, void* stream, double* out) {
    std::vector<UINT> tl;
    QS_TRY(whole_list(count, dim, "expectation_value_multi_qubit_Pauli_operator_whole_list", &tl));
    return qs_expectation_value_multi_qubit_Pauli_operator_partial_list(tl.data(), ids, count, state, dim, stream, out);
}
QS_API int qs_transition_amplitude_multi_qubit_Pauli_operator_whole_list(const QS_UINT* ids, QS_UINT count,
    const void* bra, const void* ket, QS_ITYPE dim, void* stream, double out[2]) {
    std::vector<UINT> tl;
    QS_TRY(whole_list(count, dim, "transition_amplitude_multi_qubit_Pauli_operator_whole_list", &tl));
    return qs_transition_amplitude_multi_qubit_Pauli_operator_partial_list(tl.data(), ids, count, bra, ket, dim,
        stream, out);
}

QS_API int qs_state_sampling_with_uniforms(const void* state, QS_ITYPE dim, const double* uniforms,
    QS_UINT count, QS_ITYPE* out, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    return sample_with_uniforms((const double2*)state, dim, 0, uniforms, count, out, (cudaStream_t)stream);
}

// qs_state_sampling_with_uniforms that also reports, per draw, whether it lies within `eps` of a
// cumulative boundary (near_boundary[i] in {0, 1}, may be NULL) and how many do (near_count, may be NULL).
QS_API int qs_state_sampling_with_uniforms_flagged(const void* state, QS_ITYPE dim, const double* uniforms,
    QS_UINT count, double eps, QS_ITYPE* out, unsigned char* near_boundary, QS_UINT* near_count, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (!(eps >= 0.)) return set_error(QS_ERR_INVALID_ARGUMENT, "sampling: eps must be >= 0");
    std::vector<unsigned char> flags(count);
    QS_TRY(sample_with_uniforms_t<double2>((const double2*)state, dim, 0, uniforms, count, out, (cudaStream_t)stream,
        eps, flags.data()));
    UINT c = 0;
    for (UINT i = 0; i < count; ++i) c += flags[i] ? 1 : 0;
    if (near_boundary && count) memcpy(near_boundary, flags.data(), count);
    if (near_count) *near_count = c;
    return QS_OK;
}

QS_API int qs_state_sampling(const void* state, QS_ITYPE dim, QS_UINT count, QS_UINT seed, QS_ITYPE* out,
    void* stream) {
    std::vector<double> u;
    reference_uniforms(seed, count, &u);
    return qs_state_sampling_with_uniforms(state, dim, u.data(), count, out, stream);
}

// Same result as qs_state_sampling_with_uniforms (same kernels, same order of summation), with all
// scratch in g_noalloc_sampling_scratch: no cudaMalloc, cudaFree or allocating library call.  The
// first call on a device looks up the array's device address; make that first call before any
// stream capture.
QS_API int qs_state_sampling_with_uniforms_noalloc(const void* state, QS_ITYPE dim, const double* uniforms,
    QS_UINT count, QS_ITYPE* out, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (dim > kNoAllocMaxDim)
        return set_error(QS_ERR_NOT_SUPPORTED,
            "state_sampling_with_uniforms_noalloc: state larger than 2^28 amplitudes (static scratch limit)");
    if (count > kNoAllocMaxShots)
        return set_error(QS_ERR_NOT_SUPPORTED,
            "state_sampling_with_uniforms_noalloc: more than 16384 shots (static scratch limit)");
    if (count == 0) return QS_OK;
    if (!state || !uniforms || !out) return set_error(QS_ERR_INVALID_ARGUMENT, "null pointer argument");
    double* buf = nullptr;
    QS_TRY(noalloc_scratch(&buf));
    cudaStream_t st = (cudaStream_t)stream;
    const ITYPE nchunks = (dim + kChunk - 1) / kChunk;
    double* sums = buf;
    double* incl = buf + kNoAllocChunks;
    double* du = incl + kNoAllocChunks;
    ITYPE* dout = (ITYPE*)(du + kNoAllocMaxShots);
    QS_CUDA_CHECK(cudaMemcpyAsync(du, uniforms, sizeof(double) * count, cudaMemcpyHostToDevice, st));
    k_chunk_sums<double2><<<(unsigned)nchunks, 256, 0, st>>>((const double2*)state, dim, 0, sums);
    QS_TRY(check_launch("k_chunk_sums"));
    k_scan_sums<<<1, 1024, 0, st>>>(sums, nchunks, incl);
    QS_TRY(check_launch("k_scan_sums"));
    const unsigned threads = 256;
    const unsigned blocks = (unsigned)(((ITYPE)count * 32 + threads - 1) / threads);
    k_sample<double2><<<blocks, threads, 0, st>>>((const double2*)state, dim, 0, incl, nchunks, du, count, dout);
    QS_TRY(check_launch("k_sample"));
    QS_CUDA_CHECK(cudaMemcpyAsync(out, dout, sizeof(ITYPE) * count, cudaMemcpyDeviceToHost, st));
    QS_CUDA_CHECK(cudaStreamSynchronize(st));
    return QS_OK;
}

// ---- complex64 states: FP64 accumulation over single-precision amplitudes ----
QS_API int qs_state_norm_squared_c64(const void* state, QS_ITYPE dim, void* stream, double* out) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    return prob_sum_t<float2>((const float2*)state, dim, 0, 0, (cudaStream_t)stream, out);
}
QS_API int qs_state_inner_product_c128_c64(const void* bra_c128, const void* ket_c64, QS_ITYPE dim, void* stream,
    double out[2]) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned blocks = reduce_blocks(dim);
    void* buf;
    QS_TRY(scratch(st, sizeof(double) * (2 * blocks + 2), &buf));
    k_inner_mixed<<<blocks, kRThreads, 0, st>>>((const double2*)bra_c128, (const float2*)ket_c64, dim, (double*)buf);
    QS_TRY(check_launch("k_inner_mixed"));
    return finish_reduce((double*)buf, blocks, 2, st, out);
}
QS_API int qs_expectation_value_pauli_batch_c64(const QS_ITYPE* x_masks, const QS_ITYPE* z_masks,
    const QS_UINT* y_counts, QS_UINT term_count, const void* state, QS_ITYPE dim, void* stream, double* values) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    std::vector<PauliTerm> terms(term_count);
    for (UINT k = 0; k < term_count; ++k) {
        if ((x_masks[k] | z_masks[k]) >> n)
            return set_error(QS_ERR_INVALID_ARGUMENT, "expectation_value_pauli_batch_c64: mask beyond qubit count");
        terms[k].x = x_masks[k];
        terms[k].z = z_masks[k];
        terms[k].nrot = y_counts[k];
        terms[k].pivot = x_masks[k] ? (UINT)(63 - __builtin_clzll(x_masks[k])) : 0;
    }
    return ev_batch<float2>(terms.data(), term_count, (const float2*)state, dim, (cudaStream_t)stream, values);
}
QS_API int qs_state_sampling_with_uniforms_c64(const void* state, QS_ITYPE dim, const double* uniforms,
    QS_UINT count, QS_ITYPE* out, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    return sample_with_uniforms_t<float2>((const float2*)state, dim, 0, uniforms, count, out, (cudaStream_t)stream);
}

QS_API int qs_reference_uniforms(QS_UINT seed, QS_UINT count, double* out) {
    if (!out && count) return set_error(QS_ERR_INVALID_ARGUMENT, "null output pointer");
    std::vector<double> u;
    reference_uniforms(seed, count, &u);
    for (UINT c = 0; c < count; ++c) out[c] = u[c];
    return QS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- batched expectation values
// <P_k> for the terms of MANY states in one persistent launch.  A job is either up to 16 Z-only terms
// of one state (one pass over its amplitudes) or one term with a bit flip (one pass over its pairs);
// jobs are cut into chunks of kEvChunk items, one CTA per chunk at a time; every chunk writes FP64
// partial sums, which a second kernel folds per job in chunk order (deterministic).
namespace qs {

constexpr ITYPE kEvChunk = 1 << 14;
constexpr int kEvZ = 16;

struct EvJob {
    const void* s;
    int c64;       // 1: complex64 amplitudes, 0: complex128
    ITYPE items;   // amplitudes (Z job) or pairs (X job)
    ITYPE prefix;  // first work item (chunk) of this job
    ITYPE x, z;
    UINT nrot, pivot;
    int kind;      // 0: Z batch, 1: single term with bit flip
    int nz;        // Z batch: number of terms
    UINT zoff;     // Z batch: first index into zmasks / zout
    UINT out;      // X job: output index
};

__global__ void __launch_bounds__(256) k_batch_ev(const EvJob* __restrict__ jobs, int njobs, ITYPE total,
    const ITYPE* __restrict__ zmasks, double* __restrict__ partials) {
    __shared__ double sm[32];
    __shared__ int s_job;
    for (ITYPE item = blockIdx.x; item < total; item += gridDim.x) {
        if (threadIdx.x == 0) {
            int lo = 0, hi = njobs - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) / 2;
                if (jobs[mid].prefix <= item) lo = mid;
                else hi = mid - 1;
            }
            s_job = lo;
        }
        __syncthreads();
        const EvJob& J = jobs[s_job];
        const ITYPE c0 = (item - J.prefix) * kEvChunk;
        const ITYPE c1 = min(J.items, c0 + kEvChunk);
        if (J.kind == 1) {
            double acc = 0.;
            for (ITYPE p = c0 + threadIdx.x; p < c1; p += blockDim.x) {
                const ITYPE b0 = insert0(p, J.pivot), b1 = b0 ^ J.x;
                const double2 a0 = J.c64 ? amp((const float2*)J.s + b0) : amp((const double2*)J.s + b0);
                const double2 a1 = J.c64 ? amp((const float2*)J.s + b1) : amp((const double2*)J.s + b1);
                const double2 v = cmul(a0, cconj(a1));
                const UINT r = J.nrot + 2u * (UINT)(__popcll(b0 & J.z) & 1);
                acc += 2.0 * phase_re_part(v, r);
            }
            acc = block_sum(acc, sm);
            if (threadIdx.x == 0) partials[item * kEvZ] = acc;
        } else {
            double acc[kEvZ];
            ITYPE zs[kEvZ];
#pragma unroll
            for (int w = 0; w < kEvZ; ++w) {
                acc[w] = 0.;
                zs[w] = w < J.nz ? zmasks[J.zoff + w] : 0;
            }
            for (ITYPE i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
                const double pr = norm2(J.c64 ? amp((const float2*)J.s + i) : amp((const double2*)J.s + i));
#pragma unroll
                for (int w = 0; w < kEvZ; ++w)
                    if (w < J.nz) acc[w] += (__popcll(i & zs[w]) & 1) ? -pr : pr;
            }
#pragma unroll
            for (int w = 0; w < kEvZ; ++w) {
                if (w < J.nz) {  // uniform over the CTA
                    const double v = block_sum(acc[w], sm);
                    if (threadIdx.x == 0) partials[item * kEvZ + w] = v;
                }
            }
        }
        __syncthreads();
    }
}

__global__ void k_batch_ev_fold(const EvJob* __restrict__ jobs, const double* __restrict__ partials,
    const UINT* __restrict__ zout, double* __restrict__ values) {
    __shared__ double sm[32];
    const EvJob& J = jobs[blockIdx.x];
    const ITYPE nchunks = (J.items + kEvChunk - 1) / kEvChunk;
    const int width = J.kind == 1 ? 1 : J.nz;
    for (int w = 0; w < width; ++w) {
        double v = 0.;
        for (ITYPE c = threadIdx.x; c < nchunks; c += blockDim.x) v += partials[(J.prefix + c) * kEvZ + w];
        v = block_sum(v, sm);
        if (threadIdx.x == 0) values[J.kind == 1 ? J.out : zout[J.zoff + w]] = v;
    }
}

}  // namespace qs

namespace qs {
static int batch_ev_impl(void* const* states, const QS_UINT* qubit_counts, QS_UINT count, const QS_UINT* term_offsets,
    const QS_ITYPE* x_masks, const QS_ITYPE* z_masks, const QS_UINT* y_counts, double* values, int c64,
    cudaStream_t st, bool skip_large = false);
template <class T>
int ev_weighted(const PauliTerm* terms, const double2* coefs, UINT count, const T* s, ITYPE dim, cudaStream_t st,
    double out[2], bool allow_generate);
template <class T>
int ev_weighted_many(const std::vector<const T*>& s, const std::vector<UINT>& nq,
    const std::vector<std::vector<PauliTerm>>& terms, const std::vector<const double2*>& coefs, cudaStream_t st,
    std::vector<double2>* out);
}
extern "C" QS_API int qs_batch_expectation_values(void* const* states, const QS_UINT* qubit_counts, QS_UINT count,
    const QS_UINT* term_offsets, const QS_ITYPE* x_masks, const QS_ITYPE* z_masks, const QS_UINT* y_counts,
    double* values, void* stream) {
    return qs::batch_ev_impl(states, qubit_counts, count, term_offsets, x_masks, z_masks, y_counts, values, 0,
        (cudaStream_t)stream);
}
extern "C" QS_API int qs_batch_expectation_values_c64(void* const* states, const QS_UINT* qubit_counts, QS_UINT count,
    const QS_UINT* term_offsets, const QS_ITYPE* x_masks, const QS_ITYPE* z_masks, const QS_UINT* y_counts,
    double* values, void* stream) {
    return qs::batch_ev_impl(states, qubit_counts, count, term_offsets, x_masks, z_masks, y_counts, values, 1,
        (cudaStream_t)stream);
}
namespace qs {
constexpr UINT kBatchEvSingleQubits = 18;  // states at least this large are evaluated on their own

// `skip_large`: leave the terms of states of >= kBatchEvSingleQubits qubits to the caller.
static int batch_ev_impl(void* const* states, const QS_UINT* qubit_counts, QS_UINT count, const QS_UINT* term_offsets,
    const QS_ITYPE* x_masks, const QS_ITYPE* z_masks, const QS_UINT* y_counts, double* values, int c64,
    cudaStream_t st, bool skip_large) {
    if (!states || !qubit_counts || !term_offsets || !values) return set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    std::vector<EvJob> jobs;
    std::vector<ITYPE> zm;
    std::vector<UINT> zout;
    ITYPE total = 0;
    const UINT nterms = term_offsets[count];
    for (UINT i = 0; i < count; ++i) {
        const UINT n = qubit_counts[i];
        if (n < 1 || n > 40) return set_error(QS_ERR_INVALID_ARGUMENT, "batch expectation: bad qubit count");
        const ITYPE dim = 1ULL << n;
        if (n >= kBatchEvSingleQubits) {
            if (skip_large) continue;
            // a large state: its own passes (Z-only strings 16 per pass, bit-flip strings from
            // span tiles) cost far fewer state reads than one job per bit-flip string
            const UINT k0 = term_offsets[i], nk = term_offsets[i + 1] - k0;
            std::vector<PauliTerm> pt(nk);
            for (UINT j = 0; j < nk; ++j) {
                const UINT k = k0 + j;
                if ((x_masks[k] | z_masks[k]) >> n)
                    return set_error(QS_ERR_INVALID_ARGUMENT, "batch expectation: mask beyond qubit count");
                pt[j].x = x_masks[k];
                pt[j].z = z_masks[k];
                pt[j].nrot = y_counts[k];
                pt[j].pivot = x_masks[k] ? (UINT)(63 - __builtin_clzll(x_masks[k])) : 0u;
            }
            if (nk) {
                if (c64) QS_TRY(ev_batch<float2>(pt.data(), nk, (const float2*)states[i], dim, st, values + k0));
                else QS_TRY(ev_batch<double2>(pt.data(), nk, (const double2*)states[i], dim, st, values + k0));
            }
            continue;
        }
        std::vector<UINT> zlist;
        for (UINT k = term_offsets[i]; k < term_offsets[i + 1]; ++k) {
            if ((x_masks[k] | z_masks[k]) >> n)
                return set_error(QS_ERR_INVALID_ARGUMENT, "batch expectation: mask beyond qubit count");
            if (x_masks[k] == 0) {
                zlist.push_back(k);
                continue;
            }
            EvJob J{};
            J.s = states[i];
            J.c64 = c64;
            J.items = dim / 2;
            J.prefix = total;
            J.x = x_masks[k];
            J.z = z_masks[k];
            J.nrot = y_counts[k];
            J.pivot = (UINT)(63 - __builtin_clzll(x_masks[k]));
            J.kind = 1;
            J.out = k;
            total += (J.items + kEvChunk - 1) / kEvChunk;
            jobs.push_back(J);
        }
        for (size_t z0 = 0; z0 < zlist.size(); z0 += kEvZ) {
            EvJob J{};
            J.s = states[i];
            J.c64 = c64;
            J.items = dim;
            J.prefix = total;
            J.kind = 0;
            J.nz = (int)std::min<size_t>(kEvZ, zlist.size() - z0);
            J.zoff = (UINT)zm.size();
            for (int w = 0; w < J.nz; ++w) {
                zm.push_back(z_masks[zlist[z0 + w]]);
                zout.push_back(zlist[z0 + w]);
            }
            total += (J.items + kEvChunk - 1) / kEvChunk;
            jobs.push_back(J);
        }
    }
    if (jobs.empty()) return QS_OK;
    const size_t bj = sizeof(EvJob) * jobs.size(), bz = sizeof(ITYPE) * (zm.size() + 1),
                 bo = sizeof(UINT) * (zout.size() + 1), bp = sizeof(double) * kEvZ * total,
                 bv = sizeof(double) * nterms;
    auto up = [](size_t b) { return (b + 255) / 256 * 256; };
    void* buf;
    QS_TRY(scratch(st, up(bj) + up(bz) + up(bo) + up(bp) + up(bv), &buf));
    char* p = (char*)buf;
    EvJob* dj = (EvJob*)p;
    ITYPE* dz = (ITYPE*)(p + up(bj));
    UINT* dzo = (UINT*)(p + up(bj) + up(bz));
    double* dpart = (double*)(p + up(bj) + up(bz) + up(bo));
    double* dval = (double*)(p + up(bj) + up(bz) + up(bo) + up(bp));
    QS_CUDA_CHECK(cudaMemcpyAsync(dj, jobs.data(), bj, cudaMemcpyHostToDevice, st));
    if (!zm.empty()) {
        QS_CUDA_CHECK(cudaMemcpyAsync(dz, zm.data(), sizeof(ITYPE) * zm.size(), cudaMemcpyHostToDevice, st));
        QS_CUDA_CHECK(cudaMemcpyAsync(dzo, zout.data(), sizeof(UINT) * zout.size(), cudaMemcpyHostToDevice, st));
    }
    QS_CUDA_CHECK(cudaMemsetAsync(dval, 0, bv, st));
    const unsigned grid = (unsigned)std::min<ITYPE>(total, (ITYPE)sm_count() * 8);
    k_batch_ev<<<grid, 256, 0, st>>>(dj, (int)jobs.size(), total, dz, dpart);
    QS_TRY(check_launch("k_batch_ev"));
    k_batch_ev_fold<<<(unsigned)jobs.size(), 256, 0, st>>>(dj, dpart, dzo, dval);
    QS_TRY(check_launch("k_batch_ev_fold"));
    // only the entries of the states evaluated here (large states' values are already in `values`)
    std::vector<double> hv(nterms);
    QS_CUDA_CHECK(cudaMemcpyAsync(hv.data(), dval, bv, cudaMemcpyDeviceToHost, st));
    QS_CUDA_CHECK(cudaStreamSynchronize(st));
    for (UINT i = 0; i < count; ++i)
        if (qubit_counts[i] < kBatchEvSingleQubits)
            for (UINT k = term_offsets[i]; k < term_offsets[i + 1]; ++k) values[k] = hv[k];
    return QS_OK;
}
}  // namespace qs

// sum_k c_k <P_k> per state for many states: the small states' terms in the one shared launch above
// (weighted on the host), each large state through the weighted passes (no per-term values).
extern "C" QS_API int qs_batch_expectation_weighted(void* const* states, const QS_UINT* qubit_counts, QS_UINT count,
    const QS_UINT* term_offsets, const QS_ITYPE* x_masks, const QS_ITYPE* z_masks, const QS_UINT* y_counts,
    const double* coefs, int c64, double* energies, void* stream) {
    if (!states || !qubit_counts || !term_offsets || !coefs || !energies)
        return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    for (QS_UINT i = 0; i < count; ++i)
        if (qubit_counts[i] < 1 || qubit_counts[i] > 40)
            return qs::set_error(QS_ERR_INVALID_ARGUMENT, "batch expectation: bad qubit count");
    const QS_UINT nterms = term_offsets[count];
    std::vector<double> values(nterms, 0.);
    QS_TRY(qs::batch_ev_impl(states, qubit_counts, count, term_offsets, x_masks, z_masks, y_counts, values.data(), c64,
        st, true));
    // the large states: every plan, pass and fold in one go
    std::vector<QS_UINT> large;
    std::vector<std::vector<qs::PauliTerm>> lterms;
    std::vector<UINT> lnq;
    std::vector<const double2*> lcoef;
    for (QS_UINT i = 0; i < count; ++i) {
        if (qubit_counts[i] < qs::kBatchEvSingleQubits) continue;
        const QS_UINT k0 = term_offsets[i], k1 = term_offsets[i + 1];
        std::vector<qs::PauliTerm> pt(k1 - k0);
        for (QS_UINT k = k0; k < k1; ++k) {
            if ((x_masks[k] | z_masks[k]) >> qubit_counts[i])
                return qs::set_error(QS_ERR_INVALID_ARGUMENT, "batch expectation: mask beyond qubit count");
            pt[k - k0].x = x_masks[k];
            pt[k - k0].z = z_masks[k];
            pt[k - k0].nrot = y_counts[k];
            pt[k - k0].pivot = x_masks[k] ? (QS_UINT)(63 - __builtin_clzll(x_masks[k])) : 0u;
        }
        large.push_back(i);
        lterms.push_back(std::move(pt));
        lnq.push_back(qubit_counts[i]);
        lcoef.push_back((const double2*)coefs + k0);
    }
    std::vector<double2> le;
    if (c64) {
        std::vector<const float2*> ls;
        for (QS_UINT i : large) ls.push_back((const float2*)states[i]);
        QS_TRY(qs::ev_weighted_many<float2>(ls, lnq, lterms, lcoef, st, &le));
    } else {
        std::vector<const double2*> ls;
        for (QS_UINT i : large) ls.push_back((const double2*)states[i]);
        QS_TRY(qs::ev_weighted_many<double2>(ls, lnq, lterms, lcoef, st, &le));
    }
    for (QS_UINT i = 0; i < count; ++i) {
        if (qubit_counts[i] >= qs::kBatchEvSingleQubits) continue;
        double e[2] = {0., 0.};
        for (QS_UINT k = term_offsets[i]; k < term_offsets[i + 1]; ++k) {
            e[0] += coefs[2 * k] * values[k];
            e[1] += coefs[2 * k + 1] * values[k];
        }
        energies[2 * i] = e[0];
        energies[2 * i + 1] = e[1];
    }
    for (size_t j = 0; j < large.size(); ++j) {
        energies[2 * large[j]] = le[j].x;
        energies[2 * large[j] + 1] = le[j].y;
    }
    return QS_OK;
}

// ---------------------------------------------------------------- many terms per HBM pass
// For terms with a bit flip, one pass per term costs one full read of the state per term.  Here a
// pass owns a set Q of kEvTileBits tile qubits (always including qubits 0..4) and evaluates EVERY
// term whose bit-flip mask lies inside Q: each CTA loads a tile (the 2^11 amplitudes sharing the
// values of the other qubits) into shared memory once, and warp w evaluates terms w, w + 4, ... over
// the tile's pairs.  The phase parity splits into the tile part (popcount of the tile index under the
// term's local Z mask) and the fixed part of the tile base.  Each CTA accumulates per-term FP64 sums
// over its tiles in a fixed order; a fold kernel adds the CTAs' sums in index order.
namespace qs {

constexpr int kEvTileBits = kEvTileBitsDecl;
constexpr int kEvLowFixed = 4;    // unit vectors of qubits 0..3 in every tile basis (256-byte runs)
constexpr int kEvMaxTerms = 512;  // terms per pass (shared-memory accumulators)

struct EvTileTerm {
    UINT xloc, zloc;  // masks over tile bits
    ITYPE zglob;      // full phase-flip mask (for the base parity)
    UINT nrot, pivot; // pivot: a tile bit of xloc
};

template <class T>
__device__ __forceinline__ double2 tile_amp(const T* p);
template <>
__device__ __forceinline__ double2 tile_amp<double2>(const double2* p) { return ld_stream(p); }
template <>
__device__ __forceinline__ double2 tile_amp<float2>(const float2* p) {
    const float2 v = __ldcs(p);
    return make_double2(v.x, v.y);
}

// One part (C = 0: real, 1: imaginary) of x conj(y), its sign flipped when `flip` is set.
template <int C>
__device__ __forceinline__ double part_flipped(double2 x, double2 y, UINT flip) {
    const double v = C ? fma(x.y, y.x, -(x.x * y.y)) : fma(x.x, y.x, x.y * y.y);
    return __longlong_as_double(__double_as_longlong(v) ^ ((unsigned long long)flip << 63));
}

// The sums of one string (or of two strings sharing the pairing bit, which read tile[u0] once) over
// the tile's pair bases u0 (bit `pivot` clear) of this lane.
template <int C1>
__device__ __forceinline__ double ev_single(const double2* tile, UINT half, UINT pivot, UINT x1, UINT z1) {
    double s1 = 0.;
    for (UINT p = threadIdx.x & 31; p < half; p += 32) {
        const UINT u0 = (UINT)insert0(p, pivot);
        s1 += part_flipped<C1>(tile[u0], tile[u0 ^ x1], (UINT)__popc(u0 & z1) & 1u);
    }
    return s1;
}
// The sum of one Z-only string over the tile: |tile[u]|^2 with the sign of parity(u & z1), this lane's u.
__device__ __forceinline__ double ev_diag(const double2* tile, UINT tsize, UINT z1) {
    double s1 = 0.;
    for (UINT u = threadIdx.x & 31; u < tsize; u += 32) {
        const double2 v = tile[u];
        const double p = fma(v.x, v.x, v.y * v.y);
        s1 += __longlong_as_double(__double_as_longlong(p) ^ ((unsigned long long)(__popc(u & z1) & 1u) << 63));
    }
    return s1;
}
template <int C1, int C2>
__device__ __forceinline__ void ev_pair(const double2* tile, UINT half, UINT pivot, UINT x1, UINT z1, UINT x2,
    UINT z2, double* s1, double* s2) {
    double a1 = 0., a2 = 0.;
    for (UINT p = threadIdx.x & 31; p < half; p += 32) {
        const UINT u0 = (UINT)insert0(p, pivot);
        const double2 x = tile[u0];
        a1 += part_flipped<C1>(x, tile[u0 ^ x1], (UINT)__popc(u0 & z1) & 1u);
        a2 += part_flipped<C2>(x, tile[u0 ^ x2], (UINT)__popc(u0 & z2) & 1u);
    }
    *s1 = a1;
    *s2 = a2;
}

constexpr int kEvTileCtasPerSm = 6;  // 6 x 37 KiB of shared memory; the loads go 4 rows at a time to fit

template <class T>
__global__ void __launch_bounds__(128, kEvTileCtasPerSm) k_ev_tile(const T* __restrict__ s, ITYPE tiles, const __grid_constant__ EvTileArgs a,
    const EvTileTerm* __restrict__ terms, int npairs, double* __restrict__ partials) {
    __shared__ double2 tile[1 << kEvTileBits];
    __shared__ double acc[kEvMaxTerms];
    __shared__ ITYPE hi_off[16];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m = a.m;
    const UINT tsize = 1u << m;
    for (int k = tid; k < a.nterms; k += 128) acc[k] = 0.;
    // tile index u = tid + 128 k: bits 0..6 from tid, bits 7.. from k
    if (tid < 16) {
        ITYPE o = 0;
        for (int j = 7; j < m; ++j)
            if ((tid >> (j - 7)) & 1) o ^= a.b[j];
        hi_off[tid] = o;
    }
    ITYPE lo_off = 0;
    for (int j = 0; j < 7 && j < m; ++j)
        if ((tid >> j) & 1) lo_off ^= a.b[j];
    for (ITYPE ti = blockIdx.x; ti < tiles; ti += gridDim.x) {
        ITYPE base = ti;
        for (int j = 0; j < m; ++j) base = insert0(base, a.piv_sorted[j]);
        __syncthreads();
        if constexpr (sizeof(T) == sizeof(double2)) {
            // complex128: 16-byte cp.async copies straight into shared memory, all 16 of a thread in flight
            // without holding registers
#pragma unroll
            for (int k = 0; k < 16; ++k)
                if ((UINT)tid + (UINT)k * 128 < tsize) {
                    const unsigned dst = (unsigned)__cvta_generic_to_shared(tile + tid + k * 128);
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst),
                        "l"(s + (base ^ lo_off ^ hi_off[k])) : "memory");
                }
            asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
        } else {
#pragma unroll
            for (int h = 0; h < 16; h += 4) {
                double2 v[4];  // four loads in flight per thread before the shared-memory stores
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if ((UINT)tid + (UINT)(h + k) * 128 < tsize) v[k] = tile_amp<T>(s + (base ^ lo_off ^ hi_off[h + k]));
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if ((UINT)tid + (UINT)(h + k) * 128 < tsize) tile[tid + (h + k) * 128] = v[k];
            }
        }
        __syncthreads();
        // Re(v i^r) with v = tile[u0] conj(tile[u0 ^ x]) and r = r0 + 2 parity(u0 & zloc): r0 picks the
        // real or imaginary part of v and an overall sign; the parity flips the sign per pair.  Only
        // that one part of the product is computed.  Units: terms (2w, 2w + 1) for w < npairs share
        // their pairing bit; the rest are single, the last a.nz of them Z-only strings (sum of |a|^2 with
        // the parity sign; their r is 0 or 2, so the factor is +-1 instead of +-2).
        const int nunits = npairs + (a.nterms - 2 * npairs);
        const int zfirst = nunits - a.nz;
        const UINT half = tsize >> 1;
        for (int w = warp; w < nunits; w += 4) {
            const int t1 = w < npairs ? 2 * w : npairs + w;
            const EvTileTerm m1 = terms[t1];
            const UINT r1 = (m1.nrot + 2u * (UINT)(__popcll(base & m1.zglob) & 1)) & 3u;
            double s1 = 0., s2 = 0.;
            UINT r2 = 0;
            double f1 = (r1 == 1u || r1 == 2u) ? -2.0 : 2.0;
            if (w < npairs) {
                const EvTileTerm m2 = terms[t1 + 1];
                r2 = (m2.nrot + 2u * (UINT)(__popcll(base & m2.zglob) & 1)) & 3u;
                switch (((r1 & 1u) << 1) | (r2 & 1u)) {
                    case 0: ev_pair<0, 0>(tile, half, m1.pivot, m1.xloc, m1.zloc, m2.xloc, m2.zloc, &s1, &s2); break;
                    case 1: ev_pair<0, 1>(tile, half, m1.pivot, m1.xloc, m1.zloc, m2.xloc, m2.zloc, &s1, &s2); break;
                    case 2: ev_pair<1, 0>(tile, half, m1.pivot, m1.xloc, m1.zloc, m2.xloc, m2.zloc, &s1, &s2); break;
                    default: ev_pair<1, 1>(tile, half, m1.pivot, m1.xloc, m1.zloc, m2.xloc, m2.zloc, &s1, &s2); break;
                }
            } else if (w < zfirst) {
                s1 = (r1 & 1u) ? ev_single<1>(tile, half, m1.pivot, m1.xloc, m1.zloc)
                               : ev_single<0>(tile, half, m1.pivot, m1.xloc, m1.zloc);
            } else {
                s1 = ev_diag(tile, tsize, m1.zloc);
                f1 *= 0.5;
            }
            // r0 = 0: +Re, 1: -Im, 2: -Re, 3: +Im
            s1 *= f1;
            s2 *= (r2 == 1u || r2 == 2u) ? -2.0 : 2.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                s1 += __shfl_xor_sync(0xffffffffu, s1, o);
                s2 += __shfl_xor_sync(0xffffffffu, s2, o);
            }
            if (lane == 0) {
                acc[t1] += s1;
                if (w < npairs) acc[t1 + 1] += s2;
            }
        }
    }
    __syncthreads();
    for (int k = tid; k < a.nterms; k += 128) partials[(size_t)blockIdx.x * a.nterms + k] = acc[k];
}

__global__ void k_fold_cols(const double* __restrict__ part, int rows, int cols, double* __restrict__ out,
    const UINT* __restrict__ out_index) {
    __shared__ double sm[32];
    const int c = blockIdx.x;
    double v = 0.;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) v += part[(size_t)r * cols + c];
    v = block_sum(v, sm);
    if (threadIdx.x == 0) out[out_index[c]] = v;
}

// A tile basis in reduced echelon form: b[j] has bit piv[j] set and no other mask of the basis has it,
// so reduce(x) (clear every pivot bit of x with its basis mask) is 0 exactly for x in the span.
struct EvBasis {
    std::vector<ITYPE> b;
    std::vector<int> piv;
    ITYPE reduce(ITYPE x) const {
        for (size_t j = 0; j < b.size(); ++j)
            if ((x >> piv[j]) & 1) x ^= b[j];
        return x;
    }
    void add(ITYPE r) {  // r reduced and nonzero
        const int p = 63 - __builtin_clzll(r);
        for (ITYPE& v : b)  // keep every pivot bit in exactly one basis mask
            if ((v >> p) & 1) v ^= r;
        b.push_back(r);
        piv.push_back(p);
    }
    // tile coordinates of a mask in the span: bit j <-> basis mask j
    UINT local_x(ITYPE x) const {
        UINT l = 0;
        for (size_t j = 0; j < b.size(); ++j)
            if ((x >> piv[j]) & 1) l |= 1u << j;
        return l;
    }
    // phase-flip mask over tile coordinates: bit j = parity(b[j] & z)
    UINT local_z(ITYPE z) const {
        UINT l = 0;
        for (size_t j = 0; j < b.size(); ++j)
            if (__builtin_popcountll(b[j] & z) & 1) l |= 1u << j;
        return l;
    }
    void args(EvTileArgs* a) const {
        a->m = (int)b.size();
        for (int j = 0; j < a->m; ++j) {
            a->b[j] = b[j];
            a->piv_sorted[j] = (UINT)piv[j];
        }
        std::sort(a->piv_sorted, a->piv_sorted + a->m);
    }
};

// The basis of one pass: unit vectors of qubits 0..3, then, while fewer than m, the reduced bit-flip
// mask shared by the most of `todo`'s terms not yet in the span (the first in term order on a tie: a
// term x joins the span of B + r exactly when reduce_B(x) is 0 or reduce_B(r)), then unit vectors of
// the lowest free qubits (a tile always has m basis masks).
EvBasis ev_basis(const PauliTerm* terms, const std::vector<int>& todo, UINT n, int m) {
    EvBasis B;
    for (int q = 0; q < kEvLowFixed; ++q) B.add(1ULL << q);
    std::vector<ITYPE> red(todo.size());
    for (size_t i = 0; i < todo.size(); ++i) red[i] = B.reduce(terms[todo[i]].x);
    std::unordered_map<ITYPE, int> freq;
    while ((int)B.b.size() < m) {
        freq.clear();
        ITYPE best = 0;
        int most = 0;
        for (ITYPE r : red)
            if (r) {
                const int c = ++freq[r];
                if (c > most) {
                    most = c;
                    best = r;
                }
            }
        if (!best) break;
        B.add(best);
        for (ITYPE& r : red)
            if (r) r = B.reduce(r);
    }
    for (int q = 0; q < (int)n && (int)B.b.size() < m; ++q) {
        const ITYPE r = B.reduce(1ULL << q);
        if (r) B.add(r);
    }
    return B;
}

// Host: cover the terms' bit-flip masks with tiles spanned by qubits 0..3 and up to m - 4 of the terms'
// own masks (reduced echelon form, see EvTileArgs): a pass evaluates every term whose mask lies in
// its span from shared memory.  Terms left when a pass would cover fewer than two stay in `rest`
// for the one-pass-per-term kernel.
template <class T>
int ev_tiled(const PauliTerm* terms, const std::vector<int>& xidx, UINT n, const T* s, ITYPE dim, cudaStream_t st,
    double* values, std::vector<int>* rest, std::vector<int>* zidx) {
    const int m = kEvTileBits;
    std::vector<int> todo = xidx;
    const unsigned grid = (unsigned)std::min<ITYPE>(dim >> m, (ITYPE)sm_count() * kEvTileCtasPerSm);
    constexpr size_t kMinCover = 2;  // below this a shared pass is not cheaper than one pass per term
    std::vector<double> hvals;
    while (!todo.empty()) {
        const EvBasis B = ev_basis(terms, todo, n, m);
        const std::vector<ITYPE>& basis = B.b;
        const std::vector<int>& piv = B.piv;
        auto reduce = [&](ITYPE x) { return B.reduce(x); };
        EvTileArgs a{};
        B.args(&a);
        std::vector<EvTileTerm> tt;
        std::vector<UINT> outi;
        std::vector<int> left;
        for (int k : todo) {
            if (reduce(terms[k].x) != 0 || (int)tt.size() >= kEvMaxTerms) {
                left.push_back(k);
                continue;
            }
            EvTileTerm e{};
            for (int jj = 0; jj < a.m; ++jj) {
                if ((terms[k].x >> piv[jj]) & 1) e.xloc |= 1u << jj;
                if (__builtin_popcountll(basis[jj] & terms[k].z) & 1) e.zloc |= 1u << jj;
            }
            e.zglob = terms[k].z;  // parity of rep(T) & z; the tile-element part is zloc
            e.nrot = terms[k].nrot;
            e.pivot = (UINT)(31 - __builtin_clz(e.xloc));
            tt.push_back(e);
            outi.push_back((UINT)k);
        }
        if (tt.size() < kMinCover) {  // the remaining terms go one pass each
            rest->insert(rest->end(), todo.begin(), todo.end());
            break;
        }
        // pair terms whose local X masks share a bit (it becomes both terms' pairing bit: the pair reads
        // tile[u0] once); pairs first, then the single terms with their top bit
        int npairs = 0;
        {
            std::vector<EvTileTerm> pt, st1;
            std::vector<UINT> po, so;
            std::vector<char> used(tt.size(), 0);
            for (size_t i = 0; i < tt.size(); ++i) {
                if (used[i]) continue;
                used[i] = 1;
                size_t j = i + 1;
                // a pairing bit below tile bit 3 breaks each quarter-warp's run of u0 into pieces that
                // share banks (two-way conflicts on all three loads): pair only on bits >= 3
                for (; j < tt.size(); ++j)
                    if (!used[j] && (tt[i].xloc & tt[j].xloc & ~7u)) break;
                if (j < tt.size()) {
                    used[j] = 1;
                    const UINT common = tt[i].xloc & tt[j].xloc & ~7u;
                    EvTileTerm e1 = tt[i], e2 = tt[j];
                    e1.pivot = e2.pivot = (UINT)(31 - __builtin_clz(common));
                    pt.push_back(e1);
                    pt.push_back(e2);
                    po.push_back(outi[i]);
                    po.push_back(outi[j]);
                    ++npairs;
                } else {
                    st1.push_back(tt[i]);
                    so.push_back(outi[i]);
                }
            }
            pt.insert(pt.end(), st1.begin(), st1.end());
            po.insert(po.end(), so.begin(), so.end());
            tt.swap(pt);
            outi.swap(po);
        }
        // the Z-only strings join the first pass (any tile basis serves them)
        a.nz = 0;
        if (zidx && !zidx->empty()) {
            std::vector<int> zleft;
            for (int k : *zidx) {
                if ((int)tt.size() >= kEvMaxTerms) {
                    zleft.push_back(k);
                    continue;
                }
                EvTileTerm e{};
                for (int jj = 0; jj < a.m; ++jj)
                    if (__builtin_popcountll(basis[jj] & terms[k].z) & 1) e.zloc |= 1u << jj;
                e.zglob = terms[k].z;
                e.nrot = terms[k].nrot;
                tt.push_back(e);
                outi.push_back((UINT)k);
                ++a.nz;
            }
            zidx->swap(zleft);
        }
        a.nterms = (int)tt.size();
        const size_t bt = sizeof(EvTileTerm) * tt.size(), bo = sizeof(UINT) * outi.size(),
                     bp = sizeof(double) * grid * tt.size(), bv = sizeof(double) * 1;
        auto up = [](size_t b) { return (b + 255) / 256 * 256; };
        void* buf;
        QS_TRY(scratch(st, up(bt) + up(bo) + up(bp) + up(sizeof(double) * (outi.size() + 1)) + up(bv), &buf));
        char* p = (char*)buf;
        EvTileTerm* dt = (EvTileTerm*)p;
        UINT* doi = (UINT*)(p + up(bt));
        double* dpart = (double*)(p + up(bt) + up(bo));
        double* dval = (double*)(p + up(bt) + up(bo) + up(bp));
        std::vector<UINT> seq(outi.size());
        for (size_t i = 0; i < seq.size(); ++i) seq[i] = (UINT)i;
        QS_CUDA_CHECK(cudaMemcpyAsync(dt, tt.data(), bt, cudaMemcpyHostToDevice, st));
        QS_CUDA_CHECK(cudaMemcpyAsync(doi, seq.data(), bo, cudaMemcpyHostToDevice, st));
        k_ev_tile<T><<<grid, 128, 0, st>>>(s, dim >> a.m, a, dt, npairs, dpart);
        QS_TRY(check_launch("k_ev_tile"));
        k_fold_cols<<<(unsigned)tt.size(), 256, 0, st>>>(dpart, (int)grid, (int)tt.size(), dval, doi);
        QS_TRY(check_launch("k_fold_cols"));
        hvals.resize(tt.size());
        QS_CUDA_CHECK(cudaMemcpyAsync(hvals.data(), dval, sizeof(double) * tt.size(), cudaMemcpyDeviceToHost, st));
        QS_CUDA_CHECK(cudaStreamSynchronize(st));
        for (size_t i = 0; i < outi.size(); ++i) values[outi[i]] = hvals[i];
        todo.swap(left);
    }
    return QS_OK;
}

template int ev_tiled<double2>(const PauliTerm*, const std::vector<int>&, UINT, const double2*, ITYPE, cudaStream_t,
    double*, std::vector<int>*, std::vector<int>*);
template int ev_tiled<float2>(const PauliTerm*, const std::vector<int>&, UINT, const float2*, ITYPE, cudaStream_t,
    double*, std::vector<int>*, std::vector<int>*);

}  // namespace qs

// ---------------------------------------------------------------- sum_k c_k <P_k>, register-resident tiles
// The weighted expectation value needs no per-term value, so no per-term reduction either: every
// thread folds each term's contribution into one running complex sum (FP64) across all its tiles, and
// each CTA writes one partial per pass.  Tiles use the pass bases of the per-term kernel above (2^11
// amplitudes): tile bits 0..6 are the thread index, tile bits 7..10 index 16 amplitudes held in the
// thread's registers and also stored to shared memory.  A term with bit-flip mask (xt, xr) over
// (thread bits, register bits) pairs thread t's amplitude p with amplitude p ^ xr of thread t ^ xt:
//   xt = 0:          both ends in the thread's own registers (no shared-memory read);
//   xr != 0 (K its lowest bit): thread t takes its 8 amplitudes with bit K of p clear and reads the
//                    partner end from shared memory; thread t ^ xt takes the other 8 pairs;
//   xr = 0:          thread t takes its 8 amplitudes whose bit 0 of p equals bit j of t (j the lowest
//                    bit of xt); thread t ^ xt the other 8.
// Each pair {u, u ^ x} is counted once from its own end u (2 Re(conj(a_u) P a_u^x) is the same from
// either end for a Hermitian string), so each thread reads 8 partner amplitudes per term, not 16.
// The phase parity of element u splits into the tile base's part (with the full mask), the thread
// part and the register part; the register part is folded as a +-1 butterfly over the free bits.
namespace qs {

static_assert(kEvTileBits == kEvBasisBits, "weighted and per-term passes share their tiles");

template <int C>
__device__ __forceinline__ double ew_part(double2 a, double2 b) {  // Re (C = 0) or Im (C = 1) of a conj(b)
    return C ? fma(a.y, b.x, -(a.x * b.y)) : fma(a.x, b.x, a.y * b.y);
}
// -1.0 when bit j of zr is set, else +1.0
__device__ __forceinline__ double ew_sgn(UINT zr, int j) {
    return __hiloint2double((int)(0x3FF00000u | ((zr >> j) << 31)), 0);
}
// sum_i v[i] * prod_b s_b^{bit b of i} over 8 values
__device__ __forceinline__ double ew_fold8(double (&v)[8], double s0, double s1, double s2) {
    v[0] = fma(s0, v[1], v[0]);
    v[2] = fma(s0, v[3], v[2]);
    v[4] = fma(s0, v[5], v[4]);
    v[6] = fma(s0, v[7], v[6]);
    v[0] = fma(s1, v[2], v[0]);
    v[4] = fma(s1, v[6], v[4]);
    return fma(s2, v[4], v[0]);
}
__host__ __device__ constexpr int ew_ins0(int i, int k) { return ((i >> k) << (k + 1)) | (i & ((1 << k) - 1)); }
__host__ __device__ constexpr int ew_ctz(int x) { return (x & 1) ? 0 : 1 + ew_ctz(x >> 1); }
__host__ __device__ constexpr int ew_free(int k, int b) { return b < k ? b : b + 1; }  // b-th register bit other than k

// A tile element from shared memory as FP64.
__device__ __forceinline__ double2 ew_ld(const double2* p) { return *p; }
__device__ __forceinline__ double2 ew_ld(const float2* p) {
    const float2 v = *p;
    return make_double2((double)v.x, (double)v.y);
}
// xr != 0, partner row in shared memory: own p (bit K clear) against element p ^ xr of the partner row
// (rows kRow bytes apart)
template <int K, int C, class E, int kRow>
__device__ __forceinline__ double ew_smem(const double2 (&own)[16], const char* prow, UINT xr, UINT zr) {
    double v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int p = ew_ins0(i, K);
        const double2 b = ew_ld((const E*)(prow + ((UINT)p ^ xr) * (UINT)kRow));
        v[i] = ew_part<C>(own[p], b);
    }
    return ew_fold8(v, ew_sgn(zr, ew_free(K, 0)), ew_sgn(zr, ew_free(K, 1)), ew_sgn(zr, ew_free(K, 2)));
}
// xr = 0: own p = 2i + bsel against element p of the partner row
template <int C, class E, int kRow>
__device__ __forceinline__ double ew_row(const double2 (&own)[16], const char* prow, UINT bsel, UINT zr) {
    double v[8];
    const char* pr = prow + bsel * (UINT)kRow;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const double2 a = bsel ? own[2 * i + 1] : own[2 * i];
        const double2 b = ew_ld((const E*)(pr + i * 2 * kRow));
        v[i] = ew_part<C>(a, b);
    }
    return ew_fold8(v, ew_sgn(zr, 1), ew_sgn(zr, 2), ew_sgn(zr, 3));
}
// xt = 0: both ends in registers
template <int XR, int C>
__device__ __forceinline__ double ew_reg(const double2 (&own)[16], UINT zr) {
    constexpr int K = ew_ctz(XR);
    double v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int p = ew_ins0(i, K);
        v[i] = ew_part<C>(own[p], own[p ^ XR]);
    }
    return ew_fold8(v, ew_sgn(zr, ew_free(K, 0)), ew_sgn(zr, ew_free(K, 1)), ew_sgn(zr, ew_free(K, 2)));
}
// Z-only: sum_p |own[p]|^2 (-1)^{parity(p & zr)}
__device__ __forceinline__ double ew_diag(const double2 (&own)[16], UINT zr) {
    double v[16];
#pragma unroll
    for (int p = 0; p < 16; ++p) v[p] = fma(own[p].x, own[p].x, own[p].y * own[p].y);
    const double s0 = ew_sgn(zr, 0), s1 = ew_sgn(zr, 1), s2 = ew_sgn(zr, 2), s3 = ew_sgn(zr, 3);
#pragma unroll
    for (int i = 0; i < 16; i += 2) v[i] = fma(s0, v[i + 1], v[i]);
#pragma unroll
    for (int i = 0; i < 16; i += 4) v[i] = fma(s1, v[i + 2], v[i]);
    v[0] = fma(s2, v[4], v[0]);
    v[8] = fma(s2, v[12], v[8]);
    return fma(s3, v[8], v[0]);
}

// 16- (complex128) or 8-byte (complex64) asynchronous copy global -> shared
template <int B>
__device__ __forceinline__ void ew_cp_async(unsigned dst, const void* src) {
    if constexpr (B == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}

template <int TB, class T>
constexpr size_t ew_smem_bytes() { return 2 * (size_t)(16 << TB) * sizeof(T); }  // two tiles

#define EW_REG_CASE(XR)                                            \
    case EW_REG + 2 * (XR - 1): v = ew_reg<XR, 0>(own, zr); break; \
    case EW_REG + 2 * (XR - 1) + 1: v = ew_reg<XR, 1>(own, zr); break;
#define EW_SMEM_CASE(K)                                                             \
    case EW_SMEM + 2 * K: v = ew_smem<K, 0, T, kRow>(own, prow, xr, zr); break;     \
    case EW_SMEM + 2 * K + 1: v = ew_smem<K, 1, T, kRow>(own, prow, xr, zr); break;

// Grid-stride over tiles, two tile buffers in dynamic shared memory: the copies of tile i + 1 are in
// flight (cp.async) while the terms run over tile i.
template <class T, int TB>
__global__ void __launch_bounds__(1 << TB, kEwCtasPerSm) k_ev_weighted(const T* __restrict__ s, ITYPE tiles,
    const __grid_constant__ EvTileArgs a, const EvWTerm* __restrict__ terms, int nterms,
    double2* __restrict__ partials) {
    constexpr int kThreads = 1 << TB;
    constexpr int kRow = kThreads * (int)sizeof(T);  // bytes between register rows p and p + 1
    constexpr int kTileBytes = 16 * kRow;
    extern __shared__ __align__(16) unsigned char ew_tiles[];
    __shared__ ITYPE hi_off[16];
    __shared__ double red[2][kThreads / 32];
    const UINT t = threadIdx.x;
    if (t < 16) {
        ITYPE o = 0;
        for (int j = 0; j < 4; ++j)
            if ((t >> j) & 1) o ^= a.b[TB + j];
        hi_off[t] = o;
    }
    ITYPE lo_off = 0;
    for (int j = 0; j < TB; ++j)
        if ((t >> j) & 1) lo_off ^= a.b[j];
    auto tile_base = [&](ITYPE ti) {
        ITYPE base = ti;
        for (int j = 0; j < a.m; ++j) base = insert0(base, a.piv_sorted[j]);
        return base;
    };
    const unsigned sdst = (unsigned)__cvta_generic_to_shared(ew_tiles) + t * (unsigned)sizeof(T);
    auto issue = [&](ITYPE ti, int buf) {
        const ITYPE base = tile_base(ti);
#pragma unroll
        for (int p = 0; p < 16; ++p)
            ew_cp_async<(int)sizeof(T)>(sdst + buf * kTileBytes + p * kRow, s + (base ^ lo_off ^ hi_off[p]));
    };
    __syncthreads();  // hi_off
    if ((ITYPE)blockIdx.x < tiles) issue(blockIdx.x, 0);
    asm volatile("cp.async.commit_group;" ::: "memory");
    double accr = 0., acci = 0.;
    int buf = 0;
    for (ITYPE ti = blockIdx.x; ti < tiles; ti += gridDim.x, buf ^= 1) {
        if (ti + gridDim.x < tiles) issue(ti + gridDim.x, buf ^ 1);
        asm volatile("cp.async.commit_group;\ncp.async.wait_group 1;" ::: "memory");
        __syncthreads();  // every thread's copies of tile ti landed
        const char* tb = (const char*)ew_tiles + buf * kTileBytes;
        const ITYPE base = tile_base(ti);
        double2 own[16];
#pragma unroll
        for (int p = 0; p < 16; ++p) own[p] = ew_ld((const T*)(tb + t * sizeof(T) + p * kRow));
        double2 coef_n = make_double2(0., 0.);
        ITYPE zglob_n = 0;
        UINT pk_n = 0;
        if (nterms > 0) {
            coef_n = __ldg(&terms[0].coef);
            zglob_n = __ldg(&terms[0].zglob);
            pk_n = __ldg(&terms[0].packed);
        }
        for (int k = 0; k < nterms; ++k) {
            // opaque per term: keeps the compiler from hoisting every case's products of the (term-invariant)
            // amplitudes out of the loop, which would need hundreds of registers
#pragma unroll
            for (int p = 0; p < 16; ++p) asm volatile("" : "+d"(own[p].x), "+d"(own[p].y));
            const double2 coef = coef_n;
            const ITYPE zglob = zglob_n;
            const UINT pk = pk_n;
            if (k + 1 < nterms) {  // the next descriptor in flight during this term
                coef_n = __ldg(&terms[k + 1].coef);
                zglob_n = __ldg(&terms[k + 1].zglob);
                pk_n = __ldg(&terms[k + 1].packed);
            }
            const UINT xt = pk & 0xFFu, zt = (pk >> 8) & 0xFFu, xr = (pk >> 16) & 15u, zr = (pk >> 20) & 15u;
            UINT flip = (UINT)(__popcll(base & zglob) + __popc(t & zt)) & 1u;
            const char* prow = tb + sizeof(T) * (t ^ xt);
            double v;
            switch (pk >> 24) {
                case EW_Z: v = ew_diag(own, zr); break;
                EW_SMEM_CASE(0)
                EW_SMEM_CASE(1)
                EW_SMEM_CASE(2)
                EW_SMEM_CASE(3)
                case EW_ROW:
                case EW_ROW + 1: {
                    const UINT bsel = (t >> (__ffs(xt) - 1)) & 1u;
                    flip ^= bsel & zr;
                    v = (pk >> 24) == EW_ROW ? ew_row<0, T, kRow>(own, prow, bsel, zr)
                                             : ew_row<1, T, kRow>(own, prow, bsel, zr);
                    break;
                }
                EW_REG_CASE(1) EW_REG_CASE(2) EW_REG_CASE(3) EW_REG_CASE(4) EW_REG_CASE(5)
                EW_REG_CASE(6) EW_REG_CASE(7) EW_REG_CASE(8) EW_REG_CASE(9) EW_REG_CASE(10)
                EW_REG_CASE(11) EW_REG_CASE(12) EW_REG_CASE(13) EW_REG_CASE(14) EW_REG_CASE(15)
                default: v = 0.; break;
            }
            v = __longlong_as_double(__double_as_longlong(v) ^ ((unsigned long long)(flip & 1u) << 63));
            accr = fma(coef.x, v, accr);
            acci = fma(coef.y, v, acci);
        }
        __syncthreads();  // every thread done with this buffer before the copies of tile ti + 2 overwrite it
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        accr += __shfl_xor_sync(0xffffffffu, accr, o);
        acci += __shfl_xor_sync(0xffffffffu, acci, o);
    }
    if ((t & 31) == 0) {
        red[0][t >> 5] = accr;
        red[1][t >> 5] = acci;
    }
    __syncthreads();
    if (t == 0) {
        double r = 0., i = 0.;
        for (int w = 0; w < kThreads / 32; ++w) {
            r += red[0][w];
            i += red[1][w];
        }
        partials[blockIdx.x] = make_double2(r, i);
    }
}
#undef EW_REG_CASE
#undef EW_SMEM_CASE

__global__ void k_fold_d2(const double2* __restrict__ part, int count, double* __restrict__ out) {
    __shared__ double sr[32], si[32];
    double r = 0., i = 0.;
    for (int j = threadIdx.x; j < count; j += blockDim.x) {
        r += part[j].x;
        i += part[j].y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        r += __shfl_xor_sync(0xffffffffu, r, o);
        i += __shfl_xor_sync(0xffffffffu, i, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sr[threadIdx.x >> 5] = r;
        si[threadIdx.x >> 5] = i;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0., b = 0.;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            a += sr[w];
            b += si[w];
        }
        out[0] = a;
        out[1] = b;
    }
}

// One pass of the weighted kernel: its tile basis (register bits chosen) and term descriptors.
struct EwPass {
    EvTileArgs a;
    size_t first, count;  // range in the descriptor array
};

// The descriptor of a term for a pass basis, its coefficient field holding the term's factor alone
// (+-2 for a bit flip, from i^nrot; 1 for Z-only); the coefficient c_k multiplies it per call.
static EvWTerm ew_term(const PauliTerm& pt, const EvBasis& B) {
    constexpr UINT tmask = (1u << kEwThreadBits) - 1;
    const UINT xl = B.local_x(pt.x), zl = B.local_z(pt.z);
    const UINT xt = xl & tmask, xr = xl >> kEwThreadBits, zt = zl & tmask, zr = zl >> kEwThreadBits;
    const UINT C = pt.nrot & 1u, r0 = pt.nrot & 3u;
    double f = (r0 == 1u || r0 == 2u) ? -2.0 : 2.0;  // Re(v i^r): +Re, -Im, -Re, +Im
    UINT code;
    if (!pt.x) {
        code = EW_Z;
        f = 1.0;  // nrot = 0 for a Z-only string; every element counted once
    } else if (!xt) {
        code = EW_REG + 2 * (xr - 1) + C;
    } else if (xr) {
        code = EW_SMEM + 2 * (UINT)__builtin_ctz(xr) + C;
    } else {
        code = EW_ROW + C;
    }
    EvWTerm e{};
    e.coef = make_double2(f, 0.);
    e.zglob = pt.z;
    e.packed = xt | zt << 8 | xr << 16 | zr << 20 | code << 24;
    return e;
}

// Reorder basis masks 4..m-1 so the 4 register bits (the last four) hold the most terms entirely
// (no shared-memory read), then the fewest terms with none of them (the select-based rows).
static void ew_choose_register_bits(EvBasis* B, const PauliTerm* terms, const std::vector<int>& in) {
    const int m = (int)B->b.size();
    std::vector<UINT> xl;
    for (int k : in) xl.push_back(B->local_x(terms[k].x));
    int best_set = -1;
    long best_score = -1;
    for (int set = 0; set < (1 << m); ++set) {
        if (__builtin_popcount(set) != 4 || (set & ((1 << kEvLowFixed) - 1))) continue;
        long reg = 0, row = 0;
        for (UINT l : xl) {
            reg += (l & ~(UINT)set) == 0;
            row += (l & (UINT)set) == 0;
        }
        const long score = reg * 4096 - row;
        if (score > best_score) {
            best_score = score;
            best_set = set;
        }
    }
    EvBasis R;
    for (int j = 0; j < m; ++j)
        if (!((best_set >> j) & 1)) {
            R.b.push_back(B->b[j]);
            R.piv.push_back(B->piv[j]);
        }
    for (int j = 0; j < m; ++j)
        if ((best_set >> j) & 1) {
            R.b.push_back(B->b[j]);
            R.piv.push_back(B->piv[j]);
        }
    *B = R;
}

// The plan of sum_k c_k <P_k> for a list of terms on n qubits: pass bases and descriptors (every Z-only
// term in the first pass), the term behind each descriptor, the terms left for one value each (a pass
// would cover fewer than two), and the per-pass kernels generated for it.
struct EwPlan {
    std::vector<EwPass> passes;
    std::vector<EvWTerm> desc;
    std::vector<int> term_of;
    std::vector<int> rest;
    std::mutex mu;      // guards the fields below
    int uses = 0;
    int spec_state = 0;  // 0 not generated, 1 generated, 2 generation failed
    std::vector<void*> spec;  // per pass: generated kernel, or nullptr where the generic kernel runs
    double compile_ms = 0.;
};

constexpr size_t kEvSpecMaxTerms = 192;  // larger passes keep the generic kernel (code size)
constexpr UINT kEvSpecMinQubits = 20;    // below this a pass takes microseconds: not worth a compile
std::atomic<int> g_ev_spec_mode{1};      // 0 off, 1 from the second use of a plan (n >= 20), 2 first use, any n
std::atomic<long long> g_ev_spec_launches{0};
std::atomic<double> g_ev_last_compile_ms{0.};

static void ew_build(const PauliTerm* terms, UINT count, UINT n, EwPlan* P) {
    constexpr size_t kMinCover = 2;
    std::vector<int> zidx, todo;
    for (UINT k = 0; k < count; ++k) (terms[k].x == 0 ? zidx : todo).push_back((int)k);
    if (n < (UINT)kEvTileBits || todo.size() < 4) {
        for (UINT k = 0; k < count; ++k) P->rest.push_back((int)k);
        return;
    }
    while (!todo.empty()) {
        EvBasis B = ev_basis(terms, todo, n, kEvTileBits);
        std::vector<int> in, left;
        for (int k : todo) (B.reduce(terms[k].x) == 0 ? in : left).push_back(k);
        if (in.size() < kMinCover) {
            P->rest.insert(P->rest.end(), todo.begin(), todo.end());
            break;
        }
        ew_choose_register_bits(&B, terms, in);
        EwPass pass{};
        B.args(&pass.a);
        pass.first = P->desc.size();
        auto add = [&](int k) {
            P->desc.push_back(ew_term(terms[k], B));
            P->term_of.push_back(k);
        };
        for (int k : in) add(k);
        if (P->passes.empty()) {  // the Z-only terms ride in the first pass
            for (int k : zidx) add(k);
            zidx.clear();
        }
        pass.count = P->desc.size() - pass.first;
        pass.a.nterms = (int)pass.count;
        P->passes.push_back(pass);
        todo.swap(left);
    }
    P->rest.insert(P->rest.end(), zidx.begin(), zidx.end());
}

// Plans cached by (qubit count, state type, imaginary coefficients, term masks).
static std::shared_ptr<EwPlan> ew_plan(const PauliTerm* terms, UINT count, UINT n, bool c64, bool imag) {
    std::string key;
    key.reserve(16 + (size_t)count * 20);
    const UINT head[3] = {n, (UINT)c64, (UINT)imag};
    key.append((const char*)head, sizeof(head));
    for (UINT k = 0; k < count; ++k) {
        key.append((const char*)&terms[k].x, sizeof(ITYPE));
        key.append((const char*)&terms[k].z, sizeof(ITYPE));
        key.append((const char*)&terms[k].nrot, sizeof(UINT));
    }
    static std::mutex mu;
    static std::map<std::string, std::shared_ptr<EwPlan>> cache;
    static std::deque<std::string> order;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    auto P = std::make_shared<EwPlan>();
    ew_build(terms, count, n, P.get());
    cache[key] = P;
    order.push_back(key);
    constexpr size_t kMaxPlans = 64;
    if (order.size() > kMaxPlans) {  // oldest first; a plan in use stays alive through its shared_ptr
        cache.erase(order.front());
        order.pop_front();
    }
    return P;
}

// Generate and compile the plan's per-pass kernels (in parallel), once; the first failure's status.
static int ew_specialize(EwPlan* P, bool c64, bool imag) {
    std::vector<void*> k(P->passes.size(), nullptr);
    std::vector<double> ms(P->passes.size(), 0.);
    std::vector<int> rcs(P->passes.size(), QS_OK);
    std::atomic<size_t> next{0};
    auto work = [&] {
        for (size_t i; (i = next++) < P->passes.size();) {
            const EwPass& ps = P->passes[i];
            if (ps.count > kEvSpecMaxTerms) continue;
            rcs[i] = ev_pass_kernel(P->desc.data() + ps.first, ps.count, c64, imag, &k[i], &ms[i]);
        }
    };
    const unsigned nt = std::max(1u, std::min<unsigned>((unsigned)P->passes.size(), std::min(16u,
        std::thread::hardware_concurrency())));
    std::vector<std::thread> pool;
    for (unsigned i = 1; i < nt; ++i) pool.emplace_back(work);
    work();
    for (std::thread& t : pool) t.join();
    int rc = QS_OK;
    for (size_t i = 0; i < rcs.size() && rc == QS_OK; ++i) rc = rcs[i];
    P->spec_state = rc == QS_OK ? 1 : 2;
    if (rc == QS_OK) {
        P->spec = k;
        double total = 0.;
        for (double v : ms) total += v;
        P->compile_ms = total;
        g_ev_last_compile_ms = total;
    }
    return rc;
}

// `allow_generate`: the per-pass kernels may be generated for these terms (callers that evaluate many
// different term lists once each, such as the batched energies, pass false: a compile would not pay).
template <class T>
int ev_weighted(const PauliTerm* terms, const double2* coefs, UINT count, const T* s, ITYPE dim, cudaStream_t st,
    double out[2], bool allow_generate) {
    UINT n = 0;
    while ((1ULL << n) < dim) ++n;
    constexpr bool c64 = sizeof(T) == sizeof(float2);
    bool imag = false;
    for (UINT k = 0; k < count; ++k) imag |= coefs[k].y != 0.;
    std::shared_ptr<EwPlan> P = ew_plan(terms, count, n, c64, imag);
    double sr = 0., si = 0.;
    if (!P->passes.empty()) {
        std::vector<void*> spec;
        {
            std::lock_guard<std::mutex> lk(P->mu);
            ++P->uses;
            const int mode = g_ev_spec_mode.load();
            if (allow_generate && P->spec_state == 0 &&
                (mode == 2 || (mode == 1 && n >= kEvSpecMinQubits && P->uses >= 2))) {
                const int rc = ew_specialize(P.get(), c64, imag);
                if (rc != QS_OK && mode == 2) return rc;  // required: report; by default the generic kernel runs
            }
            if (mode == 2 && P->spec_state == 2)
                return set_error(QS_ERR_NOT_SUPPORTED, "expectation: kernel generation failed earlier for these terms");
            if (mode != 0 && P->spec_state == 1) spec = P->spec;
        }
        const unsigned grid = (unsigned)std::min<ITYPE>(dim >> kEvTileBits, (ITYPE)sm_count() * kEwCtasPerSm);
        auto up = [](size_t b) { return (b + 255) / 256 * 256; };
        // descriptors with their coefficients (generic kernel) and the coefficients alone (generated kernels)
        std::vector<EvWTerm> desc = P->desc;
        std::vector<double2> cf(desc.size());
        for (size_t i = 0; i < desc.size(); ++i) {
            const double f = desc[i].coef.x;
            const double2 c = coefs[P->term_of[i]];
            cf[i] = desc[i].coef = make_double2(c.x * f, c.y * f);
        }
        const size_t bd = sizeof(EvWTerm) * desc.size(), bc = sizeof(double2) * cf.size(),
                     bp = sizeof(double2) * grid * P->passes.size();
        void* buf;
        QS_TRY(scratch(st, up(bd) + up(bc) + up(bp) + 256, &buf));
        EvWTerm* dd = (EvWTerm*)buf;
        double2* dc = (double2*)((char*)buf + up(bd));
        double2* dp = (double2*)((char*)buf + up(bd) + up(bc));
        double* dout = (double*)((char*)buf + up(bd) + up(bc) + up(bp));
        QS_CUDA_CHECK(cudaMemcpyAsync(dd, desc.data(), bd, cudaMemcpyHostToDevice, st));
        QS_CUDA_CHECK(cudaMemcpyAsync(dc, cf.data(), bc, cudaMemcpyHostToDevice, st));
        constexpr size_t smem = ew_smem_bytes<kEwThreadBits, T>();
        {  // the tile buffers exceed the default 48 KiB of dynamic shared memory: opt in once per device
            static std::mutex mu;
            static std::vector<char> ready;
            int dev = 0;
            QS_CUDA_CHECK(cudaGetDevice(&dev));
            std::lock_guard<std::mutex> lock(mu);
            if ((int)ready.size() <= dev) ready.resize(dev + 1, 0);
            if (!ready[dev]) {
                QS_CUDA_CHECK(cudaFuncSetAttribute(k_ev_weighted<T, kEwThreadBits>,
                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                ready[dev] = 1;
            }
        }
        for (size_t i = 0; i < P->passes.size(); ++i) {
            const EwPass& ps = P->passes[i];
            if (!spec.empty() && spec[i]) {
                QS_TRY(launch_ev_pass(spec[i], s, dim >> kEvTileBits, ps.a, dc + ps.first, dp + i * grid, grid, c64,
                    st));
                ++g_ev_spec_launches;
            } else {
                k_ev_weighted<T, kEwThreadBits><<<grid, 1 << kEwThreadBits, smem, st>>>(s, dim >> kEvTileBits, ps.a,
                    dd + ps.first, (int)ps.count, dp + i * grid);
                QS_TRY(check_launch("k_ev_weighted"));
            }
        }
        k_fold_d2<<<1, 256, 0, st>>>(dp, (int)(grid * P->passes.size()), dout);
        QS_TRY(check_launch("k_fold_d2"));
        double h[2];
        QS_CUDA_CHECK(cudaMemcpyAsync(h, dout, sizeof(h), cudaMemcpyDeviceToHost, st));
        QS_CUDA_CHECK(cudaStreamSynchronize(st));
        sr += h[0];
        si += h[1];
    }
    // terms evaluated one value each (ev_batch), weighted on the host
    if (!P->rest.empty()) {
        std::vector<PauliTerm> sub;
        for (int k : P->rest) sub.push_back(terms[k]);
        std::vector<double> vals(sub.size());
        QS_TRY(ev_batch<T>(sub.data(), (UINT)sub.size(), s, dim, st, vals.data()));
        for (size_t i = 0; i < P->rest.size(); ++i) {
            sr += coefs[P->rest[i]].x * vals[i];
            si += coefs[P->rest[i]].y * vals[i];
        }
    }
    out[0] = sr;
    out[1] = si;
    return QS_OK;
}

// sum_k c_k <P_k> of many states at once (each with its own terms): the plans are built on host threads
// in parallel (each term list is evaluated once, so no plan cache and no generated kernels), every
// pass of every state is launched back to back with the generic pass kernel, one fold per state, and
// one copy back; terms outside the passes are evaluated afterwards, one value each.
template <class T>
int ev_weighted_many(const std::vector<const T*>& s, const std::vector<UINT>& nq,
    const std::vector<std::vector<PauliTerm>>& terms, const std::vector<const double2*>& coefs, cudaStream_t st,
    std::vector<double2>* out) {
    const size_t S = s.size();
    out->assign(S, make_double2(0., 0.));
    if (S == 0) return QS_OK;
    std::vector<EwPlan> plans(S);
    {
        std::atomic<size_t> next{0};
        auto work = [&] {
            for (size_t i; (i = next++) < S;) ew_build(terms[i].data(), (UINT)terms[i].size(), nq[i], &plans[i]);
        };
        const unsigned nt = std::max(1u, std::min<unsigned>((unsigned)S, std::min(16u, std::thread::hardware_concurrency())));
        std::vector<std::thread> pool;
        for (unsigned t = 1; t < nt; ++t) pool.emplace_back(work);
        work();
        for (std::thread& t : pool) t.join();
    }
    std::vector<EvWTerm> desc;
    std::vector<size_t> desc0(S), part0(S + 1, 0);
    std::vector<unsigned> grid(S);
    for (size_t i = 0; i < S; ++i) {
        desc0[i] = desc.size();
        for (size_t j = 0; j < plans[i].desc.size(); ++j) {
            EvWTerm e = plans[i].desc[j];
            const double f = e.coef.x;
            const double2 c = coefs[i][plans[i].term_of[j]];
            e.coef = make_double2(c.x * f, c.y * f);
            desc.push_back(e);
        }
        const ITYPE dim = 1ULL << nq[i];
        grid[i] = (unsigned)std::min<ITYPE>(dim >> kEvTileBits, (ITYPE)sm_count() * kEwCtasPerSm);
        part0[i + 1] = part0[i] + (size_t)grid[i] * plans[i].passes.size();
    }
    if (!desc.empty()) {
        auto up = [](size_t b) { return (b + 255) / 256 * 256; };
        const size_t bd = sizeof(EvWTerm) * desc.size(), bp = sizeof(double2) * part0[S], bo = sizeof(double2) * S;
        void* buf;
        QS_TRY(scratch(st, up(bd) + up(bp) + up(bo), &buf));
        EvWTerm* dd = (EvWTerm*)buf;
        double2* dp = (double2*)((char*)buf + up(bd));
        double2* dout = (double2*)((char*)buf + up(bd) + up(bp));
        QS_CUDA_CHECK(cudaMemcpyAsync(dd, desc.data(), bd, cudaMemcpyHostToDevice, st));
        QS_CUDA_CHECK(cudaMemsetAsync(dout, 0, bo, st));
        constexpr size_t smem = ew_smem_bytes<kEwThreadBits, T>();
        {
            static std::mutex mu;
            static std::vector<char> ready;
            int dev = 0;
            QS_CUDA_CHECK(cudaGetDevice(&dev));
            std::lock_guard<std::mutex> lock(mu);
            if ((int)ready.size() <= dev) ready.resize(dev + 1, 0);
            if (!ready[dev]) {
                QS_CUDA_CHECK(cudaFuncSetAttribute(k_ev_weighted<T, kEwThreadBits>,
                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                ready[dev] = 1;
            }
        }
        for (size_t i = 0; i < S; ++i) {
            const ITYPE dim = 1ULL << nq[i];
            for (size_t p = 0; p < plans[i].passes.size(); ++p) {
                const EwPass& ps = plans[i].passes[p];
                k_ev_weighted<T, kEwThreadBits><<<grid[i], 1 << kEwThreadBits, smem, st>>>(s[i], dim >> kEvTileBits,
                    ps.a, dd + desc0[i] + ps.first, (int)ps.count, dp + part0[i] + p * grid[i]);
                QS_TRY(check_launch("k_ev_weighted"));
            }
            if (part0[i + 1] > part0[i]) {
                k_fold_d2<<<1, 256, 0, st>>>(dp + part0[i], (int)(part0[i + 1] - part0[i]), (double*)(dout + i));
                QS_TRY(check_launch("k_fold_d2"));
            }
        }
        QS_CUDA_CHECK(cudaMemcpyAsync(out->data(), dout, bo, cudaMemcpyDeviceToHost, st));
        QS_CUDA_CHECK(cudaStreamSynchronize(st));
    }
    for (size_t i = 0; i < S; ++i) {
        if (plans[i].rest.empty()) continue;
        std::vector<PauliTerm> sub;
        for (int k : plans[i].rest) sub.push_back(terms[i][k]);
        std::vector<double> vals(sub.size());
        QS_TRY(ev_batch<T>(sub.data(), (UINT)sub.size(), s[i], 1ULL << nq[i], st, vals.data()));
        for (size_t j = 0; j < sub.size(); ++j) {
            (*out)[i].x += coefs[i][plans[i].rest[j]].x * vals[j];
            (*out)[i].y += coefs[i][plans[i].rest[j]].y * vals[j];
        }
    }
    return QS_OK;
}

template int ev_weighted_many<double2>(const std::vector<const double2*>&, const std::vector<UINT>&,
    const std::vector<std::vector<PauliTerm>>&, const std::vector<const double2*>&, cudaStream_t, std::vector<double2>*);
template int ev_weighted_many<float2>(const std::vector<const float2*>&, const std::vector<UINT>&,
    const std::vector<std::vector<PauliTerm>>&, const std::vector<const double2*>&, cudaStream_t, std::vector<double2>*);

template int ev_weighted<double2>(const PauliTerm*, const double2*, UINT, const double2*, ITYPE, cudaStream_t, double*,
    bool);
template int ev_weighted<float2>(const PauliTerm*, const double2*, UINT, const float2*, ITYPE, cudaStream_t, double*,
    bool);

}  // namespace qs

// Shared argument checks of the batched Pauli entry points.
static int pauli_terms_from_masks(const QS_ITYPE* x_masks, const QS_ITYPE* z_masks, const QS_UINT* y_counts,
    QS_UINT term_count, QS_ITYPE dim, const char* what, std::vector<PauliTerm>* terms) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    terms->assign(term_count, PauliTerm{});
    for (UINT k = 0; k < term_count; ++k) {
        if ((x_masks[k] | z_masks[k]) >> n)
            return set_error(QS_ERR_INVALID_ARGUMENT, std::string(what) + ": mask beyond qubit count");
        (*terms)[k].x = x_masks[k];
        (*terms)[k].z = z_masks[k];
        (*terms)[k].nrot = y_counts[k];
        (*terms)[k].pivot = x_masks[k] ? (UINT)(63 - __builtin_clzll(x_masks[k])) : 0;
    }
    return QS_OK;
}

QS_API int qs_expectation_value_pauli_weighted(const QS_ITYPE* x_masks, const QS_ITYPE* z_masks,
    const QS_UINT* y_counts, const double* coefs, QS_UINT term_count, const void* state, QS_ITYPE dim, void* stream,
    double out[2]) {
    std::vector<PauliTerm> terms;
    QS_TRY(pauli_terms_from_masks(x_masks, z_masks, y_counts, term_count, dim, "expectation_value_pauli_weighted",
        &terms));
    return ev_weighted<double2>(terms.data(), (const double2*)coefs, term_count, (const double2*)state, dim,
        (cudaStream_t)stream, out, true);
}
QS_API int qs_expectation_value_pauli_weighted_c64(const QS_ITYPE* x_masks, const QS_ITYPE* z_masks,
    const QS_UINT* y_counts, const double* coefs, QS_UINT term_count, const void* state, QS_ITYPE dim, void* stream,
    double out[2]) {
    std::vector<PauliTerm> terms;
    QS_TRY(pauli_terms_from_masks(x_masks, z_masks, y_counts, term_count, dim,
        "expectation_value_pauli_weighted_c64", &terms));
    return ev_weighted<float2>(terms.data(), (const double2*)coefs, term_count, (const float2*)state, dim,
        (cudaStream_t)stream, out, true);
}

// Host-only plan of qs_expectation_value_pauli_weighted (no device work): passes over the state and
// how many terms each kind of evaluation takes.
QS_API int qs_expectation_value_pauli_weighted_plan(const QS_ITYPE* x_masks, const QS_ITYPE* z_masks,
    const QS_UINT* y_counts, QS_UINT term_count, QS_ITYPE dim, QS_UINT* passes_out, QS_UINT kind_counts[5]) {
    std::vector<PauliTerm> terms;
    QS_TRY(pauli_terms_from_masks(x_masks, z_masks, y_counts, term_count, dim,
        "expectation_value_pauli_weighted_plan", &terms));
    UINT n;
    QS_TRY(check_dim(dim, &n));
    EwPlan P;
    ew_build(terms.data(), term_count, n, &P);
    for (int i = 0; i < 5; ++i) kind_counts[i] = 0;
    for (const EvWTerm& e : P.desc) {
        const UINT code = e.packed >> 24;
        kind_counts[code == EW_Z ? 0 : code >= EW_REG ? 1 : code >= EW_ROW ? 3 : 2]++;
    }
    kind_counts[4] = (QS_UINT)P.rest.size();
    *passes_out = (QS_UINT)P.passes.size();
    return QS_OK;
}

QS_API int qs_set_expectation_specialized(int mode) {
    if (mode < 0 || mode > 2) return set_error(QS_ERR_INVALID_ARGUMENT, "expectation specialisation mode must be 0..2");
    g_ev_spec_mode = mode;
    return QS_OK;
}

QS_API int qs_expectation_specialized_info(unsigned long long* launches, double* compile_ms_last) {
    if (launches) *launches = (unsigned long long)g_ev_spec_launches.load();
    if (compile_ms_last) *compile_ms_last = g_ev_last_compile_ms.load();
    return QS_OK;
}

QS_API int qs_expectation_pass_source(const QS_ITYPE* x_masks, const QS_ITYPE* z_masks, const QS_UINT* y_counts,
    QS_UINT term_count, QS_ITYPE dim, QS_UINT pass, int c64, char* out, QS_ITYPE out_bytes, QS_ITYPE* needed) {
    std::vector<PauliTerm> terms;
    QS_TRY(pauli_terms_from_masks(x_masks, z_masks, y_counts, term_count, dim, "expectation_pass_source", &terms));
    UINT n;
    QS_TRY(check_dim(dim, &n));
    EwPlan P;
    ew_build(terms.data(), term_count, n, &P);
    if (pass >= P.passes.size()) return set_error(QS_ERR_INVALID_ARGUMENT, "expectation_pass_source: no such pass");
    const std::string src = ev_pass_source(P.desc.data() + P.passes[pass].first, P.passes[pass].count, c64 != 0, false);
    if (needed) *needed = src.size() + 1;
    if (out && out_bytes) {
        const size_t m = std::min<size_t>(src.size(), out_bytes - 1);
        std::memcpy(out, src.data(), m);
        out[m] = 0;
    }
    return QS_OK;
}
