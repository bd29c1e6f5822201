// Gate-by-gate complex128 kernels and their csim-named C ABI entry points.
//
// Every kernel is one streaming pass over the amplitudes it touches, with 128-bit loads/stores.
// Work items are enumerated by inserting zero bits at a sorted list of "positions" (targets and
// controls), as csim does with insert_zero_to_basis_index (csim/utility.hpp:14-19); the fixed bits
// (control values, target offsets) are then OR-ed in.  When every position is >= 5, 32 consecutive
// items of a warp touch 32 consecutive amplitudes, so each access is a fully used 512-byte run.
// Targets below 5 of an uncontrolled single-qubit gate use a warp-shuffle kernel instead: each lane
// loads its own amplitude (fully coalesced) and fetches its pair partner from lane ^ 2^t.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "qs_internal.cuh"

namespace qs {

constexpr int kThreads = 256;

struct Positions {
    int count;
    UINT pos[kMaxQubits];  // ascending; every position of a state fits
};

__device__ __forceinline__ ITYPE expand(ITYPE i, const Positions& p) {
#pragma unroll 4
    for (int j = 0; j < p.count; ++j) i = insert0(i, p.pos[j]);
    return i;
}

static Positions make_positions(std::vector<UINT> v) {
    std::sort(v.begin(), v.end());
    Positions p;
    p.count = (int)v.size();
    for (size_t i = 0; i < v.size(); ++i) p.pos[i] = v[i];
    return p;
}

// ---------------------------------------------------------------- functors
struct OpDense1 {
    Mat2 m;
    __device__ __forceinline__ void operator()(double2& a0, double2& a1) const {
        const double2 x = a0, y = a1;
        a0 = cfma(m.m[1], y, cmul(m.m[0], x));
        a1 = cfma(m.m[3], y, cmul(m.m[2], x));
    }
};
struct OpSwap {
    __device__ __forceinline__ void operator()(double2& a0, double2& a1) const {
        const double2 t = a0;
        a0 = a1;
        a1 = t;
    }
};
struct OpScale {
    double2 f;
    __device__ __forceinline__ void operator()(double2& a) const { a = cmul(f, a); }
};
struct OpNegate {
    __device__ __forceinline__ void operator()(double2& a) const { a = make_double2(-a.x, -a.y); }
};
struct OpZero {
    __device__ __forceinline__ void operator()(double2& a) const { a = make_double2(0., 0.); }
};

// ---------------------------------------------------------------- kernels
// One amplitude per item: index = expand(item) | fixed.
template <class OP, int ITEMS>
__global__ void __launch_bounds__(kThreads) k_single(
    double2* __restrict__ s, ITYPE items, const __grid_constant__ Positions pos, ITYPE fixed, OP op) {
    const ITYPE base = (ITYPE)blockIdx.x * (kThreads * ITEMS) + threadIdx.x;
    ITYPE idx[ITEMS];
    double2 v[ITEMS];
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const ITYPE it = base + (ITYPE)k * kThreads;
        idx[k] = expand(it, pos) | fixed;
        if (it < items) v[k] = ld_stream(s + idx[k]);
    }
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        if (base + (ITYPE)k * kThreads < items) {
            op(v[k]);
            st_stream(s + idx[k], v[k]);
        }
    }
}

// Two amplitudes per item: b = expand(item); (b | off0, b | off1).
template <class OP, int ITEMS>
__global__ void __launch_bounds__(kThreads) k_pair(
    double2* __restrict__ s, ITYPE items, const __grid_constant__ Positions pos, ITYPE off0, ITYPE off1, OP op) {
    const ITYPE base = (ITYPE)blockIdx.x * (kThreads * ITEMS) + threadIdx.x;
    ITYPE b[ITEMS];
    double2 v0[ITEMS], v1[ITEMS];
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const ITYPE it = base + (ITYPE)k * kThreads;
        b[k] = expand(it, pos);
        if (it < items) {
            v0[k] = ld_stream(s + (b[k] | off0));
            v1[k] = ld_stream(s + (b[k] | off1));
        }
    }
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        if (base + (ITYPE)k * kThreads < items) {
            op(v0[k], v1[k]);
            st_stream(s + (b[k] | off0), v0[k]);
            st_stream(s + (b[k] | off1), v1[k]);
        }
    }
}

// Two-qubit permutation (CNOT, SWAP) with a qubit below 5, where the pair enumeration of k_pair would
// use every 32-byte sector at half: each CTA owns 1024 amplitudes -- tile bits 0..8 are qubits 0..8
// and tile bit 9 is qubit `hq` (the pair's higher qubit when it is >= 9, else 9) -- loads them with
// fully used 512-byte runs into shared memory, and writes back amplitude x the amplitude at
// perm(x) (CNOT: x ^ t_bit when x has c_bit; SWAP: x with bits a, b exchanged).  Both qubits are tile
// bits, so every pair lies inside one tile.  Requires dim >= 1024.
constexpr int kPermTileBits = 10;
__global__ void __launch_bounds__(kThreads) k_perm2_tile(double2* __restrict__ s, UINT hq, UINT ca, UINT tb, int swap) {
    __shared__ double2 tile[1 << kPermTileBits];
    // global index of tile index x: bits 0..8 in place, tile bit 9 -> qubit hq, the block index in the
    // remaining bits (zeros inserted at 0..8 and at hq >= 9)
    const ITYPE base = insert0((ITYPE)blockIdx.x << 9, hq);
    auto gidx = [&](UINT x) { return base | (ITYPE)(x & 511u) | ((ITYPE)(x >> 9) << hq); };
    const UINT tid = threadIdx.x;
#pragma unroll
    for (int k = 0; k < (1 << kPermTileBits) / kThreads; ++k) {
        const UINT x = tid + (UINT)k * kThreads;
        tile[x] = ld_stream(s + gidx(x));
    }
    __syncthreads();
    // tile-local bit of a qubit: q itself below 9, 9 for hq
    const UINT lc = ca == hq ? 9u : ca, lt = tb == hq ? 9u : tb;
#pragma unroll
    for (int k = 0; k < (1 << kPermTileBits) / kThreads; ++k) {
        const UINT x = tid + (UINT)k * kThreads;
        UINT y = x;
        if (swap) {
            if (((x >> lc) ^ (x >> lt)) & 1u) y = x ^ (1u << lc) ^ (1u << lt);
        } else if ((x >> lc) & 1u) {
            y = x ^ (1u << lt);
        }
        st_stream(s + gidx(x), tile[y]);
    }
}

// Uncontrolled 2x2 on a target t < 5: lane-local amplitudes, partner through shuffles.
// Requires dim to be a multiple of kThreads * ITEMS.
template <int ITEMS>
__global__ void __launch_bounds__(kThreads) k_dense1_shfl(double2* __restrict__ s, UINT t, Mat2 m) {
    const ITYPE base = (ITYPE)blockIdx.x * (kThreads * ITEMS) + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int partner = lane ^ (1 << t);
    const bool hi = (lane >> t) & 1;
    const double2 self_c = hi ? m.m[3] : m.m[0];
    const double2 other_c = hi ? m.m[2] : m.m[1];
    double2 v[ITEMS];
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) v[k] = ld_stream(s + base + (ITYPE)k * kThreads);
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        double2 p;
        p.x = __shfl_sync(0xffffffffu, v[k].x, partner);
        p.y = __shfl_sync(0xffffffffu, v[k].y, partner);
        // row 0: m0 a0 + m1 a1 ; row 1: m2 a0 + m3 a1  (a_hi = self when hi)
        const double2 out = hi ? cfma(self_c, v[k], cmul(other_c, p)) : cfma(other_c, p, cmul(self_c, v[k]));
        st_stream(s + base + (ITYPE)k * kThreads, out);
    }
}

// Elementwise diagonal on one qubit.
template <int ITEMS>
__global__ void __launch_bounds__(kThreads) k_diag1(double2* __restrict__ s, ITYPE dim, UINT t, double2 d0, double2 d1) {
    const ITYPE base = (ITYPE)blockIdx.x * (kThreads * ITEMS) + threadIdx.x;
    double2 v[ITEMS];
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const ITYPE i = base + (ITYPE)k * kThreads;
        if (i < dim) v[k] = ld_stream(s + i);
    }
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const ITYPE i = base + (ITYPE)k * kThreads;
        if (i < dim) st_stream(s + i, cmul(((i >> t) & 1ULL) ? d1 : d0, v[k]));
    }
}

// Elementwise diagonal on k qubits: a[i] *= diag[bits of i at targets].
__global__ void __launch_bounds__(kThreads) k_diagK(double2* __restrict__ s, ITYPE dim, const __grid_constant__ Positions tl,
    const double2* __restrict__ diag) {
    const ITYPE stride = (ITYPE)gridDim.x * kThreads;
    for (ITYPE i = (ITYPE)blockIdx.x * kThreads + threadIdx.x; i < dim; i += stride) {
        UINT x = 0;
        for (int j = 0; j < tl.count; ++j) x |= (UINT)((i >> tl.pos[j]) & 1ULL) << j;
        st_stream(s + i, cmul(__ldg(diag + x), ld_stream(s + i)));
    }
}

// Two-qubit dense on quads: b = expand(item) | fixed, amplitudes b | off[j], j in 0..3.
template <int ITEMS>
__global__ void __launch_bounds__(kThreads) k_dense2(double2* __restrict__ s, ITYPE items, const __grid_constant__ Positions pos,
    ITYPE fixed, ITYPE m1, ITYPE m2, Mat4 m) {
    const ITYPE base = (ITYPE)blockIdx.x * (kThreads * ITEMS) + threadIdx.x;
    const ITYPE off[4] = {0, m1, m2, m1 | m2};
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const ITYPE it = base + (ITYPE)k * kThreads;
        if (it >= items) break;
        const ITYPE b = expand(it, pos) | fixed;
        double2 v[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) v[j] = ld_stream(s + (b | off[j]));
#pragma unroll
        for (int y = 0; y < 4; ++y) {
            double2 acc = cmul(m.m[y * 4], v[0]);
#pragma unroll
            for (int x = 1; x < 4; ++x) acc = cfma(m.m[y * 4 + x], v[x], acc);
            st_stream(s + (b | off[y]), acc);
        }
    }
}

// Pauli string P = i^{nY} X^x Z^z (csim/utility.cpp:12-43); P|i> = ph(i) |i ^ x>.
__device__ __forceinline__ double2 pauli_phase(ITYPE i, ITYPE zm, UINT nrot) {
    const UINT r = (nrot + 2u * (UINT)(__popcll(i & zm) & 1)) & 3u;
    return make_double2(r == 0 ? 1. : (r == 2 ? -1. : 0.), r == 1 ? 1. : (r == 3 ? -1. : 0.));
}

// rot == false: a <- P a.  rot == true: a <- (cos I + i sin P) a.
__global__ void __launch_bounds__(kThreads) k_pauli_x(double2* __restrict__ s, ITYPE items, UINT pivot,
    ITYPE xm, ITYPE zm, UINT nrot, bool rot, double c, double sn) {
    const ITYPE stride = (ITYPE)gridDim.x * kThreads;
    for (ITYPE p = (ITYPE)blockIdx.x * kThreads + threadIdx.x; p < items; p += stride) {
        const ITYPE b0 = insert0(p, pivot), b1 = b0 ^ xm;
        const double2 a0 = ld_stream(s + b0), a1 = ld_stream(s + b1);
        const double2 pa0 = cmul(pauli_phase(b1, zm, nrot), a1);  // (P a)[b0]
        const double2 pa1 = cmul(pauli_phase(b0, zm, nrot), a0);  // (P a)[b1]
        if (!rot) {
            st_stream(s + b0, pa0);
            st_stream(s + b1, pa1);
        } else {
            st_stream(s + b0, make_double2(c * a0.x - sn * pa0.y, c * a0.y + sn * pa0.x));
            st_stream(s + b1, make_double2(c * a1.x - sn * pa1.y, c * a1.y + sn * pa1.x));
        }
    }
}
__global__ void __launch_bounds__(kThreads) k_pauli_z(
    double2* __restrict__ s, ITYPE dim, ITYPE zm, bool rot, double c, double sn) {
    const ITYPE stride = (ITYPE)gridDim.x * kThreads;
    for (ITYPE i = (ITYPE)blockIdx.x * kThreads + threadIdx.x; i < dim; i += stride) {
        const double sg = (__popcll(i & zm) & 1) ? -1. : 1.;
        const double2 a = ld_stream(s + i);
        if (!rot) st_stream(s + i, make_double2(sg * a.x, sg * a.y));
        else st_stream(s + i, cmul(make_double2(c, sn * sg), a));
    }
}

// ---------------------------------------------------------------- launch helpers
static unsigned blocks_for(ITYPE items, int per_block) {
    return (unsigned)((items + per_block - 1) / per_block);
}
static unsigned grid_stride_blocks(ITYPE items) {
    ITYPE b = (items + kThreads - 1) / kThreads;
    ITYPE cap = (ITYPE)sm_count() * 16;
    return (unsigned)std::max<ITYPE>(1, std::min(b, cap));
}

int launch_dense1(UINT t, const Mat2& m, double2* s, ITYPE dim, const UINT* ctl, const UINT* cval,
    UINT nc, cudaStream_t st) {
    if (nc == 0 && t < 5 && dim >= (ITYPE)kThreads * 4) {
        k_dense1_shfl<4><<<blocks_for(dim, kThreads * 4), kThreads, 0, st>>>(s, t, m);
        return check_launch("k_dense1_shfl");
    }
    std::vector<UINT> p{t};
    ITYPE cm = 0;
    for (UINT i = 0; i < nc; ++i) {
        p.push_back(ctl[i]);
        if (cval[i]) cm |= 1ULL << ctl[i];
    }
    const ITYPE items = dim >> (1 + nc);
    k_pair<OpDense1, 2><<<blocks_for(items, kThreads * 2), kThreads, 0, st>>>(
        s, items, make_positions(p), cm, cm | (1ULL << t), OpDense1{m});
    return check_launch("k_pair<dense1>");
}

template <class OP>
static int launch_single(const std::vector<UINT>& p, ITYPE fixed, double2* s, ITYPE dim, OP op, cudaStream_t st) {
    const ITYPE items = dim >> p.size();
    k_single<OP, 4><<<blocks_for(items, kThreads * 4), kThreads, 0, st>>>(s, items, make_positions(p), fixed, op);
    return check_launch("k_single");
}

int launch_diag1(UINT t, double2 d0, double2 d1, double2* s, ITYPE dim, cudaStream_t st) {
    k_diag1<4><<<blocks_for(dim, kThreads * 4), kThreads, 0, st>>>(s, dim, t, d0, d1);
    return check_launch("k_diag1");
}

int launch_dense2(UINT t1, UINT t2, const Mat4& m, double2* s, ITYPE dim, const UINT* ctl,
    const UINT* cval, UINT nc, cudaStream_t st) {
    std::vector<UINT> p{t1, t2};
    ITYPE cm = 0;
    for (UINT i = 0; i < nc; ++i) {
        p.push_back(ctl[i]);
        if (cval[i]) cm |= 1ULL << ctl[i];
    }
    const ITYPE items = dim >> (2 + nc);
    k_dense2<2><<<blocks_for(items, kThreads * 2), kThreads, 0, st>>>(
        s, items, make_positions(p), cm, 1ULL << t1, 1ULL << t2, m);
    return check_launch("k_dense2");
}

// Register-resident k-qubit dense (3 <= K <= 6): one coset per thread.  The thread issues its 2^K
// independent 128-bit loads at once, multiplies in registers, and stores; consecutive threads own
// consecutive cosets, so accesses are coalesced whenever the lowest target is >= 5.  The matrix is
// read with warp-uniform addresses: from the kernel parameter space (constant bank) for K <= 5, from
// global memory through L1 for K = 6 (64 KiB exceeds the parameter limit).
template <int K>
struct DenseKArgs {
    ITYPE mask[1 << K];           // offset of matrix index x (bit j <-> target j)
    double2 m[K <= 5 ? (1 << (2 * K)) : 1];
};

template <int K>
__global__ void __launch_bounds__(128) k_denseK_reg(double2* __restrict__ s, ITYPE cosets,
    const __grid_constant__ Positions pos, ITYPE fixed, const __grid_constant__ DenseKArgs<K> a,
    const double2* __restrict__ gm) {
    constexpr int D = 1 << K;
    const ITYPE c = (ITYPE)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cosets) return;
    const ITYPE base = expand(c, pos) | fixed;
    double2 v[D];
#pragma unroll
    for (int x = 0; x < D; ++x) v[x] = ld_stream(s + (base | a.mask[x]));
#pragma unroll 4
    for (int y = 0; y < D; ++y) {
        double2 acc = make_double2(0., 0.);
#pragma unroll
        for (int x = 0; x < D; ++x) {
            const double2 mv = (K <= 5) ? a.m[(K <= 5 ? y * D + x : 0)] : __ldg(gm + y * D + x);
            acc = cfma(mv, v[x], acc);
        }
        st_stream(s + (base | a.mask[y]), acc);
    }
}

// k-qubit dense, register-blocked (used for k = 6, where a coset per thread in registers would spill):
// a persistent CTA (256 threads) keeps the matrix transposed in shared memory (UT[x][y] = U[y][x])
// and works through tiles of 16 CP cosets: the tile's amplitudes X[x][c] arrive by cp.async, thread
// (ty, tc) = (tid % 16, tid / 16) accumulates outputs y = ty + 16 j (j < 2^k / 16) of cosets
// c = tc + 16 i (i < CP) -- per x it reads 2^k / 16 matrix entries (the half-warps share them) and CP
// amplitudes for 2^k CP / 16 complex FMAs -- writes them back over X, and the tile leaves with the
// same coalesced pattern it came in.  k = 6: CP = 2 (2 CTAs per SM) 33 ms at 30 qubits; CP = 4
// (1 CTA per SM) 38 ms; the earlier one-output-per-thread shared-memory kernel 64 ms.
constexpr int kBlkThreads = 256;

template <int K, int CP>
__global__ void __launch_bounds__(kBlkThreads, CP <= 2 ? 2 : 1) k_denseK_blk(double2* __restrict__ s, ITYPE cosets,
    const __grid_constant__ Positions pos, ITYPE fixed, const double2* __restrict__ gm,
    const ITYPE* __restrict__ gmask) {
    constexpr int D = 1 << K, R = D / 16, C = 16 * CP;
    extern __shared__ double2 blk_smem[];
    double2* UT = blk_smem;       // D x D
    double2* X = blk_smem + D * D;  // D x C, then the outputs
    __shared__ ITYPE mask[D];
    const int tid = threadIdx.x, ty = tid & 15, tc = tid >> 4;
    for (int i = tid; i < D * D; i += kBlkThreads) UT[(i % D) * D + i / D] = __ldg(gm + i);
    for (int i = tid; i < D; i += kBlkThreads) mask[i] = gmask[i];
    __syncthreads();
    const ITYPE ntiles = (cosets + C - 1) / C;
    for (ITYPE T = blockIdx.x; T < ntiles; T += gridDim.x) {
        const ITYPE c0 = T * C;
        for (int i = tid; i < D * C; i += kBlkThreads) {  // X[x][c], c fastest: a warp reads 32 cosets
            const int x = i / C, c = i % C;
            if (c0 + c < cosets) {
                const unsigned dst = (unsigned)__cvta_generic_to_shared(X + i);
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst),
                    "l"(s + ((expand(c0 + c, pos) | fixed) | mask[x])) : "memory");
            }
        }
        asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
        __syncthreads();
        double2 acc[R][CP];
#pragma unroll
        for (int j = 0; j < R; ++j)
#pragma unroll
            for (int i = 0; i < CP; ++i) acc[j][i] = make_double2(0., 0.);
#pragma unroll 4
        for (int x = 0; x < D; ++x) {
            double2 b[CP];
#pragma unroll
            for (int i = 0; i < CP; ++i) b[i] = X[x * C + tc + 16 * i];
#pragma unroll
            for (int j = 0; j < R; ++j) {
                const double2 aj = UT[x * D + ty + 16 * j];
#pragma unroll
                for (int i = 0; i < CP; ++i) acc[j][i] = cfma(aj, b[i], acc[j][i]);
            }
        }
        __syncthreads();  // every X read done: the outputs go over it
#pragma unroll
        for (int j = 0; j < R; ++j)
#pragma unroll
            for (int i = 0; i < CP; ++i) X[(ty + 16 * j) * C + tc + 16 * i] = acc[j][i];
        __syncthreads();
        for (int i = tid; i < D * C; i += kBlkThreads) {
            const int y = i / C, c = i % C;
            if (c0 + c < cosets) st_stream(s + ((expand(c0 + c, pos) | fixed) | mask[y]), X[i]);
        }
        __syncthreads();  // the next tile's copies overwrite X
    }
}

template <int K, int CP>
static int launch_denseK_blk(const UINT* tl, const double* matrix, double2* s, const Positions& pos, ITYPE fixed,
    ITYPE cosets, cudaStream_t st) {
    QS_TRY(refuse_if_capturing("a dense gate of 6 qubits"));
    constexpr int D = 1 << K, kBlkCosets = 16 * CP;
    static std::mutex mu;
    static std::vector<char> ready;
    int dev = 0;
    QS_CUDA_CHECK(cudaGetDevice(&dev));
    const size_t smem = sizeof(double2) * ((size_t)D * D + (size_t)D * kBlkCosets);
    {
        std::lock_guard<std::mutex> lock(mu);
        if ((int)ready.size() <= dev) ready.resize(dev + 1, 0);
        if (!ready[dev]) {
            QS_CUDA_CHECK(cudaFuncSetAttribute(k_denseK_blk<K, CP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                (int)smem));
            ready[dev] = 1;
        }
    }
    std::vector<ITYPE> mk(D, 0);
    for (int x = 0; x < D; ++x)
        for (int j = 0; j < K; ++j)
            if ((x >> j) & 1) mk[x] |= 1ULL << tl[j];
    const size_t mbytes = (size_t)16 * D * D;
    void* buf = nullptr;
    QS_TRY(scratch(st, mbytes + sizeof(ITYPE) * D + 256, &buf));
    ITYPE* dmask = (ITYPE*)((char*)buf + mbytes);
    QS_CUDA_CHECK(cudaMemcpyAsync(buf, matrix, mbytes, cudaMemcpyHostToDevice, st));
    QS_CUDA_CHECK(cudaMemcpyAsync(dmask, mk.data(), sizeof(ITYPE) * D, cudaMemcpyHostToDevice, st));
    const ITYPE ntiles = (cosets + kBlkCosets - 1) / kBlkCosets;
    const unsigned grid = (unsigned)std::min<ITYPE>(ntiles, (ITYPE)sm_count() * (CP <= 2 ? 2 : 1));
    k_denseK_blk<K, CP><<<grid, kBlkThreads, smem, st>>>(s, cosets, pos, fixed, (const double2*)buf, dmask);
    return check_launch("k_denseK_blk");
}

template <int K>
static int launch_denseK_reg(const UINT* tl, const double* matrix, double2* s, ITYPE dim, const Positions& pos,
    ITYPE fixed, ITYPE cosets, cudaStream_t st) {
    constexpr int D = 1 << K;
    static thread_local DenseKArgs<K> a;  // large parameter block, filled on the host
    for (int x = 0; x < D; ++x) {
        ITYPE mk = 0;
        for (int j = 0; j < K; ++j)
            if ((x >> j) & 1) mk |= 1ULL << tl[j];
        a.mask[x] = mk;
    }
    const double2* gm = nullptr;
    if (K <= 5) {
        for (int i = 0; i < D * D; ++i) a.m[i] = make_double2(matrix[2 * i], matrix[2 * i + 1]);
    } else {
        QS_TRY(refuse_if_capturing("a dense gate of 6 qubits"));
        void* buf = nullptr;
        QS_TRY(scratch(st, (size_t)16 * D * D, &buf));
        QS_CUDA_CHECK(cudaMemcpyAsync(buf, matrix, (size_t)16 * D * D, cudaMemcpyHostToDevice, st));
        gm = (const double2*)buf;
    }
    k_denseK_reg<K><<<blocks_for(cosets, 128), 128, 0, st>>>(s, cosets, pos, fixed, a, gm);
    return check_launch("k_denseK_reg");
}

// k-qubit dense for 7 <= k <= kMaxDenseTargets: the matrix (4^k entries, 256 KiB at k = 7, 256 MiB at
// k = 12) does not fit on chip and streams from L2 / HBM, transposed on the host (UT[x][y] = U[y][x]) so
// that the lanes of a warp, which hold consecutive output rows y, read consecutive entries.  A CTA
// stages a group of kGenAmps / 2^k cosets (kGenAmps amplitudes) in shared memory as X[c][x]; thread t
// owns the outputs o = t + kGenThreads j of the group (coset o >> k, row o & (2^k - 1)), keeps them in
// registers until every thread has read the group, then writes them over it and the group leaves.
// Every group re-reads the whole matrix, so this path is bound by L2 bandwidth, not by HBM.
constexpr int kGenThreads = 256, kGenAmps = 4096, kGenOut = kGenAmps / kGenThreads;

__global__ void __launch_bounds__(kGenThreads) k_denseK_gen(double2* __restrict__ s, ITYPE cosets,
    const __grid_constant__ Positions pos, ITYPE fixed, int K, const double2* __restrict__ ut,
    const ITYPE* __restrict__ gmask) {
    extern __shared__ double2 gen_smem[];  // X[c * 2^K + x], kGenAmps entries
    const int D = 1 << K, CP = kGenAmps >> K;
    const int tid = threadIdx.x;
    const ITYPE groups = (cosets + CP - 1) / CP;
    for (ITYPE g = blockIdx.x; g < groups; g += gridDim.x) {
        const ITYPE c0 = g * (ITYPE)CP;
        for (int i = tid; i < kGenAmps; i += kGenThreads) {
            const int c = i >> K, x = i & (D - 1);
            if (c0 + c < cosets) {
                const unsigned dst = (unsigned)__cvta_generic_to_shared(gen_smem + i);
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst),
                    "l"(s + ((expand(c0 + c, pos) | fixed) | __ldg(gmask + x))) : "memory");
            }
        }
        asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
        __syncthreads();
        double2 acc[kGenOut];
#pragma unroll
        for (int j = 0; j < kGenOut; ++j) acc[j] = make_double2(0., 0.);
        for (int x = 0; x < D; ++x) {
            const double2* row = ut + (size_t)x * D;
#pragma unroll
            for (int j = 0; j < kGenOut; ++j) {
                const int o = tid + kGenThreads * j;
                acc[j] = cfma(__ldg(row + (o & (D - 1))), gen_smem[((o >> K) << K) + x], acc[j]);
            }
        }
        __syncthreads();  // every read of the group done: the outputs go over it
#pragma unroll
        for (int j = 0; j < kGenOut; ++j) gen_smem[tid + kGenThreads * j] = acc[j];
        __syncthreads();
        for (int i = tid; i < kGenAmps; i += kGenThreads) {
            const int c = i >> K, y = i & (D - 1);
            if (c0 + c < cosets) st_stream(s + ((expand(c0 + c, pos) | fixed) | __ldg(gmask + y)), gen_smem[i]);
        }
        __syncthreads();  // the next group's copies overwrite X
    }
}

static int launch_denseK_gen(const UINT* tl, UINT k, const double* matrix, double2* s, const Positions& pos,
    ITYPE fixed, ITYPE cosets, cudaStream_t st) {
    QS_TRY(refuse_if_capturing("a dense gate of 7 or more qubits"));
    const size_t D = size_t(1) << k;
    std::vector<double2> ut(D * D);
    for (size_t y = 0; y < D; ++y)
        for (size_t x = 0; x < D; ++x) ut[x * D + y] = make_double2(matrix[2 * (y * D + x)], matrix[2 * (y * D + x) + 1]);
    std::vector<ITYPE> mk(D, 0);
    for (size_t x = 0; x < D; ++x)
        for (UINT j = 0; j < k; ++j)
            if ((x >> j) & 1) mk[x] |= 1ULL << tl[j];
    const size_t ubytes = sizeof(double2) * D * D;
    void* buf = nullptr;
    QS_TRY(scratch(st, ubytes + sizeof(ITYPE) * D + 256, &buf));
    ITYPE* dmask = (ITYPE*)((char*)buf + ubytes);
    QS_CUDA_CHECK(cudaMemcpyAsync(buf, ut.data(), ubytes, cudaMemcpyHostToDevice, st));
    QS_CUDA_CHECK(cudaMemcpyAsync(dmask, mk.data(), sizeof(ITYPE) * D, cudaMemcpyHostToDevice, st));
    const int smem = (int)(sizeof(double2) * kGenAmps);
    static std::mutex mu;
    static std::vector<char> ready;
    int dev = 0;
    QS_CUDA_CHECK(cudaGetDevice(&dev));
    {
        std::lock_guard<std::mutex> lock(mu);
        if ((int)ready.size() <= dev) ready.resize(dev + 1, 0);
        if (!ready[dev]) {
            QS_CUDA_CHECK(cudaFuncSetAttribute(k_denseK_gen, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            ready[dev] = 1;
        }
    }
    const ITYPE groups = (cosets + (kGenAmps >> k) - 1) / (ITYPE)(kGenAmps >> k);
    const unsigned grid = (unsigned)std::max<ITYPE>(1, std::min<ITYPE>(groups, (ITYPE)sm_count() * 3));
    k_denseK_gen<<<grid, kGenThreads, smem, st>>>(s, cosets, pos, fixed, (int)k, (const double2*)buf, dmask);
    return check_launch("k_denseK_gen");
}

int launch_denseK(const UINT* tl, UINT k, const double* matrix, double2* s, ITYPE dim,
    const UINT* ctl, const UINT* cval, UINT nc, cudaStream_t st) {
    std::vector<UINT> p(tl, tl + k);
    ITYPE cm = 0;
    for (UINT i = 0; i < nc; ++i) {
        p.push_back(ctl[i]);
        if (cval[i]) cm |= 1ULL << ctl[i];
    }
    const ITYPE cosets = dim >> (k + nc);
    const Positions pos = make_positions(p);
    switch (k) {
        case 3: return launch_denseK_reg<3>(tl, matrix, s, dim, pos, cm, cosets, st);
        case 4: return launch_denseK_reg<4>(tl, matrix, s, dim, pos, cm, cosets, st);
        case 5: return launch_denseK_reg<5>(tl, matrix, s, dim, pos, cm, cosets, st);
        case 6: return launch_denseK_blk<6, 2>(tl, matrix, s, pos, cm, cosets, st);  // 64 register amplitudes would spill
        default:
            if (k >= 7 && k <= (UINT)kMaxDenseTargets) return launch_denseK_gen(tl, k, matrix, s, pos, cm, cosets, st);
            return set_error(QS_ERR_NOT_SUPPORTED, "dense gate: 3..12 targets expected here");
    }
}

static Mat2 mat2_from(const double* m) {
    Mat2 r;
    for (int i = 0; i < 4; ++i) r.m[i] = make_double2(m[2 * i], m[2 * i + 1]);
    return r;
}
static Mat4 mat4_from(const double* m) {
    Mat4 r;
    for (int i = 0; i < 16; ++i) r.m[i] = make_double2(m[2 * i], m[2 * i + 1]);
    return r;
}

// Reference matrices: csim/constant.cpp:4-30.
static const double kInvSqrt2 = 0.70710678118654752440;

int apply_pauli(const UINT* tl, const UINT* ids, UINT cnt, bool rot, double angle, double2* s, ITYPE dim,
    cudaStream_t st) {
    ITYPE xm = 0, zm = 0;
    UINT nrot = 0, pivot = 0;
    for (UINT i = 0; i < cnt; ++i) {
        const ITYPE b = 1ULL << tl[i];
        if (ids[i] == 1) {
            xm ^= b;
            pivot = tl[i];
        } else if (ids[i] == 2) {
            xm ^= b;
            zm ^= b;
            ++nrot;
            pivot = tl[i];
        } else if (ids[i] == 3) {
            zm ^= b;
        } else if (ids[i] != 0) {
            return set_error(QS_ERR_INVALID_ARGUMENT, "Pauli id must be 0..3");
        }
    }
    const double c = std::cos(angle / 2), sn = std::sin(angle / 2);
    if (xm == 0) {
        k_pauli_z<<<grid_stride_blocks(dim), kThreads, 0, st>>>(s, dim, zm, rot, c, sn);
        return check_launch("k_pauli_z");
    }
    k_pauli_x<<<grid_stride_blocks(dim / 2), kThreads, 0, st>>>(s, dim / 2, pivot, xm, zm, nrot, rot, c, sn);
    return check_launch("k_pauli_x");
}

}  // namespace qs

using namespace qs;

#define STATE_ARGS void *state, QS_ITYPE dim, void *stream
#define S2 ((double2*)state)
#define ST ((cudaStream_t)stream)

extern "C" {

QS_API int qs_single_qubit_dense_matrix_gate(QS_UINT t, const double matrix[8], STATE_ARGS) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    QS_TRY(check_target(t, n, "single_qubit_dense_matrix_gate"));
    return launch_dense1(t, mat2_from(matrix), S2, dim, nullptr, nullptr, 0, ST);
}

QS_API int qs_single_qubit_diagonal_matrix_gate(QS_UINT t, const double d[4], STATE_ARGS) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    QS_TRY(check_target(t, n, "single_qubit_diagonal_matrix_gate"));
    return launch_diag1(t, make_double2(d[0], d[1]), make_double2(d[2], d[3]), S2, dim, ST);
}

QS_API int qs_single_qubit_phase_gate(QS_UINT t, const double phase[2], STATE_ARGS) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    QS_TRY(check_target(t, n, "single_qubit_phase_gate"));
    return launch_single({t}, 1ULL << t, S2, dim, OpScale{make_double2(phase[0], phase[1])}, ST);
}

QS_API int qs_RX_gate(QS_UINT t, double angle, STATE_ARGS) {
    const double c = std::cos(angle / 2), s = std::sin(angle / 2);
    const double m[8] = {c, 0, 0, s, 0, s, c, 0};
    return qs_single_qubit_dense_matrix_gate(t, m, state, dim, stream);
}
QS_API int qs_RY_gate(QS_UINT t, double angle, STATE_ARGS) {
    const double c = std::cos(angle / 2), s = std::sin(angle / 2);
    const double m[8] = {c, 0, s, 0, -s, 0, c, 0};
    return qs_single_qubit_dense_matrix_gate(t, m, state, dim, stream);
}
QS_API int qs_RZ_gate(QS_UINT t, double angle, STATE_ARGS) {
    const double c = std::cos(angle / 2), s = std::sin(angle / 2);
    const double d[4] = {c, s, c, -s};
    return qs_single_qubit_diagonal_matrix_gate(t, d, state, dim, stream);
}

QS_API int qs_X_gate(QS_UINT t, STATE_ARGS) {
    const double m[8] = {0, 0, 1, 0, 1, 0, 0, 0};
    return qs_single_qubit_dense_matrix_gate(t, m, state, dim, stream);
}
QS_API int qs_Y_gate(QS_UINT t, STATE_ARGS) {
    const double m[8] = {0, 0, 0, -1, 0, 1, 0, 0};
    return qs_single_qubit_dense_matrix_gate(t, m, state, dim, stream);
}
QS_API int qs_Z_gate(QS_UINT t, STATE_ARGS) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    QS_TRY(check_target(t, n, "Z_gate"));
    return launch_single({t}, 1ULL << t, S2, dim, OpNegate{}, ST);
}
QS_API int qs_H_gate(QS_UINT t, STATE_ARGS) {
    const double h = kInvSqrt2;
    const double m[8] = {h, 0, h, 0, h, 0, -h, 0};
    return qs_single_qubit_dense_matrix_gate(t, m, state, dim, stream);
}
QS_API int qs_S_gate(QS_UINT t, STATE_ARGS) {
    const double ph[2] = {0, 1};
    return qs_single_qubit_phase_gate(t, ph, state, dim, stream);
}
QS_API int qs_Sdag_gate(QS_UINT t, STATE_ARGS) {
    const double ph[2] = {0, -1};
    return qs_single_qubit_phase_gate(t, ph, state, dim, stream);
}
QS_API int qs_T_gate(QS_UINT t, STATE_ARGS) {
    const double ph[2] = {kInvSqrt2, kInvSqrt2};
    return qs_single_qubit_phase_gate(t, ph, state, dim, stream);
}
QS_API int qs_Tdag_gate(QS_UINT t, STATE_ARGS) {
    const double ph[2] = {kInvSqrt2, -kInvSqrt2};
    return qs_single_qubit_phase_gate(t, ph, state, dim, stream);
}
QS_API int qs_sqrtX_gate(QS_UINT t, STATE_ARGS) {
    const double m[8] = {0.5, 0.5, 0.5, -0.5, 0.5, -0.5, 0.5, 0.5};
    return qs_single_qubit_dense_matrix_gate(t, m, state, dim, stream);
}
QS_API int qs_sqrtXdag_gate(QS_UINT t, STATE_ARGS) {
    const double m[8] = {0.5, -0.5, 0.5, 0.5, 0.5, 0.5, 0.5, -0.5};
    return qs_single_qubit_dense_matrix_gate(t, m, state, dim, stream);
}
QS_API int qs_sqrtY_gate(QS_UINT t, STATE_ARGS) {
    const double m[8] = {0.5, 0.5, -0.5, -0.5, 0.5, 0.5, 0.5, 0.5};
    return qs_single_qubit_dense_matrix_gate(t, m, state, dim, stream);
}
QS_API int qs_sqrtYdag_gate(QS_UINT t, STATE_ARGS) {
    const double m[8] = {0.5, -0.5, 0.5, -0.5, -0.5, 0.5, 0.5, -0.5};
    return qs_single_qubit_dense_matrix_gate(t, m, state, dim, stream);
}
QS_API int qs_P0_gate(QS_UINT t, STATE_ARGS) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    QS_TRY(check_target(t, n, "P0_gate"));
    return launch_single({t}, 1ULL << t, S2, dim, OpZero{}, ST);
}
QS_API int qs_P1_gate(QS_UINT t, STATE_ARGS) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    QS_TRY(check_target(t, n, "P1_gate"));
    return launch_single({t}, 0, S2, dim, OpZero{}, ST);
}

QS_API int qs_CNOT_gate(QS_UINT c, QS_UINT t, STATE_ARGS) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    const UINT l[2] = {c, t};
    QS_TRY(check_distinct(l, 2, n, "CNOT_gate"));
    if (std::min(c, t) < 5 && dim >= (1ULL << kPermTileBits)) {
        const UINT hq = std::max(std::max(c, t), 9u);
        k_perm2_tile<<<(unsigned)(dim >> kPermTileBits), kThreads, 0, ST>>>(S2, hq, c, t, 0);
        return check_launch("k_perm2_tile<CNOT>");
    }
    const ITYPE cm = 1ULL << c;
    const ITYPE items = dim >> 2;
    k_pair<OpSwap, 2><<<blocks_for(items, kThreads * 2), kThreads, 0, ST>>>(
        S2, items, make_positions({c, t}), cm, cm | (1ULL << t), OpSwap{});
    return check_launch("k_pair<CNOT>");
}
QS_API int qs_CZ_gate(QS_UINT c, QS_UINT t, STATE_ARGS) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    const UINT l[2] = {c, t};
    QS_TRY(check_distinct(l, 2, n, "CZ_gate"));
    return launch_single({c, t}, (1ULL << c) | (1ULL << t), S2, dim, OpNegate{}, ST);
}
QS_API int qs_SWAP_gate(QS_UINT a, QS_UINT b, STATE_ARGS) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    const UINT l[2] = {a, b};
    QS_TRY(check_distinct(l, 2, n, "SWAP_gate"));
    if (std::min(a, b) < 5 && dim >= (1ULL << kPermTileBits)) {
        const UINT hq = std::max(std::max(a, b), 9u);
        k_perm2_tile<<<(unsigned)(dim >> kPermTileBits), kThreads, 0, ST>>>(S2, hq, a, b, 1);
        return check_launch("k_perm2_tile<SWAP>");
    }
    const ITYPE items = dim >> 2;
    k_pair<OpSwap, 2><<<blocks_for(items, kThreads * 2), kThreads, 0, ST>>>(
        S2, items, make_positions({a, b}), 1ULL << a, 1ULL << b, OpSwap{});
    return check_launch("k_pair<SWAP>");
}

QS_API int qs_double_qubit_dense_matrix_gate_c(QS_UINT t1, QS_UINT t2, const double matrix[32], STATE_ARGS) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    const UINT l[2] = {t1, t2};
    QS_TRY(check_distinct(l, 2, n, "double_qubit_dense_matrix_gate_c"));
    return launch_dense2(t1, t2, mat4_from(matrix), S2, dim, nullptr, nullptr, 0, ST);
}

static int dense_dispatch(const UINT* tl, UINT k, const double* matrix, const UINT* ctl, const UINT* cval,
    UINT nc, double2* s, ITYPE dim, cudaStream_t st, const char* what) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (k < 1 || k > (UINT)kMaxDenseTargets)
        return set_error(QS_ERR_NOT_SUPPORTED, std::string(what) + ": target count must be 1..12");
    std::vector<UINT> all(tl, tl + k);
    for (UINT i = 0; i < nc; ++i) {
        if (cval[i] > 1) return set_error(QS_ERR_INVALID_ARGUMENT, "control value must be 0 or 1");
        all.push_back(ctl[i]);
    }
    QS_TRY(check_distinct(all.data(), (UINT)all.size(), n, what));
    if (k == 1) return launch_dense1(tl[0], mat2_from(matrix), s, dim, ctl, cval, nc, st);
    if (k == 2) return launch_dense2(tl[0], tl[1], mat4_from(matrix), s, dim, ctl, cval, nc, st);
    return launch_denseK(tl, k, matrix, s, dim, ctl, cval, nc, st);
}

QS_API int qs_multi_qubit_dense_matrix_gate(const QS_UINT* tl, QS_UINT k, const double* matrix, STATE_ARGS) {
    return dense_dispatch(tl, k, matrix, nullptr, nullptr, 0, S2, dim, ST, "multi_qubit_dense_matrix_gate");
}
QS_API int qs_single_qubit_control_single_qubit_dense_matrix_gate(
    QS_UINT c, QS_UINT cv, QS_UINT t, const double matrix[8], STATE_ARGS) {
    return dense_dispatch(&t, 1, matrix, &c, &cv, 1, S2, dim, ST,
        "single_qubit_control_single_qubit_dense_matrix_gate");
}
QS_API int qs_multi_qubit_control_single_qubit_dense_matrix_gate(const QS_UINT* cl, const QS_UINT* cv,
    QS_UINT nc, QS_UINT t, const double matrix[8], STATE_ARGS) {
    return dense_dispatch(&t, 1, matrix, cl, cv, nc, S2, dim, ST,
        "multi_qubit_control_single_qubit_dense_matrix_gate");
}
QS_API int qs_multi_qubit_control_multi_qubit_dense_matrix_gate(const QS_UINT* cl, const QS_UINT* cv,
    QS_UINT nc, const QS_UINT* tl, QS_UINT nt, const double* matrix, STATE_ARGS) {
    return dense_dispatch(tl, nt, matrix, cl, cv, nc, S2, dim, ST,
        "multi_qubit_control_multi_qubit_dense_matrix_gate");
}

QS_API int qs_multi_qubit_diagonal_matrix_gate(const QS_UINT* tl, QS_UINT k, const double* diag, STATE_ARGS) {
    QS_TRY(refuse_if_capturing("a multi-qubit diagonal gate"));
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (k < 1 || k > 20) return set_error(QS_ERR_NOT_SUPPORTED, "multi_qubit_diagonal_matrix_gate: 1..20 targets");
    QS_TRY(check_distinct(tl, k, n, "multi_qubit_diagonal_matrix_gate"));
    const size_t bytes = (size_t)16 << k;
    void* buf = nullptr;
    QS_TRY(scratch(ST, bytes, &buf));
    QS_CUDA_CHECK(cudaMemcpyAsync(buf, diag, bytes, cudaMemcpyHostToDevice, ST));
    Positions p;
    p.count = (int)k;
    for (UINT i = 0; i < k; ++i) p.pos[i] = tl[i];  // kept in list order: bit j <-> tl[j]
    k_diagK<<<grid_stride_blocks(dim), kThreads, 0, ST>>>(S2, dim, p, (const double2*)buf);
    return check_launch("k_diagK");
}

QS_API int qs_multi_qubit_Pauli_gate_partial_list(const QS_UINT* tl, const QS_UINT* ids, QS_UINT cnt, STATE_ARGS) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    QS_TRY(check_distinct(tl, cnt, n, "multi_qubit_Pauli_gate_partial_list"));
    return apply_pauli(tl, ids, cnt, false, 0., S2, dim, ST);
}
QS_API int qs_multi_qubit_Pauli_rotation_gate_partial_list(
    const QS_UINT* tl, const QS_UINT* ids, QS_UINT cnt, double angle, STATE_ARGS) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    QS_TRY(check_distinct(tl, cnt, n, "multi_qubit_Pauli_rotation_gate_partial_list"));
    return apply_pauli(tl, ids, cnt, true, angle, S2, dim, ST);
}

// Whole-list forms (update_ops_pauli_multi.cpp): id j acts on qubit j.
static int whole_list_targets(QS_UINT count, ITYPE dim, const char* what, std::vector<UINT>* tl) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (count > n) return set_error(QS_ERR_INVALID_ARGUMENT, std::string(what) + ": more Pauli ids than qubits");
    tl->resize(count);
    for (UINT j = 0; j < count; ++j) (*tl)[j] = j;
    return QS_OK;
}
QS_API int qs_multi_qubit_Pauli_gate_whole_list(const QS_UINT* ids, QS_UINT count, STATE_ARGS) {
    std::vector<UINT> tl;
    QS_TRY(whole_list_targets(count, dim, "multi_qubit_Pauli_gate_whole_list", &tl));
    return apply_pauli(tl.data(), ids, count, false, 0., S2, dim, ST);
}
QS_API int qs_multi_qubit_Pauli_rotation_gate_whole_list(const QS_UINT* ids, QS_UINT count, double angle,
    STATE_ARGS) {
    std::vector<UINT> tl;
    QS_TRY(whole_list_targets(count, dim, "multi_qubit_Pauli_rotation_gate_whole_list", &tl));
    return apply_pauli(tl.data(), ids, count, true, angle, S2, dim, ST);
}

QS_API int qs_single_qubit_Pauli_gate(QS_UINT t, QS_UINT id, STATE_ARGS) {
    switch (id) {
        case 0: {
            UINT n;
            QS_TRY(check_dim(dim, &n));
            return check_target(t, n, "single_qubit_Pauli_gate");
        }
        case 1: return qs_X_gate(t, state, dim, stream);
        case 2: return qs_Y_gate(t, state, dim, stream);
        case 3: return qs_Z_gate(t, state, dim, stream);
        default: return set_error(QS_ERR_INVALID_ARGUMENT, "single_qubit_Pauli_gate: Pauli id must be 0..3");
    }
}
QS_API int qs_single_qubit_Pauli_rotation_gate(QS_UINT t, QS_UINT id, double angle, STATE_ARGS) {
    switch (id) {
        case 0: {
            UINT n;
            QS_TRY(check_dim(dim, &n));
            return check_target(t, n, "single_qubit_Pauli_rotation_gate");
        }
        case 1: return qs_RX_gate(t, angle, state, dim, stream);
        case 2: return qs_RY_gate(t, angle, state, dim, stream);
        case 3: return qs_RZ_gate(t, angle, state, dim, stream);
        default: return set_error(QS_ERR_INVALID_ARGUMENT, "single_qubit_Pauli_rotation_gate: Pauli id must be 0..3");
    }
}

QS_API int qs_single_qubit_control_multi_qubit_dense_matrix_gate(QS_UINT c, QS_UINT cv, const QS_UINT* tl, QS_UINT k,
    const double* matrix, STATE_ARGS) {
    const UINT ctl[1] = {c}, val[1] = {cv};
    return dense_dispatch(tl, k, matrix, ctl, val, 1, S2, dim, ST, "single_qubit_control_multi_qubit_dense_matrix_gate");
}

// The controlled diagonal as one diagonal over (targets, controls): entry y + 2^k c is diagonal[y] where the
// control bits c spell the control values and 1 elsewhere (update_ops_matrix_diagonal_multi.cpp:60-112
// multiplies only the amplitudes whose control bits match).
QS_API int qs_multi_qubit_control_multi_qubit_diagonal_matrix_gate(const QS_UINT* ctl, const QS_UINT* cval, QS_UINT nc,
    const QS_UINT* tl, QS_UINT k, const double* diag, STATE_ARGS) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    const UINT total = k + nc;
    if (k < 1 || total > 20)
        return set_error(QS_ERR_NOT_SUPPORTED, "multi_qubit_control_multi_qubit_diagonal_matrix_gate: 1..20 qubits");
    std::vector<UINT> all(tl, tl + k);
    size_t cbits = 0;
    for (UINT j = 0; j < nc; ++j) {
        if (cval[j] > 1) return set_error(QS_ERR_INVALID_ARGUMENT, "control value must be 0 or 1");
        if (cval[j]) cbits |= size_t(1) << j;
        all.push_back(ctl[j]);
    }
    QS_TRY(check_distinct(all.data(), total, n, "multi_qubit_control_multi_qubit_diagonal_matrix_gate"));
    const size_t full = size_t(1) << total, md = size_t(1) << k;
    std::vector<double> d(2 * full);
    for (size_t i = 0; i < full; ++i) {
        const bool on = (i >> k) == cbits;
        d[2 * i] = on ? diag[2 * (i & (md - 1))] : 1.0;
        d[2 * i + 1] = on ? diag[2 * (i & (md - 1)) + 1] : 0.0;
    }
    return qs_multi_qubit_diagonal_matrix_gate(all.data(), total, d.data(), state, dim, stream);
}

}  // extern "C"
