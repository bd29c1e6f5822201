// Fused reduced-precision executor: complex64 state, gates fused into 6-qubit blocks applied on the
// 5th-generation tensor cores (tcgen05.mma, kind::f16 with bf16 operands, FP32 accumulation in TMEM).
//
// Host side (FP64): the pass scheduler groups gates into tile passes (13 tile qubits, qubits 0..4
// always included so every HBM access is a >= 256-byte run); inside a pass, gates are fused greedily
// into blocks of 6 qubits and each block's 64x64 complex matrix is composed in FP64.  The matrix is
// made real, [[Re U, -Im U], [Im U, Re U]] (128 x 128), and split into bf16 hi + lo parts, written
// in the canonical K-major no-swizzle UMMA shared-memory layout (8-row x 16-byte core matrices).
//
// Device side: one persistent CTA per SM.  For each tile (2^13 amplitudes = 64 KiB in shared memory):
// per block, the 128 cosets x 64 amplitudes are gathered into the B operand (bf16 hi and lo of the
// real and imaginary parts, K-major), one thread issues 8 K-steps x 3 products
// (A_hi B_hi + A_hi B_lo + A_lo B_hi) of tcgen05.mma M=128 N=128 K=16 into a 128 x 128 FP32 TMEM
// accumulator, commits to an mbarrier, and all warps read the accumulator back with tcgen05.ld into
// the tile.  Every wait is bounded; on expiry the kernel records an error, frees its TMEM and returns.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>

#include "circuit.hpp"
#include "qs_internal.cuh"

namespace qs {

constexpr int kFTileMax = 13;      // tile qubits (2^13 c64 amplitudes = 64 KiB)
constexpr int kFLow = 5;            // qubits 0..4 always in a tile
constexpr int kFBlock = 6;          // qubits per fused block
constexpr int kFThreads = 512;
constexpr int kFTidBits = 9;      // log2(kFThreads)
constexpr int kARows = 128, kAK = 128;           // real-ified block matrix
constexpr int kAImageBytes = kARows * kAK * 2;   // one bf16 image (hi or lo): 32 KiB
constexpr long long kWaitLimit = 4000000000LL;   // ~2 s of clock64 at 2 GHz

// canonical K-major, no swizzle: element (r, k) of a rows x 128 bf16 operand
__host__ __device__ __forceinline__ uint32_t kmajor_off(uint32_t r, uint32_t k) {
    return (r >> 3) * 2048u + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

struct FusedPassArgs {
    int m;                        // tile qubits
    int nblocks;
    UINT q[kFTileMax];            // global qubit of tile bit j (ascending)
    const uint8_t* block_bits;    // nblocks x 6 tile-local bits (ascending)
    const uint4* images;          // nblocks x (hi image | lo image)
    float2* state;
    ITYPE tiles;
    int* err;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Tile layout swizzle: XOR tile bits 5..12 into bits 1..4 (bit 0 untouched, so amplitude pairs stay
// adjacent for 16-byte copies), spreading block-bit strides over the shared-memory banks.
__device__ __forceinline__ uint32_t tswz(uint32_t u) { return u ^ ((((u >> 5) ^ (u >> 9)) & 15u) << 1); }

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem_dst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Two floats -> packed bf16 pairs (a in the low half): hi = RN(v), lo = RN(v - hi).
__device__ __forceinline__ void split2_bf16(float a, float b, uint32_t* hi, uint32_t* lo) {
    uint32_t h;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(h) : "f"(b), "f"(a));
    const float ha = __uint_as_float(h << 16), hb = __uint_as_float(h & 0xFFFF0000u);
    uint32_t l;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(l) : "f"(b - hb), "f"(a - ha));
    *hi = h;
    *lo = l;
}

// UMMA shared-memory descriptor: start >> 4 [0,14), LBO >> 4 [16,30), SBO >> 4 [32,46),
// version 1 [46,48), layout SWIZZLE_NONE (0) [61,64).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor, kind::f16: D = F32 [4,6), A = B = BF16 [7,10) [10,13), K-major A/B,
// N >> 3 [17,23), M >> 4 [24,29).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
    const long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            "selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(mbar), "r"(phase)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > kWaitLimit) return false;
    }
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void split_bf16(float v, __nv_bfloat16_raw* hi, __nv_bfloat16_raw* lo);

__global__ void __launch_bounds__(kFThreads, 1) k_fused_pass(const __grid_constant__ FusedPassArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int m = a.m;
    const uint32_t tsize = 1u << m;
    const uint32_t N = tsize >> kFBlock;  // cosets per block = MMA N
    unsigned char* sA = smem;                                  // A hi | A lo   (64 KiB)
    unsigned char* sB = sA + 2 * kAImageBytes;                 // B hi | B lo   (2 x N x 256 B)
    const uint32_t bimg = N * 256u;
    float2* tile = (float2*)(sB + 2 * bimg);                   // c64 tile (tsize x 8 B)
    uint32_t* dep_x = (uint32_t*)(tile + tsize);               // 64 entries
    uint32_t* dep_c = dep_x + 64;                              // N entries
    uint64_t* mbar = (uint64_t*)(dep_c + 256);
    uint32_t* tmem_slot = (uint32_t*)(mbar + 1);
    int* s_err = (int*)(tmem_slot + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t ncols = N < 32 ? 32u : N;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;");
        *s_err = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tmem_slot;
    const uint32_t mb = smem_u32(mbar);
    uint32_t phase = 0;
    const uint32_t idesc = idesc_bf16(kARows, (int)N);
    const uint32_t aaddr = smem_u32(sA), baddr = smem_u32(sB);

    // Tile loads/stores move amplitude pairs (tile bit 0 = qubit 0), 16 B each: pair p = tid + 512 k
    // holds tile bits 1..9 from tid and bits 10.. from k.
    ITYPE lo_off = 0;
    for (int j = 1; j <= kFTidBits && j < m; ++j)
        if ((tid >> (j - 1)) & 1) lo_off |= 1ULL << a.q[j];
    const uint32_t npairs = tsize >> 1;

    for (ITYPE T = blockIdx.x; T < a.tiles; T += gridDim.x) {
        ITYPE base = T;
        for (int j = 0; j < m; ++j) base = insert0(base, a.q[j]);
        // load tile: all pairs in flight at once (cp.async, 16 B)
#pragma unroll 4
        for (uint32_t k = 0; k * kFThreads < npairs; ++k) {
            const uint32_t pidx = tid + k * kFThreads;
            if (pidx < npairs) {
                ITYPE off = lo_off;
                for (int j = kFTidBits + 1; j < m; ++j)
                    if ((k >> (j - kFTidBits - 1)) & 1) off |= 1ULL << a.q[j];
                cp_async16(tile + tswz(2 * pidx), a.state + (base | off));
            }
        }
        cp_async_wait_all();
        __syncthreads();
        for (int b = 0; b < a.nblocks; ++b) {
            const uint8_t* bb = a.block_bits + b * kFBlock;
            // A images for this block: asynchronous copy, overlapped with the B gather below
            const uint4* img = a.images + (size_t)b * (2 * kAImageBytes / 16);
            for (int i = tid; i < 2 * kAImageBytes / 16; i += kFThreads) cp_async16((uint4*)sA + i, img + i);
            // deposit tables, pre-swizzled (tswz is XOR-linear, so the swizzled index of coset c and
            // block index x is sdep_c[c] ^ sdep_x[x]): x over the 6 block bits, c over the other bits
            if (tid < 64) {
                uint32_t d = 0;
                for (int j = 0; j < kFBlock; ++j)
                    if ((tid >> j) & 1) d |= 1u << bb[j];
                dep_x[tid] = tswz(d);
            }
            if ((uint32_t)tid < N) {
                uint32_t d = 0, bit = 0;
                for (int j = 0; j < m; ++j) {
                    bool inb = false;
                    for (int q = 0; q < kFBlock; ++q) inb |= (bb[q] == j);
                    if (!inb) {
                        if ((tid >> bit) & 1) d |= 1u << j;
                        ++bit;
                    }
                }
                dep_c[tid] = tswz(d);
            }
            __syncthreads();
            // gather B: row c (coset), K = x (real part) and 64 + x (imaginary part), hi and lo.
            // Thread t owns block indices x = 2j, 2j + 1 with j = bits 3..7 of t, and cosets
            // c = (t & 7) + 8 (t >> 8) + 16 i: its B offsets are fixed up to i * 4096, and within a warp
            // the 32 4-byte stores cover 128 distinct bytes.
            {
                const uint32_t j = ((tid >> 3) & 3u) | (((tid >> 5) & 7u) << 2);
                const uint32_t c0 = (tid & 7u) | ((uint32_t)(tid >> 8) << 3);
                const uint32_t sx0 = dep_x[2 * j], sx1 = dep_x[2 * j + 1];
                unsigned char* ore = sB + kmajor_off(c0, 2 * j);
                unsigned char* oim = sB + kmajor_off(c0, 64 + 2 * j);
#pragma unroll 2
                for (uint32_t i = 0; c0 + 16 * i < N; ++i) {
                    const uint32_t cb = dep_c[c0 + 16 * i];
                    const float2 v0 = tile[cb ^ sx0];
                    const float2 v1 = tile[cb ^ sx1];
                    uint32_t hi, lo;
                    split2_bf16(v0.x, v1.x, &hi, &lo);
                    *(uint32_t*)(ore + i * 4096) = hi;
                    *(uint32_t*)(ore + bimg + i * 4096) = lo;
                    split2_bf16(v0.y, v1.y, &hi, &lo);
                    *(uint32_t*)(oim + i * 4096) = hi;
                    *(uint32_t*)(oim + bimg + i * 4096) = lo;
                }
            }
            cp_async_wait_all();
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncthreads();
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;");
                // K-step s covers K = 16 s .. 16 s + 15: two 16-byte core-matrix columns, LBO = 128 B,
                // SBO = 2048 B (16 core matrices of one 8-row group along K)
#pragma unroll 1
                for (int s = 0; s < kAK / 16; ++s) {
                    const uint64_t ahi = umma_desc(aaddr + s * 256, 128, 2048);
                    const uint64_t alo = umma_desc(aaddr + kAImageBytes + s * 256, 128, 2048);
                    const uint64_t bhi = umma_desc(baddr + s * 256, 128, 2048);
                    const uint64_t blo = umma_desc(baddr + bimg + s * 256, 128, 2048);
                    mma_bf16(tmem, ahi, bhi, idesc, s > 0 ? 1u : 0u);
                    mma_bf16(tmem, ahi, blo, idesc, 1u);
                    mma_bf16(tmem, alo, bhi, idesc, 1u);
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mb)
                             : "memory");
            }
            const bool ok = mbar_wait(mb, phase);
            phase ^= 1u;
            if (!ok) *s_err = 1;
            asm volatile("tcgen05.fence::after_thread_sync;");
            // warp w reads TMEM lanes 32 (w % 4) .. +31 (rows y) and column part w / 4
            const uint32_t y = 32u * (warp & 3) + lane;
            const uint32_t parts = N >= 64 ? 4u : N / 16;
            const uint32_t cw = N / parts;
            const uint32_t c_begin = (uint32_t)(warp >> 2) < parts ? (warp >> 2) * cw : 0;
            const uint32_t c_end = (uint32_t)(warp >> 2) < parts ? c_begin + cw : 0;
            const uint32_t xo = dep_x[y & 63u];
            for (uint32_t c0 = c_begin; c0 < c_end; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + ((32u * (warp & 3)) << 16) + c0, v);
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    float* dst = (float*)&tile[dep_c[c0 + i] ^ xo];
                    dst[y >> 6] = v[i];
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncthreads();
            if (*s_err) break;
        }
        if (*s_err) break;
        // store tile (16-byte pairs)
        for (uint32_t k = 0; k * kFThreads < npairs; ++k) {
            const uint32_t pidx = tid + k * kFThreads;
            if (pidx < npairs) {
                ITYPE off = lo_off;
                for (int j = kFTidBits + 1; j < m; ++j)
                    if ((k >> (j - kFTidBits - 1)) & 1) off |= 1ULL << a.q[j];
                const float4 v = *(const float4*)(tile + tswz(2 * pidx));
                __stcs((float4*)(a.state + (base | off)), v);
            }
        }
        __syncthreads();
    }
    if (tid == 0 && *s_err) atomicExch(a.err, 1);
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

__device__ __forceinline__ void split_bf16(float v, __nv_bfloat16_raw* hi, __nv_bfloat16_raw* lo) {
    // round to nearest even: hi = bf16(v), lo = bf16(v - hi)
    uint32_t u = __float_as_uint(v);
    uint32_t r = u + 0x7FFFu + ((u >> 16) & 1u);
    const uint16_t h = (uint16_t)(r >> 16);
    const float hf = __uint_as_float((uint32_t)h << 16);
    const float rem = v - hf;
    uint32_t u2 = __float_as_uint(rem);
    uint32_t r2 = u2 + 0x7FFFu + ((u2 >> 16) & 1u);
    hi->x = h;
    lo->x = (uint16_t)(r2 >> 16);
}

// ---------------------------------------------------------------- host planning
using cd = std::complex<double>;

static uint16_t host_bf16(float v) {
    uint32_t u;
    memcpy(&u, &v, 4);
    uint32_t r = u + 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(r >> 16);
}
static float host_bf16_to_float(uint16_t h) {
    uint32_t u = (uint32_t)h << 16;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

// Apply a gate (dense on `pos` = positions of its qubits within the 6-bit block index, targets first
// then controls with their values) to every column of the 64x64 matrix U (U <- G U).
static void apply_to_block(std::vector<cd>& U, const GateRec& g, const std::vector<int>& pos) {
    const std::vector<cd> gm = g.dense_matrix();
    const int nt = (int)g.targets.size();
    const int nc = (int)g.controls.size();
    const int md = 1 << nt;
    std::vector<cd> tmp(md);
    for (int col = 0; col < 64; ++col) {
        for (int base = 0; base < 64; ++base) {
            bool is_base = true;
            for (int j = 0; j < nt; ++j)
                if ((base >> pos[j]) & 1) is_base = false;
            if (!is_base) continue;
            bool active = true;
            for (int j = 0; j < nc; ++j)
                if (((base >> pos[nt + j]) & 1) != (int)g.control_values[j]) active = false;
            if (!active) continue;
            for (int y = 0; y < md; ++y) {
                cd acc = 0.;
                for (int x = 0; x < md; ++x) {
                    int idx = base;
                    for (int j = 0; j < nt; ++j)
                        if ((x >> j) & 1) idx |= 1 << pos[j];
                    acc += gm[y * md + x] * U[idx * 64 + col];
                }
                tmp[y] = acc;
            }
            for (int y = 0; y < md; ++y) {
                int idx = base;
                for (int j = 0; j < nt; ++j)
                    if ((y >> j) & 1) idx |= 1 << pos[j];
                U[idx * 64 + col] = tmp[y];
            }
        }
    }
}

static ITYPE gate_mask(const GateRec& g) {
    ITYPE m = 0;
    for (UINT q : g.qubits()) m |= 1ULL << q;
    return m;
}

static bool fusable(const GateRec& g) {
    if (g.kind == QS_GATE_DEPOLARIZING) return false;
    if (g.kind == QS_GATE_DIAGONAL && g.targets.size() > 6) return false;
    return g.qubits().size() <= (size_t)kFBlock;
}

struct FusedBlock {
    uint8_t bits[kFBlock];
    std::vector<uint16_t> image;  // hi image then lo image (kAImageBytes / 2 each)
    std::vector<cd> U;            // FP64 block matrix, row-major, bit j <-> bits[j]
    int ngates;
};
struct FusedPass {
    std::vector<UINT> q;
    std::vector<FusedBlock> blocks;
};

struct FusedPlanHost {
    std::vector<FusedPass> passes;
    size_t nblocks = 0;
};

// Greedy absorption in program order: gates whose qubits lie in `allowed` and are not blocked by
// an earlier skipped gate on a shared qubit.
static std::vector<int> absorb_mask(const std::vector<GateRec>& G, const std::vector<int>& todo, ITYPE allowed) {
    std::vector<int> out;
    ITYPE blocked = 0;
    for (int gi : todo) {
        const ITYPE gm = gate_mask(G[gi]);
        if ((gm & blocked) || (gm & ~allowed)) {
            blocked |= gm;
            continue;
        }
        out.push_back(gi);
    }
    return out;
}
static ITYPE greedy_set(const std::vector<GateRec>& G, const std::vector<int>& todo, ITYPE start, int cap) {
    ITYPE S = start, blocked = 0;
    for (int gi : todo) {
        const ITYPE gm = gate_mask(G[gi]);
        if (gm & blocked) {
            blocked |= gm;
            continue;
        }
        if ((gm & ~S) == 0) continue;
        if (__builtin_popcountll(S | gm) <= cap) S |= gm;
        else blocked |= gm;
    }
    return S;
}

static void build_image(const std::vector<cd>& U, std::vector<uint16_t>* img) {
    img->assign(kAImageBytes, 0);  // 2 images x kAImageBytes / 2 uint16
    uint16_t* hi = img->data();
    uint16_t* lo = img->data() + kAImageBytes / 2;
    for (int r = 0; r < 128; ++r)
        for (int k = 0; k < 128; ++k) {
            const cd u = U[(r & 63) * 64 + (k & 63)];
            double v;
            if (r < 64) v = (k < 64) ? u.real() : -u.imag();
            else v = (k < 64) ? u.imag() : u.real();
            const float f = (float)v;
            const uint16_t h = host_bf16(f);
            const uint16_t l = host_bf16((float)(v - (double)host_bf16_to_float(h)));
            hi[kmajor_off(r, k) / 2] = h;
            lo[kmajor_off(r, k) / 2] = l;
        }
}

int fused_plan_host(const Circuit& c, FusedPlanHost* P) {
    const UINT n = c.n;
    for (const GateRec& g : c.gates)
        if (!fusable(g)) return set_error(QS_ERR_NOT_SUPPORTED, "fused path: gate over more than 6 qubits or a noise channel");
    const int m = (int)std::min<UINT>(kFTileMax, n);
    const ITYPE low = (1ULL << std::min(kFLow, m)) - 1;
    std::vector<int> pending(c.gates.size());
    for (size_t i = 0; i < c.gates.size(); ++i) pending[i] = (int)i;
    while (!pending.empty()) {
        // tile set: best of greedy and windows of consecutive qubits
        std::vector<ITYPE> cands{greedy_set(c.gates, pending, low, m)};
        const int free = m - __builtin_popcountll(low);
        for (int a0 = __builtin_popcountll(low); a0 + free <= (int)n; ++a0) {
            ITYPE Q = low;
            for (int j = 0; j < free; ++j) Q |= 1ULL << (a0 + j);
            cands.push_back(Q);
        }
        std::vector<int> best;
        ITYPE bestQ = 0;
        for (ITYPE Q : cands) {
            std::vector<int> got = absorb_mask(c.gates, pending, Q);
            if (got.size() > best.size()) {
                best = got;
                bestQ = Q;
            }
        }
        for (UINT q = 0; q < n && __builtin_popcountll(bestQ) < m; ++q) bestQ |= 1ULL << q;
        FusedPass fp;
        for (UINT q = 0; q < n; ++q)
            if (bestQ >> q & 1ULL) fp.q.push_back(q);
        auto local = [&](UINT gq) {
            for (size_t j = 0; j < fp.q.size(); ++j)
                if (fp.q[j] == gq) return (int)j;
            return -1;
        };
        // blocks of 6 tile qubits inside the pass (masks over global qubits)
        std::vector<int> todo = best;
        while (!todo.empty()) {
            std::vector<ITYPE> bc{greedy_set(c.gates, todo, 0, kFBlock)};
            for (int a0 = 0; a0 + kFBlock <= m; ++a0) {
                ITYPE B = 0;
                for (int j = 0; j < kFBlock; ++j) B |= 1ULL << fp.q[a0 + j];
                bc.push_back(B);
            }
            std::vector<int> bg;
            ITYPE bestB = 0;
            for (ITYPE B : bc) {
                std::vector<int> got = absorb_mask(c.gates, todo, B);
                if (got.size() > bg.size()) {
                    bg = got;
                    bestB = B;
                }
            }
            for (size_t j = 0; j < fp.q.size() && __builtin_popcountll(bestB) < kFBlock; ++j) bestB |= 1ULL << fp.q[j];
            FusedBlock blk;
            std::vector<UINT> bq;  // global qubits of block bit j (ascending tile-local == ascending global)
            for (UINT q = 0; q < n; ++q)
                if (bestB >> q & 1ULL) bq.push_back(q);
            for (int j = 0; j < kFBlock; ++j) blk.bits[j] = (uint8_t)local(bq[j]);
            std::vector<cd> U(64 * 64, 0.);
            for (int i = 0; i < 64; ++i) U[i * 64 + i] = 1.;
            for (int gi : bg) {
                const GateRec& g = c.gates[gi];
                std::vector<int> pos;
                for (UINT gq : g.qubits())
                    for (int j = 0; j < kFBlock; ++j)
                        if (bq[j] == gq) pos.push_back(j);
                apply_to_block(U, g, pos);
            }
            build_image(U, &blk.image);
            blk.U = U;
            blk.ngates = (int)bg.size();
            fp.blocks.push_back(std::move(blk));
            std::vector<char> taken(c.gates.size(), 0);
            for (int gi : bg) taken[gi] = 1;
            std::vector<int> rest;
            for (int gi : todo)
                if (!taken[gi]) rest.push_back(gi);
            todo.swap(rest);
        }
        P->nblocks += fp.blocks.size();
        P->passes.push_back(std::move(fp));
        std::vector<char> taken(c.gates.size(), 0);
        for (int gi : best) taken[gi] = 1;
        std::vector<int> rest;
        for (int gi : pending)
            if (!taken[gi]) rest.push_back(gi);
        pending.swap(rest);
    }
    return QS_OK;
}

struct FusedPlanDev {
    ITYPE dim = 0;
    std::vector<FusedPassArgs> passes;
    void* dev = nullptr;
    int* err = nullptr;
    ~FusedPlanDev() {
        if (dev) cudaFree(dev);
    }
};

static size_t fused_smem_bytes(int m) {
    const size_t tsize = size_t(1) << m, N = tsize >> kFBlock;
    return 2 * kAImageBytes + 2 * N * 256 + tsize * 8 + (64 + 256) * 4 + 64;
}

// Device plan cached on the circuit (dropped when a gate is added).
static int fused_plan_dev(Circuit& c, ITYPE dim, std::shared_ptr<FusedPlanDev>* out) {
    if (c.fused && c.fused_dim == dim) {
        *out = std::static_pointer_cast<FusedPlanDev>(c.fused);
        return QS_OK;
    }
    FusedPlanHost H;
    QS_TRY(fused_plan_host(c, &H));
    auto D = std::make_shared<FusedPlanDev>();
    D->dim = dim;
    size_t bits_bytes = (H.nblocks * kFBlock + 255) / 256 * 256;
    size_t img_bytes = H.nblocks * (size_t)(2 * kAImageBytes);
    QS_CUDA_CHECK(cudaMalloc(&D->dev, bits_bytes + img_bytes + 256));
    std::vector<unsigned char> host(bits_bytes + img_bytes + 256, 0);
    size_t bi = 0, ii = 0;
    std::vector<std::pair<size_t, size_t>> offs;
    for (const FusedPass& p : H.passes) {
        offs.push_back({bi, ii});
        for (const FusedBlock& b : p.blocks) {
            memcpy(host.data() + bi, b.bits, kFBlock);
            bi += kFBlock;
            memcpy(host.data() + bits_bytes + ii, b.image.data(), 2 * kAImageBytes);
            ii += 2 * kAImageBytes;
        }
    }
    QS_CUDA_CHECK(cudaMemcpy(D->dev, host.data(), host.size(), cudaMemcpyHostToDevice));
    D->err = (int*)((char*)D->dev + bits_bytes + img_bytes);
    QS_CUDA_CHECK(cudaMemset(D->err, 0, sizeof(int)));
    for (size_t i = 0; i < H.passes.size(); ++i) {
        FusedPassArgs a{};
        a.m = (int)H.passes[i].q.size();
        a.nblocks = (int)H.passes[i].blocks.size();
        for (int j = 0; j < a.m; ++j) a.q[j] = H.passes[i].q[j];
        a.block_bits = (const uint8_t*)D->dev + offs[i].first;
        a.images = (const uint4*)((const char*)D->dev + bits_bytes + offs[i].second);
        a.tiles = dim >> a.m;
        a.err = D->err;
        D->passes.push_back(a);
    }
    c.fused = D;
    c.fused_dim = dim;
    *out = D;
    return QS_OK;
}

int run_fused_c64(Circuit& c, void* state, ITYPE dim, cudaStream_t st) {
    if (c.n < 10) return set_error(QS_ERR_NOT_SUPPORTED, "fused path needs at least 10 qubits");
    std::shared_ptr<FusedPlanDev> D;
    QS_TRY(fused_plan_dev(c, dim, &D));
    for (const FusedPassArgs& p0 : D->passes) {
        FusedPassArgs p = p0;
        p.state = (float2*)state;
        const size_t smem = fused_smem_bytes(p.m);
        QS_CUDA_CHECK(cudaFuncSetAttribute(k_fused_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const unsigned grid = (unsigned)std::min<ITYPE>(p.tiles, (ITYPE)sm_count());
        k_fused_pass<<<grid, kFThreads, smem, st>>>(p);
        QS_TRY(check_launch("k_fused_pass"));
    }
    int err = 0;
    QS_CUDA_CHECK(cudaMemcpyAsync(&err, D->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    QS_CUDA_CHECK(cudaStreamSynchronize(st));
    if (err) return set_error(QS_ERR_TIMEOUT, "fused pass: tensor-core completion wait expired");
    return QS_OK;
}

// Host-only export of fused block `index` (in application order): the pass's tile qubits, the
// block's 6 tile-local bits, its FP64 matrix and its bf16 hi|lo operand image.
int fused_block_export(Circuit& c, UINT index, UINT* tile_qubits, int* m_out, UINT* bits, double* U_out,
    uint16_t* image_out) {
    FusedPlanHost H;
    QS_TRY(fused_plan_host(c, &H));
    UINT k = 0;
    for (const FusedPass& p : H.passes)
        for (const FusedBlock& b : p.blocks) {
            if (k++ != index) continue;
            *m_out = (int)p.q.size();
            for (size_t j = 0; j < p.q.size(); ++j) tile_qubits[j] = p.q[j];
            for (int j = 0; j < kFBlock; ++j) bits[j] = b.bits[j];
            if (image_out) memcpy(image_out, b.image.data(), 2 * kAImageBytes);
            if (U_out) memcpy(U_out, b.U.data(), sizeof(cd) * 64 * 64);
            return QS_OK;
        }
    return set_error(QS_ERR_INVALID_ARGUMENT, "fused block index out of range");
}

int fused_stats(Circuit& c, UINT* passes, UINT* blocks) {
    FusedPlanHost H;
    QS_TRY(fused_plan_host(c, &H));
    *passes = (UINT)H.passes.size();
    *blocks = (UINT)H.nblocks;
    return QS_OK;
}

}  // namespace qs

extern "C" {

QS_API int qs_circuit_update_quantum_state_fused_c64(qs_circuit_t circuit, void* state_c64, QS_ITYPE dim, void* stream) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null circuit");
    if (dim != (1ULL << c->n))
        return qs::set_error(QS_ERR_INVALID_ARGUMENT, "state dimension does not match the circuit's qubit count");
    return qs::run_fused_c64(*c, state_c64, dim, (cudaStream_t)stream);
}

QS_API int qs_circuit_fused_block_export(qs_circuit_t circuit, QS_UINT index, QS_UINT* tile_qubits, int* tile_qubit_count,
    QS_UINT* block_bits, double* matrix, unsigned short* operand_image) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c || !tile_qubits || !tile_qubit_count || !block_bits) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    return qs::fused_block_export(*c, index, tile_qubits, tile_qubit_count, block_bits, matrix, operand_image);
}

QS_API int qs_circuit_fused_stats(qs_circuit_t circuit, QS_UINT* passes, QS_UINT* blocks) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c || !passes || !blocks) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    return qs::fused_stats(*c, passes, blocks);
}

}  // extern "C"
