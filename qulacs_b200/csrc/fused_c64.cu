// Fused reduced-precision executor: complex64 state, gates fused into 6-qubit blocks applied on the
// 5th-generation tensor cores (tcgen05.mma, kind::f16 with bf16 operands, FP32 accumulation in TMEM).
//
// Host side (FP64): the pass scheduler groups gates into tile passes (13 tile qubits, qubits 0..4
// always included so every HBM access is a >= 256-byte run); inside a pass, gates are fused greedily
// into blocks of 6 qubits and each block's 64x64 complex matrix is composed in FP64.  The matrix is
// made real, [[Re U, -Im U], [Im U, Re U]] (128 x 128), and split into bf16 hi + lo parts, written
// in the UMMA K-major shared-memory layout with the 128-byte swizzle.  Per block the host also picks
// the operand orders (rows, K, cosets) that make the kernel's warp-wide shared-memory accesses
// conflict-free, and emits them as XOR tables.
//
// Device side: one persistent CTA (512 threads) per SM takes its tiles in pairs that go through the
// pass's blocks in lockstep and share each block's A image (bulk async copy).  Per block, one thread
// issues for each tile 8 K-steps x 3 products (A_hi B_hi + A_hi B_lo + A_lo B_hi) of tcgen05.mma
// M=128 N=128 K=16 into its 128 x 128 FP32 TMEM accumulator and commits to an mbarrier; the other
// warps move one tile's accumulator (tcgen05.ld) into its next B operand while the other tile's MMAs
// run.  Tiles are gathered straight from HBM; after the last block each becomes a complex64
// tile stored to HBM.  Every wait is bounded; on expiry the kernel records an error, frees its TMEM
// and returns.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "circuit.hpp"
#include "qs_internal.cuh"

namespace qs {

constexpr int kFTileMax = 13;      // tile qubits (2^13 c64 amplitudes = 64 KiB)
constexpr int kFLow = 5;            // qubits 0..4 always in a tile
constexpr int kFBlock = 6;          // qubits per fused block
constexpr int kFThreads = 512;
constexpr int kARows = 128, kAK = 128;           // real-ified block matrix
constexpr int kAImageBytes = kARows * kAK * 2;   // one bf16 image (hi or lo): 32 KiB
constexpr long long kWaitLimit = 4000000000LL;   // ~2 s of clock64 at 2 GHz
// Per-block index tables (u32 words): rowtab[128] | coltab[128] | gn[128] (u64) | gj[64] (u64)
constexpr int kTabRow = 0, kTabCol = 128, kTabGn = 256, kTabGj = 512, kTabWords = 640;
constexpr int kTabBytes = kTabWords * 4;
constexpr int kRecordBytes = 2 * kAImageBytes + kTabBytes;  // one block record in global memory

// K-major with the 128-byte swizzle: element (r, k) of a rows x 128 bf16 operand.  Atoms of 8 rows x
// 64 K (8 rows of 128 B = 1024 B, 1024-byte aligned); atom (r / 8, k / 64) at ((r / 8) * 2 + k / 64) KiB;
// in an atom, row r % 8 at 128 (r % 8) and its 16-byte chunk (k / 8) % 8 at chunk ((k / 8) % 8) ^ (r % 8).
// A bit placement with an XOR, so offsets of XORed indices XOR.
__host__ __device__ __forceinline__ uint32_t kmajor_off(uint32_t r, uint32_t k) {
    return ((r >> 3) * 2u + (k >> 6)) * 1024u + (r & 7u) * 128u + ((((k >> 3) & 7u) ^ (r & 7u)) << 4) +
           (k & 7u) * 2u;
}

struct FusedPassArgs {
    int m;                        // tile qubits
    int nblocks;
    UINT q[kFTileMax];            // global qubit of tile bit j (ascending)
    const unsigned char* records; // nblocks x (A hi | A lo | tables), kRecordBytes each
    float2* state;
    ITYPE tiles;
    int* err;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Tile layout swizzle: XOR tile bits 5..12 into bits 1..4 (bit 0 untouched, so amplitude pairs stay
// adjacent for 16-byte copies), spreading block-bit strides over the shared-memory banks.
__host__ __device__ __forceinline__ uint32_t tswz(uint32_t u) { return u ^ ((((u >> 5) ^ (u >> 9)) & 15u) << 1); }

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

// UMMA shared-memory descriptor for the swizzled K-major operands above: start >> 4 [0,14),
// LBO field 1 [16,30) (unused by swizzled K-major layouts), SBO >> 4 = 2048 B between 8-row groups
// [32,46), version 1 [46,48), base offset 0 (1024-byte aligned atoms), layout SWIZZLE_128B (2) [61,64).
// K-step s (K = 16 s .. 16 s + 15) starts at atom column s / 4 (+1 KiB) and 32 B (s % 4) into the row.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(2048u >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
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

// One block record: A image (hi | lo, 64 KiB) into `dst_a` and its index tables into `dst_t`, with bulk
// async copies completing on `mbar` (issued by one thread; the phase completes when all bytes landed).
__device__ __forceinline__ void bulk_load_block(uint32_t dst_a, uint32_t dst_t, const unsigned char* rec,
                                                uint32_t mbar) {
    asm volatile(
        "{\n.reg .b64 st;\nmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(mbar),
        "r"(2 * kAImageBytes + kTabBytes)
        : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst_a),
                 "l"(rec), "r"(2 * kAImageBytes), "r"(mbar)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst_t),
                 "l"(rec + 2 * kAImageBytes), "r"(kTabBytes), "r"(mbar)
                 : "memory");
}

// Two tiles in flight.  A CTA takes its tiles in pairs (X, Y) that go through the pass's blocks in
// lockstep and share each block's A operand: X's and Y's MMAs go into two TMEM accumulators, X's
// accumulator moves run while Y's MMAs do, and Y's moves run while the next block's A image (bulk
// copy) lands and X's next MMAs run.  A tile is gathered straight from HBM into its B operand
// (bf16 hi / lo) through 64-bit offset tables; after the last block its accumulator becomes a
// complex64 tile over its own B region, stored with 16-byte streaming stores.
// Every in-tile data movement is a table XOR: element (row y, column n) of a block's accumulator goes
// to byte rowtab[y] ^ coltab[n] of the next B operand (float rowtab[y] ^ coltab[n] of the output
// tile after the last block).
//
// The per-pair work is written once (fused_pair) and shared by the single-circuit kernel
// (k_fused_pass: all tile pairs of one pass) and the multi-circuit kernel (k_fused_batch: work items of
// many circuits' passes).  Shared memory is laid out for the largest tile (N = 128 cosets), so passes
// of any tile size fit the same layout.

// Shared-memory regions of a fused CTA and the TMEM allocation.
struct FusedSmem {
    unsigned char* sA;   // A hi | A lo (64 KiB)
    unsigned char* sB0;  // tile X: B hi | B lo, then its output tile
    unsigned char* sB1;  // tile Y
    uint32_t* tabs;      // [2][kTabWords]
    uint64_t* dep;       // [kDepChunks][64]: tile-index bits -> global offset (see fused_addr_tables)
    uint64_t* runoff;    // [256]: 256-byte run index (tile bits 5..12) -> global offset
    uint64_t* mbar;      // [0] MMA X, [1] MMA Y, [2] block record
    int* s_err;
    uint32_t tmem, ncols, mb0, mb1, mba, aaddr, taddr;
};
// Completion-barrier phases and the record pipeline, identical in every thread of the CTA.
struct FusedPipe {
    uint32_t ph0 = 0, ph1 = 0, pha = 0;
    bool a_pending = false;  // a block record copy is in flight on mba
    int slot = 0;            // table slot of the current block's record
    int loads = 0;           // records issued so far (the next one goes to slot loads & 1)
};

constexpr uint32_t kFNMax = 1u << (kFTileMax - kFBlock);  // 128 cosets per block at the largest tile
// Tile indices have at most kDepChunks x 6 bits (the host refuses larger states).
constexpr int kDepChunks = 4;
constexpr int kAddrTabBytes = (kDepChunks * 64 + 256) * 8;

__device__ __forceinline__ FusedSmem fused_setup(unsigned char* smem, uint32_t ncols) {
    FusedSmem S;
    const uint32_t bimg_max = kFNMax * 256u;
    S.sA = smem;
    S.sB0 = S.sA + 2 * kAImageBytes;
    S.sB1 = S.sB0 + 2 * bimg_max;
    S.tabs = (uint32_t*)(S.sB1 + 2 * bimg_max);
    S.dep = (uint64_t*)(S.tabs + 2 * kTabWords);
    S.runoff = S.dep + kDepChunks * 64;
    S.mbar = S.runoff + 256;
    uint32_t* tmem_slot = (uint32_t*)(S.mbar + 3);
    S.s_err = (int*)(tmem_slot + 1);
    S.ncols = ncols;
    const int tid = threadIdx.x, warp = tid >> 5;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int i = 0; i < 3; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(S.mbar + i)));
        asm volatile("fence.mbarrier_init.release.cluster;");
        *S.s_err = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    S.tmem = *tmem_slot;
    S.mb0 = smem_u32(S.mbar);
    S.mb1 = smem_u32(S.mbar + 1);
    S.mba = smem_u32(S.mbar + 2);
    S.aaddr = smem_u32(S.sA);
    S.taddr = smem_u32(S.tabs);
    return S;
}

// No copy in flight, the error flag published, TMEM freed.
__device__ __forceinline__ void fused_teardown(const FusedSmem& S, FusedPipe& P, int* err) {
    if (P.a_pending && !mbar_wait(S.mba, P.pha)) *S.s_err = 1;
    P.a_pending = false;
    if (threadIdx.x == 0 && *S.s_err) atomicExch(err, 1);
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(S.tmem), "r"(S.ncols));
}

// A pass's address tables, filled by the whole CTA (a barrier must follow before use): dep[c][v] is
// the global offset of tile index v << 6c (its bits deposited into the non-tile qubits, in ascending
// order), so tile T starts at the OR of four lookups; runoff[r] is the offset of 256-byte run r (its
// bits at tile qubits q[5..m-1]; qubits 0..4 are the run).  This replaces per-pair bit loops over the
// pass's qubit list.
__device__ __forceinline__ void fused_addr_tables(const FusedSmem& S, const FusedPassArgs& a) {
    const int t = threadIdx.x;
    if (t < kDepChunks * 64) {
        ITYPE base = (ITYPE)(t & 63) << (6 * (t >> 6));
        for (int j = 0; j < a.m; ++j) base = insert0(base, a.q[j]);
        S.dep[t] = base;
    } else if (t < kDepChunks * 64 + 256) {
        const uint32_t r = (uint32_t)t - kDepChunks * 64;
        ITYPE off = 0;
        for (int j = kFLow; j < a.m; ++j)
            if ((r >> (j - kFLow)) & 1u) off |= 1ULL << a.q[j];
        S.runoff[r] = off;
    }
}

__device__ __forceinline__ ITYPE fused_tile_base(const FusedSmem& S, ITYPE T) {
    return S.dep[T & 63] | S.dep[64 + ((T >> 6) & 63)] | S.dep[128 + ((T >> 12) & 63)] | S.dep[192 + ((T >> 18) & 63)];
}

__device__ __forceinline__ const unsigned char* fused_record(const FusedPassArgs& a, int b) {
    return a.records + (size_t)b * kRecordBytes;
}

// Issue block b's record into the next table slot (one thread copies; every thread tracks the state).
__device__ __forceinline__ void fused_load_record(const FusedSmem& S, FusedPipe& P, const FusedPassArgs& a, int b,
                                                  bool set_slot) {
    const int nslot = P.loads & 1;
    if (threadIdx.x == 0) bulk_load_block(S.aaddr, S.taddr + nslot * kTabBytes, fused_record(a, b), S.mba);
    P.a_pending = true;
    ++P.loads;
    if (set_slot) P.slot = nslot;
}

__device__ __forceinline__ void fused_wait_record(const FusedSmem& S, FusedPipe& P) {
    if (P.a_pending) {
        if (!mbar_wait(S.mba, P.pha)) *S.s_err = 1;
        P.pha ^= 1u;
        P.a_pending = false;
    }
}

// One tile pair (TX and, if hasY, TY) through every block of pass `a`.  On entry block 0's record is
// loaded or in flight in slot P.slot.  `next_pair` (>= 0): another pair of the same pass follows, so
// block 0's record is reloaded after the last block (tile `next_pair` and its partner are prefetched
// into L2 meanwhile).  Returns false when a bounded wait expired (the CTA must stop).
__device__ __forceinline__ bool fused_pair(const FusedPassArgs& a, const FusedSmem& S, FusedPipe& P, ITYPE TX, ITYPE TY, bool hasY,
                           long long next_pair, ITYPE pair_stride) {
    const int m = a.m;
    const uint32_t tsize = 1u << m;
    const uint32_t N = tsize >> kFBlock;  // cosets per block = MMA N
    const uint32_t bimg = N * 256u;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t idesc = idesc_bf16(kARows, (int)N);
    unsigned char* sB0 = S.sB0;
    unsigned char* sB1 = S.sB1;
    const uint32_t* tabs = S.tabs;

    // output stores move amplitude pairs (tile bit 0 = qubit 0), 16 B each: pair p = tid + 512 k is
    // amplitude 2 (p % 16) of 256-byte run p / 16
    const uint32_t npairs = tsize >> 1;
    auto tile_base = [&](ITYPE T) { return fused_tile_base(S, T); };

    // accumulator reads: warp w >= 1 reads TMEM lanes 32 (w % 4) .. +31 (rows y); the 16-column chunks
    // are split over the mover warps of each lane quarter (three in quarter 0: warp 0 issues the MMAs)
    const uint32_t y = 32u * (warp & 3) + lane;
    const bool mover = warp != 0;
    const uint32_t nchunks = N / 16;
    const uint32_t nq = (warp & 3) == 0 ? 3u : 4u;
    const uint32_t rq = mover ? ((warp & 3) == 0 ? (uint32_t)(warp >> 2) - 1u : (uint32_t)(warp >> 2)) : 0u;
    const uint32_t c_begin = mover ? 16u * ((rq * nchunks) / nq) : 0u;
    const uint32_t c_end = mover ? 16u * (((rq + 1u) * nchunks) / nq) : 0u;
    // gather: thread t owns B rows n = (t & 7) + 8 i and K pair j = bits 3..8 of t
    const uint32_t g_n0 = tid & 7u, g_j = (uint32_t)tid >> 3;
    const uint32_t g_off = kmajor_off(g_n0, 2 * g_j);

    // tiles -> B operands straight from HBM: 64-bit offsets of coset n (gn) and block index j (gj);
    // both tiles' loads are in flight together
    auto gather = [&](int slot) {
        const uint64_t* gn = (const uint64_t*)(tabs + slot * kTabWords + kTabGn);
        const ITYPE gj = ((const uint64_t*)(tabs + slot * kTabWords + kTabGj))[g_j];
        const ITYPE bx = tile_base(TX) | gj, by = hasY ? (tile_base(TY) | gj) : bx;
        float2 vx[16], vy[16];
#pragma unroll
        for (uint32_t i = 0; i < 16; ++i)
            if (g_n0 + 8 * i < N) {
                const ITYPE o = gn[g_n0 + 8 * i];
                vx[i] = __ldcs(a.state + (bx | o));
                if (hasY) vy[i] = __ldcs(a.state + (by | o));
            }
        auto put = [&](unsigned char* sB, const float2 (&v)[16]) {
#pragma unroll
            for (uint32_t i = 0; i < 16; ++i)
                if (g_n0 + 8 * i < N) {
                    uint32_t hi, lo;
                    split2_bf16(v[i].x, v[i].y, &hi, &lo);
                    *(uint32_t*)(sB + g_off + i * 2048) = hi;
                    *(uint32_t*)(sB + bimg + g_off + i * 2048) = lo;
                }
        };
        put(sB0, vx);
        if (hasY) put(sB1, vy);
    };
    auto issue_mma = [&](unsigned char* sB, uint32_t dcol, uint32_t mbar_addr) {
        const uint32_t baddr = smem_u32(sB);
        // shared addresses are below 256 KiB, so the 14-bit start-address field never wraps: the
        // descriptor of K-step s is the K-step-0 descriptor plus its start offset >> 4
        const uint64_t ahi0 = umma_desc(S.aaddr), alo0 = umma_desc(S.aaddr + kAImageBytes);
        const uint64_t bhi0 = umma_desc(baddr), blo0 = umma_desc(baddr + bimg);
#pragma unroll
        for (int s = 0; s < kAK / 16; ++s) {
            const uint64_t ds = (uint64_t)(((s >> 2) * 1024 + (s & 3) * 32) >> 4);
            mma_bf16(S.tmem + dcol, ahi0 + ds, bhi0 + ds, idesc, s > 0 ? 1u : 0u);
            mma_bf16(S.tmem + dcol, ahi0 + ds, blo0 + ds, idesc, 1u);
            mma_bf16(S.tmem + dcol, alo0 + ds, bhi0 + ds, idesc, 1u);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar_addr)
                     : "memory");
    };
    // accumulator (TMEM columns dcol..) -> next B operand in sB, or -> complex64 output tile over sB.
    // Row bit 0 is the real/imaginary part: lanes 2j and 2j + 1 swap halves of their 16 columns with one
    // shuffle each, so the even lane holds (re, im) of columns 0..7 of the chunk and the odd lane of
    // columns 8..15, and each amplitude is stored as one word: bf16x2 hi and lo (re in the low half,
    // the next operand's K bit 0) or a float2 of the output tile.
    auto move = [&](unsigned char* sB, uint32_t dcol, int slot, bool last) {
        const uint32_t* rt = tabs + slot * kTabWords + kTabRow;
        const uint32_t* ct = tabs + slot * kTabWords + kTabCol;
        const bool odd = lane & 1;
        const uint32_t ybase = rt[y & ~1u];  // the pair's real-part row
        float* outt = (float*)sB;
        for (uint32_t cc = c_begin; cc < c_end; cc += 16) {
            float v[16];
            tmem_ld16(S.tmem + ((32u * (warp & 3)) << 16) + dcol + cc, v);
            float re[8], im[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const float got = __shfl_xor_sync(0xffffffffu, odd ? v[i] : v[8 + i], 1);
                re[i] = odd ? got : v[i];
                im[i] = odd ? v[8 + i] : got;
            }
            const uint32_t c0 = cc + (odd ? 8u : 0u);
            uint32_t o[8];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const uint4 t4 = *(const uint4*)(ct + c0 + 4 * q);
                o[4 * q] = t4.x ^ ybase;
                o[4 * q + 1] = t4.y ^ ybase;
                o[4 * q + 2] = t4.z ^ ybase;
                o[4 * q + 3] = t4.w ^ ybase;
            }
            if (last) {
#pragma unroll
                for (int i = 0; i < 8; ++i) *(float2*)(outt + o[i]) = make_float2(re[i], im[i]);
            } else {
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    uint32_t hi, lo;
                    split2_bf16(re[i], im[i], &hi, &lo);
                    *(uint32_t*)(sB + o[i]) = hi;
                    *(uint32_t*)(sB + bimg + o[i]) = lo;
                }
            }
        }
    };
    auto store_out = [&](ITYPE T, const unsigned char* sB) {
        const ITYPE base = tile_base(T);
        const float* outt = (const float*)sB;
        for (uint32_t k = 0; k * kFThreads < npairs; ++k) {
            const uint32_t pidx = tid + k * kFThreads;
            if (pidx < npairs) {
                const float4 v = *(const float4*)(outt + 2 * tswz(2 * pidx));
                __stcs((float4*)(a.state + (base | S.runoff[pidx >> 4] | ((pidx & 15u) << 1))), v);
            }
        }
    };

    fused_wait_record(S, P);  // block 0's record: its gather tables
    __syncthreads();
    if (*S.s_err) return false;
    gather(P.slot);
    if (next_pair >= 0) {  // the next pair's 256-byte runs into L2 while this pair's blocks run
        const ITYPE T2 = (ITYPE)next_pair + (tid >= 256 ? pair_stride : 0);
        const uint32_t r = (uint32_t)tid & 255u;
        if (T2 < a.tiles && r < (tsize >> kFLow))
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], 256;" ::"l"(a.state + (tile_base(T2) | S.runoff[r]))
                         : "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();  // the gathered B operands are visible to the tensor cores
    // Block loop, software-pipelined: X(b) is issued as soon as block b's record has landed, while the
    // mover warps still turn Y's accumulator of block b - 1 into its next operand; Y(b) follows once
    // that is done, and X's accumulator moves run under Y(b)'s MMAs.  Warp 0 only issues.
    for (int b = 0; b < a.nblocks; ++b) {
        const bool last = b + 1 == a.nblocks;
        const int cur = P.slot;
        fused_wait_record(S, P);  // block b's A image and tables (every thread observes the copy)
        if (tid == 0 && !*S.s_err) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            issue_mma(sB0, 0, S.mb0);  // sB0 and D_X were released at the previous barrier
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();  // Y's operand of block b written (and proxy-fenced), D_Y read
        if (tid == 0 && !*S.s_err && hasY) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            issue_mma(sB1, N, S.mb1);
        }
        if (!mbar_wait(S.mb0, P.ph0)) *S.s_err = 1;
        P.ph0 ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (mover) move(sB0, 0, cur, last);  // while Y's MMAs run
        if (hasY) {
            if (!mbar_wait(S.mb1, P.ph1)) *S.s_err = 1;
            P.ph1 ^= 1u;
            asm volatile("tcgen05.fence::after_thread_sync;");
        }
        const int nxt = b + 1 < a.nblocks ? b + 1 : (next_pair >= 0 ? 0 : -1);
        const bool reload = nxt >= 0 && nxt != b;  // a single-block pass keeps its record resident
        // Thread 0 has seen both MMA groups complete, so A is free, and the other table slot was
        // released at the first barrier: the next record's copy starts before the second barrier.
        // Every thread books it after that barrier, ahead of the error exit, so a teardown waits for it.
        if (reload && tid == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            bulk_load_block(S.aaddr, S.taddr + (P.loads & 1) * kTabBytes, fused_record(a, nxt), S.mba);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();  // both MMAs done (A and the other table slot free); X's next operand written
        if (reload) {
            P.slot = P.loads & 1;
            ++P.loads;
            P.a_pending = true;
        }
        if (*S.s_err) return false;
        if (hasY && mover) move(sB1, N, cur, last);  // while the next record lands and X(b + 1) runs
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    store_out(TX, sB0);
    if (hasY) store_out(TY, sB1);
    __syncthreads();  // the next pair's gather overwrites the output tiles
    return true;
}

__global__ void __launch_bounds__(kFThreads, 1) k_fused_pass(const __grid_constant__ FusedPassArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const uint32_t N = (1u << a.m) >> kFBlock;
    FusedSmem S = fused_setup(smem, 2 * N < 32 ? 32u : 2 * N);  // D_X at column 0, D_Y at column N
    fused_addr_tables(S, a);
    __syncthreads();
    FusedPipe P;
    if ((ITYPE)blockIdx.x < a.tiles) fused_load_record(S, P, a, 0, true);
    const ITYPE stride = 2 * (ITYPE)gridDim.x;
    for (ITYPE TX = blockIdx.x; TX < a.tiles; TX += stride) {
        const ITYPE TY = TX + gridDim.x;
        const bool has_next = TX + stride < a.tiles;
        if (!fused_pair(a, S, P, TX, TY, TY < a.tiles, has_next ? (long long)(TX + stride) : -1, gridDim.x)) break;
    }
    fused_teardown(S, P, a.err);
}

// ---- many circuits in one persistent launch
// Work records are (circuit, pass) in pass-round-robin order; a record's work items are its tile pairs
// (tiles 2i and 2i + 1).  A CTA takes the next item with an atomic counter and, for a pass after a
// circuit's first, waits until every tile of the circuit's previous pass is done (acquire load of that
// record's counter, bounded by a %globaltimer deadline).  Items are handed out in queue order and a
// dependency always points to an earlier record whose items resident CTAs already hold, so the wait
// ends; on expiry the CTA records an error and leaves.
struct FusedBatchRec {
    FusedPassArgs args;  // state, records, m, q, nblocks, tiles
    ITYPE prefix;        // first work item of this record
    int dep;             // record of the circuit's previous pass, -1 for its first
};

__device__ __forceinline__ unsigned ld_acquire_u32_f(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long fused_global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__global__ void __launch_bounds__(kFThreads, 1) k_fused_batch(const FusedBatchRec* __restrict__ recs, int nrec,
    ITYPE total, unsigned long long* head, unsigned* done, int* err, unsigned long long wait_ns) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ ITYPE s_item;
    __shared__ int s_rec, s_abort;
    FusedSmem S = fused_setup(smem, 2 * kFNMax);
    FusedPipe P;
    int tab_rec = -1;  // record whose address tables are in shared memory
    const int tid = threadIdx.x;
    while (true) {
        if (tid == 0) {
            s_abort = 0;
            s_item = atomicAdd(head, 1ULL);
            if (s_item < total) {
                int lo = 0, hi = nrec - 1;  // last record with prefix <= item
                while (lo < hi) {
                    const int mid = (lo + hi + 1) / 2;
                    if (recs[mid].prefix <= s_item) lo = mid;
                    else hi = mid - 1;
                }
                s_rec = lo;
                const int dep = recs[lo].dep;
                if (dep >= 0) {
                    const unsigned need = (unsigned)recs[dep].args.tiles;
                    const unsigned long long t0 = fused_global_ns();
                    while (ld_acquire_u32_f(done + dep) < need) {
                        if (fused_global_ns() - t0 > wait_ns) {
                            s_abort = 1;
                            *S.s_err = 1;
                            break;
                        }
                        __nanosleep(128);
                    }
                }
            }
        }
        __syncthreads();
        if (s_item >= total || s_abort) break;
        const FusedPassArgs a = recs[s_rec].args;
        if (s_rec != tab_rec) {  // every thread left the previous pair's last table use behind a barrier
            fused_addr_tables(S, a);
            __syncthreads();
            tab_rec = s_rec;
        }
        const ITYPE TX = 2 * (s_item - recs[s_rec].prefix), TY = TX + 1;
        const bool hasY = TY < a.tiles;
        fused_load_record(S, P, a, 0, true);
        if (!fused_pair(a, S, P, TX, TY, hasY, -1, 0)) break;
        if (tid == 0) {
            __threadfence();
            atomicAdd(done + s_rec, hasY ? 2u : 1u);
        }
    }
    fused_teardown(S, P, err);
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

// Operand orders of one block.  All are bit placements, so every index map between the tile, the
// B operand and the accumulator is an XOR of per-bit terms (two table lookups on the device).
//   row_src[i]    : source of accumulator row bit i (block-local bit 0..5, or 6 = real/imaginary part)
//   k_src[i]      : block-local bit at K bit 1 + i of the operands (K bit 0 = real/imaginary part)
//   coset_bits[i] : tile bit at bit i of the coset index (the MMA N index)
struct BlockLayout {
    int row_src[7];
    int k_src[kFBlock];
    std::vector<int> coset_bits;
};

struct FusedBlock {
    uint8_t bits[kFBlock];        // tile-local bits (ascending); block-local bit j <-> bits[j]
    BlockLayout lay;
    std::vector<uint16_t> image;  // hi image then lo image (kAImageBytes / 2 each), in `lay` order
    std::vector<uint32_t> tabs;   // kTabWords: rowtab | coltab | gn | gj
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

// A operand of a block: row y = (real/imaginary part, output index) by lay.row_src, column K =
// (part, input index) by lay.k_src; entries of [[Re U, -Im U], [Im U, Re U]].
static void build_image(const std::vector<cd>& U, const BlockLayout& lay, std::vector<uint16_t>* img) {
    img->assign(kAImageBytes, 0);  // 2 images x kAImageBytes / 2 uint16
    uint16_t* hi = img->data();
    uint16_t* lo = img->data() + kAImageBytes / 2;
    for (int r = 0; r < 128; ++r)
        for (int k = 0; k < 128; ++k) {
            int xo = 0, po = 0, xi = 0;
            for (int i = 0; i < 7; ++i) {
                const int bit = (r >> i) & 1;
                if (lay.row_src[i] == 6) po = bit;
                else xo |= bit << lay.row_src[i];
            }
            const int pi = k & 1;
            for (int i = 0; i < kFBlock; ++i) xi |= ((k >> (1 + i)) & 1) << lay.k_src[i];
            const cd u = U[xo * 64 + xi];
            double v;
            if (po == 0) v = (pi == 0) ? u.real() : -u.imag();
            else v = (pi == 0) ? u.imag() : u.real();
            const float f = (float)v;
            const uint16_t h = host_bf16(f);
            const uint16_t l = host_bf16((float)(v - (double)host_bf16_to_float(h)));
            hi[kmajor_off(r, k) / 2] = h;
            lo[kmajor_off(r, k) / 2] = l;
        }
}

// ---- operand layouts: chosen per block so that the warp-wide shared-memory accesses of the gather,
// the accumulator -> next-operand moves and the output scatter hit distinct banks.

// Largest number of distinct 4-byte words any bank receives (accesses to one word do not conflict).
static int bank_degree(const uint32_t* word, int count) {
    int worst = 0;
    for (uint32_t bank = 0; bank < 32; ++bank) {
        uint32_t seen[64];
        int cnt = 0;
        for (int l = 0; l < count; ++l) {
            if ((word[l] & 31u) != bank) continue;
            bool dup = false;
            for (int q = 0; q < cnt; ++q) dup |= seen[q] == word[l];
            if (!dup) seen[cnt++] = word[l];
        }
        worst = std::max(worst, cnt);
    }
    return worst;
}

static std::vector<int> coset_bits_of(const FusedBlock& b, int m) {
    std::vector<int> v;
    for (int j = 0; j < m; ++j)
        if (std::find(b.bits, b.bits + kFBlock, (uint8_t)j) == b.bits + kFBlock) v.push_back(j);
    return v;
}
// `first` in the given order, then the rest of `all` ascending
static std::vector<int> order_with_prefix(const std::vector<int>& first, const std::vector<int>& all) {
    std::vector<int> v = first;
    for (int x : all)
        if (std::find(first.begin(), first.end(), x) == first.end()) v.push_back(x);
    return v;
}
// tile index and part of accumulator row y
static uint32_t row_tile_index(const uint8_t* bits, const BlockLayout& L, uint32_t y, uint32_t* part) {
    uint32_t u = 0;
    *part = 0;
    for (int i = 0; i < 7; ++i) {
        const uint32_t bit = (y >> i) & 1u;
        if (L.row_src[i] == 6) *part = bit;
        else u |= bit << bits[L.row_src[i]];
    }
    return u;
}
static uint32_t coset_tile_index(const BlockLayout& L, uint32_t n) {
    uint32_t u = 0;
    for (size_t i = 0; i < L.coset_bits.size(); ++i) u |= ((n >> i) & 1u) << L.coset_bits[i];
    return u;
}
static uint32_t k_tile_index(const FusedBlock& b, uint32_t j) {  // j = K >> 1
    uint32_t u = 0;
    for (int i = 0; i < kFBlock; ++i) u |= ((j >> i) & 1u) << b.bits[b.lay.k_src[i]];
    return u;
}
// byte offset of (tile index u, part) in the B operand of a block on `bits` with layout L
static uint32_t b_operand_off(const uint8_t* bits, const BlockLayout& L, uint32_t u, uint32_t part) {
    uint32_t n = 0, k = part;
    for (size_t i = 0; i < L.coset_bits.size(); ++i) n |= ((u >> L.coset_bits[i]) & 1u) << i;
    for (int i = 0; i < kFBlock; ++i) k |= ((u >> bits[L.k_src[i]]) & 1u) << (1 + i);
    return kmajor_off(n, k);
}

static void choose_layouts(FusedPass& fp) {
    const int m = (int)fp.q.size();
    std::vector<int> locals(kFBlock);
    for (int j = 0; j < kFBlock; ++j) locals[j] = j;
    // block 0's gather straight from HBM: lanes 0..2 = coset index bits 0..2, lanes 3..4 = K pair bits
    // 0..1; pick them so a warp's 32 eight-byte loads touch the fewest 32-byte sectors (8 at best)
    {
        FusedBlock& b0 = fp.blocks[0];
        const std::vector<int> cos = coset_bits_of(b0, m);
        int best = 1 << 30;
        std::vector<int> bc, bk;
        const int nc = (int)cos.size();
        for (int c0 = 0; c0 < nc; ++c0)
            for (int c1 = c0 + 1; c1 < nc; ++c1)
                for (int c2 = c1 + 1; c2 < nc; ++c2)
                    for (int k0 = 0; k0 < kFBlock; ++k0)
                        for (int k1 = k0 + 1; k1 < kFBlock; ++k1) {
                            const int lb[5] = {cos[c0], cos[c1], cos[c2], b0.bits[k0], b0.bits[k1]};
                            std::vector<ITYPE> sectors;
                            for (int lane = 0; lane < 32; ++lane) {
                                ITYPE g = 0;
                                for (int i = 0; i < 5; ++i)
                                    if ((lane >> i) & 1) g |= 1ULL << fp.q[lb[i]];
                                sectors.push_back(g >> 2);  // 4 complex64 amplitudes per 32-byte sector
                            }
                            std::sort(sectors.begin(), sectors.end());
                            const int cost = (int)(std::unique(sectors.begin(), sectors.end()) - sectors.begin());
                            if (cost < best) {
                                best = cost;
                                bc = {cos[c0], cos[c1], cos[c2]};
                                bk = {k0, k1};
                            }
                        }
        b0.lay.coset_bits = order_with_prefix(bc, cos);
        const std::vector<int> ks = order_with_prefix(bk, locals);
        std::copy(ks.begin(), ks.end(), b0.lay.k_src);
    }
    // accumulator rows of block b: lanes 0..4 of a warp are rows y bits 0..4.  Lane bit 0 is always the
    // real/imaginary part, so lanes 2j and 2j + 1 hold the two parts of one output amplitude and the
    // device stores them as one word (bf16x2, or float2 after the last block); pick the other 4 lane
    // sources (of the 6 block bits) and the next block's K / coset orders that minimise the bank
    // conflicts of those paired stores.
    for (size_t b = 0; b < fp.blocks.size(); ++b) {
        FusedBlock& cb = fp.blocks[b];
        const bool last = b + 1 == fp.blocks.size();
        FusedBlock* nb = last ? nullptr : &fp.blocks[b + 1];
        const std::vector<int> ncos = last ? std::vector<int>() : coset_bits_of(*nb, m);
        int best = 1 << 30;
        BlockLayout best_next;
        int best_rows[7] = {6, 0, 1, 2, 3, 4, 5};
        for (int e1 = 0; e1 < kFBlock; ++e1)
            for (int e2 = e1 + 1; e2 < kFBlock; ++e2) {
                int rows[7], r = 1;
                rows[0] = 6;
                for (int s = 0; s < kFBlock; ++s)
                    if (s != e1 && s != e2) rows[r++] = s;
                rows[5] = e1;
                rows[6] = e2;
                BlockLayout trial_next;
                if (!last) {
                    std::vector<int> kpre, cpre;
                    for (int i = 0; i < 5; ++i) {
                        if (rows[i] == 6) continue;
                        const uint8_t tb = cb.bits[rows[i]];
                        const uint8_t* at = std::find(nb->bits, nb->bits + kFBlock, tb);
                        if (at != nb->bits + kFBlock) kpre.push_back((int)(at - nb->bits));
                        else cpre.push_back(tb);
                    }
                    trial_next.coset_bits = order_with_prefix(cpre, ncos);
                    const std::vector<int> ks = order_with_prefix(kpre, locals);
                    std::copy(ks.begin(), ks.end(), trial_next.k_src);
                }
                BlockLayout probe = cb.lay;
                std::copy(rows, rows + 7, probe.row_src);
                // one paired store instruction: lane l writes the amplitude of row pair l / 2 at column
                // 0 (even lanes) or 8 (odd lanes); offsets are XOR-linear, so column 0 stands for all
                const uint32_t u8 = coset_tile_index(cb.lay, 8);
                uint32_t words[64];
                int nwords = 0;
                for (uint32_t lane = 0; lane < 32; ++lane) {
                    uint32_t part;
                    const uint32_t u = row_tile_index(cb.bits, probe, lane & ~1u, &part) ^ ((lane & 1) ? u8 : 0u);
                    if (last) {  // float2 of (re, im): two words
                        words[nwords++] = 2 * tswz(u);
                        words[nwords++] = 2 * tswz(u) + 1;
                    } else {     // bf16x2 of (re, im): one word
                        words[nwords++] = b_operand_off(nb->bits, trial_next, u, 0) >> 2;
                    }
                }
                const int cost = bank_degree(words, nwords);
                if (cost < best) {
                    best = cost;
                    std::copy(rows, rows + 7, best_rows);
                    if (!last) best_next = trial_next;
                }
            }
        std::copy(best_rows, best_rows + 7, cb.lay.row_src);
        if (!last) {
            std::copy(best_next.k_src, best_next.k_src + kFBlock, nb->lay.k_src);
            nb->lay.coset_bits = best_next.coset_bits;
        }
    }
}

// Device tables of block b (rowtab / coltab into the next block's B operand, or into the output tile
// after the last block; gn / gj for the tile -> B gather of a pass's first block).
static void build_tables(const FusedPass& fp, size_t b, int m, std::vector<uint32_t>* t) {
    const FusedBlock& cb = fp.blocks[b];
    const FusedBlock* nb = b + 1 < fp.blocks.size() ? &fp.blocks[b + 1] : nullptr;
    const uint32_t N = 1u << (m - kFBlock);
    t->assign(kTabWords, 0);
    for (uint32_t y = 0; y < 128; ++y) {
        uint32_t part;
        const uint32_t u = row_tile_index(cb.bits, cb.lay, y, &part);
        (*t)[kTabRow + y] = nb ? b_operand_off(nb->bits, nb->lay, u, part) : (2 * tswz(u) | part);
    }
    // global amplitude offset of tile index u (tile bit j <-> qubit q[j])
    auto global_off = [&](uint32_t u) {
        ITYPE g = 0;
        for (int j = 0; j < m; ++j)
            if ((u >> j) & 1) g |= 1ULL << fp.q[j];
        return g;
    };
    auto put64 = [&](int word, ITYPE v) {
        (*t)[word] = (uint32_t)v;
        (*t)[word + 1] = (uint32_t)(v >> 32);
    };
    for (uint32_t n = 0; n < N; ++n) {
        const uint32_t u = coset_tile_index(cb.lay, n);
        (*t)[kTabCol + n] = nb ? b_operand_off(nb->bits, nb->lay, u, 0) : 2 * tswz(u);
        put64(kTabGn + 2 * n, global_off(u));
    }
    for (uint32_t j = 0; j < 64; ++j) put64(kTabGj + 2 * j, global_off(k_tile_index(cb, j)));
}

int fused_plan_host(const Circuit& c, FusedPlanHost* P) {
    const UINT n = c.n;
    for (const GateRec& g : c.gates)
        if (!fusable(g)) return set_error(QS_ERR_NOT_SUPPORTED, "fused path: gate over more than 6 qubits or a noise channel");
    const int m = (int)std::min<UINT>(kFTileMax, n);
    if ((int)n - m > 6 * kDepChunks) return set_error(QS_ERR_NOT_SUPPORTED, "fused path: too many tiles");
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
                apply_gate_to_block(U, kFBlock, g, pos);
            }
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
        choose_layouts(fp);
        for (size_t b = 0; b < fp.blocks.size(); ++b) {
            build_image(fp.blocks[b].U, fp.blocks[b].lay, &fp.blocks[b].image);
            build_tables(fp, b, (int)fp.q.size(), &fp.blocks[b].tabs);
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

// Shared memory of a fused CTA: A (hi | lo), two B / output tiles laid out for the largest tile (every
// pass uses the same layout), two table slots, the pass's address tables, 3 mbarriers, the TMEM slot
// and the error flag.
static size_t fused_smem_bytes() {
    return 2 * kAImageBytes + 2 * (2 * (size_t)kFNMax * 256) + 2 * kTabBytes + kAddrTabBytes + 64;
}

// The kernel's dynamic shared-memory limit is a process-wide attribute: set it once per device to
// the largest tile's need (a launch may use less), never per launch, so concurrent host threads
// launching passes of different tile sizes cannot undo each other's setting.
static int fused_allow_smem() {
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    QS_CUDA_CHECK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 0 || dev >= 64) return set_error(QS_ERR_NOT_SUPPORTED, "device index");
    if (!done[dev]) {
        QS_CUDA_CHECK(cudaFuncSetAttribute(k_fused_pass, cudaFuncAttributeMaxDynamicSharedMemorySize,
            (int)fused_smem_bytes()));
        QS_CUDA_CHECK(cudaFuncSetAttribute(k_fused_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
            (int)fused_smem_bytes()));
        done[dev] = true;
    }
    return QS_OK;
}

static int upload_fused_plan(Circuit& c, ITYPE dim, const FusedPlanHost& H, std::shared_ptr<FusedPlanDev>* out);

// Device plan cached on the circuit (dropped when a gate is added).
static int fused_plan_dev(Circuit& c, ITYPE dim, std::shared_ptr<FusedPlanDev>* out) {
    if (c.fused && c.fused_dim == dim) {
        *out = std::static_pointer_cast<FusedPlanDev>(c.fused);
        return QS_OK;
    }
    FusedPlanHost H;
    QS_TRY(fused_plan_host(c, &H));
    return upload_fused_plan(c, dim, H, out);
}

static int upload_fused_plan(Circuit& c, ITYPE dim, const FusedPlanHost& H, std::shared_ptr<FusedPlanDev>* out) {
    auto D = std::make_shared<FusedPlanDev>();
    D->dim = dim;
    const size_t rec_bytes = H.nblocks * (size_t)kRecordBytes;
    QS_CUDA_CHECK(cudaMalloc(&D->dev, rec_bytes + 256));
    std::vector<unsigned char> host(rec_bytes + 256, 0);
    size_t ri = 0;
    std::vector<size_t> offs;
    for (const FusedPass& p : H.passes) {
        offs.push_back(ri);
        for (const FusedBlock& b : p.blocks) {
            memcpy(host.data() + ri, b.image.data(), 2 * kAImageBytes);
            memcpy(host.data() + ri + 2 * kAImageBytes, b.tabs.data(), kTabBytes);
            ri += kRecordBytes;
        }
    }
    QS_CUDA_CHECK(cudaMemcpy(D->dev, host.data(), host.size(), cudaMemcpyHostToDevice));
    D->err = (int*)((char*)D->dev + rec_bytes);
    QS_CUDA_CHECK(cudaMemset(D->err, 0, sizeof(int)));
    for (size_t i = 0; i < H.passes.size(); ++i) {
        FusedPassArgs a{};
        a.m = (int)H.passes[i].q.size();
        a.nblocks = (int)H.passes[i].blocks.size();
        for (int j = 0; j < a.m; ++j) a.q[j] = H.passes[i].q[j];
        a.records = (const unsigned char*)D->dev + offs[i];
        a.tiles = dim >> a.m;
        a.err = D->err;
        D->passes.push_back(a);
    }
    c.fused = D;
    c.fused_dim = dim;
    *out = D;
    return QS_OK;
}

// Many circuits, each on its own complex64 state: the plans missing from the circuits' caches are
// built on host threads in parallel (the FP64 block composition and layout search dominate a small
// circuit's cost), then every circuit's passes run in ONE persistent launch of k_fused_batch (work
// items: tile pairs of (circuit, pass) records in pass-round-robin order, bounded dependency waits),
// with one error-flag read.
constexpr unsigned long long kFusedBatchWaitNs = 2000000000ULL;

int batch_update_fused_c64(Circuit* const* cs, void* const* states, UINT count, cudaStream_t st,
    unsigned long long wait_ns, int self_dep) {
    for (UINT i = 0; i < count; ++i) {
        if (!cs[i] || !states[i]) return set_error(QS_ERR_INVALID_ARGUMENT, "null circuit or state");
        if (cs[i]->n < 10) return set_error(QS_ERR_NOT_SUPPORTED, "fused path needs at least 10 qubits");
    }
    if (count == 0) return QS_OK;
    // 1. host plans in parallel
    std::vector<FusedPlanHost> H(count);
    std::vector<int> rc(count, QS_OK), need(count, 0);
    for (UINT i = 0; i < count; ++i) {
        const ITYPE dim = 1ULL << cs[i]->n;
        need[i] = !(cs[i]->fused && cs[i]->fused_dim == dim);
        for (UINT j = 0; j < i && need[i]; ++j)  // the same circuit twice: build once
            if (cs[j] == cs[i]) need[i] = 0;
    }
    {
        std::atomic<UINT> next{0};
        const unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nt; ++t)
            pool.emplace_back([&] {
                for (UINT i; (i = next.fetch_add(1)) < count;)
                    if (need[i]) rc[i] = fused_plan_host(*cs[i], &H[i]);
            });
        for (std::thread& t : pool) t.join();
    }
    for (UINT i = 0; i < count; ++i)
        if (rc[i] != QS_OK) {  // rebuild here so that the error message is this thread's
            FusedPlanHost again;
            return fused_plan_host(*cs[i], &again);
        }
    // 2. uploads (device calls from this thread)
    std::vector<std::shared_ptr<FusedPlanDev>> D(count);
    for (UINT i = 0; i < count; ++i) {
        const ITYPE dim = 1ULL << cs[i]->n;
        if (need[i]) QS_TRY(upload_fused_plan(*cs[i], dim, H[i], &D[i]));
        else QS_TRY(fused_plan_dev(*cs[i], dim, &D[i]));
    }
    QS_TRY(fused_allow_smem());
    // 3. work records, pass-round-robin over the circuits
    size_t maxp = 0;
    for (UINT i = 0; i < count; ++i) maxp = std::max(maxp, D[i]->passes.size());
    std::vector<FusedBatchRec> recs;
    std::vector<int> last(count, -1);
    ITYPE total = 0;
    for (size_t p = 0; p < maxp; ++p)
        for (UINT i = 0; i < count; ++i) {
            if (p >= D[i]->passes.size()) continue;
            FusedBatchRec r{};
            r.args = D[i]->passes[p];
            r.args.state = (float2*)states[i];
            r.prefix = total;
            r.dep = last[i];
            last[i] = (int)recs.size();
            total += (r.args.tiles + 1) / 2;  // tile pairs
            recs.push_back(r);
        }
    if (recs.empty()) return QS_OK;
    if (self_dep >= 0) {
        if (self_dep >= (int)recs.size()) return set_error(QS_ERR_INVALID_ARGUMENT, "batch: no such work record");
        recs[self_dep].dep = self_dep;
    }
    const size_t brec = sizeof(FusedBatchRec) * recs.size(), bdone = sizeof(unsigned) * recs.size();
    void* buf = nullptr;
    QS_TRY(scratch(st, brec + bdone + 256, &buf));
    FusedBatchRec* drec = (FusedBatchRec*)buf;
    unsigned* ddone = (unsigned*)((char*)buf + brec);
    unsigned long long* dhead = (unsigned long long*)((char*)buf + ((brec + bdone + 15) / 16 * 16));
    int* derr = (int*)(dhead + 1);
    QS_CUDA_CHECK(cudaMemcpyAsync(drec, recs.data(), brec, cudaMemcpyHostToDevice, st));
    QS_CUDA_CHECK(cudaMemsetAsync(ddone, 0, (brec + bdone + 256) - brec, st));
    int per_sm = 0;
    QS_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fused_batch, kFThreads, fused_smem_bytes()));
    const ITYPE resident = (ITYPE)std::max(1, per_sm) * sm_count();
    const unsigned grid = (unsigned)std::min<ITYPE>(resident, total);
    k_fused_batch<<<grid, kFThreads, fused_smem_bytes(), st>>>(drec, (int)recs.size(), total, dhead, ddone, derr,
        wait_ns);
    QS_TRY(check_launch("k_fused_batch"));
    int err = 0;
    QS_CUDA_CHECK(cudaMemcpyAsync(&err, derr, sizeof(int), cudaMemcpyDeviceToHost, st));
    QS_CUDA_CHECK(cudaStreamSynchronize(st));
    if (err) return set_error(QS_ERR_TIMEOUT, "fused batch: a bounded wait expired");
    return QS_OK;
}

int run_fused_c64(Circuit& c, void* state, ITYPE dim, cudaStream_t st) {
    if (c.n < 10) return set_error(QS_ERR_NOT_SUPPORTED, "fused path needs at least 10 qubits");
    std::shared_ptr<FusedPlanDev> D;
    QS_TRY(fused_plan_dev(c, dim, &D));
    QS_TRY(fused_allow_smem());
    for (const FusedPassArgs& p0 : D->passes) {
        FusedPassArgs p = p0;
        p.state = (float2*)state;
        const size_t smem = fused_smem_bytes();
        const unsigned grid = (unsigned)std::min<ITYPE>((p.tiles + 1) / 2, (ITYPE)sm_count());  // tile pairs
        k_fused_pass<<<grid, kFThreads, smem, st>>>(p);
        QS_TRY(check_launch("k_fused_pass"));
    }
    int err = 0;
    QS_CUDA_CHECK(cudaMemcpyAsync(&err, D->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    QS_CUDA_CHECK(cudaStreamSynchronize(st));
    if (err) return set_error(QS_ERR_TIMEOUT, "fused pass: tensor-core completion wait expired");
    return QS_OK;
}

// Whether the tensor-core executor takes the circuit: >= 10 qubits, every gate on <= 6 qubits, no
// noise channel.
bool fused_c64_accepts(const Circuit& c) {
    if (c.n < 10) return false;
    for (const GateRec& g : c.gates)
        if (!fusable(g)) return false;
    return true;
}

// The executor of a single complex64 run: forced, or the tensor cores whenever they take the circuit,
// else FP64 passes.  Measured on a B200 over HEA, U3+CZ and layered circuits of 12..30 qubits (depth
// 4..20), the tensor-core run was the faster or equal one in 13 of 15 and at most 7 % slower in the
// other two; the FP64 passes take circuits below 10 qubits.  (Batches choose differently, see
// qs_batch_update_quantum_states_c64: there many circuits fill the device and the FP64 passes' cheaper
// small tiles win.)
int choose_c64_executor(Circuit& c, int* exec) {
    if (c.c64_exec >= 0) {
        *exec = c.c64_exec;
    } else if (fused_c64_accepts(c)) {
        *exec = 0;
    } else if (c.n >= 4) {  // the FP64 passes hold 16 amplitudes per thread
        *exec = 1;
    } else {
        return set_error(QS_ERR_NOT_SUPPORTED, "complex64 states need at least 4 qubits");
    }
    c.c64_chosen = *exec;
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

// Host-only export of fused block `index`'s operand layout and device index tables.
int fused_block_layout(Circuit& c, UINT index, int* row_source, int* k_source, UINT* coset_bits, uint32_t* tables) {
    FusedPlanHost H;
    QS_TRY(fused_plan_host(c, &H));
    UINT k = 0;
    for (const FusedPass& p : H.passes)
        for (const FusedBlock& b : p.blocks) {
            if (k++ != index) continue;
            for (int i = 0; i < 7; ++i) row_source[i] = b.lay.row_src[i];
            for (int i = 0; i < kFBlock; ++i) k_source[i] = b.lay.k_src[i];
            for (size_t i = 0; i < b.lay.coset_bits.size(); ++i) coset_bits[i] = (UINT)b.lay.coset_bits[i];
            if (tables) memcpy(tables, b.tabs.data(), kTabBytes);
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

QS_API int qs_circuit_set_c64_executor(qs_circuit_t circuit, int mode) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null circuit");
    if (mode < -1 || mode > 1) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "complex64 executor must be -1, 0 or 1");
    c->c64_exec = mode;
    return QS_OK;
}

QS_API int qs_circuit_update_quantum_state_c64(qs_circuit_t circuit, void* state_c64, QS_ITYPE dim, void* stream) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c || !state_c64) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    if (dim != (1ULL << c->n)) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "dim differs from 2^qubit_count");
    int exec = 0;
    QS_TRY(qs::choose_c64_executor(*c, &exec));
    return exec == 0 ? qs::run_fused_c64(*c, state_c64, dim, (cudaStream_t)stream)
                     : qs::run_staged_c64(*c, state_c64, dim, (cudaStream_t)stream);
}

QS_API int qs_circuit_c64_executor_info(qs_circuit_t circuit, int* chosen) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c || !chosen) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    *chosen = c->c64_chosen;
    return QS_OK;
}

QS_API int qs_circuit_update_quantum_state_fused_c64(qs_circuit_t circuit, void* state_c64, QS_ITYPE dim, void* stream) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null circuit");
    if (dim != (1ULL << c->n))
        return qs::set_error(QS_ERR_INVALID_ARGUMENT, "state dimension does not match the circuit's qubit count");
    return qs::run_fused_c64(*c, state_c64, dim, (cudaStream_t)stream);
}

QS_API int qs_batch_update_quantum_states_c64(qs_circuit_t const* circuits, void* const* states_c64, QS_UINT count,
    int exec, void* stream) {
    if (!circuits || !states_c64) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    if (exec < -1 || exec > 1) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "complex64 executor must be -1, 0 or 1");
    auto cs = reinterpret_cast<qs::Circuit* const*>(circuits);
    for (QS_UINT i = 0; i < count; ++i)
        if (!cs[i] || !states_c64[i]) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null circuit or state");
    if (exec == 0)
        return qs::batch_update_fused_c64(cs, states_c64, count, (cudaStream_t)stream, qs::kFusedBatchWaitNs, -1);
    const int rc = qs::batch_update(cs, states_c64, count, (cudaStream_t)stream, qs::kBatchWaitNs, -1, true);
    if (rc != QS_ERR_NOT_SUPPORTED || exec == 1) return rc;
    // some circuit has a gate the FP64 passes cannot stage (refused before any launch): tensor cores
    return qs::batch_update_fused_c64(cs, states_c64, count, (cudaStream_t)stream, qs::kFusedBatchWaitNs, -1);
}

QS_API int qs_batch_update_quantum_states_fused_c64(qs_circuit_t const* circuits, void* const* states_c64,
    QS_UINT count, void* stream) {
    if (!circuits || !states_c64) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    return qs::batch_update_fused_c64(reinterpret_cast<qs::Circuit* const*>(circuits), states_c64, count,
        (cudaStream_t)stream, qs::kFusedBatchWaitNs, -1);
}

// Failure-path check of the complex64 batch kernel's bounded dependency wait (the same construction as
// qs_debug_batch_wait_expiry): `circuit` on `state_c64` as a one-circuit batch whose last pass waits on
// its own completion counter, with the wait bounded by wait_limit_us.
QS_API int qs_debug_batch_wait_expiry_fused_c64(qs_circuit_t circuit, void* state_c64, QS_UINT wait_limit_us,
    void* stream) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c || !state_c64) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null circuit or state");
    if (wait_limit_us == 0 || wait_limit_us > 2000000u)
        return qs::set_error(QS_ERR_INVALID_ARGUMENT, "wait limit must be 1 us .. 2 s");
    if (c->n < 10) return qs::set_error(QS_ERR_NOT_SUPPORTED, "fused path needs at least 10 qubits");
    qs::FusedPlanHost H;
    QS_TRY(qs::fused_plan_host(*c, &H));
    if (H.passes.empty()) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "circuit has no passes");
    qs::Circuit* cs[1] = {c};
    void* ss[1] = {state_c64};
    return qs::batch_update_fused_c64(cs, ss, 1, (cudaStream_t)stream, 1000ULL * wait_limit_us,
        (int)H.passes.size() - 1);
}

QS_API int qs_circuit_fused_block_export(qs_circuit_t circuit, QS_UINT index, QS_UINT* tile_qubits, int* tile_qubit_count,
    QS_UINT* block_bits, double* matrix, unsigned short* operand_image) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c || !tile_qubits || !tile_qubit_count || !block_bits) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    return qs::fused_block_export(*c, index, tile_qubits, tile_qubit_count, block_bits, matrix, operand_image);
}

QS_API int qs_circuit_fused_block_layout(qs_circuit_t circuit, QS_UINT index, int* row_source, int* k_source,
    QS_UINT* coset_bits, unsigned int* tables) {
    auto* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c || !row_source || !k_source || !coset_bits) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    return qs::fused_block_layout(*c, index, row_source, k_source, coset_bits, tables);
}

QS_API int qs_circuit_fused_stats(qs_circuit_t circuit, QS_UINT* passes, QS_UINT* blocks) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c || !passes || !blocks) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    return qs::fused_stats(*c, passes, blocks);
}

}  // extern "C"
