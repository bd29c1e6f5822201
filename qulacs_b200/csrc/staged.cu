// Staged executor: several gates per HBM pass, each gate applied with its own (unfused) arithmetic.
//
// A pass owns a set Q of m "tile qubits" (always including qubits 0..3, so every HBM access is a
// run of >= 16 contiguous amplitudes = 256 B).  Each CTA loads one tile -- the 2^m amplitudes that
// share the values of the other n - m qubits -- into shared memory, applies every gate of the pass
// (all of whose qubits lie in Q), and writes the tile back: one read and one write of the state per
// pass instead of one per gate.  Inside the tile, gates are grouped into "phases" of at most 4 tile
// qubits: each thread gathers the 16 amplitudes of its 4-qubit coset into registers, applies all the
// phase's gates there, and scatters them back, so shared memory is touched once per phase, not once
// per gate.  The host scheduler (below) builds passes and phases greedily from the gate list; a gate
// is only moved past gates on disjoint qubits, so the result equals gate-by-gate application up to
// rounding order (~1e-16).  Gates the pass kernel does not cover (more than 2 targets, controls,
// Pauli strings, multi-qubit diagonals) run between passes with the gate-by-gate kernels.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <memory>
#include <string>
#include <mutex>
#include <thread>
#include <vector>

#include "circuit.hpp"
#include "qs_internal.cuh"
#include "staged.hpp"

namespace qs {

struct StPassArgs {
    int m;                 // tile bits (<= kTileBits)
    int nphases;
    int io;                // bit 0: the first phase gathers from HBM; bit 1: the last phase scatters to HBM
    UINT q[kTileBits];     // global qubit of tile bit j, ascending, q[j] = j for j < kLowFixed
    const StPhase* phases;
    const StOp* ops;
    const double2* pool;
};

// ---------------------------------------------------------------- register ops
template <int B>
__device__ __forceinline__ void r_dense1(double2 (&r)[16], const double2* __restrict__ p) {
    const double2 m0 = p[0], m1 = p[1], m2 = p[2], m3 = p[3];
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (!(j & (1 << B))) {
            const double2 x = r[j], y = r[j | (1 << B)];
            r[j] = cfma(m1, y, cmul(m0, x));
            r[j | (1 << B)] = cfma(m3, y, cmul(m2, x));
        }
}
template <int B>
__device__ __forceinline__ void r_diag1(double2 (&r)[16], const double2* __restrict__ p) {
    const double2 d0 = p[0], d1 = p[1];
#pragma unroll
    for (int j = 0; j < 16; ++j) r[j] = cmul((j & (1 << B)) ? d1 : d0, r[j]);
}
// RX: {c, i s; i s, c}
template <int B>
__device__ __forceinline__ void r_rx(double2 (&r)[16], const double2* __restrict__ p) {
    const double c = p[0].x, s = p[0].y;
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (!(j & (1 << B))) {
            const double2 x = r[j], y = r[j | (1 << B)];
            r[j] = make_double2(fma(c, x.x, -s * y.y), fma(c, x.y, s * y.x));
            r[j | (1 << B)] = make_double2(fma(c, y.x, -s * x.y), fma(c, y.y, s * x.x));
        }
}
// RY: {c, s; -s, c}
template <int B>
__device__ __forceinline__ void r_ry(double2 (&r)[16], const double2* __restrict__ p) {
    const double c = p[0].x, s = p[0].y;
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (!(j & (1 << B))) {
            const double2 x = r[j], y = r[j | (1 << B)];
            r[j] = make_double2(fma(c, x.x, s * y.x), fma(c, x.y, s * y.y));
            r[j | (1 << B)] = make_double2(fma(c, y.x, -s * x.x), fma(c, y.y, -s * x.y));
        }
}
template <int C, int T>
__device__ __forceinline__ void r_cnot(double2 (&r)[16]) {
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if ((j & (1 << C)) && !(j & (1 << T))) {
            const double2 t = r[j];
            r[j] = r[j | (1 << T)];
            r[j | (1 << T)] = t;
        }
}
template <int A, int B>
__device__ __forceinline__ void r_cz(double2 (&r)[16]) {
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if ((j & (1 << A)) && (j & (1 << B))) r[j] = make_double2(-r[j].x, -r[j].y);
}
template <int A, int B>
__device__ __forceinline__ void r_swap(double2 (&r)[16]) {
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if ((j & (1 << A)) && !(j & (1 << B))) {
            const int k = j ^ (1 << A) ^ (1 << B);
            const double2 t = r[j];
            r[j] = r[k];
            r[k] = t;
        }
}
// matrix-index bit 0 <-> register bit A (first target), bit 1 <-> B
template <int A, int B>
__device__ __forceinline__ void r_dense2(double2 (&r)[16], const double2* __restrict__ p) {
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (!(j & (1 << A)) && !(j & (1 << B))) {
            const int o[4] = {j, j | (1 << A), j | (1 << B), j | (1 << A) | (1 << B)};
            double2 v[4];
#pragma unroll
            for (int x = 0; x < 4; ++x) v[x] = r[o[x]];
#pragma unroll
            for (int y = 0; y < 4; ++y) {
                double2 acc = cmul(p[y * 4], v[0]);
#pragma unroll
                for (int x = 1; x < 4; ++x) acc = cfma(p[y * 4 + x], v[x], acc);
                r[o[y]] = acc;
            }
        }
}

// Dense 2x2 along register bit A with the matrix chosen by register bit B: p[0..3] where bit B is 0,
// p[4..7] where it is 1 (a one-qubit gate on the target of a CNOT, with the CNOT folded in).
template <int A, int B>
__device__ __forceinline__ void r_csel1(double2 (&r)[16], const double2* __restrict__ p) {
    const double2 m0 = p[0], m1 = p[1], m2 = p[2], m3 = p[3];
    const double2 n0 = p[4], n1 = p[5], n2 = p[6], n3 = p[7];
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (!(j & (1 << A))) {
            const double2 x = r[j], y = r[j | (1 << A)];
            const bool hi = (j >> B) & 1;
            r[j] = cfma(hi ? n1 : m1, y, cmul(hi ? n0 : m0, x));
            r[j | (1 << A)] = cfma(hi ? n3 : m3, y, cmul(hi ? n2 : m2, x));
        }
}
// A one-qubit dense gate U on the control A of CNOT(A -> B), CNOT first: for j with bits A, B clear
// and t in {0, B}, out[j^t] = U00 in[j^t] + U01 in[j^t^A^B], out[j^t^A] = U10 in[j^t] + U11 in[j^t^A^B].
template <int A, int B>
__device__ __forceinline__ void r_d1_in(double2 (&r)[16], const double2* __restrict__ p) {
    const double2 m0 = p[0], m1 = p[1], m2 = p[2], m3 = p[3];
    double2 o[16];
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (!(j & (1 << A))) {
            const int k = j ^ (1 << A) ^ (1 << B);
            const double2 x = r[j], y = r[k];
            o[j] = cfma(m1, y, cmul(m0, x));
            o[j | (1 << A)] = cfma(m3, y, cmul(m2, x));
        }
#pragma unroll
    for (int j = 0; j < 16; ++j) r[j] = o[j];
}
// The same gate with the CNOT second: out[j^t] = U00 in[j^t] + U01 in[j^t^A],
// out[j^t^A^B] = U10 in[j^t] + U11 in[j^t^A].
template <int A, int B>
__device__ __forceinline__ void r_d1_out(double2 (&r)[16], const double2* __restrict__ p) {
    const double2 m0 = p[0], m1 = p[1], m2 = p[2], m3 = p[3];
    double2 o[16];
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (!(j & (1 << A))) {
            const double2 x = r[j], y = r[j | (1 << A)];
            o[j] = cfma(m1, y, cmul(m0, x));
            o[j ^ (1 << A) ^ (1 << B)] = cfma(m3, y, cmul(m2, x));
        }
#pragma unroll
    for (int j = 0; j < 16; ++j) r[j] = o[j];
}

// One indirect branch per op: the host encodes code = kind * 16 + a * 4 + b (op_code), and every code
// has its own fully specialised register code (unused codes are empty).  One-qubit kinds use b = a;
// their b != a codes hold the CNOT-folded ops (DENSE1: ST_CSEL1, DIAG1: ST_D1_IN, RX: ST_D1_OUT), which
// keeps the switch at 128 codes -- more codes made every pass slower.  Passes without folded ops run
// the FOLDS = false build, whose switch holds only the plain ops (the folded code placed among the
// plain one-qubit cases slowed unfused schedules by 12 %).
template <int CODE, bool FOLDS>
__device__ __forceinline__ void run_code(double2 (&r)[16], const double2* p) {
    constexpr int kind = CODE >> 4, A = (CODE >> 2) & 3, B = CODE & 3;
    if constexpr (kind == ST_DENSE1 && B == A) r_dense1<A>(r, p);
    else if constexpr (FOLDS && kind == ST_DENSE1) r_csel1<A, B>(r, p);
    else if constexpr (kind == ST_DIAG1 && B == A) r_diag1<A>(r, p);
    else if constexpr (FOLDS && kind == ST_DIAG1) r_d1_in<A, B>(r, p);
    else if constexpr (kind == ST_RX && B == A) r_rx<A>(r, p);
    else if constexpr (FOLDS && kind == ST_RX) r_d1_out<A, B>(r, p);
    else if constexpr (kind == ST_RY && B == A) r_ry<A>(r, p);
    else if constexpr (kind == ST_CNOT && A != B) r_cnot<A, B>(r);
    else if constexpr (kind == ST_CZ && A != B) r_cz<A, B>(r);
    else if constexpr (kind == ST_SWAP && A != B) r_swap<A, B>(r);
    else if constexpr (kind == ST_DENSE2 && A != B) r_dense2<A, B>(r, p);
}
#define QS_CODE1(c) \
    case c: run_code<c, FOLDS>(r, p); break;
#define QS_CODE4(c) QS_CODE1(c) QS_CODE1(c + 1) QS_CODE1(c + 2) QS_CODE1(c + 3)
#define QS_CODE16(c) QS_CODE4(c) QS_CODE4(c + 4) QS_CODE4(c + 8) QS_CODE4(c + 12)
template <bool FOLDS>
__device__ __forceinline__ void apply_op(const StOp& op, double2 (&r)[16], const double2* pool) {
    const double2* p = pool + op.param;
    switch (op.pad) {
        QS_CODE16(0)
        QS_CODE16(16)
        QS_CODE16(32)
        QS_CODE16(48)
        QS_CODE16(64)
        QS_CODE16(80)
        QS_CODE16(96)
        QS_CODE16(112)
        default: break;
    }
}
#undef QS_CODE16
#undef QS_CODE4
#undef QS_CODE1

// XOR swizzle of the tile index for conflict-free 16-byte shared-memory accesses (linear over XOR,
// so swz(a | b) = swz(a) ^ swz(b) for disjoint bit sets).
__device__ __forceinline__ UINT swz(UINT u) { return u ^ (((u >> 4) ^ (u >> 7) ^ (u >> 10)) & 7u); }

// Tile index u = tid + k * kStThreads (k < 2^(m-7)) has global offset base | lo_off | hi_off[k]:
// lo_off takes tid's bits 0..6 to the tile qubits q[0..6], hi_off[k] takes k's bits to q[7..].

// Global rows of 16 amplitudes per thread from the swizzled tile to HBM (rows k0 .. k0 + 15).
template <class T>
__device__ __forceinline__ void tile_rows_store(T* __restrict__ s, const double2* tile, ITYPE off,
    const ITYPE* hi_off, UINT tsize, int k0) {
    const UINT tid = threadIdx.x;
    double2 v[16];
#pragma unroll
    for (int k = 0; k < 16; ++k)
        if (tid + (UINT)(k0 + k) * kStThreads < tsize) v[k] = tile[swz(tid + (UINT)(k0 + k) * kStThreads)];
#pragma unroll
    for (int k = 0; k < 16; ++k)
        if (tid + (UINT)(k0 + k) * kStThreads < tsize) st_amp(s + (off | hi_off[k0 + k]), v[k]);
}

// One tile of one pass: load, apply every phase, store.  Shared by the per-pass kernel and the
// persistent multi-circuit kernel.  `tile` holds 2^m amplitudes (m <= kTileBits) in FP64 whatever the
// state's type E (complex128, or complex64 widened on load and rounded on store).  Ends with a CTA
// barrier so the shared buffers can be reused immediately.
template <int MAX_BITS, bool FOLDS, class E>
__device__ __forceinline__ void staged_tile(E* __restrict__ s, const StPassArgs& a, ITYPE T, double2* tile,
    ITYPE* hi_off) {
    const int m = a.m;
    const UINT tsize = 1u << m;
    // base: insert zeros at the tile qubits into the tile index
    ITYPE base = T;
    for (int j = 0; j < m; ++j) base = insert0(base, a.q[j]);
    const int tid = threadIdx.x;
    const bool hbm_first = a.io & 1, hbm_last = (a.io >> 1) & 1;
    ITYPE lo_off = 0;
    if (!hbm_first || !hbm_last) {
        if (tid < (1 << (MAX_BITS - 7))) {
            ITYPE o = 0;
            for (int j = 7; j < m; ++j)
                if ((tid >> (j - 7)) & 1) o |= 1ULL << a.q[j];
            hi_off[tid] = o;
        }
        for (int j = 0; j < 7 && j < m; ++j)
            if ((tid >> j) & 1) lo_off |= 1ULL << a.q[j];
        __syncthreads();
    }
    if (!hbm_first) {
        const ITYPE off = base | lo_off;
        if constexpr (sizeof(E) == sizeof(double2)) {
            // 16-byte cp.async copies straight into the swizzled tile: every copy of a thread in flight at
            // once, without holding registers
#pragma unroll
            for (int k = 0; k < (1 << (MAX_BITS - 7)); ++k)
                if ((UINT)tid + (UINT)k * kStThreads < tsize) {
                    const unsigned dst =
                        (unsigned)__cvta_generic_to_shared(tile + swz((UINT)tid + (UINT)k * kStThreads));
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(s + (off | hi_off[k]))
                                 : "memory");
                }
            asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
        } else {
            // complex64: widened in registers, 4 loads in flight per thread before their stores
#pragma unroll
            for (int k0 = 0; k0 < (1 << (MAX_BITS - 7)); k0 += 4) {
                double2 v[4];
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if ((UINT)tid + (UINT)(k0 + k) * kStThreads < tsize) v[k] = ld_amp(s + (off | hi_off[k0 + k]));
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if ((UINT)tid + (UINT)(k0 + k) * kStThreads < tsize)
                        tile[swz((UINT)tid + (UINT)(k0 + k) * kStThreads)] = v[k];
            }
        }
        __syncthreads();
    }
    const UINT ncos = tsize >> kPhaseBits;  // cosets per phase
    char* tile_bytes = reinterpret_cast<char*>(tile);
    for (int ph = 0; ph < a.nphases; ++ph) {
        const StPhase P = a.phases[ph];
        // The first phase may gather its cosets straight from HBM and the last scatter them straight to
        // HBM (the host sets this when the phase's bits are all >= 4, so that a coset's lanes 0..15 cover
        // 16 consecutive amplitudes): no tile load or store round through shared memory.
        const bool from_hbm = hbm_first && ph == 0, to_hbm = hbm_last && ph == a.nphases - 1;
        // Byte offset of register amplitude j from the coset's first one: the XOR of sb[p] over the set
        // bits p of j (the swizzle is XOR-linear); in HBM, the XOR of gb[p].  The 16 amplitudes are
        // visited in Gray-code order so that each address is the previous one with one offset XORed in.
        UINT sb[4];
        ITYPE gb[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            sb[p] = swz(1u << P.bits[p]) << 4;
            gb[p] = 1ULL << a.q[P.bits[p]];
        }
        for (UINT c = tid; c < ncos; c += kStThreads) {
            UINT u0 = c;
#pragma unroll
            for (int p = 0; p < 4; ++p) u0 = (UINT)insert0(u0, P.bits[p]);
            ITYPE g0 = base;  // global index of the coset's first amplitude (only for HBM phases)
            if (from_hbm || to_hbm)
                for (int j = 0; j < m; ++j)
                    if ((u0 >> j) & 1) g0 |= 1ULL << a.q[j];
            double2 r[16];
            UINT addr = swz(u0) << 4;
            if (from_hbm) {
                ITYPE gi = g0;
#pragma unroll
                for (int g = 0; g < 16; ++g) {
                    if (g) gi ^= gb[(g & 1) ? 0 : (g & 2) ? 1 : (g & 4) ? 2 : 3];
                    r[g ^ (g >> 1)] = ld_amp(s + gi);
                }
            } else {
#pragma unroll
                for (int g = 0; g < 16; ++g) {
                    if (g) addr ^= sb[(g & 1) ? 0 : (g & 2) ? 1 : (g & 4) ? 2 : 3];
                    r[g ^ (g >> 1)] = *reinterpret_cast<const double2*>(tile_bytes + addr);
                }
                addr = swz(u0) << 4;
            }
            for (UINT o = 0; o < P.op_count; ++o) apply_op<FOLDS>(a.ops[P.op_begin + o], r, a.pool);
            if (to_hbm) {
                ITYPE gi = g0;
#pragma unroll
                for (int g = 0; g < 16; ++g) {
                    if (g) gi ^= gb[(g & 1) ? 0 : (g & 2) ? 1 : (g & 4) ? 2 : 3];
                    st_amp(s + gi, r[g ^ (g >> 1)]);
                }
            } else {
#pragma unroll
                for (int g = 0; g < 16; ++g) {
                    if (g) addr ^= sb[(g & 1) ? 0 : (g & 2) ? 1 : (g & 4) ? 2 : 3];
                    *reinterpret_cast<double2*>(tile_bytes + addr) = r[g ^ (g >> 1)];
                }
            }
        }
        if (!to_hbm) __syncthreads();
    }
    if (!hbm_last) {
        tile_rows_store(s, tile, base | lo_off, hi_off, tsize, 0);
        if constexpr (MAX_BITS > 11)
            if (tsize > 16 * kStThreads) tile_rows_store(s, tile, base | lo_off, hi_off, tsize, 16);
    }
    __syncthreads();
}

// One CTA per tile; the tile (2^m x 16 bytes, up to 64 KiB) is dynamic shared memory.
template <bool FOLDS, class E>
__global__ void __launch_bounds__(kStThreads, 3) k_staged_pass(E* __restrict__ s, const __grid_constant__ StPassArgs a) {
    extern __shared__ double2 st_tile[];
    __shared__ ITYPE hi_off[1 << (kTileBits - 7)];
    staged_tile<kTileBits, FOLDS>(s, a, blockIdx.x, st_tile, hi_off);
}

// Opt k_staged_pass in to 64 KiB of dynamic shared memory, once per device.
static int staged_allow_smem() {
    static std::mutex mu;
    static std::vector<char> done;
    int dev = 0;
    QS_CUDA_CHECK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if ((int)done.size() <= dev) done.resize(dev + 1, 0);
    if (!done[dev]) {
        QS_CUDA_CHECK(cudaFuncSetAttribute(k_staged_pass<false, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
            (int)(sizeof(double2) << kTileBits)));
        QS_CUDA_CHECK(cudaFuncSetAttribute(k_staged_pass<true, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
            (int)(sizeof(double2) << kTileBits)));
        QS_CUDA_CHECK(cudaFuncSetAttribute(k_staged_pass<false, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
            (int)(sizeof(double2) << kTileBits)));
        QS_CUDA_CHECK(cudaFuncSetAttribute(k_staged_pass<true, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
            (int)(sizeof(double2) << kTileBits)));
        done[dev] = 1;
    }
    return QS_OK;
}


// ---------------------------------------------------------------- host scheduler
using cd = std::complex<double>;

static bool stageable(const GateRec& g) {
    if (!g.controls.empty()) return false;
    switch (g.kind) {
        case QS_GATE_RX:
        case QS_GATE_RY:
        case QS_GATE_RZ:
        case QS_GATE_CNOT:
        case QS_GATE_CZ:
        case QS_GATE_SWAP: return true;
        case QS_GATE_DENSE: return g.targets.size() <= 2;
        case QS_GATE_DIAGONAL: return g.targets.size() == 1;
        default: return false;
    }
}

static ITYPE qmask(const std::vector<UINT>& qs) {
    ITYPE m = 0;
    for (UINT q : qs) m |= 1ULL << q;
    return m;
}

struct PassPlan {
    bool single = false;  // a gate run by the gate-by-gate kernels
    int gate = -1;
    std::vector<UINT> q;  // tile qubits (ascending)
    std::vector<int> gates;
};

// Absorb greedily in program order with a fixed tile set; returns the absorbed gate indices.
static std::vector<int> absorb(const std::vector<GateRec>& G, const std::vector<int>& pending, ITYPE Q, UINT n) {
    std::vector<int> out;
    ITYPE blocked = 0;
    const ITYPE all = (n >= 64) ? ~0ULL : ((1ULL << n) - 1);
    for (int gi : pending) {
        const ITYPE gm = qmask(G[gi].qubits());
        if ((gm & blocked) || !stageable(G[gi]) || (gm & ~Q)) {
            blocked |= gm;
            if ((blocked & all) == all) break;
            continue;
        }
        out.push_back(gi);
    }
    return out;
}

// Grow Q greedily in program order (capacity m), absorbing as we go.
static ITYPE greedy_q(const std::vector<GateRec>& G, const std::vector<int>& pending, ITYPE Q, int m) {
    ITYPE blocked = 0;
    for (int gi : pending) {
        const ITYPE gm = qmask(G[gi].qubits());
        if ((gm & blocked) || !stageable(G[gi])) {
            blocked |= gm;
            continue;
        }
        if ((gm & ~Q) == 0) continue;
        if (__builtin_popcountll(Q | gm) <= m) Q |= gm;
        else blocked |= gm;
    }
    return Q;
}

static std::vector<PassPlan> plan_passes(const std::vector<GateRec>& G, UINT n, int tile_bits) {
    std::vector<PassPlan> plan;
    std::vector<int> pending(G.size());
    for (size_t i = 0; i < G.size(); ++i) pending[i] = (int)i;
    const int m = (int)std::min<UINT>((UINT)tile_bits, n);
    const int low = std::min(kLowFixed, m);
    const ITYPE lowmask = (1ULL << low) - 1;
    while (!pending.empty()) {
        if (!stageable(G[pending[0]])) {
            PassPlan p;
            p.single = true;
            p.gate = pending[0];
            plan.push_back(p);
            pending.erase(pending.begin());
            continue;
        }
        // candidate tile sets: greedy in program order, and windows of consecutive high qubits
        std::vector<ITYPE> cands;
        cands.push_back(greedy_q(G, pending, lowmask, m));
        for (int a = low; a + (m - low) <= (int)n; ++a) {
            ITYPE Q = lowmask;
            for (int j = 0; j < m - low; ++j) Q |= 1ULL << (a + j);
            cands.push_back(Q);
        }
        std::vector<int> best;
        ITYPE bestQ = 0;
        for (ITYPE Q : cands) {
            std::vector<int> got = absorb(G, pending, Q, n);
            if (got.size() > best.size()) {
                best = got;
                bestQ = Q;
            }
        }
        if (best.empty()) {  // cannot happen for a stageable front gate; keep progress anyway
            PassPlan p;
            p.single = true;
            p.gate = pending[0];
            plan.push_back(p);
            pending.erase(pending.begin());
            continue;
        }
        // pad Q to m qubits with the lowest unused ones
        for (UINT q = 0; q < n && __builtin_popcountll(bestQ) < m; ++q) bestQ |= 1ULL << q;
        PassPlan p;
        for (UINT q = 0; q < n; ++q)
            if (bestQ >> q & 1ULL) p.q.push_back(q);
        p.gates = best;
        plan.push_back(p);
        std::vector<char> taken(G.size(), 0);
        for (int gi : best) taken[gi] = 1;
        std::vector<int> rest;
        for (int gi : pending)
            if (!taken[gi]) rest.push_back(gi);
        pending.swap(rest);
    }
    return plan;
}

struct DevPass {
    bool single;
    bool folds;  // the pass has CNOT-folded ops
    int gate;
    StPassArgs args;
    size_t phase_begin = 0;  // the pass's phases in StagedPlan::phases
    void* spec = nullptr;    // specialised kernel of this pass (pass_codegen.cpp), if compiled
    std::vector<double2> spec_params;  // its parameter block
};

template <class E>
static void launch_pass(E* state, const DevPass& d, ITYPE tiles, cudaStream_t st) {
    const size_t smem = sizeof(double2) << d.args.m;  // the tile is FP64 for either state type
    if (d.folds) k_staged_pass<true, E><<<(unsigned)tiles, kStThreads, smem, st>>>(state, d.args);
    else k_staged_pass<false, E><<<(unsigned)tiles, kStThreads, smem, st>>>(state, d.args);
}

struct StagedPlan {
    ITYPE dim = 0;
    std::vector<DevPass> passes;
    void* dev = nullptr;  // phases | ops | pool
    // host copies of the schedule (for specialised pass kernels)
    std::vector<StPhase> phases;
    std::vector<StOp> ops;
    std::vector<double2> pool;
    bool specialized = false;  // every pass has its specialised kernel
    double compile_ms = 0.;    // wall time of compiling them
    ~StagedPlan() {
        if (dev) cudaFree(dev);
    }
};

// Tile-local bit of a global qubit.
static int local_bit(const std::vector<UINT>& q, UINT g) {
    for (size_t j = 0; j < q.size(); ++j)
        if (q[j] == g) return (int)j;
    return -1;
}

// Dispatch code of an op (see run_code).
static uint8_t op_code(const StOp& o) {
    int kind = o.kind;
    if (kind == ST_CSEL1) kind = ST_DENSE1;
    else if (kind == ST_D1_IN) kind = ST_DIAG1;
    else if (kind == ST_D1_OUT) kind = ST_RX;
    return (uint8_t)(kind * 16 + o.a * 4 + o.b);
}

// Fold CNOTs into a neighbouring one-qubit dense op of the same phase (ops [begin, end) of `ops`, in
// program order), which costs the CNOT's register moves and dispatch nothing: a CNOT whose nearest
// earlier op on its two register bits is a dense op U (on either bit) runs at U's place, after it;
// failing that, one whose nearest later op on them is a dense op runs at that op's place, before it.
// A folded CNOT takes its host op's place in the order, so a CNOT is not moved past an earlier folded
// CNOT on the same bits.
// On the target T: CNOT.U_T = U (control 0) / X U (control 1); U_T.CNOT = U / U X (ST_CSEL1).  On the
// control C: U_C.CNOT pairs (c, t) with (c^1, t^1) on input (ST_D1_IN), CNOT.U_C on output (ST_D1_OUT).
// A CZ folds the same way into a dense op on either of its qubits: CZ.U = U / Z U, U.CZ = U / U Z.
static void absorb_cnots(std::vector<StOp>& ops, std::vector<double2>& pool, size_t begin) {
    auto touches = [](const StOp& o, int bit) {
        const bool two = o.kind == ST_CNOT || o.kind == ST_CZ || o.kind == ST_SWAP || o.kind == ST_DENSE2 ||
                         o.kind == ST_CSEL1 || o.kind == ST_D1_IN || o.kind == ST_D1_OUT;
        return o.a == bit || (two && o.b == bit);
    };
    const size_t end = ops.size();
    std::vector<char> dead(end, 0);
    std::vector<size_t> at_op(end);  // place of each op in the order (a folded CNOT: its host op)
    for (size_t i = begin; i < end; ++i) at_op[i] = i;
    for (size_t i = begin; i < end; ++i) {
        if (ops[i].kind != ST_CNOT && ops[i].kind != ST_CZ) continue;
        const bool cz = ops[i].kind == ST_CZ;
        const int c = ops[i].a, t = ops[i].b;
        // a folded CNOT on c or t placed strictly between lo and hi forbids the move
        auto blocked = [&](size_t lo, size_t hi) {
            for (size_t j = begin; j < end; ++j)
                if (dead[j] && at_op[j] > lo && at_op[j] < hi && (touches(ops[j], c) || touches(ops[j], t)))
                    return true;
            return false;
        };
        auto fold = [&](size_t k, bool cnot_first) {
            StOp& u = ops[k];
            const double2 m0 = pool[u.param], m1 = pool[u.param + 1], m2 = pool[u.param + 2], m3 = pool[u.param + 3];
            const uint32_t at = (uint32_t)pool.size();
            const double2 n0 = make_double2(-m0.x, -m0.y), n1 = make_double2(-m1.x, -m1.y),
                          n2 = make_double2(-m2.x, -m2.y), n3 = make_double2(-m3.x, -m3.y);
            if (cz) {  // the other qubit selects U or its sign-flipped form
                u.kind = ST_CSEL1;
                u.b = (uint8_t)(u.a == t ? c : t);
                for (const double2& v : {m0, m1, m2, m3}) pool.push_back(v);
                if (cnot_first) for (const double2& v : {m0, n1, m2, n3}) pool.push_back(v);  // U Z
                else for (const double2& v : {m0, m1, n2, n3}) pool.push_back(v);             // Z U
            } else if (u.a == t) {
                u.kind = ST_CSEL1;
                u.b = (uint8_t)c;
                for (const double2& v : {m0, m1, m2, m3}) pool.push_back(v);
                if (cnot_first) for (const double2& v : {m1, m0, m3, m2}) pool.push_back(v);  // U X
                else for (const double2& v : {m2, m3, m0, m1}) pool.push_back(v);             // X U
            } else {
                u.kind = cnot_first ? ST_D1_IN : ST_D1_OUT;
                u.b = (uint8_t)t;
                for (const double2& v : {m0, m1, m2, m3}) pool.push_back(v);
            }
            u.param = at;
            dead[i] = 1;
            at_op[i] = k;
        };
        for (size_t k = i; k-- > begin;) {
            if (dead[k] || !(touches(ops[k], c) || touches(ops[k], t))) continue;
            if (ops[k].kind == ST_DENSE1 && !blocked(k, i)) fold(k, false);
            break;
        }
        if (dead[i]) continue;
        for (size_t k = i + 1; k < end; ++k) {
            if (dead[k] || !(touches(ops[k], c) || touches(ops[k], t))) continue;
            if (ops[k].kind == ST_DENSE1 && !blocked(i, k)) fold(k, true);
            break;
        }
    }
    size_t w = begin;
    for (size_t i = begin; i < end; ++i)
        if (!dead[i]) {
            ops[i].pad = op_code(ops[i]);
            ops[w++] = ops[i];
        }
    ops.resize(w);
}

struct HostPlan {
    std::vector<PassPlan> passes;
    std::vector<StPhase> phases;
    std::vector<StOp> ops;
    std::vector<double2> pool;
    struct Range {
        size_t phase_begin, nphases;
    };
    std::vector<Range> pp;
};

// Host-only part of planning: passes, phases and encoded ops (no device calls).
static void make_host_plan(const std::vector<GateRec>& gates, UINT n, HostPlan* H, int tile_bits = kTileBits) {
    H->passes = plan_passes(gates, n, tile_bits);
    const std::vector<PassPlan>& passes = H->passes;
    std::vector<StPhase>& phases = H->phases;
    std::vector<StOp>& ops = H->ops;
    std::vector<double2>& pool = H->pool;
    std::vector<HostPlan::Range>& pp = H->pp;
    for (const PassPlan& p : passes) {
        if (p.single) {
            pp.push_back({0, 0});
            continue;
        }
        const size_t ph0 = phases.size();
        // phases: greedy over the pass's gates (program order) with 4 register bits each
        std::vector<int> todo = p.gates;
        const int m = (int)p.q.size();
        while (!todo.empty()) {
            std::vector<int> lb;  // per gate: its tile-local bits
            // candidates: greedy in order, and windows of 4 consecutive tile bits
            auto bits_of = [&](int gi) {
                ITYPE bm = 0;
                for (UINT g : gates[gi].qubits()) bm |= 1ULL << local_bit(p.q, g);
                return bm;
            };
            auto take = [&](ITYPE R, std::vector<int>* got) {
                ITYPE blocked = 0;
                for (int gi : todo) {
                    const ITYPE bm = bits_of(gi);
                    if ((bm & blocked) || (bm & ~R)) {
                        blocked |= bm;
                        continue;
                    }
                    got->push_back(gi);
                }
            };
            std::vector<ITYPE> cands;
            {
                ITYPE R = 0, blocked = 0;
                for (int gi : todo) {
                    const ITYPE bm = bits_of(gi);
                    if (bm & blocked) {
                        blocked |= bm;
                        continue;
                    }
                    if (__builtin_popcountll(R | bm) <= kPhaseBits) R |= bm;
                    else blocked |= bm;
                }
                cands.push_back(R);
            }
            for (int a0 = 0; a0 + kPhaseBits <= m; ++a0) cands.push_back(((1ULL << kPhaseBits) - 1) << a0);
            std::vector<int> best;
            ITYPE bestR = 0;
            for (ITYPE R : cands) {
                std::vector<int> got;
                take(R, &got);
                if (got.size() > best.size()) {
                    best = got;
                    bestR = R;
                }
            }
            for (int b = 0; b < m && __builtin_popcountll(bestR) < kPhaseBits; ++b) bestR |= 1ULL << b;
            StPhase ph;
            int nb = 0;
            int regbit[64];
            for (int b = 0; b < m; ++b)
                if (bestR >> b & 1ULL) {
                    regbit[b] = nb;
                    ph.bits[nb++] = (uint8_t)b;
                }
            ph.op_begin = (uint32_t)ops.size();
            for (int gi : best) {
                const GateRec& g = gates[gi];
                StOp op{};
                auto rb = [&](UINT gq) { return (uint8_t)regbit[local_bit(p.q, gq)]; };
                op.param = (uint32_t)pool.size();
                const double ang = g.angle;
                switch (g.kind) {
                    case QS_GATE_RX:
                        op.kind = ST_RX;
                        op.a = rb(g.targets[0]);
                        pool.push_back(make_double2(std::cos(ang / 2), std::sin(ang / 2)));
                        break;
                    case QS_GATE_RY:
                        op.kind = ST_RY;
                        op.a = rb(g.targets[0]);
                        pool.push_back(make_double2(std::cos(ang / 2), std::sin(ang / 2)));
                        break;
                    case QS_GATE_RZ:
                        op.kind = ST_DIAG1;
                        op.a = rb(g.targets[0]);
                        pool.push_back(make_double2(std::cos(ang / 2), std::sin(ang / 2)));
                        pool.push_back(make_double2(std::cos(ang / 2), -std::sin(ang / 2)));
                        break;
                    case QS_GATE_CNOT:
                        op.kind = ST_CNOT;
                        op.a = rb(g.targets[0]);
                        op.b = rb(g.targets[1]);
                        break;
                    case QS_GATE_CZ:
                        op.kind = ST_CZ;
                        op.a = rb(g.targets[0]);
                        op.b = rb(g.targets[1]);
                        break;
                    case QS_GATE_SWAP:
                        op.kind = ST_SWAP;
                        op.a = rb(g.targets[0]);
                        op.b = rb(g.targets[1]);
                        break;
                    case QS_GATE_DIAGONAL:
                        op.kind = ST_DIAG1;
                        op.a = rb(g.targets[0]);
                        for (int i = 0; i < 2; ++i) pool.push_back(make_double2(g.matrix[i].real(), g.matrix[i].imag()));
                        break;
                    default:  // dense 1 or 2 targets
                        if (g.targets.size() == 1) {
                            op.kind = ST_DENSE1;
                            op.a = rb(g.targets[0]);
                            for (int i = 0; i < 4; ++i) pool.push_back(make_double2(g.matrix[i].real(), g.matrix[i].imag()));
                        } else {
                            op.kind = ST_DENSE2;
                            op.a = rb(g.targets[0]);
                            op.b = rb(g.targets[1]);
                            for (int i = 0; i < 16; ++i) pool.push_back(make_double2(g.matrix[i].real(), g.matrix[i].imag()));
                        }
                        break;
                }
                if (op.kind == ST_DENSE1 || op.kind == ST_DIAG1 || op.kind == ST_RX || op.kind == ST_RY)
                    op.b = op.a;  // one-qubit ops: b = a (see run_code)
                op.pad = op_code(op);
                ops.push_back(op);
            }
            absorb_cnots(ops, pool, ph.op_begin);
            ph.op_count = (uint32_t)(ops.size() - ph.op_begin);
            phases.push_back(ph);
            std::vector<char> taken(gates.size(), 0);
            for (int gi : best) taken[gi] = 1;
            std::vector<int> rest;
            for (int gi : todo)
                if (!taken[gi]) rest.push_back(gi);
            todo.swap(rest);
        }
        pp.push_back({ph0, phases.size() - ph0});
    }
}

static int upload_plan(const HostPlan& H, ITYPE dim, std::shared_ptr<StagedPlan>* out);

static int build_plan(const std::vector<GateRec>& gates, UINT n, ITYPE dim, std::shared_ptr<StagedPlan>* out,
    int tile_bits = kTileBits) {
    HostPlan H;
    make_host_plan(gates, n, &H, tile_bits);
    return upload_plan(H, dim, out);
}

// Device copy of a host plan (phases | ops | parameter pool in one allocation) and its launch args.
static int upload_plan(const HostPlan& H, ITYPE dim, std::shared_ptr<StagedPlan>* out) {
    auto P = std::make_shared<StagedPlan>();
    P->dim = dim;
    P->phases = H.phases;
    P->ops = H.ops;
    P->pool = H.pool;
    const std::vector<PassPlan>& passes = H.passes;
    const std::vector<StPhase>& phases = H.phases;
    const std::vector<StOp>& ops = H.ops;
    const std::vector<double2>& pool = H.pool;
    const std::vector<HostPlan::Range>& pp = H.pp;
    // upload
    const size_t bph = sizeof(StPhase) * phases.size(), bop = sizeof(StOp) * ops.size(),
                 bpo = sizeof(double2) * pool.size();
    const size_t o_ops = (bph + 255) / 256 * 256, o_pool = o_ops + (bop + 255) / 256 * 256;
    const size_t total = o_pool + bpo + 256;
    QS_CUDA_CHECK(cudaMalloc(&P->dev, total));
    std::vector<char> host(total, 0);
    if (bph) memcpy(host.data(), phases.data(), bph);
    if (bop) memcpy(host.data() + o_ops, ops.data(), bop);
    if (bpo) memcpy(host.data() + o_pool, pool.data(), bpo);
    QS_CUDA_CHECK(cudaMemcpy(P->dev, host.data(), total, cudaMemcpyHostToDevice));
    const StPhase* dph = (const StPhase*)P->dev;
    const StOp* dop = (const StOp*)((char*)P->dev + o_ops);
    const double2* dpo = (const double2*)((char*)P->dev + o_pool);
    for (size_t i = 0; i < passes.size(); ++i) {
        DevPass d{};
        d.single = passes[i].single;
        d.gate = passes[i].gate;
        if (!d.single) {
            d.args.m = (int)passes[i].q.size();
            for (int j = 0; j < d.args.m; ++j) d.args.q[j] = passes[i].q[j];
            d.args.nphases = (int)pp[i].nphases;
            auto high_bits = [&](const StPhase& ph) {  // all of the phase's tile bits >= 4
                for (int p = 0; p < 4; ++p)
                    if (ph.bits[p] < kLowFixed) return false;
                return true;
            };
            if (pp[i].nphases) {
                if (high_bits(phases[pp[i].phase_begin])) d.args.io |= 1;
                if (high_bits(phases[pp[i].phase_begin + pp[i].nphases - 1])) d.args.io |= 2;
            }
            d.args.phases = dph + pp[i].phase_begin;
            d.phase_begin = pp[i].phase_begin;
            for (size_t ph = pp[i].phase_begin; ph < pp[i].phase_begin + pp[i].nphases; ++ph)
                for (uint32_t o = phases[ph].op_begin; o < phases[ph].op_begin + phases[ph].op_count; ++o)
                    d.folds = d.folds || ops[o].kind == ST_CSEL1 || ops[o].kind == ST_D1_IN || ops[o].kind == ST_D1_OUT;
            d.args.ops = dop;
            d.args.pool = dpo;
        }
        P->passes.push_back(d);
    }
    *out = P;
    return QS_OK;
}

static int run_plan(const std::vector<GateRec>& gates, const StagedPlan& P, void* state, ITYPE dim, cudaStream_t st) {
    QS_TRY(staged_allow_smem());
    for (const DevPass& d : P.passes) {
        if (d.single) {
            QS_TRY(apply_gate_by_gate(gates[d.gate], state, dim, st));
            continue;
        }
        const ITYPE tiles = dim >> d.args.m;
        if (d.spec) {
            QS_TRY(launch_specialized_pass(d.spec, (double2*)state, d.spec_params.empty() ? nullptr : d.spec_params.data(),
                tiles, d.args.m, st));
            continue;
        }
        launch_pass((double2*)state, d, tiles, st);
        QS_TRY(check_launch("k_staged_pass"));
    }
    return QS_OK;
}

// The pass as the code generator sees it.
static PassDesc pass_desc(const StagedPlan& P, const DevPass& d) {
    PassDesc pd;
    pd.m = d.args.m;
    pd.io = d.args.io;
    for (int j = 0; j < d.args.m; ++j) pd.q[j] = d.args.q[j];
    pd.phases.assign(P.phases.begin() + d.phase_begin, P.phases.begin() + d.phase_begin + d.args.nphases);
    pd.ops = P.ops.data();
    pd.pool = P.pool.data();
    return pd;
}

// Specialised kernels for every pass of a plan, compiled on host threads in parallel.  On failure the
// plan keeps the generic pass kernel for every pass and the error is returned.
static int specialize_plan(StagedPlan& P) {
    if (P.specialized) return QS_OK;
    std::vector<size_t> todo;
    for (size_t i = 0; i < P.passes.size(); ++i)
        if (!P.passes[i].single && P.passes[i].args.nphases > 0) todo.push_back(i);
    std::vector<void*> handles(P.passes.size(), nullptr);
    std::vector<std::vector<double2>> params(P.passes.size());
    std::vector<int> rcs(P.passes.size(), QS_OK);
    std::vector<std::string> errs(P.passes.size());
    std::atomic<size_t> next{0};
    const auto t0 = std::chrono::steady_clock::now();
    const unsigned nt = std::max(1u, std::min<unsigned>((unsigned)todo.size(), std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nt; ++t)
        pool.emplace_back([&] {
            for (size_t j; (j = next.fetch_add(1)) < todo.size();) {
                const size_t i = todo[j];
                rcs[i] = specialized_pass_kernel(pass_desc(P, P.passes[i]), &handles[i], &params[i], nullptr);
                if (rcs[i] != QS_OK) errs[i] = qs_get_last_error();
            }
        });
    for (std::thread& t : pool) t.join();
    for (size_t i : todo)
        if (rcs[i] != QS_OK) return set_error(rcs[i], errs[i]);
    for (size_t i : todo) {
        P.passes[i].spec = handles[i];
        P.passes[i].spec_params = std::move(params[i]);
    }
    P.specialized = true;
    P.compile_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return QS_OK;
}

// Whether a circuit's single-state passes use specialised kernels: forced on or off per circuit, else
// for states of at least 2^kSpecializeMinQubits amplitudes (where a pass runs long enough to repay its
// compile time).
constexpr UINT kSpecializeMinQubits = 22;
static bool want_specialized(const Circuit& c, ITYPE dim) {
    if (c.specialize >= 0) return c.specialize == 1;
    return dim >= (1ULL << kSpecializeMinQubits);
}

static int ensure_plan(Circuit& c, ITYPE dim) {
    if (!c.plan || c.plan->dim != dim) QS_TRY(build_plan(c.gates, c.n, dim, &c.plan));
    if (want_specialized(c, dim)) QS_TRY(specialize_plan(*c.plan));
    return QS_OK;
}


int run_staged(Circuit& c, void* state, ITYPE dim, cudaStream_t st) {
    if (c.n < kPhaseBits) {  // too small for a 4-qubit register phase
        for (const GateRec& g : c.gates) QS_TRY(apply_gate_by_gate(g, state, dim, st));
        return QS_OK;
    }
    QS_TRY(ensure_plan(c, dim));
    return run_plan(c.gates, *c.plan, state, dim, st);
}

// ---- FP64 gate fusion + staged passes, block size and tile shape chosen by measurement.
// The autotuner fuses the gate list for each candidate block size k = 0..6 (0 = unfused), builds its
// staged schedule with 2^12-amplitude tiles, and times every pass's kernel -- the specialised kernel
// when the circuit runs specialised passes, else the generic one -- on a scratch buffer of whole tiles
// (the pass's ops only see tile-local bits, so its tile qubits are remapped to 0..m-1); a pass costs at
// least its HBM time, and gates left outside passes cost one HBM pass each (dense 5- and 6-qubit
// kernels more).  The best k is then also tried with 2^11-amplitude tiles (the tile shape).
constexpr int kTuneMaxK = 6;
constexpr int kTuneSlots = kTuneMaxK + 2;  // k = 0..6 at 2^12 tiles, then the best k at 2^11 tiles
constexpr double kTuneHbmBytesPerSec = 6.5e12;  // B200 streaming copy bandwidth

static double single_gate_factor(const GateRec& g) {
    const size_t k = g.targets.size() + g.controls.size();
    if (g.kind == QS_GATE_DENSE && k == 5) return 2.0;
    if (g.kind == QS_GATE_DENSE && k >= 6) return 6.5;  // k_denseK_blk: 33 ms against a 5.3 ms pass at 30 qubits
    return 1.0;
}

static int estimate_plan_ms(const std::vector<GateRec>& gates, const StagedPlan& P, ITYPE dim, cudaStream_t st,
    bool specialized, double* out_ms) {
    const double hbm_ms = 2.0 * 16.0 * (double)dim / kTuneHbmBytesPerSec * 1e3;
    QS_TRY(staged_allow_smem());
    // specialised kernels of the remapped passes, compiled on host threads in parallel
    std::vector<void*> spec(P.passes.size(), nullptr);
    std::vector<std::vector<double2>> sparams(P.passes.size());
    if (specialized) {
        std::vector<size_t> todo;
        for (size_t i = 0; i < P.passes.size(); ++i)
            if (!P.passes[i].single && P.passes[i].args.nphases > 0) todo.push_back(i);
        std::vector<int> rcs(P.passes.size(), QS_OK);
        std::vector<std::string> errs(P.passes.size());
        std::atomic<size_t> next{0};
        const unsigned nt =
            std::max(1u, std::min<unsigned>((unsigned)todo.size(), std::thread::hardware_concurrency()));
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nt; ++t)
            pool.emplace_back([&] {
                for (size_t j; (j = next.fetch_add(1)) < todo.size();) {
                    const size_t i = todo[j];
                    PassDesc pd = pass_desc(P, P.passes[i]);
                    for (int b = 0; b < pd.m; ++b) pd.q[b] = (UINT)b;
                    rcs[i] = specialized_pass_kernel(pd, &spec[i], &sparams[i], nullptr);
                    if (rcs[i] != QS_OK) errs[i] = qs_get_last_error();
                }
            });
        for (std::thread& t : pool) t.join();
        for (size_t i : todo)
            if (rcs[i] != QS_OK) return set_error(rcs[i], errs[i]);
    }
    double total = 0.;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    QS_CUDA_CHECK(cudaEventCreate(&e0));
    QS_CUDA_CHECK(cudaEventCreate(&e1));
    int rc = QS_OK;
    for (size_t i = 0; i < P.passes.size(); ++i) {
        const DevPass& d = P.passes[i];
        if (d.single) {
            total += hbm_ms * single_gate_factor(gates[d.gate]);
            continue;
        }
        const ITYPE tiles = dim >> d.args.m;
        const ITYPE tt = std::min<ITYPE>(tiles, (ITYPE)sm_count() * 3 * 4);
        void* buf = nullptr;
        rc = scratch(st, (size_t)(tt << d.args.m) * sizeof(double2), &buf);
        if (rc != QS_OK) break;
        StPassArgs a = d.args;
        for (int j = 0; j < a.m; ++j) a.q[j] = (UINT)j;
        DevPass dt = d;
        dt.args = a;
        auto launch = [&]() -> int {
            if (spec[i])
                return launch_specialized_pass(spec[i], (double2*)buf, sparams[i].empty() ? nullptr : sparams[i].data(),
                    tt, a.m, st);
            launch_pass((double2*)buf, dt, tt, st);
            return check_launch("k_staged_pass");
        };
        rc = launch();  // warm-up
        if (rc != QS_OK) break;
        cudaEventRecord(e0, st);
        rc = launch();
        cudaEventRecord(e1, st);
        if (rc != QS_OK) break;
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            rc = set_error(QS_ERR_CUDA, "autotune: event synchronize failed");
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        total += std::max((double)ms * (double)tiles / (double)tt, hbm_ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *out_ms = total;
    return rc;
}

static int ensure_fused_plan(Circuit& c, ITYPE dim, cudaStream_t st) {
    if (c.fplan && c.fplan->dim == dim) return QS_OK;
    const bool spec = want_specialized(c, dim);
    if (c.fusion_k >= 0) {
        c.fgates = fuse_gates(c.gates, c.fusion_k);
        c.fused_k = c.fusion_k;
        c.fused_tile_bits = kTileBits;
        QS_TRY(build_plan(c.fgates, c.n, dim, &c.fplan));
        if (spec) QS_TRY(specialize_plan(*c.fplan));
        return QS_OK;
    }
    c.tune_ms.assign(kTuneSlots, -1.);
    double best = 0.;
    auto consider = [&](int k, int tile_bits, int slot) -> int {
        std::vector<GateRec> fg = fuse_gates(c.gates, k);
        std::shared_ptr<StagedPlan> P;
        QS_TRY(build_plan(fg, c.n, dim, &P, tile_bits));
        double ms = 0.;
        QS_TRY(estimate_plan_ms(fg, *P, dim, st, spec, &ms));
        c.tune_ms[slot] = ms;
        if (!c.fplan || ms < best) {
            best = ms;
            c.fgates.swap(fg);
            c.fplan = P;
            c.fused_k = k;
            c.fused_tile_bits = tile_bits;
        }
        return QS_OK;
    };
    for (int k = 0; k <= kTuneMaxK; ++k) QS_TRY(consider(k, kTileBits, k));
    if (c.n > (UINT)kTileBits - 1) QS_TRY(consider(c.fused_k, kTileBits - 1, kTuneMaxK + 1));
    if (spec) QS_TRY(specialize_plan(*c.fplan));
    return QS_OK;
}

int run_staged_fused(Circuit& c, void* state, ITYPE dim, cudaStream_t st) {
    if (c.n < kPhaseBits) {
        for (const GateRec& g : c.gates) QS_TRY(apply_gate_by_gate(g, state, dim, st));
        return QS_OK;
    }
    QS_TRY(ensure_fused_plan(c, dim, st));
    return run_plan(c.fgates, *c.fplan, state, dim, st);
}

// ---------------------------------------------------------------- complex64 states, FP64 passes
// The staged schedule over a complex64 state: each tile is widened to FP64 in shared memory, every
// phase runs in FP64 (the generic pass kernel's code), and the tile is rounded back on the store, so a
// pass moves half the bytes of the complex128 pass.  Gates are fused into blocks of at most 2 qubits
// (a forced QS_EXEC_STAGED_FUSED size of 0..2 is kept) so that every block is a pass op.  The same
// schedule (it does not depend on the state type) runs the large circuits of a batch.
static int c64_block_size(const Circuit& c) { return (c.fusion_k >= 0 && c.fusion_k <= 2) ? c.fusion_k : 2; }

static int ensure_c64_plan(Circuit& c, ITYPE dim) {
    const int k = c64_block_size(c);
    if (c.cplan && c.cplan->dim == dim && c.ck == k) return QS_OK;
    c.cgates = fuse_gates(c.gates, k);
    c.ck = k;
    QS_TRY(build_plan(c.cgates, c.n, dim, &c.cplan));
    for (const DevPass& d : c.cplan->passes)
        if (d.single) {
            c.cplan.reset();
            return set_error(QS_ERR_NOT_SUPPORTED,
                "complex64 FP64 passes: every gate must be stageable (<= 2 targets and controls together)");
        }
    return QS_OK;
}

int run_staged_c64(Circuit& c, void* state, ITYPE dim, cudaStream_t st) {
    if (c.n < kPhaseBits) return set_error(QS_ERR_NOT_SUPPORTED, "complex64 FP64 passes need at least 4 qubits");
    QS_TRY(ensure_c64_plan(c, dim));
    QS_TRY(staged_allow_smem());
    for (const DevPass& d : c.cplan->passes) {
        launch_pass((float2*)state, d, dim >> d.args.m, st);
        QS_TRY(check_launch("k_staged_pass"));
    }
    return QS_OK;
}

int staged_pass_count(Circuit& c, ITYPE dim, UINT* out) {
    if (c.n < kPhaseBits) {
        *out = (UINT)c.gates.size();
        return QS_OK;
    }
    HostPlan H;
    make_host_plan(c.gates, c.n, &H);
    *out = (UINT)H.passes.size();
    return QS_OK;
}

}  // namespace qs

// Host-only statistics of the staged schedule: HBM passes, register phases, operations in phases,
// and gates run by the gate-by-gate kernels between passes.
extern "C" QS_API int qs_circuit_staged_stats(qs_circuit_t circuit, QS_UINT* passes, QS_UINT* phases, QS_UINT* ops,
    QS_UINT* single_gates) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c || !passes || !phases || !ops || !single_gates) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    qs::HostPlan H;
    qs::make_host_plan(c->gates, c->n, &H);
    UINT single = 0;
    for (const qs::PassPlan& p : H.passes) single += p.single ? 1 : 0;
    *passes = (QS_UINT)H.passes.size();
    *phases = (QS_UINT)H.phases.size();
    *ops = (QS_UINT)H.ops.size();
    *single_gates = single;
    return QS_OK;
}

// Block size, gate count and HBM passes of the FP64-fused schedule last built for QS_EXEC_STAGED_FUSED
// (k = -1 before the first run), and the autotuner's estimates (ms; < 0 when not tried, e.g. with a
// forced k): estimates_ms[k] for k = 0..6 with 2^12-amplitude tiles, estimates_ms[7] for the best k
// with 2^11-amplitude tiles (the schedule uses those tiles when that estimate is the smallest).
extern "C" QS_API int qs_circuit_fusion_info(qs_circuit_t circuit, int* k, QS_UINT* gate_count, QS_UINT* passes,
    double* estimates_ms) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c || !k || !gate_count || !passes) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    *k = c->fplan ? c->fused_k : -1;
    *gate_count = c->fplan ? (QS_UINT)c->fgates.size() : 0;
    *passes = c->fplan ? (QS_UINT)c->fplan->passes.size() : 0;
    if (estimates_ms)
        for (int i = 0; i < qs::kTuneSlots; ++i)
            estimates_ms[i] = i < (int)c->tune_ms.size() ? c->tune_ms[i] : -1.;
    return QS_OK;
}

// Specialised pass kernels for this circuit's single-state staged modes: 1 = always, 0 = never (the
// generic pass kernel), -1 = for states of at least 2^22 amplitudes (default).
extern "C" QS_API int qs_circuit_set_specialized(qs_circuit_t circuit, int mode) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null circuit");
    if (mode < -1 || mode > 1) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "specialised mode must be -1, 0 or 1");
    c->specialize = mode;
    c->plan.reset();
    c->fplan.reset();
    c->fgates.clear();
    c->fused_k = -1;
    c->tune_ms.clear();
    return QS_OK;
}

// Whether the last-built QS_EXEC_STAGED and QS_EXEC_STAGED_FUSED schedules run specialised kernels, and
// the wall time their compilation took (ms, both schedules; 0 when served from the kernel cache).
extern "C" QS_API int qs_circuit_specialized_info(qs_circuit_t circuit, int* staged, int* staged_fused,
    double* compile_ms) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c || !staged || !staged_fused) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    *staged = c->plan && c->plan->specialized;
    *staged_fused = c->fplan && c->fplan->specialized;
    if (compile_ms)
        *compile_ms = (c->plan ? c->plan->compile_ms : 0.) + (c->fplan ? c->fplan->compile_ms : 0.);
    return QS_OK;
}

// CUDA C source of the specialised kernel of pass `pass` of the circuit's QS_EXEC_STAGED schedule at
// `dim` amplitudes (host only).  With buf == NULL, *size receives the length + 1; otherwise up to *size
// bytes are written, NUL-terminated.
extern "C" QS_API int qs_circuit_specialized_source(qs_circuit_t circuit, QS_ITYPE dim, QS_UINT pass, char* buf,
    QS_ITYPE* size) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c || !size) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    if (dim != (1ULL << c->n)) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "dim differs from 2^qubit_count");
    if (c->n < (UINT)qs::kPhaseBits + 3) return qs::set_error(QS_ERR_NOT_SUPPORTED, "fewer than 7 qubits");
    qs::HostPlan H;
    qs::make_host_plan(c->gates, c->n, &H);
    if (pass >= H.passes.size() || H.passes[pass].single)
        return qs::set_error(QS_ERR_INVALID_ARGUMENT, "no such staged pass");
    qs::StagedPlan P;
    P.phases = H.phases;
    P.ops = H.ops;
    P.pool = H.pool;
    qs::DevPass d{};
    d.args.m = (int)H.passes[pass].q.size();
    for (int j = 0; j < d.args.m; ++j) d.args.q[j] = H.passes[pass].q[j];
    d.args.nphases = (int)H.pp[pass].nphases;
    d.phase_begin = H.pp[pass].phase_begin;
    if (d.args.nphases) {
        auto high_bits = [&](const qs::StPhase& ph) {
            for (int p = 0; p < 4; ++p)
                if (ph.bits[p] < qs::kLowFixed) return false;
            return true;
        };
        if (high_bits(H.phases[d.phase_begin])) d.args.io |= 1;
        if (high_bits(H.phases[d.phase_begin + d.args.nphases - 1])) d.args.io |= 2;
    }
    const std::string src = qs::specialized_pass_source(qs::pass_desc(P, d));
    if (!buf) {
        *size = src.size() + 1;
        return QS_OK;
    }
    if (*size == 0) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "zero-size buffer");
    const size_t n = std::min<size_t>(src.size(), (size_t)*size - 1);
    memcpy(buf, src.data(), n);
    buf[n] = '\0';
    return QS_OK;
}

// Force the FP64 fusion block size of QS_EXEC_STAGED_FUSED (0..6; 0 = no fusion) or, with -1, let
// the autotuner choose on the next run.
extern "C" QS_API int qs_circuit_set_fusion(qs_circuit_t circuit, int k) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null circuit");
    if (k < -1 || k > 6) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "fusion block size must be -1..6");
    c->fusion_k = k;
    c->dm_vec.reset();
    c->fplan.reset();
    c->fgates.clear();
    c->fused_k = -1;
    c->tune_ms.clear();
    return QS_OK;
}

// ---------------------------------------------------------------- batched execution
// Many circuits (each on its own state, of any size >= 4 qubits) in ONE persistent launch.  Work
// items are (circuit, pass, tile); the queue lists every circuit's pass 0, then every circuit's
// pass 1, and so on.  A CTA takes the next item with an atomic counter and, for pass p > 0, waits
// until all tiles of pass p - 1 of the same circuit are done (acquire load of a per-pass counter).
// Dependencies only point to earlier queue items, which resident CTAs already hold, so the wait
// always ends; it is still bounded (a %globaltimer deadline, 2 s) and reports QS_ERR_TIMEOUT through an
// error flag, after which the CTA leaves without touching the item.
namespace qs {

struct BatchRec {
    StPassArgs args;
    void* state;  // complex128 or complex64 (one type per launch)
    ITYPE tiles;
    ITYPE prefix;  // first work item of this record
    int dep;       // record of the previous pass of the same circuit, -1 for pass 0
};


__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <class E>
__global__ void __launch_bounds__(kStThreads, 3) k_batch_staged(const BatchRec* __restrict__ recs, int nrec,
    ITYPE total, unsigned long long* head, unsigned* done, int* err, unsigned long long wait_ns) {
    __shared__ double2 tile[1 << kBatchTileBits];
    __shared__ ITYPE hi_off[1 << (kBatchTileBits - 7)];
    __shared__ ITYPE s_item;
    __shared__ int s_rec, s_abort;
    __shared__ StPassArgs s_args;  // the record's pass, copied so the tile code indexes shared memory
    __shared__ E* s_state;
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
                    const unsigned need = (unsigned)recs[dep].tiles;
                    const unsigned long long t0 = global_ns();
                    while (ld_acquire_u32(done + dep) < need) {
                        if (global_ns() - t0 > wait_ns) {
                            atomicExch(err, 1);
                            s_abort = 1;
                            break;
                        }
                        __nanosleep(64);
                    }
                }
            }
        }
        __syncthreads();
        if (s_item >= total || s_abort) break;
        if (tid == 0) {
            s_args = recs[s_rec].args;
            s_state = (E*)recs[s_rec].state;
        }
        __syncthreads();
        staged_tile<kBatchTileBits, true>(s_state, s_args, s_item - recs[s_rec].prefix, tile, hi_off);
        if (tid == 0) {
            __threadfence();
            atomicAdd(done + s_rec, 1u);
        }
    }
}

// Block size of batched execution: the circuit's forced QS_EXEC_STAGED_FUSED size when it is at most 2,
// else 2 (autotuning each circuit of a batch would cost more than it saves; k <= 2 keeps every fused
// block a pass op).
static int batch_block_size(const Circuit& c) { return (c.fusion_k >= 0 && c.fusion_k <= 2) ? c.fusion_k : 2; }

static int ensure_batch_plan(Circuit& c, ITYPE dim) {
    const int k = batch_block_size(c);
    if (c.bplan && c.bplan->dim == dim && c.bk == k) return QS_OK;
    c.bgates = fuse_gates(c.gates, k);
    c.bk = k;
    return build_plan(c.bgates, c.n, dim, &c.bplan, kBatchTileBits);
}

// `wait_ns`: the dependency wait limit; `self_dep` >= 0 makes that work record depend on itself (a
// counter nothing can complete), which only the wait-expiry check below uses.
// The work records of a batch (plans missing from the circuits' caches built first: FP64 fusion and
// host planning on host threads in parallel, uploads afterwards) and the number of work items.
static int batch_records(Circuit* const* cs, void* const* states, UINT count, std::vector<BatchRec>* recs,
    ITYPE* total_out) {
    for (UINT i = 0; i < count; ++i)
        if (cs[i]->n < kPhaseBits) return set_error(QS_ERR_NOT_SUPPORTED, "batch: circuits need at least 4 qubits");
    {
        std::vector<char> need(count, 0);
        for (UINT i = 0; i < count; ++i) {
            const Circuit& c = *cs[i];
            need[i] = !(c.bplan && c.bplan->dim == (1ULL << c.n) && c.bk == batch_block_size(c));
            for (UINT j = 0; j < i && need[i]; ++j)
                if (cs[j] == cs[i]) need[i] = 0;
        }
        std::vector<std::vector<GateRec>> fg(count);
        std::vector<HostPlan> hp(count);
        std::atomic<UINT> next{0};
        const unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nt; ++t)
            pool.emplace_back([&] {
                for (UINT i; (i = next.fetch_add(1)) < count;)
                    if (need[i]) {
                        fg[i] = fuse_gates(cs[i]->gates, batch_block_size(*cs[i]));
                        make_host_plan(fg[i], cs[i]->n, &hp[i], kBatchTileBits);
                    }
            });
        for (std::thread& t : pool) t.join();
        for (UINT i = 0; i < count; ++i)
            if (need[i]) {
                Circuit& c = *cs[i];
                c.bgates = std::move(fg[i]);
                c.bk = batch_block_size(c);
                QS_TRY(upload_plan(hp[i], 1ULL << c.n, &c.bplan));
            }
    }
    std::vector<std::vector<const DevPass*>> passes(count);
    size_t maxp = 0;
    for (UINT i = 0; i < count; ++i) {
        Circuit& c = *cs[i];
        QS_TRY(ensure_batch_plan(c, 1ULL << c.n));
        for (const DevPass& d : c.bplan->passes) {
            if (d.single)
                return set_error(QS_ERR_NOT_SUPPORTED,
                    "batch: every gate must be stageable (<= 2 targets, no controls, no Pauli strings)");
            passes[i].push_back(&d);
        }
        maxp = std::max(maxp, passes[i].size());
    }
    recs->clear();
    std::vector<int> last(count, -1);
    ITYPE total = 0;
    for (size_t p = 0; p < maxp; ++p)
        for (UINT i = 0; i < count; ++i) {
            if (p >= passes[i].size()) continue;
            BatchRec r{};
            r.args = passes[i][p]->args;
            r.state = states[i];
            r.tiles = (1ULL << cs[i]->n) >> r.args.m;
            r.prefix = total;
            r.dep = last[i];
            last[i] = (int)recs->size();
            total += r.tiles;
            recs->push_back(r);
        }
    *total_out = total;
    return QS_OK;
}

// Device buffer of a batch launch: records | per-record done counters | (16-byte aligned) work head |
// error flag.  Everything after the records must be zero before a launch.
struct BatchLayout {
    size_t brec, zero_bytes, bytes;
    explicit BatchLayout(size_t nrec) {
        brec = sizeof(BatchRec) * nrec;
        const size_t bdone = sizeof(unsigned) * nrec;
        bytes = brec + bdone + 256;
        zero_bytes = bytes - brec;
    }
    unsigned* done(void* b) const { return (unsigned*)((char*)b + brec); }
    unsigned long long* head(void* b) const {
        return (unsigned long long*)((char*)b + ((brec + (bytes - 256 - brec) + 15) / 16 * 16));
    }
    int* err(void* b) const { return (int*)(head(b) + 1); }
};

static int batch_kernel(void* buf, const BatchLayout& L, int nrec, ITYPE total, unsigned long long wait_ns, bool c64,
    cudaStream_t st) {
    int per_sm = 0;
    if (c64)
        QS_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_staged<float2>, kStThreads, 0));
    else
        QS_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_staged<double2>, kStThreads, 0));
    const ITYPE resident = (ITYPE)std::max(1, per_sm) * sm_count();
    const unsigned grid = (unsigned)std::min<ITYPE>(resident, total);
    const BatchRec* drec = (const BatchRec*)buf;
    if (c64)
        k_batch_staged<float2><<<grid, kStThreads, 0, st>>>(drec, nrec, total, L.head(buf), L.done(buf), L.err(buf), wait_ns);
    else
        k_batch_staged<double2><<<grid, kStThreads, 0, st>>>(drec, nrec, total, L.head(buf), L.done(buf), L.err(buf), wait_ns);
    return check_launch("k_batch_staged");
}

// Circuits of at least this many qubits leave the persistent launch: a pass of theirs has >= 1024
// tiles of 2^11 amplitudes, enough to fill the device alone, so they run as their own staged passes
// with 2^12-amplitude tiles (fewer passes, no dependency waits), on the same stream.
constexpr UINT kBatchSoloQubits = 21;

int batch_update(Circuit* const* cs, void* const* states, UINT count, cudaStream_t st, unsigned long long wait_ns,
    int self_dep, bool c64) {
    if (count == 0) return QS_OK;
    std::vector<Circuit*> shared_cs, solo_cs;
    std::vector<void*> shared_st, solo_st;
    for (UINT i = 0; i < count; ++i) {
        const bool solo = self_dep < 0 && cs[i]->n >= kBatchSoloQubits;
        (solo ? solo_cs : shared_cs).push_back(cs[i]);
        (solo ? solo_st : shared_st).push_back(states[i]);
    }
    // every plan first (a refusal comes before any launch)
    for (size_t i = 0; i < solo_cs.size(); ++i) QS_TRY(ensure_c64_plan(*solo_cs[i], 1ULL << solo_cs[i]->n));
    std::vector<BatchRec> recs;
    ITYPE total = 0;
    if (!shared_cs.empty())
        QS_TRY(batch_records(shared_cs.data(), shared_st.data(), (UINT)shared_cs.size(), &recs, &total));
    if (!solo_cs.empty()) QS_TRY(staged_allow_smem());
    for (size_t i = 0; i < solo_cs.size(); ++i) {
        const ITYPE dim = 1ULL << solo_cs[i]->n;
        for (const DevPass& d : solo_cs[i]->cplan->passes) {
            if (c64) launch_pass((float2*)solo_st[i], d, dim >> d.args.m, st);
            else launch_pass((double2*)solo_st[i], d, dim >> d.args.m, st);
            QS_TRY(check_launch("k_staged_pass"));
        }
    }
    if (recs.empty()) {
        QS_CUDA_CHECK(cudaStreamSynchronize(st));
        return QS_OK;
    }
    if (self_dep >= 0) {
        if (self_dep >= (int)recs.size()) return set_error(QS_ERR_INVALID_ARGUMENT, "batch: no such work record");
        recs[self_dep].dep = self_dep;
    }
    const BatchLayout L(recs.size());
    void* buf = nullptr;
    QS_TRY(scratch(st, L.bytes, &buf));
    QS_CUDA_CHECK(cudaMemcpyAsync(buf, recs.data(), L.brec, cudaMemcpyHostToDevice, st));
    QS_CUDA_CHECK(cudaMemsetAsync(L.done(buf), 0, L.zero_bytes, st));
    QS_TRY(batch_kernel(buf, L, (int)recs.size(), total, wait_ns, c64, st));
    int err = 0;
    QS_CUDA_CHECK(cudaMemcpyAsync(&err, L.err(buf), sizeof(int), cudaMemcpyDeviceToHost, st));
    QS_CUDA_CHECK(cudaStreamSynchronize(st));
    if (err) return set_error(QS_ERR_TIMEOUT, "batch: dependency wait expired");
    return QS_OK;
}

// ---------------------------------------------------------------- captured CUDA graphs
// A circuit (or a batch) applied to fixed device states, recorded once as a CUDA graph and replayed
// with one cudaGraphLaunch: the host planning, parameter uploads and per-pass launches of a call are
// paid once.  Plans (and the autotuner, and specialised kernels) are prepared before the capture;
// the capture records only stream work.  Work that copies from pageable host memory during a run (a
// dense gate of >= 6 qubits left outside the staged passes, a multi-qubit diagonal) refuses to be
// recorded: creation then fails with QS_ERR_NOT_SUPPORTED.
struct GraphExec {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    void* dev = nullptr;       // batch graphs: work records and counters
    int* host_err = nullptr;   // batch graphs: the wait-expiry flag, copied back by the graph (pinned)
    long long kernels = 0;     // kernel launches one replay performs
    ~GraphExec() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (dev) cudaFree(dev);
        if (host_err) cudaFreeHost(host_err);
    }
};

// Records `work` on a capturing stream (the caller's, or a private one for the legacy default stream)
// into G.  Capture is thread-local, so other threads' unrelated CUDA calls are not affected.
template <class F>
static int capture_graph(cudaStream_t user, GraphExec* G, F work) {
    cudaStream_t st = user;
    cudaStream_t own = nullptr;
    if (!st) {  // the legacy default stream cannot capture
        QS_TRY(qs_stream_create((void**)&own));
        st = own;
    }
    const unsigned long long l0 = qs_launch_count();
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        if (own) qs_stream_destroy(own);
        return check_cuda(e, "cudaStreamBeginCapture");
    }
    set_capturing(true);
    int rc = work(st);
    set_capturing(false);
    std::string msg = rc == QS_OK ? std::string() : std::string(qs_get_last_error());
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(st, &g);
    G->kernels = (long long)(qs_launch_count() - l0);
    count_launches(-G->kernels);  // recorded, not run
    if (own) qs_stream_destroy(own);  // with any scratch the capture allocated for it
    if (rc != QS_OK || e != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();  // clear the capture error
        return set_error(QS_ERR_NOT_SUPPORTED,
            "graph capture: this work cannot be recorded (" + (msg.empty() ? std::string(cudaGetErrorString(e)) : msg) +
            ")");
    }
    G->graph = g;
    e = cudaGraphInstantiate(&G->exec, g, 0);
    if (e != cudaSuccess) return check_cuda(e, "cudaGraphInstantiate");
    return QS_OK;
}

}  // namespace qs

extern "C" QS_API int qs_circuit_graph_create(qs_circuit_t circuit, void* state, QS_ITYPE dim, int mode, int reset_state,
    void* stream, qs_graph_t* out) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c || !state || !out) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    if (dim != (1ULL << c->n)) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "dim differs from 2^qubit_count");
    if (mode != QS_EXEC_GATE_BY_GATE && mode != QS_EXEC_STAGED && mode != QS_EXEC_STAGED_FUSED)
        return qs::set_error(QS_ERR_INVALID_ARGUMENT, "unknown execution mode");
    cudaStream_t st = (cudaStream_t)stream;
    // plans, autotuning and specialised kernels first: they synchronise and allocate
    if (c->n >= (UINT)qs::kPhaseBits) {
        if (mode == QS_EXEC_STAGED) QS_TRY(qs::ensure_plan(*c, dim));
        if (mode == QS_EXEC_STAGED_FUSED) QS_TRY(qs::ensure_fused_plan(*c, dim, st));
    }
    QS_TRY(qs::staged_allow_smem());
    auto G = std::make_unique<qs::GraphExec>();
    QS_TRY(qs::capture_graph(st, G.get(), [&](cudaStream_t cs) -> int {
        if (reset_state) QS_TRY(qs_initialize_quantum_state(state, dim, cs));
        if (mode == QS_EXEC_STAGED) return qs::run_staged(*c, state, dim, cs);
        if (mode == QS_EXEC_STAGED_FUSED) return qs::run_staged_fused(*c, state, dim, cs);
        for (const qs::GateRec& g : c->gates) QS_TRY(qs::apply_gate_by_gate(g, state, dim, cs));
        return QS_OK;
    }));
    *out = reinterpret_cast<qs_graph_t>(G.release());
    return QS_OK;
}

extern "C" QS_API int qs_batch_graph_create(const qs_circuit_t* circuits, void* const* states, QS_UINT count, int c64,
    int reset_states, void* stream, qs_graph_t* out) {
    if (!circuits || !states || !out || count == 0) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    std::vector<qs::Circuit*> cs(count);
    for (QS_UINT i = 0; i < count; ++i) {
        cs[i] = reinterpret_cast<qs::Circuit*>(circuits[i]);
        if (!cs[i] || !states[i]) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null circuit or state");
    }
    std::vector<qs::BatchRec> recs;
    ITYPE total = 0;
    QS_TRY(qs::batch_records(cs.data(), states, count, &recs, &total));
    if (recs.empty()) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "batch graph: no passes to run");
    auto G = std::make_unique<qs::GraphExec>();
    const qs::BatchLayout L(recs.size());
    QS_CUDA_CHECK(cudaMalloc(&G->dev, L.bytes));
    QS_CUDA_CHECK(cudaMemcpy(G->dev, recs.data(), L.brec, cudaMemcpyHostToDevice));
    QS_CUDA_CHECK(cudaMallocHost((void**)&G->host_err, sizeof(int)));
    *G->host_err = 0;
    void* dev = G->dev;
    int* host_err = G->host_err;
    QS_TRY(qs::capture_graph((cudaStream_t)stream, G.get(), [&](cudaStream_t st) -> int {
        if (reset_states)
            for (QS_UINT i = 0; i < count; ++i) {
                const QS_ITYPE dim = 1ULL << cs[i]->n;
                QS_TRY(c64 ? qs_initialize_quantum_state_c64(states[i], dim, st)
                           : qs_initialize_quantum_state(states[i], dim, st));
            }
        QS_CUDA_CHECK(cudaMemsetAsync(L.done(dev), 0, L.zero_bytes, st));
        QS_TRY(qs::batch_kernel(dev, L, (int)recs.size(), total, qs::kBatchWaitNs, c64 != 0, st));
        QS_CUDA_CHECK(cudaMemcpyAsync(host_err, L.err(dev), sizeof(int), cudaMemcpyDeviceToHost, st));
        return QS_OK;
    }));
    *out = reinterpret_cast<qs_graph_t>(G.release());
    return QS_OK;
}

extern "C" QS_API int qs_graph_launch(qs_graph_t graph, void* stream) {
    qs::GraphExec* G = reinterpret_cast<qs::GraphExec*>(graph);
    if (!G || !G->exec) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null graph");
    cudaStream_t st = (cudaStream_t)stream;
    QS_CUDA_CHECK(cudaGraphLaunch(G->exec, st));
    qs::count_launches(G->kernels);
    if (G->host_err) {  // a batch graph: its wait-expiry flag arrives with the graph's last node
        QS_CUDA_CHECK(cudaStreamSynchronize(st));
        if (*G->host_err) return qs::set_error(QS_ERR_TIMEOUT, "batch graph: dependency wait expired");
    }
    return QS_OK;
}

extern "C" QS_API int qs_graph_kernel_count(qs_graph_t graph, QS_ITYPE* kernels) {
    qs::GraphExec* G = reinterpret_cast<qs::GraphExec*>(graph);
    if (!G || !kernels) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    *kernels = (QS_ITYPE)G->kernels;
    return QS_OK;
}

extern "C" QS_API int qs_graph_destroy(qs_graph_t graph) {
    delete reinterpret_cast<qs::GraphExec*>(graph);
    return QS_OK;
}

namespace qs {
}  // namespace qs

extern "C" QS_API int qs_batch_update_quantum_states(const qs_circuit_t* circuits, void* const* states, QS_UINT count,
    void* stream) {
    if (!circuits || !states) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    std::vector<qs::Circuit*> cs(count);
    for (QS_UINT i = 0; i < count; ++i) {
        cs[i] = reinterpret_cast<qs::Circuit*>(circuits[i]);
        if (!cs[i] || !states[i]) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null circuit or state");
    }
    return qs::batch_update(cs.data(), states, count, (cudaStream_t)stream, qs::kBatchWaitNs, -1, false);
}

// Failure-path check of the batch executor's bounded dependency wait: runs `circuit` on `state` as a
// one-circuit batch whose last pass waits on its own completion counter, which never completes, with
// a wait limit of `wait_limit_us`.  Every CTA that takes a tile of that pass gives up after the limit,
// sets the error flag and leaves, so the call returns QS_ERR_TIMEOUT and the context stays usable; the
// state is left with all passes but the last applied.
extern "C" QS_API int qs_debug_batch_wait_expiry(qs_circuit_t circuit, void* state, QS_UINT wait_limit_us,
    void* stream) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c || !state) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null circuit or state");
    if (wait_limit_us == 0 || wait_limit_us > 2000000u)
        return qs::set_error(QS_ERR_INVALID_ARGUMENT, "wait limit must be 1 us .. 2 s");
    qs::Circuit* cs[1] = {c};
    void* ss[1] = {state};
    // the last record of a one-circuit batch is its last pass
    UINT passes = 0;
    {
        qs::HostPlan H;
        std::vector<qs::GateRec> fg = qs::fuse_gates(c->gates, qs::batch_block_size(*c));
        qs::make_host_plan(fg, c->n, &H, qs::kBatchTileBits);
        passes = (UINT)H.passes.size();
    }
    if (passes == 0) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "circuit has no passes");
    return qs::batch_update(cs, ss, 1, (cudaStream_t)stream, 1000ULL * wait_limit_us, (int)passes - 1, false);
}

