// Per-pass kernels of the weighted Pauli expectation value, generated as CUDA C from the pass's terms
// and compiled for sm_100a with NVRTC (csrc/pass_codegen.cpp keeps the compiler and the cache).
//
// The generic pass kernel (k_ev_weighted, csrc/stats_c128.cu) reads each term's descriptor, unpacks
// its masks and branches through a 42-case switch, so every term costs the same dispatch work and the
// terms run one after another.  Here each term's masks, evaluation kind, register indices, partner
// offsets and butterfly signs are compile-time constants: a term is its pair products, a butterfly
// of adds and subtracts, and one parity of the tile element's index, in straight-line code that the
// compiler can interleave across terms.  Z-only strings read one 16-point Walsh-Hadamard transform of
// the thread's probabilities.  The per-pair arithmetic is the generic kernel's (same products); the
// sums are formed in another order, so results agree to rounding.
#include <algorithm>
#include <cstdio>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/qulacs_b200.h"
#include "codegen.hpp"
#include "ev_spec.hpp"

namespace qs {

int set_error(int code, const std::string& msg);

namespace {

const char* kEvPrelude = R"(
typedef unsigned long long u64;
struct __align__(16) D2 { double x, y; };
struct __align__(8) F2 { float x, y; };
struct EvArgs {
    int m;
    u64 b[11];
    unsigned piv[11];
    int nterms;
    int nz;
};
__device__ __forceinline__ D2 mk(double x, double y) { D2 v; v.x = x; v.y = y; return v; }
__device__ __forceinline__ D2 ldd(const D2* p) { return *p; }
__device__ __forceinline__ D2 ldd(const F2* p) { const F2 v = *p; return mk((double)v.x, (double)v.y); }
// Re (C = 0) or Im (C = 1) of a conj(b)
__device__ __forceinline__ double part0(D2 a, D2 b) { return fma(a.x, b.x, a.y * b.y); }
__device__ __forceinline__ double part1(D2 a, D2 b) { return fma(a.y, b.x, -(a.x * b.y)); }
// A coefficient read at its use (volatile: not hoisted out of the tile loop, where every coefficient of
// the pass would stay live in registers).
__device__ __forceinline__ D2 ldc(const D2* p) {
    D2 v;
    asm volatile("ld.global.nc.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
}
__device__ __forceinline__ u64 ins0(u64 i, unsigned q) { return ((i >> q) << (q + 1)) | (i & ((1ULL << q) - 1ULL)); }
__device__ __forceinline__ double flip(double v, unsigned par) {
    return __longlong_as_double(__double_as_longlong(v) ^ ((u64)(par & 1u) << 63));
}
)";

std::string hex32(unsigned v) {
    char buf[24];
    std::snprintf(buf, sizeof(buf), "0x%xu", v);
    return buf;
}

int ctz(unsigned x) { return __builtin_ctz(x); }
int ins0(int i, int k) { return ((i >> k) << (k + 1)) | (i & ((1 << k) - 1)); }
int free_bit(int k, int b) { return b < k ? b : b + 1; }  // b-th register bit other than k

// v0..v7 (bit b of the index <-> register bit bits[b]) folded with the signs of zr's bits.
void emit_fold8(std::ostringstream& o, UINT zr, const int bits[3]) {
    auto op = [&](int b) { return ((zr >> bits[b]) & 1) ? " - " : " + "; };
    o << "    v0 = v0" << op(0) << "v1; v2 = v2" << op(0) << "v3; v4 = v4" << op(0) << "v5; v6 = v6" << op(0)
      << "v7;\n";
    o << "    v0 = v0" << op(1) << "v2; v4 = v4" << op(1) << "v6;\n";
    o << "    double v = v0" << op(2) << "v4;\n";
}

// The tile element's index parity with the full phase-flip mask (g0 = index of register 0 of this thread).
std::string parity(ITYPE z) {
    const unsigned lo = (unsigned)z, hi = (unsigned)(z >> 32);
    std::string s;
    if (lo) s = "__popc(gl & " + hex32(lo) + ")";
    if (hi) s += std::string(s.empty() ? "" : " + ") + "__popc(gh & " + hex32(hi) + ")";
    return s.empty() ? "0u" : s;
}

void emit_term(std::ostringstream& o, const EvWTerm& e, size_t k, int row_bytes, int elem_shift, bool imag) {
    const UINT pk = e.packed;
    const UINT xt = pk & 0xFFu, xr = (pk >> 16) & 15u, zr = (pk >> 20) & 15u, code = pk >> 24;
    o << "  {  // term " << k << "\n    const D2 c = ldc(coef + " << k << ");\n";
    std::string par = parity(e.zglob);
    if (code == EW_Z) {
        o << "    double v = w[" << zr << "];\n";
    } else if (code >= EW_REG) {
        const int C = (int)((code - EW_REG) & 1u), K = ctz(xr);
        for (int i = 0; i < 8; ++i) {
            const int p = ins0(i, K);
            o << "    double v" << i << " = part" << C << "(o[" << p << "], o[" << (p ^ (int)xr) << "]);\n";
        }
        const int bits[3] = {free_bit(K, 0), free_bit(K, 1), free_bit(K, 2)};
        emit_fold8(o, zr, bits);
    } else if (code >= EW_ROW) {
        const int C = (int)(code - EW_ROW), J = ctz(xt);
        o << "    const unsigned bs = (t >> " << J << ") & 1u;\n";
        o << "    const char* pr = tb + ((t ^ " << hex32(xt) << ") << " << elem_shift << ") + bs * " << row_bytes
          << "u;\n";
        for (int i = 0; i < 8; ++i)
            o << "    double v" << i << " = part" << C << "(bs ? o[" << (2 * i + 1) << "] : o[" << (2 * i)
              << "], ldd((const ELEM*)(pr + " << (2 * i * row_bytes) << ")));\n";
        const int bits[3] = {1, 2, 3};
        emit_fold8(o, zr, bits);
        if (zr & 1u) par += " + bs";
    } else {
        const int K = (int)((code - EW_SMEM) >> 1), C = (int)((code - EW_SMEM) & 1u);
        o << "    const char* pr = tb + ((t ^ " << hex32(xt) << ") << " << elem_shift << ");\n";
        for (int i = 0; i < 8; ++i) {
            const int p = ins0(i, K);
            o << "    double v" << i << " = part" << C << "(o[" << p << "], ldd((const ELEM*)(pr + "
              << ((p ^ (int)xr) * row_bytes) << ")));\n";
        }
        const int bits[3] = {free_bit(K, 0), free_bit(K, 1), free_bit(K, 2)};
        emit_fold8(o, zr, bits);
    }
    o << "    v = flip(v, " << par << ");\n    ar = fma(c.x, v, ar);\n";
    if (imag) o << "    ai = fma(c.y, v, ai);\n";
    o << "  }\n";
}

}  // namespace

size_t ev_pass_smem_bytes(bool c64) { return 2 * (size_t)(16 << kEwThreadBits) * (c64 ? 8 : 16); }

std::string ev_pass_source(const EvWTerm* terms, size_t count, bool c64, bool imag) {
    const int elem = c64 ? 8 : 16, elem_shift = c64 ? 3 : 4;
    const int threads = 1 << kEwThreadBits, row_bytes = threads * elem, tile_bytes = 16 * row_bytes;
    std::ostringstream o;
    o << kEvPrelude;
    // the same members in the same order as EvTileArgs (the kernel receives it as a parameter)
    o << "static_assert(sizeof(EvArgs) == " << sizeof(EvTileArgs) << ", \"EvTileArgs layout\");\n";
    o << "typedef " << (c64 ? "F2" : "D2") << " ELEM;\n";
    bool has_z = false;
    for (size_t k = 0; k < count; ++k) has_z |= (terms[k].packed >> 24) == EW_Z;
    o << "extern \"C\" __global__ void __launch_bounds__(" << threads << ", " << kEwCtasPerSm
      << ") k_ev_spec(const ELEM* __restrict__ s, u64 tiles, const __grid_constant__ EvArgs a,\n"
         "    const D2* __restrict__ coef, D2* __restrict__ partials) {\n"
         "  extern __shared__ __align__(16) unsigned char ev_tiles[];\n"
         "  __shared__ u64 hi_off[16];\n"
         "  __shared__ double red[2]["
      << threads / 32
      << "];\n"
         "  const unsigned t = threadIdx.x;\n"
         "  if (t < 16) {\n"
         "    u64 h = 0;\n"
         "    for (int j = 0; j < 4; ++j) if ((t >> j) & 1) h ^= a.b["
      << kEwThreadBits
      << " + j];\n"
         "    hi_off[t] = h;\n"
         "  }\n"
         "  u64 lo_off = 0;\n"
         "  for (int j = 0; j < "
      << kEwThreadBits
      << "; ++j) if ((t >> j) & 1) lo_off ^= a.b[j];\n"
         "  const unsigned sdst = (unsigned)__cvta_generic_to_shared(ev_tiles) + t * "
      << elem
      << "u;\n"
         "  __syncthreads();\n"
         "  auto tile_base = [&](u64 ti) { for (int j = 0; j < a.m; ++j) ti = ins0(ti, a.piv[j]); return ti; };\n"
         "  auto issue = [&](u64 ti, int buf) {\n"
         "    const u64 base = tile_base(ti);\n"
         "#pragma unroll\n"
         "    for (int p = 0; p < 16; ++p) {\n"
         "      const unsigned dst = sdst + buf * "
      << tile_bytes << " + p * " << row_bytes
      << ";\n"
         "      const ELEM* src = s + (base ^ lo_off ^ hi_off[p]);\n"
      << (c64 ? "      asm volatile(\"cp.async.ca.shared.global [%0], [%1], 8;\" :: \"r\"(dst), \"l\"(src) : \"memory\");\n"
              : "      asm volatile(\"cp.async.cg.shared.global [%0], [%1], 16;\" :: \"r\"(dst), \"l\"(src) : \"memory\");\n")
      << "    }\n"
         "  };\n"
         "  if ((u64)blockIdx.x < tiles) issue(blockIdx.x, 0);\n"
         "  asm volatile(\"cp.async.commit_group;\" ::: \"memory\");\n"
         "  double ar = 0., ai = 0.;\n"
         "  int buf = 0;\n"
         "  for (u64 ti = blockIdx.x; ti < tiles; ti += gridDim.x, buf ^= 1) {\n"
         "    if (ti + gridDim.x < tiles) issue(ti + gridDim.x, buf ^ 1);\n"
         "    asm volatile(\"cp.async.commit_group;\\ncp.async.wait_group 1;\" ::: \"memory\");\n"
         "    __syncthreads();\n"
         "    const char* tb = (const char*)ev_tiles + buf * "
      << tile_bytes
      << ";\n"
         "    const u64 g0 = tile_base(ti) ^ lo_off;\n"
         "    const unsigned gl = (unsigned)g0, gh = (unsigned)(g0 >> 32);\n"
         "    D2 o[16];\n"
         "#pragma unroll\n"
         "    for (int p = 0; p < 16; ++p) o[p] = ldd((const ELEM*)(tb + t * "
      << elem << "u + p * " << row_bytes << "));\n";
    if (has_z) {
        o << "    double w[16];\n"
             "#pragma unroll\n"
             "    for (int p = 0; p < 16; ++p) w[p] = fma(o[p].x, o[p].x, o[p].y * o[p].y);\n"
             "#pragma unroll\n"
             "    for (int h = 1; h < 16; h <<= 1)\n"
             "#pragma unroll\n"
             "      for (int i = 0; i < 16; ++i)\n"
             "        if (!(i & h)) { const double x = w[i], y = w[i | h]; w[i] = x + y; w[i | h] = x - y; }\n";
    }
    // Z-only terms first: the transform's 16 values die before the bit-flip terms run.  Every
    // kSegment terms sit in a block behind a branch the compiler cannot resolve (a.nterms is the term
    // count): that bounds how far it interleaves terms, which would otherwise keep the partner
    // amplitudes of many terms live at once and spill.
    constexpr size_t kSegment = 8;
    std::vector<size_t> order;
    for (size_t k = 0; k < count; ++k)
        if ((terms[k].packed >> 24) == EW_Z) order.push_back(k);
    for (size_t k = 0; k < count; ++k)
        if ((terms[k].packed >> 24) != EW_Z) order.push_back(k);
    for (size_t j = 0; j < order.size(); j += kSegment) {
        o << "  if (a.nterms > " << j << ") {\n";
        for (size_t i = j; i < std::min(order.size(), j + kSegment); ++i)
            emit_term(o, terms[order[i]], order[i], row_bytes, elem_shift, imag);
        o << "  }\n";
    }
    o << "    __syncthreads();\n"
         "  }\n"
         "  asm volatile(\"cp.async.wait_group 0;\" ::: \"memory\");\n"
         "#pragma unroll\n"
         "  for (int d = 16; d > 0; d >>= 1) {\n"
         "    ar += __shfl_xor_sync(0xffffffffu, ar, d);\n"
         "    ai += __shfl_xor_sync(0xffffffffu, ai, d);\n"
         "  }\n"
         "  if ((t & 31) == 0) { red[0][t >> 5] = ar; red[1][t >> 5] = ai; }\n"
         "  __syncthreads();\n"
         "  if (t == 0) {\n"
         "    double r = 0., i = 0.;\n"
         "    for (int w2 = 0; w2 < "
      << threads / 32
      << "; ++w2) { r += red[0][w2]; i += red[1][w2]; }\n"
         "    partials[blockIdx.x] = mk(r, i);\n"
         "  }\n"
         "}\n";
    return o.str();
}

int ev_pass_kernel(const EvWTerm* terms, size_t count, bool c64, bool imag, void** kernel, double* compile_ms) {
    return nvrtc_kernel(ev_pass_source(terms, count, c64, imag), "k_ev_spec", kernel, compile_ms);
}

int launch_ev_pass(void* kernel, const void* state, ITYPE tiles, const EvTileArgs& a, const double2* coef,
    double2* partials, unsigned grid, bool c64, cudaStream_t st) {
    void* args[] = {&state, &tiles, const_cast<EvTileArgs*>(&a), &coef, &partials};
    const size_t smem = ev_pass_smem_bytes(c64);
    return launch_nvrtc_kernel(kernel, dim3(grid), dim3(1u << kEwThreadBits), args, smem, smem, st, "k_ev_spec");
}

}  // namespace qs
