// Weighted Pauli expectation value, shared by the generic pass kernel (csrc/stats_c128.cu) and the
// per-pass kernels generated at run time (csrc/ev_codegen.cpp).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include <string>

typedef unsigned long long ITYPE;
typedef unsigned int UINT;

namespace qs {

constexpr int kEvBasisBits = 11;  // tile qubits of a pass: 2^11 amplitudes

// A tile is a coset of the span of m basis masks b_j over the index bits, in reduced echelon form:
// b_j has bit piv_j set and no other basis mask has it.  Tile element u (bit j <-> b_j) of tile T is
// index rep(T) ^ XOR_{j in u} b_j, rep(T) = T with zeros inserted at the pivots (ascending in
// `piv_sorted`).  With unit vectors the tile is the usual set of tile qubits.
struct EvTileArgs {
    int m;
    ITYPE b[kEvBasisBits];
    UINT piv_sorted[kEvBasisBits];
    int nterms;
    int nz;  // the last nz terms are Z-only strings (no bit flip)
};

// Weighted passes: tile bits 0..6 are the thread index, tile bits 7..10 index 16 amplitudes held in a
// thread's registers.
constexpr int kEwThreadBits = 7;
constexpr int kEwCtasPerSm = 3;  // 64 KiB of tile buffers each (complex128)
static_assert(kEwThreadBits + 4 == kEvBasisBits, "16 register amplitudes per thread");

struct EvWTerm {  // 32 bytes, read warp-uniformly by the generic kernel
    double2 coef;  // c_k times the term's factor: +-2 for a bit flip (i^nrot picks the part and sign), 1 for Z-only
    ITYPE zglob;   // phase-flip mask over the full index (its parity with the tile element's index)
    UINT packed;   // xt | zt << 8 | xr << 16 | zr << 20 | code << 24
    UINT pad;
};
// code: 0 Z-only; 2 + 2K + C: xt, xr != 0 (K = lowest bit of xr); 10 + C: xr = 0;
// 12 + 2 (xr - 1) + C: xt = 0.  C = 1 takes the imaginary part of a conj(b) (odd Y count).
enum : UINT { EW_Z = 0, EW_SMEM = 2, EW_ROW = 10, EW_REG = 12 };

// csrc/ev_codegen.cpp: one pass's kernel with its terms' masks compiled in (the coefficients stay a
// device array, so a kernel serves any coefficients of the same strings).  `c64`: complex64 state.
// `imag`: some coefficient has an imaginary part.
std::string ev_pass_source(const EvWTerm* terms, size_t count, bool c64, bool imag);
int ev_pass_kernel(const EvWTerm* terms, size_t count, bool c64, bool imag, void** kernel, double* compile_ms);
// grid CTAs of 2^kEwThreadBits threads over `tiles` tiles; partials[blockIdx] = the CTA's (re, im) sum.
int launch_ev_pass(void* kernel, const void* state, ITYPE tiles, const EvTileArgs& a, const double2* coef,
    double2* partials, unsigned grid, bool c64, cudaStream_t st);
size_t ev_pass_smem_bytes(bool c64);

}  // namespace qs
