// Specialised staged-pass kernels: one kernel per pass, generated as CUDA C from the pass's schedule and
// compiled for sm_100a with NVRTC at plan time.
//
// The generic pass kernel (k_staged_pass, staged.cu) interprets each phase's op list: per op it loads
// the op record and its matrix from memory, branches through a 128-case switch, and returns its 16
// amplitudes to the registers the switch fixed, which costs register moves at every op boundary and an
// instruction footprint larger than the instruction cache.  Here every tile qubit, phase bit, Gray-code
// address offset and matrix entry is a compile-time constant: the phases become straight-line code,
// matrix entries are read as constant-bank operands, and the compiler allocates registers across op
// boundaries.  The arithmetic of each op is the generic kernel's (same fma sequence, same order), and
// the tile load/store, HBM-direct first/last phases and 16-byte swizzle are the same.
//
// NVRTC is opened at run time (libnvrtc.so.12); the compiled cubin is loaded with cudaLibraryLoadData,
// which makes it available to every device context.  Kernels are cached by source text for the life of
// the process.
#include <dlfcn.h>

#include <chrono>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/qulacs_b200.h"
#include "codegen.hpp"
#include "staged.hpp"

namespace qs {

int set_error(int code, const std::string& msg);
int check_cuda(cudaError_t e, const char* what);
int check_launch(const char* kernel);

namespace {

// ---------------------------------------------------------------- NVRTC, opened at run time
typedef int nvrtcResult_t;
typedef struct _nvrtcProgram* nvrtcProgram_t;
struct Nvrtc {
    void* h = nullptr;
    nvrtcResult_t (*create)(nvrtcProgram_t*, const char*, const char*, int, const char* const*, const char* const*) =
        nullptr;
    nvrtcResult_t (*compile)(nvrtcProgram_t, int, const char* const*) = nullptr;
    nvrtcResult_t (*cubin_size)(nvrtcProgram_t, size_t*) = nullptr;
    nvrtcResult_t (*cubin)(nvrtcProgram_t, char*) = nullptr;
    nvrtcResult_t (*log_size)(nvrtcProgram_t, size_t*) = nullptr;
    nvrtcResult_t (*log)(nvrtcProgram_t, char*) = nullptr;
    nvrtcResult_t (*destroy)(nvrtcProgram_t*) = nullptr;
    std::string error;
};

Nvrtc* nvrtc() {
    static Nvrtc N;
    static std::once_flag once;
    std::call_once(once, [] {
        std::vector<std::string> names;
        for (const char* env : {"CUDA_HOME", "CUDA_PATH"})
            if (const char* p = std::getenv(env)) names.push_back(std::string(p) + "/lib64/libnvrtc.so.12");
        names.push_back("libnvrtc.so.12");
        names.push_back("libnvrtc.so");
        for (const std::string& nm : names) {
            N.h = dlopen(nm.c_str(), RTLD_NOW | RTLD_LOCAL);
            if (N.h) break;
        }
        if (!N.h) {
            N.error = "NVRTC (libnvrtc.so.12) not found";
            return;
        }
        auto sym = [&](const char* s) { return dlsym(N.h, s); };
        N.create = (decltype(N.create))sym("nvrtcCreateProgram");
        N.compile = (decltype(N.compile))sym("nvrtcCompileProgram");
        N.cubin_size = (decltype(N.cubin_size))sym("nvrtcGetCUBINSize");
        N.cubin = (decltype(N.cubin))sym("nvrtcGetCUBIN");
        N.log_size = (decltype(N.log_size))sym("nvrtcGetProgramLogSize");
        N.log = (decltype(N.log))sym("nvrtcGetProgramLog");
        N.destroy = (decltype(N.destroy))sym("nvrtcDestroyProgram");
        if (!N.create || !N.compile || !N.cubin_size || !N.cubin || !N.log_size || !N.log || !N.destroy) {
            N.error = "NVRTC lacks the CUBIN entry points";
            N.h = nullptr;
        }
    });
    return &N;
}

// ---------------------------------------------------------------- kernel source
// The device helpers every generated kernel shares.  The register ops mirror staged.cu's r_* ops, with
// the matrix entries passed by value so that literal arguments become constants.
const char* kPrelude = R"(
typedef unsigned long long u64;
struct __align__(16) D2 { double x, y; };
__device__ __forceinline__ D2 mk(double x, double y) { D2 v; v.x = x; v.y = y; return v; }
__device__ __forceinline__ D2 cmul(D2 a, D2 b) { return mk(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x)); }
__device__ __forceinline__ D2 cfma(D2 a, D2 b, D2 acc) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
    return acc;
}
__device__ __forceinline__ D2 ldcs(const D2* p) {
    D2 v;
    asm volatile("ld.global.cs.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
}
__device__ __forceinline__ void stcs(D2* p, D2 v) {
    asm volatile("st.global.cs.v2.f64 [%0], {%1, %2};" ::"l"(p), "d"(v.x), "d"(v.y) : "memory");
}
// A parameter read at its use (volatile: not hoisted out of the coset loop, where every parameter of
// the pass would stay live in registers).
__device__ __forceinline__ D2 ldp(const D2* p) {
    D2 v;
    asm volatile("ld.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
}
__device__ __forceinline__ unsigned swz(unsigned u) { return u ^ (((u >> 4) ^ (u >> 7) ^ (u >> 10)) & 7u); }
__device__ __forceinline__ u64 ins0(u64 i, unsigned q) { return ((i >> q) << (q + 1)) | (i & ((1ULL << q) - 1ULL)); }

template <int B> __device__ __forceinline__ void r_dense1(D2 (&r)[16], D2 m0, D2 m1, D2 m2, D2 m3) {
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (!(j & (1 << B))) {
            const D2 x = r[j], y = r[j | (1 << B)];
            r[j] = cfma(m1, y, cmul(m0, x));
            r[j | (1 << B)] = cfma(m3, y, cmul(m2, x));
        }
}
template <int B> __device__ __forceinline__ void r_diag1(D2 (&r)[16], D2 d0, D2 d1) {
#pragma unroll
    for (int j = 0; j < 16; ++j) r[j] = cmul((j & (1 << B)) ? d1 : d0, r[j]);
}
template <int B> __device__ __forceinline__ void r_rx(D2 (&r)[16], double c, double s) {
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (!(j & (1 << B))) {
            const D2 x = r[j], y = r[j | (1 << B)];
            r[j] = mk(fma(c, x.x, -s * y.y), fma(c, x.y, s * y.x));
            r[j | (1 << B)] = mk(fma(c, y.x, -s * x.y), fma(c, y.y, s * x.x));
        }
}
template <int B> __device__ __forceinline__ void r_ry(D2 (&r)[16], double c, double s) {
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (!(j & (1 << B))) {
            const D2 x = r[j], y = r[j | (1 << B)];
            r[j] = mk(fma(c, x.x, s * y.x), fma(c, x.y, s * y.y));
            r[j | (1 << B)] = mk(fma(c, y.x, -s * x.x), fma(c, y.y, -s * x.y));
        }
}
template <int C, int T> __device__ __forceinline__ void r_cnot(D2 (&r)[16]) {
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if ((j & (1 << C)) && !(j & (1 << T))) {
            const D2 t = r[j];
            r[j] = r[j | (1 << T)];
            r[j | (1 << T)] = t;
        }
}
template <int A, int B> __device__ __forceinline__ void r_cz(D2 (&r)[16]) {
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if ((j & (1 << A)) && (j & (1 << B))) r[j] = mk(-r[j].x, -r[j].y);
}
template <int A, int B> __device__ __forceinline__ void r_swap(D2 (&r)[16]) {
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if ((j & (1 << A)) && !(j & (1 << B))) {
            const int k = j ^ (1 << A) ^ (1 << B);
            const D2 t = r[j];
            r[j] = r[k];
            r[k] = t;
        }
}
template <int A, int B> __device__ __forceinline__ void r_dense2(D2 (&r)[16], const D2 (&p)[16]) {
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (!(j & (1 << A)) && !(j & (1 << B))) {
            const int o[4] = {j, j | (1 << A), j | (1 << B), j | (1 << A) | (1 << B)};
            D2 v[4];
#pragma unroll
            for (int x = 0; x < 4; ++x) v[x] = r[o[x]];
#pragma unroll
            for (int y = 0; y < 4; ++y) {
                D2 acc = cmul(p[y * 4], v[0]);
#pragma unroll
                for (int x = 1; x < 4; ++x) acc = cfma(p[y * 4 + x], v[x], acc);
                r[o[y]] = acc;
            }
        }
}
// r_dense2 with the matrix read from a parameter block at each use (volatile loads: only the entries
// of the row being computed are live).
template <int A, int B> __device__ __forceinline__ void r_dense2p(D2 (&r)[16], const D2* p) {
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (!(j & (1 << A)) && !(j & (1 << B))) {
            const int o[4] = {j, j | (1 << A), j | (1 << B), j | (1 << A) | (1 << B)};
            D2 v[4];
#pragma unroll
            for (int x = 0; x < 4; ++x) v[x] = r[o[x]];
#pragma unroll
            for (int y = 0; y < 4; ++y) {
                D2 acc = cmul(ldp(p + y * 4), v[0]);
#pragma unroll
                for (int x = 1; x < 4; ++x) acc = cfma(ldp(p + y * 4 + x), v[x], acc);
                r[o[y]] = acc;
            }
        }
}
template <int A, int B> __device__ __forceinline__ void r_csel1(D2 (&r)[16], D2 m0, D2 m1, D2 m2, D2 m3, D2 n0, D2 n1,
                                                                D2 n2, D2 n3) {
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (!(j & (1 << A))) {
            const D2 x = r[j], y = r[j | (1 << A)];
            const bool hi = (j >> B) & 1;
            r[j] = cfma(hi ? n1 : m1, y, cmul(hi ? n0 : m0, x));
            r[j | (1 << A)] = cfma(hi ? n3 : m3, y, cmul(hi ? n2 : m2, x));
        }
}
template <int A, int B> __device__ __forceinline__ void r_d1_in(D2 (&r)[16], D2 m0, D2 m1, D2 m2, D2 m3) {
    D2 o[16];
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (!(j & (1 << A))) {
            const int k = j ^ (1 << A) ^ (1 << B);
            const D2 x = r[j], y = r[k];
            o[j] = cfma(m1, y, cmul(m0, x));
            o[j | (1 << A)] = cfma(m3, y, cmul(m2, x));
        }
#pragma unroll
    for (int j = 0; j < 16; ++j) r[j] = o[j];
}
template <int A, int B> __device__ __forceinline__ void r_d1_out(D2 (&r)[16], D2 m0, D2 m1, D2 m2, D2 m3) {
    D2 o[16];
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (!(j & (1 << A))) {
            const D2 x = r[j], y = r[j | (1 << A)];
            o[j] = cfma(m1, y, cmul(m0, x));
            o[j ^ (1 << A) ^ (1 << B)] = cfma(m3, y, cmul(m2, x));
        }
#pragma unroll
    for (int j = 0; j < 16; ++j) r[j] = o[j];
}
)";

// An exact C++17 hexadecimal literal of a double.
std::string lit(double v) {
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%a", v);
    return buf;
}
// Gate parameters of a generated kernel: written into the source as literals, or (when `bank` is set)
// referenced as P.v[i] of the kernel's __grid_constant__ parameter block and collected into `bank`, so
// the kernel depends only on the pass's structure and is shared by circuits that differ in angles.
struct ParamSink {
    std::vector<double2>* bank = nullptr;
    std::string d2(const double2& v) {
        if (!bank) return "mk(" + lit(v.x) + ", " + lit(v.y) + ")";
        bank->push_back(v);
        return "ldp(&P.v[" + std::to_string(bank->size() - 1) + "])";
    }
};

std::string u64hex(ITYPE v) {
    char buf[40];
    std::snprintf(buf, sizeof(buf), "0x%llxULL", (unsigned long long)v);
    return buf;
}

int gray_bit(int g) { return (g & 1) ? 0 : (g & 2) ? 1 : (g & 4) ? 2 : 3; }

unsigned swz_host(unsigned u) { return u ^ (((u >> 4) ^ (u >> 7) ^ (u >> 10)) & 7u); }

void emit_op(std::ostringstream& o, const StOp& op, const double2* pool, ParamSink& ps) {
    const double2* p = pool + op.param;
    const int a = op.a, b = op.b;
    auto d2 = [&](const double2& v) { return ps.d2(v); };
    switch (op.kind) {
        case ST_DENSE1:
            o << "      r_dense1<" << a << ">(r, " << d2(p[0]) << ", " << d2(p[1]) << ", " << d2(p[2]) << ", " << d2(p[3])
              << ");\n";
            break;
        case ST_DIAG1: o << "      r_diag1<" << a << ">(r, " << d2(p[0]) << ", " << d2(p[1]) << ");\n"; break;
        case ST_RX:
        case ST_RY:
            o << "      { const D2 cs = " << d2(p[0]) << "; r_" << (op.kind == ST_RX ? "rx" : "ry") << "<" << a
              << ">(r, cs.x, cs.y); }\n";
            break;
        case ST_CNOT: o << "      r_cnot<" << a << ", " << b << ">(r);\n"; break;
        case ST_CZ: o << "      r_cz<" << a << ", " << b << ">(r);\n"; break;
        case ST_SWAP: o << "      r_swap<" << a << ", " << b << ">(r);\n"; break;
        case ST_DENSE2: {
            if (ps.bank) {  // the 16 entries as one run of the parameter block, read row by row
                const size_t first = ps.bank->size();
                for (int i = 0; i < 16; ++i) ps.bank->push_back(p[i]);
                o << "      r_dense2p<" << a << ", " << b << ">(r, &P.v[" << first << "]);\n";
                break;
            }
            o << "      { const D2 m[16] = {";
            for (int i = 0; i < 16; ++i) o << (i ? ", " : "") << d2(p[i]);
            o << "}; r_dense2<" << a << ", " << b << ">(r, m); }\n";
            break;
        }
        case ST_CSEL1:
            o << "      r_csel1<" << a << ", " << b << ">(r";
            for (int i = 0; i < 8; ++i) o << ", " << d2(p[i]);
            o << ");\n";
            break;
        case ST_D1_IN:
        case ST_D1_OUT:
            o << "      r_d1_" << (op.kind == ST_D1_IN ? "in" : "out") << "<" << a << ", " << b << ">(r, " << d2(p[0])
              << ", " << d2(p[1]) << ", " << d2(p[2]) << ", " << d2(p[3]) << ");\n";
            break;
        default: o << "      /* unknown op */\n"; break;
    }
}

// Largest parameter block passed to a kernel (within the classic 4 KB kernel-parameter space, with
// room for the state pointer); a pass with more parameters gets them as literals instead.
constexpr size_t kMaxParamBytes = 4000;

// CUDA C of one pass; mirrors staged_tile (staged.cu) with every schedule quantity a constant.  With
// `params`, gate parameters come from the kernel's parameter block (their values appended to *params);
// without, they are literals.
std::string pass_source(const PassDesc& d, std::vector<double2>* params) {
    const int m = d.m;
    const unsigned tsize = 1u << m, ncos = tsize >> kPhaseBits;
    const bool hbm_first = d.io & 1, hbm_last = (d.io >> 1) & 1;
    const int rows = 1 << (m - 7);  // tile rows of kStThreads amplitudes
    ParamSink ps;
    ps.bank = params;
    std::ostringstream o;  // kernel body (the parameter block's size is known once it is written)
    o << ") {\n";
    o << "  extern __shared__ D2 tile[];\n  char* tb = reinterpret_cast<char*>(tile);\n";
    o << "  const unsigned tid = threadIdx.x;\n  u64 base = blockIdx.x;\n";
    for (int j = 0; j < m; ++j) o << "  base = ins0(base, " << d.q[j] << "u);\n";
    if (!hbm_first || !hbm_last) {
        o << "  u64 lo = 0;\n";
        for (int j = 0; j < 7 && j < m; ++j) o << "  lo |= (u64)((tid >> " << j << ") & 1u) << " << d.q[j] << ";\n";
    }
    if (!hbm_first) {
        o << "  {\n";
        for (int k = 0; k < rows; ++k) {
            ITYPE hi = 0;
            for (int j = 7; j < m; ++j)
                if ((k >> (j - 7)) & 1) hi |= 1ULL << d.q[j];
            o << "    asm volatile(\"cp.async.cg.shared.global [%0], [%1], 16;\" :: \"r\"((unsigned)__cvta_generic_to_shared("
              << "tile + swz(tid + " << k * kStThreads << "u))), \"l\"(s + (base | lo | " << u64hex(hi) << ")) : \"memory\");\n";
        }
        o << "    asm volatile(\"cp.async.commit_group;\\ncp.async.wait_group 0;\" ::: \"memory\");\n    __syncthreads();\n  }\n";
    }
    const int np = (int)d.phases.size();
    for (int ph = 0; ph < np; ++ph) {
        const StPhase& P = d.phases[ph];
        const bool from_hbm = hbm_first && ph == 0, to_hbm = hbm_last && ph == np - 1;
        o << "  // phase " << ph << ": tile bits " << (int)P.bits[0] << "," << (int)P.bits[1] << "," << (int)P.bits[2] << ","
          << (int)P.bits[3] << ", " << P.op_count << " ops\n";
        o << "#pragma unroll 1\n  for (unsigned c = tid; c < " << ncos << "u; c += " << kStThreads << "u) {\n";
        o << "    unsigned u0 = c;\n";
        for (int p = 0; p < 4; ++p) o << "    u0 = (unsigned)ins0(u0, " << (int)P.bits[p] << "u);\n";
        o << "    D2 r[16];\n";
        if (from_hbm || to_hbm) {
            o << "    u64 g0 = base;\n";
            for (int j = 0; j < m; ++j) o << "    g0 |= (u64)((u0 >> " << j << ") & 1u) << " << d.q[j] << ";\n";
        }
        if (from_hbm) {
            o << "    { u64 gi = g0;\n";
            for (int g = 0; g < 16; ++g) {
                if (g) o << "      gi ^= " << u64hex(1ULL << d.q[P.bits[gray_bit(g)]]) << ";\n";
                o << "      r[" << (g ^ (g >> 1)) << "] = ldcs(s + gi);\n";
            }
            o << "    }\n";
        } else {
            o << "    { unsigned a = swz(u0) << 4;\n";
            for (int g = 0; g < 16; ++g) {
                if (g) o << "      a ^= " << (swz_host(1u << P.bits[gray_bit(g)]) << 4) << "u;\n";
                o << "      r[" << (g ^ (g >> 1)) << "] = *reinterpret_cast<const D2*>(tb + a);\n";
            }
            o << "    }\n";
        }
        for (uint32_t i = 0; i < P.op_count; ++i) emit_op(o, d.ops[P.op_begin + i], d.pool, ps);
        if (to_hbm) {
            o << "    { u64 gi = g0;\n";
            for (int g = 0; g < 16; ++g) {
                if (g) o << "      gi ^= " << u64hex(1ULL << d.q[P.bits[gray_bit(g)]]) << ";\n";
                o << "      stcs(s + gi, r[" << (g ^ (g >> 1)) << "]);\n";
            }
            o << "    }\n";
        } else {
            o << "    { unsigned a = swz(u0) << 4;\n";
            for (int g = 0; g < 16; ++g) {
                if (g) o << "      a ^= " << (swz_host(1u << P.bits[gray_bit(g)]) << 4) << "u;\n";
                o << "      *reinterpret_cast<D2*>(tb + a) = r[" << (g ^ (g >> 1)) << "];\n";
            }
            o << "    }\n";
        }
        o << "  }\n";
        if (!to_hbm) o << "  __syncthreads();\n";
    }
    if (!hbm_last) {
        // batches of 16 rows per thread: the batch's shared-memory loads first, then its streaming
        // stores; row k's global offset takes k's bits to the tile qubits q[7..]
        const int batch = rows < 16 ? rows : 16;
        o << "#pragma unroll 1\n  for (unsigned k0 = 0; k0 < " << rows << "u; k0 += " << batch << "u) {\n";
        o << "    D2 v[" << batch << "];\n#pragma unroll\n    for (unsigned k = 0; k < " << batch
          << "u; ++k) v[k] = tile[swz(tid + (k0 + k) * " << kStThreads << "u)];\n";
        o << "#pragma unroll\n    for (unsigned k = 0; k < " << batch << "u; ++k) {\n      const unsigned row = k0 + k;\n"
          << "      u64 hi = 0;\n";
        for (int j = 7; j < m; ++j) o << "      hi |= (u64)((row >> " << j - 7 << ") & 1u) << " << d.q[j] << ";\n";
        o << "      stcs(s + (base | lo | hi), v[k]);\n    }\n  }\n";
    }
    o << "}\n";
    std::ostringstream h;
    h << kPrelude;
    if (params) h << "struct PassParams { D2 v[" << std::max<size_t>(1, params->size()) << "]; };\n";
    h << "extern \"C\" __global__ void __launch_bounds__(" << kStThreads << ", 3) k_pass_spec(D2* __restrict__ s";
    if (params) h << ", const __grid_constant__ PassParams P";
    return h.str() + o.str();
}

struct Compiled {
    cudaLibrary_t lib = nullptr;
    cudaKernel_t kernel = nullptr;
    bool has_params = false;  // takes a parameter block after the state pointer
    std::set<int> smem_set;  // devices on which the dynamic shared-memory limit is raised
};

std::mutex g_mu;
std::map<std::string, std::shared_ptr<Compiled>> g_cache;
std::map<std::string, std::shared_ptr<std::mutex>> g_building;  // one compile per source at a time

int compile(const std::string& src, const char* name, std::vector<char>* cubin) {
    Nvrtc* N = nvrtc();
    if (!N->h) return set_error(QS_ERR_NOT_SUPPORTED, "specialised kernels: " + N->error);
    nvrtcProgram_t prog = nullptr;
    const std::string file = std::string(name) + ".cu";
    if (N->create(&prog, src.c_str(), file.c_str(), 0, nullptr, nullptr) != 0)
        return set_error(QS_ERR_CUDA, "specialised kernels: nvrtcCreateProgram failed");
    const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17"};
    const int rc = N->compile(prog, 2, opts);
    if (rc != 0) {
        size_t n = 0;
        N->log_size(prog, &n);
        std::string log(n, '\0');
        if (n) N->log(prog, &log[0]);
        N->destroy(&prog);
        return set_error(QS_ERR_CUDA, std::string(name) + ": NVRTC compile failed: " + log.substr(0, 2000));
    }
    size_t n = 0;
    N->cubin_size(prog, &n);
    cubin->resize(n);
    N->cubin(prog, cubin->data());
    N->destroy(&prog);
    return QS_OK;
}

}  // namespace

int nvrtc_kernel(const std::string& src, const char* name, void** kernel, double* compile_ms) {
    std::shared_ptr<std::mutex> build_mu;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_cache.find(src);
        if (it != g_cache.end()) {
            *kernel = it->second.get();
            if (compile_ms) *compile_ms = 0.;
            return QS_OK;
        }
        auto& b = g_building[src];
        if (!b) b = std::make_shared<std::mutex>();
        build_mu = b;
    }
    std::lock_guard<std::mutex> blk(*build_mu);
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_cache.find(src);
        if (it != g_cache.end()) {
            *kernel = it->second.get();
            if (compile_ms) *compile_ms = 0.;
            return QS_OK;
        }
    }
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<char> cubin;
    int rc = compile(src, name, &cubin);
    if (rc != QS_OK) return rc;
    auto C = std::make_shared<Compiled>();
    cudaError_t e = cudaLibraryLoadData(&C->lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e != cudaSuccess) return check_cuda(e, "cudaLibraryLoadData (specialised kernel)");
    e = cudaLibraryGetKernel(&C->kernel, C->lib, name);
    if (e != cudaSuccess) return check_cuda(e, "cudaLibraryGetKernel (specialised kernel)");
    if (compile_ms)
        *compile_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    std::lock_guard<std::mutex> lk(g_mu);
    g_cache[src] = C;  // entries live for the process, so the handle stays valid
    g_building.erase(src);
    *kernel = C.get();
    return QS_OK;
}

int launch_nvrtc_kernel(void* handle, dim3 grid, dim3 block, void** args, size_t smem, size_t smem_limit,
    cudaStream_t st, const char* what) {
    Compiled* C = static_cast<Compiled*>(handle);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return check_cuda(e, "cudaGetDevice");
    {
        // raise the kernel's dynamic shared-memory limit once per device
        std::lock_guard<std::mutex> lk(g_mu);
        if (!C->smem_set.count(dev)) {
            e = cudaFuncSetAttribute((const void*)C->kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                (int)smem_limit);
            if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute (specialised kernel)");
            C->smem_set.insert(dev);
        }
    }
    e = cudaLaunchKernel((const void*)C->kernel, grid, block, args, smem, st);
    if (e != cudaSuccess) return check_cuda(e, what);
    return check_launch(what);
}

int specialized_pass_kernel(const PassDesc& d, void** kernel, std::vector<double2>* params, double* compile_ms) {
    if (d.m < 7 || d.m > kTileBits || d.phases.empty())
        return set_error(QS_ERR_NOT_SUPPORTED, "specialised passes need 7..12 tile qubits and a phase");
    params->clear();
    std::string src = pass_source(d, params);
    if (params->empty() || params->size() * sizeof(double2) > kMaxParamBytes) {
        // no parameters (the kernel takes only the state), or too many for a parameter block: literals
        params->clear();
        src = pass_source(d, nullptr);
    }
    const int rc = nvrtc_kernel(src, "k_pass_spec", kernel, compile_ms);
    if (rc != QS_OK) return rc;
    static_cast<Compiled*>(*kernel)->has_params = !params->empty();  // a property of the source
    return QS_OK;
}

int launch_specialized_pass(void* handle, double2* state, const double2* params, ITYPE tiles, int m, cudaStream_t st) {
    Compiled* C = static_cast<Compiled*>(handle);
    if (C->has_params && !params) return set_error(QS_ERR_INVALID_ARGUMENT, "specialised pass: no parameter block");
    void* args[] = {&state, const_cast<double2*>(params)};  // the parameter block is copied at launch
    return launch_nvrtc_kernel(handle, dim3((unsigned)tiles), dim3(kStThreads), args, sizeof(double2) << m,
        sizeof(double2) << kTileBits, st, "k_pass_spec");
}

std::string specialized_pass_source(const PassDesc& d) {
    std::vector<double2> params;
    return pass_source(d, &params);
}

}  // namespace qs
