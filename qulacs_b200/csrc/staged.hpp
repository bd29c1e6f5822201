// Host-visible description of a staged pass (csrc/staged.cu builds it; csrc/pass_codegen.cpp turns one
// pass into a specialised kernel).  A pass owns m tile qubits q[0..m-1] (ascending, q[j] = j for
// j < kLowFixed); its gates run in phases of 4 tile bits, each phase a list of register ops on a
// thread's 16-amplitude coset.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

typedef unsigned long long ITYPE;
typedef unsigned int UINT;

namespace qs {

constexpr int kLowFixed = 4;        // qubits 0..3 always belong to a tile
constexpr int kTileBits = 12;       // pass kernel: 2^12 amplitudes = 64 KiB of shared memory per CTA
constexpr int kBatchTileBits = 11;  // multi-circuit kernel: 2^11 amplitudes = 32 KiB
constexpr int kStThreads = 128;     // 16 (m = 11) or 32 (m = 12) amplitudes per thread; 1 or 2 cosets per phase
constexpr int kPhaseBits = 4;       // 16 amplitudes in registers per thread

// ST_CSEL1, ST_D1_IN and ST_D1_OUT are a one-qubit dense gate with a CNOT (or CZ) folded in.
enum StKind : uint8_t {
    ST_DENSE1 = 0, ST_DIAG1, ST_RX, ST_RY, ST_CNOT, ST_CZ, ST_SWAP, ST_DENSE2, ST_CSEL1, ST_D1_IN, ST_D1_OUT
};

struct StOp {
    uint8_t kind, a, b, pad;  // a, b: register-bit indices 0..3 within the phase; pad: dispatch code
    uint32_t param;           // index into the parameter pool (double2)
};
struct StPhase {
    uint8_t bits[4];  // tile-local bit positions, ascending
    uint32_t op_begin, op_count;
};

// One pass as the code generator sees it: tile qubits, the HBM-direct first/last phase flags, and the
// host copies of its phases, ops and parameters.
struct PassDesc {
    int m = 0;
    int io = 0;  // bit 0: the first phase gathers from HBM; bit 1: the last phase scatters to HBM
    UINT q[kTileBits] = {};
    std::vector<StPhase> phases;  // op_begin indexes `ops`
    const StOp* ops = nullptr;
    const double2* pool = nullptr;
};

// csrc/pass_codegen.cpp: a kernel for one pass with its tile qubits, phase bits and op list compiled
// in (NVRTC, sm_100a), cached by source for the life of the process.  `handle` receives the
// cache entry (valid until exit), launched over dim >> m CTAs of kStThreads threads with 16 << m bytes
// of dynamic shared memory.  QS_ERR_NOT_SUPPORTED when NVRTC cannot be loaded.
// The kernel depends only on the pass's structure: its gate parameters are a kernel-parameter block
// whose values `params` receives (empty when the pass has too many and they are literals instead), to
// be passed at every launch.
int specialized_pass_kernel(const PassDesc& d, void** handle, std::vector<double2>* params, double* compile_ms);
int launch_specialized_pass(void* handle, double2* state, const double2* params, ITYPE tiles, int m, cudaStream_t st);
std::string specialized_pass_source(const PassDesc& d);

}  // namespace qs
