// Host-side circuit representation shared by the executors.
#pragma once

#include <cuda_runtime.h>

#include <complex>
#include <memory>
#include <vector>

typedef unsigned long long ITYPE;
typedef unsigned int UINT;

namespace qs {

constexpr int kMaxQubits = 40;        // largest state (2^40 amplitudes) any entry point accepts
constexpr int kMaxDenseTargets = 12;  // dense gates: 1..12 targets (4^12 matrix entries = 256 MiB)

struct GateRec {
    int kind = 0;
    std::vector<UINT> targets, controls, control_values;
    std::vector<std::complex<double>> matrix;  // dense: 4^k row-major; diagonal: 2^k entries
    std::vector<UINT> pauli_ids;
    double angle = 0.;
    double prob = 0.;

    std::vector<UINT> qubits() const;                      // targets then controls
    std::vector<std::complex<double>> dense_matrix() const;  // on targets only
};

struct StagedPlan;  // staged.cpp

struct Circuit {
    UINT n = 0;
    std::vector<GateRec> gates;
    // cached staged schedule (built on first staged run for a given dim)
    std::shared_ptr<StagedPlan> plan;
    // cached fused complex64 plan (fused_c64.cu)
    std::shared_ptr<void> fused;
    ITYPE fused_dim = 0;
    // FP64-fused gate list and its staged schedule (QS_EXEC_STAGED_FUSED, staged.cu)
    int fusion_k = -1;              // forced block size, or -1: the autotuner chooses
    int fused_k = -1;               // block size of fgates (valid while fplan is set)
    int fused_tile_bits = 12;       // tile qubits of fplan's passes
    std::vector<GateRec> fgates;
    std::shared_ptr<StagedPlan> fplan;
    std::vector<double> tune_ms;    // autotuner estimate per candidate block size (ms; < 0: not tried)
    int specialize = -1;            // single-state passes as specialised kernels: 1 on, 0 off, -1 by state size
    // the circuit acting on a density matrix seen as a 2n-qubit vector (circuit.cpp), for the staged
    // executors of qs_circuit_update_density_matrix
    std::shared_ptr<Circuit> dm_vec;
    // batched execution (qs_batch_update_quantum_states): the gate list fused at a fixed block size
    // (<= 2, so every block stays a pass op) and its staged schedule
    int bk = -1;
    std::vector<GateRec> bgates;
    std::shared_ptr<StagedPlan> bplan;
    // complex64 states: the executor (-1: tensor cores when they take the circuit, else FP64 passes;
    // 0: 6-qubit blocks on the tensor cores, fused_c64.cu; 1: FP64 passes over the complex64 state,
    // staged.cu), the executor of the last run, and the FP64 passes' gate list (blocks of <= 2 qubits)
    // and schedule
    int c64_exec = -1;
    int c64_chosen = -1;
    int ck = -1;
    std::vector<GateRec> cgates;
    std::shared_ptr<StagedPlan> cplan;
    void invalidate() {
        cplan.reset();
        cgates.clear();
        ck = -1;
        c64_chosen = -1;
        dm_vec.reset();
        bplan.reset();
        bgates.clear();
        bk = -1;
        plan.reset();
        fused.reset();
        fused_dim = 0;
        fplan.reset();
        fgates.clear();
        fused_k = -1;
        tune_ms.clear();
    }
};

int apply_gate_by_gate(const GateRec& g, void* state, ITYPE dim, cudaStream_t st);
int apply_gate_dm(const GateRec& g, void* rho, ITYPE dim, cudaStream_t st);
// A density-matrix circuit on n qubits as gates on the 2n-qubit vector rho[row * 2^n + col]
// (column = bits 0..n-1, row = bits n..2n-1): a gate U -> U on the row bits and conj(U) on the
// column bits; a noise channel -> its superoperator sum_k p_k K_k (x) conj(K_k) on its column bits
// then row bits.
std::vector<GateRec> dm_vector_gates(const std::vector<GateRec>& G, UINT n);
int run_staged(Circuit& c, void* state, ITYPE dim, cudaStream_t st);
int run_staged_fused(Circuit& c, void* state, ITYPE dim, cudaStream_t st);
int staged_pass_count(Circuit& c, ITYPE dim, UINT* out);
// staged.cu: the circuit as FP64 passes over a complex64 state (blocks of <= 2 qubits; every gate must
// be stageable)
int run_staged_c64(Circuit& c, void* state_c64, ITYPE dim, cudaStream_t st);
// fused_c64.cu: the tensor-core executor, and whether it takes the circuit
int run_fused_c64(Circuit& c, void* state, ITYPE dim, cudaStream_t st);
bool fused_c64_accepts(const Circuit& c);
// Persistent multi-circuit launches (one state per circuit): staged.cu's FP64 passes over complex128
// or (c64) complex64 states, and fused_c64.cu's tensor-core blocks over complex64 states.  Dependency
// waits are bounded by wait_ns; self_dep >= 0 makes that work record wait on itself (expiry checks).
constexpr unsigned long long kBatchWaitNs = 2000000000ULL;
int batch_update(Circuit* const* cs, void* const* states, UINT count, cudaStream_t st, unsigned long long wait_ns,
    int self_dep, bool c64);
int batch_update_fused_c64(Circuit* const* cs, void* const* states, UINT count, cudaStream_t st,
    unsigned long long wait_ns, int self_dep);

// fusion.cpp: U <- G U for gate g on block-local bit positions `pos` (targets then controls) of a
// kb-qubit block matrix U (2^kb x 2^kb, row-major); and the greedy k-qubit fusion of a gate list.
void apply_gate_to_block(std::vector<std::complex<double>>& U, int kb, const GateRec& g, const std::vector<int>& pos);
std::vector<GateRec> fuse_gates(const std::vector<GateRec>& G, int k);

}  // namespace qs
