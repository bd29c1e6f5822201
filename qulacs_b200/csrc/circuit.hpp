// Host-side circuit representation shared by the executors.
#pragma once

#include <cuda_runtime.h>

#include <complex>
#include <memory>
#include <vector>

typedef unsigned long long ITYPE;
typedef unsigned int UINT;

namespace qs {

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
    void invalidate() {
        plan.reset();
        fused.reset();
        fused_dim = 0;
    }
};

int apply_gate_by_gate(const GateRec& g, void* state, ITYPE dim, cudaStream_t st);
int apply_gate_dm(const GateRec& g, void* rho, ITYPE dim, cudaStream_t st);
int run_staged(Circuit& c, void* state, ITYPE dim, cudaStream_t st);
int staged_pass_count(Circuit& c, ITYPE dim, UINT* out);

}  // namespace qs
