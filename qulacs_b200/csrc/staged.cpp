// Staged executor (placeholder until the multi-gate pass kernel lands): gate by gate.
#include "circuit.hpp"

#include "../../include/qulacs_b200.h"

namespace qs {

struct StagedPlan {};

int run_staged(Circuit& c, void* state, ITYPE dim, cudaStream_t st) {
    for (const GateRec& g : c.gates) {
        int rc = apply_gate_by_gate(g, state, dim, st);
        if (rc != QS_OK) return rc;
    }
    return QS_OK;
}

int staged_pass_count(Circuit& c, ITYPE, UINT* out) {
    *out = (UINT)c.gates.size();
    return QS_OK;
}

}  // namespace qs
