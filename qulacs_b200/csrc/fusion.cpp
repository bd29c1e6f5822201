// Host gate fusion for the executors: runs of gates whose qubits fit in k qubits are composed in
// FP64 into one dense k-qubit block.  The semantics are the reference's gate::merge
// (gate_merge.cpp:316-356: the later gate's matrix times the earlier one's, both expanded to the union
// of their qubits), computed with a plain dense product instead of Eigen.
#include <algorithm>
#include <cstring>

#include "circuit.hpp"
#include "../../include/qulacs_b200.h"

namespace qs {

using cd = std::complex<double>;

static ITYPE qubit_mask(const GateRec& g) {
    ITYPE m = 0;
    for (UINT q : g.qubits()) m |= 1ULL << q;
    return m;
}

void apply_gate_to_block(std::vector<cd>& U, int kb, const GateRec& g, const std::vector<int>& pos) {
    const int md = 1 << kb;
    const std::vector<cd> gm = g.dense_matrix();
    const int nt = (int)g.targets.size(), nc = (int)g.controls.size();
    const int gd = 1 << nt;
    int tmask = 0, cmask = 0, cval = 0;
    for (int j = 0; j < nt; ++j) tmask |= 1 << pos[j];
    for (int j = 0; j < nc; ++j) {
        cmask |= 1 << pos[nt + j];
        if (g.control_values[j]) cval |= 1 << pos[nt + j];
    }
    std::vector<int> off(gd, 0);
    for (int x = 0; x < gd; ++x)
        for (int j = 0; j < nt; ++j)
            if ((x >> j) & 1) off[x] |= 1 << pos[j];
    // plain real arithmetic: std::complex's operator* goes through the library's inf/nan-checking
    // routine, which dominated the cost of composing large blocks
    std::vector<double> tr(gd), ti(gd);
    for (int base = 0; base < md; ++base) {
        if ((base & tmask) || (base & cmask) != cval) continue;
        for (int col = 0; col < md; ++col) {
            for (int y = 0; y < gd; ++y) {
                double ar = 0., ai = 0.;
                for (int x = 0; x < gd; ++x) {
                    const cd m = gm[y * gd + x], u = U[(size_t)(base | off[x]) * md + col];
                    ar += m.real() * u.real() - m.imag() * u.imag();
                    ai += m.real() * u.imag() + m.imag() * u.real();
                }
                tr[y] = ar;
                ti[y] = ai;
            }
            for (int y = 0; y < gd; ++y) U[(size_t)(base | off[y]) * md + col] = cd(tr[y], ti[y]);
        }
    }
}

static bool fusable(const GateRec& g, int k) {
    return g.kind != QS_GATE_DEPOLARIZING && (int)g.qubits().size() <= k;
}

// One block -> one gate: the original gate when the block holds one, else a dense (or, when the
// product is diagonal on one qubit, a diagonal) gate on the block's qubits in ascending order.
static GateRec block_gate(const std::vector<GateRec>& G, ITYPE mask, const std::vector<int>& members) {
    if (members.size() == 1) return G[members[0]];
    std::vector<UINT> qs;
    for (UINT q = 0; q < 64; ++q)
        if ((mask >> q) & 1ULL) qs.push_back(q);
    const int kb = (int)qs.size(), md = 1 << kb;
    std::vector<cd> U((size_t)md * md, 0.);
    for (int i = 0; i < md; ++i) U[(size_t)i * md + i] = 1.;
    for (int gi : members) {
        std::vector<int> pos;
        for (UINT gq : G[gi].qubits()) pos.push_back((int)(std::find(qs.begin(), qs.end(), gq) - qs.begin()));
        apply_gate_to_block(U, kb, G[gi], pos);
    }
    GateRec r;
    r.targets = qs;
    bool diag = true;
    for (int y = 0; y < md && diag; ++y)
        for (int x = 0; x < md; ++x)
            if (x != y && U[(size_t)y * md + x] != cd(0.)) {
                diag = false;
                break;
            }
    if (diag && kb == 1) {
        r.kind = QS_GATE_DIAGONAL;
        r.matrix = {U[0], U[3]};
    } else {
        r.kind = QS_GATE_DENSE;
        r.matrix = U;
    }
    return r;
}

std::vector<GateRec> fuse_gates(const std::vector<GateRec>& G, int k) {
    if (k <= 0) return G;
    struct Block {
        ITYPE mask;
        std::vector<int> members;
    };
    std::vector<Block> open;  // pairwise disjoint qubit sets
    std::vector<GateRec> out;
    for (int i = 0; i < (int)G.size(); ++i) {
        const ITYPE gm = qubit_mask(G[i]);
        ITYPE um = gm;
        std::vector<size_t> touch;
        for (size_t j = 0; j < open.size(); ++j)
            if (open[j].mask & gm) {
                touch.push_back(j);
                um |= open[j].mask;
            }
        const bool fits = fusable(G[i], k) && __builtin_popcountll(um) <= k;
        Block merged{um, {}};
        for (size_t j : touch) {
            if (fits) merged.members.insert(merged.members.end(), open[j].members.begin(), open[j].members.end());
            else out.push_back(block_gate(G, open[j].mask, open[j].members));
        }
        for (size_t t = touch.size(); t-- > 0;) open.erase(open.begin() + (long)touch[t]);
        if (fits) {
            merged.members.push_back(i);
            open.push_back(merged);
        } else if (fusable(G[i], k)) {
            open.push_back({gm, {i}});
        } else {
            out.push_back(G[i]);
        }
    }
    for (const Block& b : open) out.push_back(block_gate(G, b.mask, b.members));
    return out;
}

}  // namespace qs
