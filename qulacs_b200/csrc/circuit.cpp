// Host-side circuit object: the gate list of cppsim's QuantumCircuit (cppsim/circuit.hpp) and its
// executors.  QS_EXEC_GATE_BY_GATE launches one kernel per gate, the reference's method
// (QuantumCircuit::update_quantum_state, circuit.cpp:46-57, dispatching each gate to its csim
// kernel).  QS_EXEC_STAGED hands the list to the pass scheduler (staged.cpp), which applies several
// gates per HBM pass with the same per-gate arithmetic.
#include "circuit.hpp"

#include <cmath>
#include <complex>
#include <string>
#include <vector>

#include "../../include/qulacs_b200.h"

namespace qs {
int set_error(int code, const std::string& msg);
}

using qs::Circuit;
using qs::GateRec;
using cd = std::complex<double>;

#define QS_TRY(expr)                 \
    do {                             \
        int _rc = (expr);            \
        if (_rc != QS_OK) return _rc; \
    } while (0)

namespace qs {

std::vector<UINT> GateRec::qubits() const {
    std::vector<UINT> q = targets;
    q.insert(q.end(), controls.begin(), controls.end());
    return q;
}

// Dense matrix of a gate on its targets (controls excluded), row-major, bit j <-> targets[j].
std::vector<cd> GateRec::dense_matrix() const {
    switch (kind) {
        case QS_GATE_DENSE: return matrix;
        case QS_GATE_DIAGONAL: {
            const size_t md = matrix.size();
            std::vector<cd> m(md * md, 0.);
            for (size_t i = 0; i < md; ++i) m[i * md + i] = matrix[i];
            return m;
        }
        case QS_GATE_RX: {
            const double c = std::cos(angle / 2), s = std::sin(angle / 2);
            return {c, cd(0, s), cd(0, s), c};
        }
        case QS_GATE_RY: {
            const double c = std::cos(angle / 2), s = std::sin(angle / 2);
            return {c, s, -s, c};
        }
        case QS_GATE_RZ: {
            const double c = std::cos(angle / 2), s = std::sin(angle / 2);
            return {cd(c, s), 0., 0., cd(c, -s)};
        }
        case QS_GATE_CNOT:  // targets = {control, target}: bit0 <-> control, bit1 <-> target
            return {1, 0, 0, 0, 0, 0, 0, 1, 0, 0, 1, 0, 0, 1, 0, 0};
        case QS_GATE_CZ: return {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, -1};
        case QS_GATE_SWAP: return {1, 0, 0, 0, 0, 0, 1, 0, 0, 1, 0, 0, 0, 0, 0, 1};
        default: break;
    }
    // Pauli string / rotation: build from the ids (targets in list order).
    const size_t k = targets.size(), md = size_t(1) << k;
    std::vector<cd> p(md * md, 0.);
    static const cd P[4][4] = {{1, 0, 0, 1}, {0, 1, 1, 0}, {0, cd(0, -1), cd(0, 1), 0}, {1, 0, 0, -1}};
    for (size_t y = 0; y < md; ++y)
        for (size_t x = 0; x < md; ++x) {
            cd v = 1.;
            for (size_t j = 0; j < k; ++j) v *= P[pauli_ids[j]][((y >> j) & 1) * 2 + ((x >> j) & 1)];
            p[y * md + x] = v;
        }
    if (kind == QS_GATE_PAULI) return p;
    // exp(i angle P / 2) = cos I + i sin P
    const double c = std::cos(angle / 2), s = std::sin(angle / 2);
    for (size_t i = 0; i < md * md; ++i) p[i] *= cd(0, s);
    for (size_t i = 0; i < md; ++i) p[i * md + i] += c;
    return p;
}

int apply_gate_by_gate(const GateRec& g, void* state, ITYPE dim, cudaStream_t st) {
    void* sp = (void*)st;
    const UINT* t = g.targets.data();
    const UINT nt = (UINT)g.targets.size();
    switch (g.kind) {
        case QS_GATE_RX: return qs_RX_gate(t[0], g.angle, state, dim, sp);
        case QS_GATE_RY: return qs_RY_gate(t[0], g.angle, state, dim, sp);
        case QS_GATE_RZ: return qs_RZ_gate(t[0], g.angle, state, dim, sp);
        case QS_GATE_CNOT: return qs_CNOT_gate(t[0], t[1], state, dim, sp);
        case QS_GATE_CZ: return qs_CZ_gate(t[0], t[1], state, dim, sp);
        case QS_GATE_SWAP: return qs_SWAP_gate(t[0], t[1], state, dim, sp);
        case QS_GATE_PAULI:
            return qs_multi_qubit_Pauli_gate_partial_list(t, g.pauli_ids.data(), nt, state, dim, sp);
        case QS_GATE_PAULI_ROTATION:
            return qs_multi_qubit_Pauli_rotation_gate_partial_list(t, g.pauli_ids.data(), nt, g.angle, state, dim, sp);
        case QS_GATE_DIAGONAL:
            if (nt == 1) return qs_single_qubit_diagonal_matrix_gate(t[0], (const double*)g.matrix.data(), state, dim, sp);
            return qs_multi_qubit_diagonal_matrix_gate(t, nt, (const double*)g.matrix.data(), state, dim, sp);
        case QS_GATE_DENSE: {
            const double* m = (const double*)g.matrix.data();
            if (g.controls.empty()) {
                if (nt == 1) return qs_single_qubit_dense_matrix_gate(t[0], m, state, dim, sp);
                if (nt == 2) return qs_double_qubit_dense_matrix_gate_c(t[0], t[1], m, state, dim, sp);
                return qs_multi_qubit_dense_matrix_gate(t, nt, m, state, dim, sp);
            }
            if (nt == 1)
                return qs_multi_qubit_control_single_qubit_dense_matrix_gate(g.controls.data(), g.control_values.data(),
                    (UINT)g.controls.size(), t[0], m, state, dim, sp);
            return qs_multi_qubit_control_multi_qubit_dense_matrix_gate(g.controls.data(), g.control_values.data(),
                (UINT)g.controls.size(), t, nt, m, state, dim, sp);
        }
        case QS_GATE_DEPOLARIZING:
            return set_error(QS_ERR_NOT_SUPPORTED,
                "depolarizing noise on a state vector needs a random branch; apply it to a density matrix");
        default: return set_error(QS_ERR_INVALID_ARGUMENT, "unknown gate kind");
    }
}

int apply_gate_dm(const GateRec& g, void* rho, ITYPE dim, cudaStream_t st) {
    void* sp = (void*)st;
    const UINT* t = g.targets.data();
    const UINT nt = (UINT)g.targets.size();
    switch (g.kind) {
        case QS_GATE_CNOT: return qs_dm_CNOT_gate(t[0], t[1], rho, dim, sp);
        case QS_GATE_CZ: return qs_dm_CZ_gate(t[0], t[1], rho, dim, sp);
        case QS_GATE_DEPOLARIZING:
            if (nt == 1) return qs_dm_depolarizing_noise(t[0], g.prob, rho, dim, sp);
            return qs_dm_two_qubit_depolarizing_noise(t[0], t[1], g.prob, rho, dim, sp);
        default: break;
    }
    if (!g.controls.empty()) {
        // controlled dense: expand to a matrix over targets + controls
        const std::vector<cd> u = g.dense_matrix();
        const UINT nc = (UINT)g.controls.size(), k = nt + nc;
        if (k > (UINT)kMaxDenseTargets)
            return set_error(QS_ERR_NOT_SUPPORTED, "density matrix: controlled gate over more than 12 qubits");
        const size_t md = size_t(1) << k, mt = size_t(1) << nt;
        std::vector<cd> full(md * md, 0.);
        size_t cmask = 0;
        for (UINT j = 0; j < nc; ++j)
            if (g.control_values[j]) cmask |= size_t(1) << (nt + j);
        for (size_t y = 0; y < md; ++y)
            for (size_t x = 0; x < md; ++x) {
                const bool active = ((y >> nt) << nt) == cmask;
                if ((y >> nt) != (x >> nt)) continue;
                if (active) full[y * md + x] = u[(y & (mt - 1)) * mt + (x & (mt - 1))];
                else if (y == x) full[y * md + x] = 1.;
            }
        std::vector<UINT> q = g.qubits();
        return qs_dm_multi_qubit_dense_matrix_gate(q.data(), k, (const double*)full.data(), rho, dim, sp);
    }
    const std::vector<cd> u = g.dense_matrix();
    return qs_dm_multi_qubit_dense_matrix_gate(t, nt, (const double*)u.data(), rho, dim, sp);
}

static GateRec shifted(const GateRec& g, UINT by) {
    GateRec r = g;
    for (UINT& t : r.targets) t += by;
    for (UINT& c : r.controls) c += by;
    return r;
}

// Kraus weights and operators of the reference's depolarizing channels (gate_factory.cpp:451-500):
// one qubit {1 - p: I, p/3: X, Z, Y}; two qubits {1 - p: I, p/15: each non-identity Pauli pair}.
static std::vector<cd> depolarizing_superoperator(UINT k, double p) {
    static const cd P[4][4] = {{1, 0, 0, 1}, {0, 1, 1, 0}, {0, cd(0, -1), cd(0, 1), 0}, {1, 0, 0, -1}};
    const size_t md = size_t(1) << k, sd = md * md;  // Kraus dim, superoperator dim
    const UINT nterms = k == 1 ? 4 : 16;
    std::vector<cd> S(sd * sd, 0.);
    for (UINT t = 0; t < nterms; ++t) {
        const double w = t == 0 ? 1. - p : p / (double)(nterms - 1);
        if (w == 0.) continue;
        std::vector<cd> K(md * md);
        for (size_t y = 0; y < md; ++y)
            for (size_t x = 0; x < md; ++x) {
                cd v = 1.;
                for (UINT j = 0; j < k; ++j) v *= P[(t >> (2 * j)) & 3][((y >> j) & 1) * 2 + ((x >> j) & 1)];
                K[y * md + x] = v;
            }
        // index = col + (row << k): S[(r, c), (r', c')] += w K[r][r'] conj(K[c][c'])
        for (size_t r = 0; r < md; ++r)
            for (size_t c = 0; c < md; ++c)
                for (size_t r2 = 0; r2 < md; ++r2)
                    for (size_t c2 = 0; c2 < md; ++c2)
                        S[(c + (r << k)) * sd + (c2 + (r2 << k))] += w * K[r * md + r2] * std::conj(K[c * md + c2]);
    }
    return S;
}

std::vector<GateRec> dm_vector_gates(const std::vector<GateRec>& G, UINT n) {
    std::vector<GateRec> out;
    for (const GateRec& g : G) {
        if (g.kind == QS_GATE_DEPOLARIZING) {
            const UINT k = (UINT)g.targets.size();
            GateRec s;
            s.kind = QS_GATE_DENSE;
            for (UINT t : g.targets) s.targets.push_back(t);
            for (UINT t : g.targets) s.targets.push_back(t + n);
            s.matrix = depolarizing_superoperator(k, g.prob);
            out.push_back(s);
            continue;
        }
        GateRec row = shifted(g, n), col = g;
        switch (g.kind) {
            case QS_GATE_RX:
            case QS_GATE_RZ: col.angle = -g.angle; break;  // conj(exp(i a P / 2)) = exp(-i a P / 2) for X, Z
            case QS_GATE_RY:
            case QS_GATE_CNOT:
            case QS_GATE_CZ:
            case QS_GATE_SWAP: break;  // real matrices
            case QS_GATE_DENSE:
            case QS_GATE_DIAGONAL:
                for (cd& v : col.matrix) v = std::conj(v);
                break;
            case QS_GATE_PAULI:
            case QS_GATE_PAULI_ROTATION: {
                // conj(P) = (-1)^{#Y} P
                UINT ny = 0;
                for (UINT id : g.pauli_ids) ny += id == 2 ? 1 : 0;
                if (g.kind == QS_GATE_PAULI_ROTATION) {
                    col.angle = (ny & 1) ? g.angle : -g.angle;
                } else if (ny & 1) {
                    GateRec sign;  // the global -1 of P (x) conj(P)
                    sign.kind = QS_GATE_DIAGONAL;
                    sign.targets = {g.targets[0]};
                    sign.matrix = {cd(-1.), cd(-1.)};
                    out.push_back(sign);
                }
                break;
            }
            default: break;
        }
        out.push_back(row);
        out.push_back(col);
    }
    return out;
}

}  // namespace qs

extern "C" {

QS_API int qs_circuit_create(QS_UINT qubit_count, qs_circuit_t* out) {
    if (!out) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null output pointer");
    if (qubit_count < 1 || qubit_count > 40) return qs::set_error(QS_ERR_NOT_SUPPORTED, "qubit count must be 1..40");
    Circuit* c = new Circuit();
    c->n = qubit_count;
    *out = reinterpret_cast<qs_circuit_t>(c);
    return QS_OK;
}

QS_API int qs_circuit_destroy(qs_circuit_t circuit) {
    delete reinterpret_cast<Circuit*>(circuit);
    return QS_OK;
}

QS_API int qs_circuit_add_gate(qs_circuit_t circuit, int kind, const QS_UINT* targets, QS_UINT nt,
    const QS_UINT* controls, const QS_UINT* control_values, QS_UINT nc, const double* params, QS_UINT np) {
    Circuit* c = reinterpret_cast<Circuit*>(circuit);
    if (!c) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null circuit");
    GateRec g;
    g.kind = kind;
    g.targets.assign(targets, targets + nt);
    if (nc) {
        g.controls.assign(controls, controls + nc);
        g.control_values.assign(control_values, control_values + nc);
    }
    // qubit checks (the reference throws on out-of-range or duplicated indices)
    std::vector<UINT> all = g.qubits();
    unsigned long long seen = 0;
    for (UINT q : all) {
        if (q >= c->n) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "gate qubit index >= circuit qubit count");
        if (seen & (1ULL << q)) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "gate has duplicated qubit indices");
        seen |= 1ULL << q;
    }
    for (UINT j = 0; j < nc; ++j)
        if (control_values[j] > 1) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "control value must be 0 or 1");
    auto need = [&](QS_UINT k) -> int {
        return np < k ? qs::set_error(QS_ERR_INVALID_ARGUMENT, "too few gate parameters") : QS_OK;
    };
    switch (kind) {
        case QS_GATE_DENSE: {
            if (nt < 1 || nt > (QS_UINT)qs::kMaxDenseTargets)
                return qs::set_error(QS_ERR_NOT_SUPPORTED, "dense gate: 1..12 targets");
            const size_t md = size_t(1) << nt;
            QS_TRY(need((QS_UINT)(2 * md * md)));
            g.matrix.resize(md * md);
            for (size_t i = 0; i < md * md; ++i) g.matrix[i] = cd(params[2 * i], params[2 * i + 1]);
            break;
        }
        case QS_GATE_DIAGONAL: {
            if (nt < 1 || nt > 20) return qs::set_error(QS_ERR_NOT_SUPPORTED, "diagonal gate: 1..20 targets");
            const size_t md = size_t(1) << nt;
            QS_TRY(need((QS_UINT)(2 * md)));
            g.matrix.resize(md);
            for (size_t i = 0; i < md; ++i) g.matrix[i] = cd(params[2 * i], params[2 * i + 1]);
            if (nc) return qs::set_error(QS_ERR_NOT_SUPPORTED, "controlled diagonal gate");
            break;
        }
        case QS_GATE_RX:
        case QS_GATE_RY:
        case QS_GATE_RZ:
            if (nt != 1 || nc) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "rotation gate takes one target");
            QS_TRY(need(1));
            g.angle = params[0];
            break;
        case QS_GATE_CNOT:
        case QS_GATE_CZ:
        case QS_GATE_SWAP:
            if (nt != 2 || nc) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "two-qubit named gate takes two qubits");
            break;
        case QS_GATE_PAULI:
        case QS_GATE_PAULI_ROTATION:
            if (nt < 1 || nc) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "Pauli gate needs targets");
            QS_TRY(need(kind == QS_GATE_PAULI ? nt : nt + 1));
            for (UINT j = 0; j < nt; ++j) {
                const double v = params[j];
                if (!(v == 0 || v == 1 || v == 2 || v == 3)) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "Pauli id must be 0..3");
                g.pauli_ids.push_back((UINT)v);
            }
            if (kind == QS_GATE_PAULI_ROTATION) g.angle = params[nt];
            break;
        case QS_GATE_DEPOLARIZING:
            if ((nt != 1 && nt != 2) || nc) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "depolarizing: 1 or 2 targets");
            QS_TRY(need(1));
            if (!(params[0] >= 0. && params[0] <= 1.)) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "probability outside [0, 1]");
            g.prob = params[0];
            break;
        default: return qs::set_error(QS_ERR_INVALID_ARGUMENT, "unknown gate kind");
    }
    c->gates.push_back(std::move(g));
    c->invalidate();
    return QS_OK;
}

QS_API int qs_circuit_gate_count(qs_circuit_t circuit, QS_UINT* out) {
    Circuit* c = reinterpret_cast<Circuit*>(circuit);
    if (!c || !out) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    *out = (QS_UINT)c->gates.size();
    return QS_OK;
}

QS_API int qs_circuit_update_quantum_state(qs_circuit_t circuit, void* state, QS_ITYPE dim, int mode, void* stream) {
    Circuit* c = reinterpret_cast<Circuit*>(circuit);
    if (!c) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null circuit");
    if (dim != (1ULL << c->n))
        return qs::set_error(QS_ERR_INVALID_ARGUMENT, "state dimension does not match the circuit's qubit count");
    if (mode == QS_EXEC_STAGED) return qs::run_staged(*c, state, dim, (cudaStream_t)stream);
    if (mode == QS_EXEC_STAGED_FUSED) return qs::run_staged_fused(*c, state, dim, (cudaStream_t)stream);
    if (mode != QS_EXEC_GATE_BY_GATE) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "unknown execution mode");
    for (const GateRec& g : c->gates) QS_TRY(qs::apply_gate_by_gate(g, state, dim, (cudaStream_t)stream));
    return QS_OK;
}

QS_API int qs_circuit_fuse(qs_circuit_t circuit, int k, qs_circuit_t* out) {
    Circuit* c = reinterpret_cast<Circuit*>(circuit);
    if (!c || !out) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    if (k < 0 || k > 6) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "fusion block size must be 0..6");
    Circuit* f = new (std::nothrow) Circuit();
    if (!f) return qs::set_error(QS_ERR_OUT_OF_MEMORY, "circuit");
    f->n = c->n;
    f->gates = qs::fuse_gates(c->gates, k);
    *out = reinterpret_cast<qs_circuit_t>(f);
    return QS_OK;
}

QS_API int qs_circuit_density_matrix_as_vector(qs_circuit_t circuit, qs_circuit_t* out) {
    Circuit* c = reinterpret_cast<Circuit*>(circuit);
    if (!c || !out) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    if (2 * c->n > 40) return qs::set_error(QS_ERR_NOT_SUPPORTED, "density matrix: at most 20 qubits");
    Circuit* v = new (std::nothrow) Circuit();
    if (!v) return qs::set_error(QS_ERR_OUT_OF_MEMORY, "circuit");
    v->n = 2 * c->n;
    v->gates = qs::dm_vector_gates(c->gates, c->n);
    *out = reinterpret_cast<qs_circuit_t>(v);
    return QS_OK;
}

QS_API int qs_circuit_gate_matrix(qs_circuit_t circuit, QS_UINT index, QS_UINT* qubits, QS_UINT* qubit_count,
    double* matrix) {
    Circuit* c = reinterpret_cast<Circuit*>(circuit);
    if (!c || !qubits || !qubit_count || !matrix) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    if (index >= c->gates.size()) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "gate index out of range");
    const GateRec& g = c->gates[index];
    if (g.kind == QS_GATE_DEPOLARIZING) return qs::set_error(QS_ERR_NOT_SUPPORTED, "noise channel has no unitary matrix");
    const std::vector<UINT> q = g.qubits();
    if (q.size() > 6) return qs::set_error(QS_ERR_NOT_SUPPORTED, "gate matrix export: at most 6 qubits");
    const int kb = (int)q.size(), md = 1 << kb;
    std::vector<cd> U((size_t)md * md, 0.);
    for (int i = 0; i < md; ++i) U[(size_t)i * md + i] = 1.;
    std::vector<int> pos(kb);
    for (int j = 0; j < kb; ++j) pos[j] = j;
    qs::apply_gate_to_block(U, kb, g, pos);
    for (int j = 0; j < kb; ++j) qubits[j] = q[j];
    *qubit_count = (QS_UINT)kb;
    for (size_t i = 0; i < U.size(); ++i) {
        matrix[2 * i] = U[i].real();
        matrix[2 * i + 1] = U[i].imag();
    }
    return QS_OK;
}

QS_API int qs_circuit_pass_count(qs_circuit_t circuit, QS_ITYPE dim, QS_UINT* out) {
    Circuit* c = reinterpret_cast<Circuit*>(circuit);
    if (!c || !out) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    return qs::staged_pass_count(*c, dim, out);
}

QS_API int qs_circuit_update_density_matrix(qs_circuit_t circuit, void* rho, QS_ITYPE dim, int mode, void* stream) {
    Circuit* c = reinterpret_cast<Circuit*>(circuit);
    if (!c) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null circuit");
    if (dim != (1ULL << c->n))
        return qs::set_error(QS_ERR_INVALID_ARGUMENT, "density matrix dimension does not match the circuit");
    if (mode == QS_EXEC_GATE_BY_GATE) {
        for (const GateRec& g : c->gates) QS_TRY(qs::apply_gate_dm(g, rho, dim, (cudaStream_t)stream));
        return QS_OK;
    }
    if (mode != QS_EXEC_STAGED && mode != QS_EXEC_STAGED_FUSED)
        return qs::set_error(QS_ERR_INVALID_ARGUMENT, "unknown execution mode");
    if (2 * c->n > 40) return qs::set_error(QS_ERR_NOT_SUPPORTED, "density matrix: at most 20 qubits");
    if (!c->dm_vec) {
        auto v = std::make_shared<Circuit>();
        v->n = 2 * c->n;
        v->gates = qs::dm_vector_gates(c->gates, c->n);
        v->fusion_k = c->fusion_k;
        c->dm_vec = v;
    }
    if (mode == QS_EXEC_STAGED) return qs::run_staged(*c->dm_vec, rho, dim * dim, (cudaStream_t)stream);
    return qs::run_staged_fused(*c->dm_vec, rho, dim * dim, (cudaStream_t)stream);
}

}  // extern "C"
