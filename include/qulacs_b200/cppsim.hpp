// cppsim.hpp -- header-only C++ surface over the qulacs_b200 C ABI.
//
// Mirrors the reference's cppsim classes that sit on the state-update path, so C++ code written
// against them needs only this header and libqulacs_b200.so:
//   QuantumState         (cppsim/state.hpp:419-1006; device-resident, get_device_name() == "gpu")
//   DensityMatrix        (cppsim/state_dm.hpp)
//   QuantumGateBase and the gate:: factory (cppsim/gate.hpp:83-310, cppsim/gate_factory.cpp)
//   QuantumCircuit       (cppsim/circuit.hpp; update_quantum_state as circuit.cpp:46-57)
//   PauliOperator, Observable (cppsim/pauli_operator.cpp, cppsim/general_quantum_operator.cpp)
// Ownership follows the reference: gate:: factories return raw new'd pointers owned by the caller;
// QuantumCircuit::add_gate takes ownership, add_gate_copy copies.  Errors are thrown as std
// exceptions (the reference throws typed std:: exceptions, cppsim/exception.hpp).
#pragma once

#include <cmath>
#include <complex>
#include <cstdint>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../qulacs_b200.h"

namespace qulacs_b200 {

using CPPCTYPE = std::complex<double>;
using ComplexVector = std::vector<CPPCTYPE>;
using UINT = QS_UINT;
using ITYPE = QS_ITYPE;

inline void check(int rc, const char* what) {
    if (rc == QS_OK) return;
    const std::string msg = std::string(what) + ": " + qs_get_last_error();
    switch (rc) {
        case QS_ERR_INVALID_ARGUMENT: throw std::invalid_argument(msg);
        case QS_ERR_OUT_OF_MEMORY: throw std::bad_alloc();
        case QS_ERR_NOT_SUPPORTED: throw std::domain_error(msg);
        default: throw std::runtime_error(msg);
    }
}

// ------------------------------------------------------------------ states
class QuantumStateBase {
public:
    const UINT qubit_count;
    const ITYPE dim;
    explicit QuantumStateBase(UINT n, ITYPE d) : qubit_count(n), dim(d) {}
    virtual ~QuantumStateBase() = default;
    virtual bool is_state_vector() const = 0;
    virtual void* data() const = 0;
    virtual void* get_cuda_stream() const { return stream_; }
    virtual std::string get_device_name() const { return "gpu"; }
    virtual void set_zero_state() = 0;
    virtual double get_squared_norm() const = 0;

protected:
    void* stream_ = nullptr;
};

class QuantumState : public QuantumStateBase {
public:
    explicit QuantumState(UINT qubit_count, void* stream = nullptr)
        : QuantumStateBase(qubit_count, ITYPE(1) << qubit_count) {
        stream_ = stream;
        check(qs_allocate_quantum_state(dim, &ptr_), "QuantumState");
        set_zero_state();
    }
    ~QuantumState() override { qs_release_quantum_state(ptr_); }
    QuantumState(const QuantumState&) = delete;
    QuantumState& operator=(const QuantumState&) = delete;

    bool is_state_vector() const override { return true; }
    void* data() const override { return ptr_; }
    void set_zero_state() override { check(qs_initialize_quantum_state(ptr_, dim, stream_), "set_zero_state"); }
    void set_computational_basis(ITYPE basis) {
        check(qs_set_computational_basis(basis, ptr_, dim, stream_), "set_computational_basis");
    }
    void load(const ComplexVector& v) {
        if (v.size() != dim) throw std::invalid_argument("load: vector size differs from dim");
        check(qs_load_state(v.data(), ptr_, dim, stream_), "load");
        check(qs_stream_synchronize(stream_), "load");
    }
    void load(const QuantumState& other) {
        if (other.dim != dim) throw std::invalid_argument("load: dimension mismatch");
        load(other.get_vector());
    }
    ComplexVector get_vector() const {
        ComplexVector v(dim);
        check(qs_get_state(ptr_, v.data(), dim, stream_), "get_vector");
        return v;
    }
    QuantumState* copy() const {
        auto* s = new QuantumState(qubit_count, stream_);
        s->load(*this);
        return s;
    }
    double get_squared_norm() const override {
        double out = 0;
        check(qs_state_norm_squared(ptr_, dim, stream_, &out), "get_squared_norm");
        return out;
    }
    double get_zero_probability(UINT target) const {
        double out = 0;
        check(qs_M0_prob(target, ptr_, dim, stream_, &out), "get_zero_probability");
        return out;
    }
    // measured_values[i] in {0, 1, 2}; 2 = not measured (cppsim QuantumStateBase::get_marginal_probability)
    double get_marginal_probability(const std::vector<UINT>& measured_values) const {
        std::vector<UINT> tl, vals;
        for (UINT i = 0; i < measured_values.size(); ++i)
            if (measured_values[i] <= 1) {
                tl.push_back(i);
                vals.push_back(measured_values[i]);
            }
        double out = 0;
        check(qs_marginal_prob(tl.data(), vals.data(), (UINT)tl.size(), ptr_, dim, stream_, &out),
            "get_marginal_probability");
        return out;
    }
    // cppsim/state.hpp:899-992: mt19937_64(seed) uniforms, lower_bound over the FP64 prefix sums
    std::vector<ITYPE> sampling(UINT count, UINT seed) const {
        std::vector<ITYPE> out(count);
        check(qs_state_sampling(ptr_, dim, count, seed, out.data(), stream_), "sampling");
        return out;
    }
    std::vector<ITYPE> sampling_with_uniforms(const std::vector<double>& uniforms) const {
        std::vector<ITYPE> out(uniforms.size());
        check(qs_state_sampling_with_uniforms(ptr_, dim, uniforms.data(), (UINT)uniforms.size(), out.data(), stream_),
            "sampling_with_uniforms");
        return out;
    }

private:
    void* ptr_ = nullptr;
};

inline CPPCTYPE inner_product(const QuantumState& bra, const QuantumState& ket) {
    double out[2];
    check(qs_state_inner_product(bra.data(), ket.data(), bra.dim, bra.get_cuda_stream(), out), "inner_product");
    return {out[0], out[1]};
}

// cppsim state::tensor_product / permutate_qubit / drop_qubit (cppsim/state.cpp; csim stat_ops.cpp:111-158):
// new states the caller owns, as cppsim's return raw new'd pointers.
namespace state {
inline CPPCTYPE inner_product(const QuantumState& bra, const QuantumState& ket) { return qulacs_b200::inner_product(bra, ket); }
// The result is held by a unique_ptr until the C call succeeds, so a rejected call frees its device memory.
inline QuantumState* tensor_product(const QuantumState& left, const QuantumState& right) {
    std::unique_ptr<QuantumState> out(new QuantumState(left.qubit_count + right.qubit_count, left.get_cuda_stream()));
    if (right.get_cuda_stream() != left.get_cuda_stream())  // the right state's last writes must be done
        check(qs_stream_synchronize(right.get_cuda_stream()), "tensor_product");
    check(qs_state_tensor_product(left.data(), left.dim, right.data(), right.dim, out->data(), left.get_cuda_stream()),
        "tensor_product");
    return out.release();
}
inline QuantumState* permutate_qubit(const QuantumState& src, const std::vector<UINT>& qubit_order) {
    if (qubit_order.size() != src.qubit_count)  // cppsim/state.cpp: the order lists every qubit
        throw std::invalid_argument("permutate_qubit: qubit_order must list every qubit once");
    std::unique_ptr<QuantumState> out(new QuantumState(src.qubit_count, src.get_cuda_stream()));
    check(qs_state_permutate_qubit(qubit_order.data(), src.data(), out->data(), (UINT)qubit_order.size(), src.dim,
              src.get_cuda_stream()),
        "permutate_qubit");
    return out.release();
}
inline QuantumState* drop_qubit(const QuantumState& src, const std::vector<UINT>& target,
    const std::vector<UINT>& projection) {
    if (target.size() != projection.size()) throw std::invalid_argument("drop_qubit: size mismatch");
    if (target.size() >= src.qubit_count)  // cppsim/state.cpp:70: at least one qubit must remain
        throw std::invalid_argument("drop_qubit: cannot drop every qubit");
    std::unique_ptr<QuantumState> out(new QuantumState(src.qubit_count - (UINT)target.size(), src.get_cuda_stream()));
    check(qs_state_drop_qubits(target.data(), projection.data(), (UINT)target.size(), src.data(), out->data(), src.dim,
              src.get_cuda_stream()),
        "drop_qubit");
    return out.release();
}
}  // namespace state

class DensityMatrix : public QuantumStateBase {
public:
    explicit DensityMatrix(UINT qubit_count, void* stream = nullptr)
        : QuantumStateBase(qubit_count, ITYPE(1) << qubit_count) {
        stream_ = stream;
        check(qs_dm_allocate(dim, &ptr_), "DensityMatrix");
        set_zero_state();
    }
    ~DensityMatrix() override { qs_release_quantum_state(ptr_); }
    DensityMatrix(const DensityMatrix&) = delete;
    DensityMatrix& operator=(const DensityMatrix&) = delete;

    bool is_state_vector() const override { return false; }
    void* data() const override { return ptr_; }
    void set_zero_state() override { check(qs_dm_initialize_quantum_state(ptr_, dim, stream_), "set_zero_state"); }
    void load(const QuantumState& pure) {
        check(qs_dm_initialize_with_pure_state(ptr_, pure.data(), dim, stream_), "load");
    }
    ComplexVector get_matrix() const {  // row-major dim x dim
        ComplexVector v(dim * dim);
        check(qs_get_state(ptr_, v.data(), dim * dim, stream_), "get_matrix");
        return v;
    }
    double get_squared_norm() const override {  // trace, as the reference's density-matrix norm
        double out = 0;
        check(qs_dm_state_norm_squared(ptr_, dim, stream_, &out), "get_squared_norm");
        return out;
    }

private:
    void* ptr_ = nullptr;
};

// ------------------------------------------------------------------ gates
class QuantumGateBase {
public:
    QuantumGateBase(int kind, std::vector<UINT> targets, std::vector<double> params, std::string name)
        : kind_(kind), targets_(std::move(targets)), params_(std::move(params)), name_(std::move(name)) {}
    virtual ~QuantumGateBase() = default;
    std::vector<UINT> get_target_index_list() const { return targets_; }
    std::vector<UINT> get_control_index_list() const { return controls_; }
    std::string get_name() const { return name_; }
    QuantumGateBase* copy() const { return new QuantumGateBase(*this); }
    void add_control_qubit(UINT qubit, UINT value) {
        if (kind_ != QS_GATE_DENSE) throw std::domain_error("add_control_qubit: DenseMatrix gates only");
        controls_.push_back(qubit);
        control_values_.push_back(value);
    }
    // Adds this gate to a C-ABI circuit handle.
    void add_to(qs_circuit_t c) const {
        check(qs_circuit_add_gate(c, kind_, targets_.data(), (UINT)targets_.size(), controls_.data(),
                  control_values_.data(), (UINT)controls_.size(), params_.data(), (UINT)params_.size()),
            "add_gate");
    }
    // cppsim QuantumGateBase::update_quantum_state (gate.hpp:159): state vector or density matrix.
    // One csim-named C-ABI call per gate (the reference's gate classes call csim the same way,
    // gate_named_one.hpp:41-63, gate_matrix.cpp:69-332); no circuit object is built.
    void update_quantum_state(QuantumStateBase* state) const {
        if (state->is_state_vector()) check(apply_state_vector(state->data(), state->dim, state->get_cuda_stream()),
                                          "update_quantum_state");
        else check(apply_density_matrix(state->data(), state->dim, state->get_cuda_stream()), "update_quantum_state");
    }

private:
    std::vector<UINT> pauli_ids() const {
        std::vector<UINT> ids;
        for (size_t i = 0; i < targets_.size(); ++i) ids.push_back((UINT)params_[i]);
        return ids;
    }
    int apply_state_vector(void* s, ITYPE dim, void* st) const {
        const UINT* t = targets_.data();
        const UINT nt = (UINT)targets_.size();
        const double* m = params_.data();
        switch (kind_) {
            case QS_GATE_RX: return qs_RX_gate(t[0], params_[0], s, dim, st);
            case QS_GATE_RY: return qs_RY_gate(t[0], params_[0], s, dim, st);
            case QS_GATE_RZ: return qs_RZ_gate(t[0], params_[0], s, dim, st);
            case QS_GATE_CNOT: return qs_CNOT_gate(t[0], t[1], s, dim, st);
            case QS_GATE_CZ: return qs_CZ_gate(t[0], t[1], s, dim, st);
            case QS_GATE_SWAP: return qs_SWAP_gate(t[0], t[1], s, dim, st);
            case QS_GATE_PAULI: {
                const std::vector<UINT> ids = pauli_ids();
                return qs_multi_qubit_Pauli_gate_partial_list(t, ids.data(), nt, s, dim, st);
            }
            case QS_GATE_PAULI_ROTATION: {
                const std::vector<UINT> ids = pauli_ids();
                return qs_multi_qubit_Pauli_rotation_gate_partial_list(t, ids.data(), nt, params_[nt], s, dim, st);
            }
            case QS_GATE_DIAGONAL:
                if (nt == 1) return qs_single_qubit_diagonal_matrix_gate(t[0], m, s, dim, st);
                return qs_multi_qubit_diagonal_matrix_gate(t, nt, m, s, dim, st);
            case QS_GATE_DENSE:
                if (controls_.empty()) {
                    if (nt == 1) return qs_single_qubit_dense_matrix_gate(t[0], m, s, dim, st);
                    if (nt == 2) return qs_double_qubit_dense_matrix_gate_c(t[0], t[1], m, s, dim, st);
                    return qs_multi_qubit_dense_matrix_gate(t, nt, m, s, dim, st);
                }
                if (nt == 1)
                    return qs_multi_qubit_control_single_qubit_dense_matrix_gate(controls_.data(), control_values_.data(),
                        (UINT)controls_.size(), t[0], m, s, dim, st);
                return qs_multi_qubit_control_multi_qubit_dense_matrix_gate(controls_.data(), control_values_.data(),
                    (UINT)controls_.size(), t, nt, m, s, dim, st);
            default: return via_circuit(s, dim, st, true);  // depolarizing: the circuit path reports the error
        }
    }
    int apply_density_matrix(void* r, ITYPE dim, void* st) const {
        const UINT* t = targets_.data();
        const UINT nt = (UINT)targets_.size();
        switch (kind_) {
            case QS_GATE_RX: return qs_dm_RX_gate(t[0], params_[0], r, dim, st);
            case QS_GATE_RY: return qs_dm_RY_gate(t[0], params_[0], r, dim, st);
            case QS_GATE_RZ: return qs_dm_RZ_gate(t[0], params_[0], r, dim, st);
            case QS_GATE_CNOT: return qs_dm_CNOT_gate(t[0], t[1], r, dim, st);
            case QS_GATE_CZ: return qs_dm_CZ_gate(t[0], t[1], r, dim, st);
            case QS_GATE_SWAP: return qs_dm_SWAP_gate(t[0], t[1], r, dim, st);
            case QS_GATE_PAULI: {
                const std::vector<UINT> ids = pauli_ids();
                return qs_dm_multi_qubit_Pauli_gate_partial_list(t, ids.data(), nt, r, dim, st);
            }
            case QS_GATE_PAULI_ROTATION: {
                const std::vector<UINT> ids = pauli_ids();
                return qs_dm_multi_qubit_Pauli_rotation_gate_partial_list(t, ids.data(), nt, params_[nt], r, dim, st);
            }
            case QS_GATE_DEPOLARIZING:
                if (nt == 1) return qs_dm_depolarizing_noise(t[0], params_[0], r, dim, st);
                return qs_dm_two_qubit_depolarizing_noise(t[0], t[1], params_[0], r, dim, st);
            case QS_GATE_DENSE:
                if (controls_.empty()) {
                    if (nt == 1) return qs_dm_single_qubit_dense_matrix_gate(t[0], params_.data(), r, dim, st);
                    return qs_dm_multi_qubit_dense_matrix_gate(t, nt, params_.data(), r, dim, st);
                }
                return qs_dm_multi_qubit_control_multi_qubit_dense_matrix_gate(controls_.data(), control_values_.data(),
                    (UINT)controls_.size(), t, nt, params_.data(), r, dim, st);
            default: return via_circuit(r, dim, st, false);  // diagonal gates: expanded by the circuit path
        }
    }
    int via_circuit(void* s, ITYPE dim, void* st, bool vector) const {
        UINT n = 0;
        while ((ITYPE(1) << n) < dim) ++n;
        qs_circuit_t c = nullptr;
        int rc = qs_circuit_create(n, &c);
        if (rc != QS_OK) return rc;
        std::unique_ptr<void, void (*)(void*)> guard(c, [](void* p) { qs_circuit_destroy((qs_circuit_t)p); });
        rc = qs_circuit_add_gate(c, kind_, targets_.data(), (UINT)targets_.size(), controls_.data(),
            control_values_.data(), (UINT)controls_.size(), params_.data(), (UINT)params_.size());
        if (rc != QS_OK) return rc;
        return vector ? qs_circuit_update_quantum_state(c, s, dim, QS_EXEC_GATE_BY_GATE, st)
                      : qs_circuit_update_density_matrix(c, s, dim, QS_EXEC_GATE_BY_GATE, st);
    }

    int kind_;
    std::vector<UINT> targets_, controls_, control_values_;
    std::vector<double> params_;
    std::string name_;
};

using QuantumGateMatrix = QuantumGateBase;

namespace gate {
inline std::vector<double> flat(const ComplexVector& m) {
    std::vector<double> p(2 * m.size());
    for (size_t i = 0; i < m.size(); ++i) {
        p[2 * i] = m[i].real();
        p[2 * i + 1] = m[i].imag();
    }
    return p;
}
// row-major matrix; bit j of the index <-> targets[j]
inline QuantumGateBase* DenseMatrix(const std::vector<UINT>& targets, const ComplexVector& matrix) {
    const size_t md = size_t(1) << targets.size();
    if (matrix.size() != md * md) throw std::invalid_argument("DenseMatrix: matrix size");
    return new QuantumGateBase(QS_GATE_DENSE, targets, flat(matrix), "DenseMatrix");
}
inline QuantumGateBase* DenseMatrix(UINT t, const ComplexVector& m) { return DenseMatrix(std::vector<UINT>{t}, m); }
inline QuantumGateBase* DiagonalMatrix(const std::vector<UINT>& targets, const ComplexVector& diag) {
    if (diag.size() != (size_t(1) << targets.size())) throw std::invalid_argument("DiagonalMatrix: size");
    return new QuantumGateBase(QS_GATE_DIAGONAL, targets, flat(diag), "DiagonalMatrix");
}
// named gates: csim/constant.cpp:4-30
inline QuantumGateBase* X(UINT t) { return DenseMatrix(t, {0, 1, 1, 0}); }
inline QuantumGateBase* Y(UINT t) { return DenseMatrix(t, {0, CPPCTYPE(0, -1), CPPCTYPE(0, 1), 0}); }
inline QuantumGateBase* Z(UINT t) { return DiagonalMatrix({t}, {1, -1}); }
inline QuantumGateBase* H(UINT t) {
    const double h = 1.0 / std::sqrt(2.0);
    return DenseMatrix(t, {h, h, h, -h});
}
inline QuantumGateBase* S(UINT t) { return DiagonalMatrix({t}, {1, CPPCTYPE(0, 1)}); }
inline QuantumGateBase* Sdag(UINT t) { return DiagonalMatrix({t}, {1, CPPCTYPE(0, -1)}); }
inline QuantumGateBase* T(UINT t) { return DiagonalMatrix({t}, {1, CPPCTYPE(1, 1) / std::sqrt(2.0)}); }
inline QuantumGateBase* Tdag(UINT t) { return DiagonalMatrix({t}, {1, CPPCTYPE(1, -1) / std::sqrt(2.0)}); }
// exp(+i angle P / 2) (csim/update_ops_pauli_single.cpp:54-120); RotX = RX(-angle) (gate_factory.cpp:152-163)
inline QuantumGateBase* RX(UINT t, double a) { return new QuantumGateBase(QS_GATE_RX, {t}, {a}, "X-rotation"); }
inline QuantumGateBase* RY(UINT t, double a) { return new QuantumGateBase(QS_GATE_RY, {t}, {a}, "Y-rotation"); }
inline QuantumGateBase* RZ(UINT t, double a) { return new QuantumGateBase(QS_GATE_RZ, {t}, {a}, "Z-rotation"); }
inline QuantumGateBase* RotX(UINT t, double a) { return RX(t, -a); }
inline QuantumGateBase* RotY(UINT t, double a) { return RY(t, -a); }
inline QuantumGateBase* RotZ(UINT t, double a) { return RZ(t, -a); }
// cppsim get_IBMQ_matrix (gate_factory.cpp:165-179)
inline QuantumGateBase* U3(UINT t, double theta, double phi, double lambda) {
    const CPPCTYPE e1 = std::exp(CPPCTYPE(0, phi)), e2 = std::exp(CPPCTYPE(0, lambda));
    const double c = std::cos(theta / 2), s = std::sin(theta / 2);
    return DenseMatrix(t, {c, -e2 * s, e1 * s, e1 * e2 * c});
}
inline QuantumGateBase* CNOT(UINT control, UINT target) {
    if (control == target) throw std::invalid_argument("CNOT: control and target are the same qubit");
    return new QuantumGateBase(QS_GATE_CNOT, {control, target}, {}, "CNOT");
}
inline QuantumGateBase* CZ(UINT control, UINT target) {
    if (control == target) throw std::invalid_argument("CZ: control and target are the same qubit");
    return new QuantumGateBase(QS_GATE_CZ, {control, target}, {}, "CZ");
}
inline QuantumGateBase* SWAP(UINT a, UINT b) {
    if (a == b) throw std::invalid_argument("SWAP: duplicated qubit");
    return new QuantumGateBase(QS_GATE_SWAP, {a, b}, {}, "SWAP");
}
inline QuantumGateBase* Pauli(const std::vector<UINT>& targets, const std::vector<UINT>& ids) {
    return new QuantumGateBase(QS_GATE_PAULI, targets, std::vector<double>(ids.begin(), ids.end()), "Pauli");
}
inline QuantumGateBase* PauliRotation(const std::vector<UINT>& targets, const std::vector<UINT>& ids, double a) {
    std::vector<double> p(ids.begin(), ids.end());
    p.push_back(a);
    return new QuantumGateBase(QS_GATE_PAULI_ROTATION, targets, p, "PauliRotation");
}
// exact channels on a DensityMatrix (gate_factory.cpp:451-500)
inline QuantumGateBase* DepolarizingNoise(UINT t, double p) {
    return new QuantumGateBase(QS_GATE_DEPOLARIZING, {t}, {p}, "DepolarizingNoise");
}
inline QuantumGateBase* TwoQubitDepolarizingNoise(UINT t1, UINT t2, double p) {
    if (t1 == t2) throw std::invalid_argument("TwoQubitDepolarizingNoise: duplicated qubit");
    return new QuantumGateBase(QS_GATE_DEPOLARIZING, {t1, t2}, {p}, "TwoQubitDepolarizingNoise");
}
}  // namespace gate

// ------------------------------------------------------------------ circuit
class QuantumCircuit {
public:
    explicit QuantumCircuit(UINT qubit_count) : qubit_count(qubit_count) {
        check(qs_circuit_create(qubit_count, &h_), "QuantumCircuit");
    }
    ~QuantumCircuit() {
        for (auto* g : gate_list) delete g;
        qs_circuit_destroy(h_);
    }
    QuantumCircuit(const QuantumCircuit&) = delete;
    QuantumCircuit& operator=(const QuantumCircuit&) = delete;

    const UINT qubit_count;
    std::vector<QuantumGateBase*> gate_list;

    void add_gate(QuantumGateBase* g) {  // takes ownership (circuit.hpp:72-100)
        g->add_to(h_);
        gate_list.push_back(g);
    }
    void add_gate_copy(const QuantumGateBase* g) { add_gate(g->copy()); }
    void add_noise_gate(QuantumGateBase* g, const std::string& noise_type, double p) {  // circuit.cpp:167-190
        if (noise_type != "Depolarizing") throw std::domain_error("add_noise_gate: " + noise_type);
        std::vector<UINT> q = g->get_target_index_list();
        for (UINT c : g->get_control_index_list()) q.push_back(c);
        add_gate(g);
        if (q.size() == 1) add_gate(gate::DepolarizingNoise(q[0], p));
        else if (q.size() == 2) add_gate(gate::TwoQubitDepolarizingNoise(q[0], q[1], p));
        else throw std::invalid_argument("add_noise_gate: depolarizing noise can be used up to 2 qubits");
    }
    UINT get_gate_count() const { return (UINT)gate_list.size(); }
    qs_circuit_t handle() const { return h_; }
    // block size of QS_EXEC_STAGED_FUSED: 0..6, or -1 (default) for the autotuner's choice
    void set_fusion(int k) { check(qs_circuit_set_fusion(h_, k), "set_fusion"); }
    // exec_mode: QS_EXEC_STAGED (default), QS_EXEC_STAGED_FUSED (FP64 k-qubit fusion, autotuned k) or
    // QS_EXEC_GATE_BY_GATE
    void update_quantum_state(QuantumStateBase* state, int exec_mode = QS_EXEC_STAGED) {
        if (state->qubit_count != qubit_count)
            throw std::invalid_argument("update_quantum_state: qubit count differs");
        if (state->is_state_vector())
            check(qs_circuit_update_quantum_state(h_, state->data(), state->dim, exec_mode, state->get_cuda_stream()),
                "update_quantum_state");
        else
            check(qs_circuit_update_density_matrix(h_, state->data(), state->dim, exec_mode, state->get_cuda_stream()),
                "update_quantum_state");
    }

private:
    qs_circuit_t h_ = nullptr;
};

// ------------------------------------------------------------------ noisy sampling
// cppsim NoiseSimulator (noisesimulator.hpp): trajectories drawn as the reference draws them, distinct
// ones simulated once on the device.  The reference seeds from std::random_device; here the seed is
// an argument (reproducible runs).
class NoiseSimulator {
public:
    struct Result {
        std::vector<std::pair<QuantumState*, UINT>> result;
        Result() = default;
        Result(const Result&) = delete;
        Result& operator=(const Result&) = delete;
        ~Result() {
            for (auto& p : result) delete p.first;
        }
        std::vector<ITYPE> sampling(UINT seed = 0) const {
            std::vector<ITYPE> out;
            UINT i = 0;
            for (const auto& p : result) {
                const std::vector<ITYPE> s = p.first->sampling(p.second, seed + i++);
                out.insert(out.end(), s.begin(), s.end());
            }
            return out;
        }
    };

    explicit NoiseSimulator(const QuantumCircuit* circuit, const QuantumState* init_state = nullptr, UINT seed = 0)
        : circuit_(circuit), init_(init_state), seed_(seed) {}

    std::vector<ITYPE> execute(UINT sample_count) {
        std::vector<ITYPE> out(sample_count);
        check(qs_noise_simulator_execute(circuit_->handle(), init_ ? init_->data() : nullptr,
                  ITYPE(1) << circuit_->qubit_count, sample_count, seed_, out.data(), nullptr, stream()),
            "NoiseSimulator::execute");
        return out;
    }
    // caller deletes the result (as the reference's execute_and_get_result)
    Result* execute_and_get_result(UINT execution_count) {
        UINT count = 0;
        check(qs_noise_simulator_trajectories(circuit_->handle(), execution_count, seed_, &count, nullptr),
            "NoiseSimulator::execute_and_get_result");
        std::vector<UINT> shots(count);
        check(qs_noise_simulator_trajectories(circuit_->handle(), execution_count, seed_, &count, shots.data()),
            "NoiseSimulator::execute_and_get_result");
        auto* r = new Result();
        std::vector<void*> ptrs;
        for (UINT i = 0; i < count; ++i) {
            r->result.push_back({new QuantumState(circuit_->qubit_count, stream()), shots[i]});
            ptrs.push_back(r->result.back().first->data());
        }
        const int rc = qs_noise_simulator_execute(circuit_->handle(), init_ ? init_->data() : nullptr,
            ITYPE(1) << circuit_->qubit_count, execution_count, seed_, nullptr, ptrs.data(), stream());
        if (rc != QS_OK) {
            delete r;
            check(rc, "NoiseSimulator::execute_and_get_result");
        }
        return r;
    }

private:
    void* stream() const { return init_ ? init_->get_cuda_stream() : nullptr; }
    const QuantumCircuit* circuit_;
    const QuantumState* init_;
    UINT seed_;
};

// ------------------------------------------------------------------ operators
class PauliOperator {
public:
    // "X 0 Y 3 Z 5" (pauli_operator.cpp)
    explicit PauliOperator(const std::string& s, CPPCTYPE coef = 1.0) : coef_(coef) {
        std::istringstream is(s);
        std::string p;
        UINT q;
        while (is >> p >> q) {
            const char c = (char)std::toupper(p[0]);
            const UINT id = c == 'I' ? 0 : c == 'X' ? 1 : c == 'Y' ? 2 : c == 'Z' ? 3 : 4;
            if (id == 4) throw std::invalid_argument("PauliOperator: bad Pauli symbol " + p);
            targets_.push_back(q);
            ids_.push_back(id);
        }
    }
    PauliOperator(std::vector<UINT> targets, std::vector<UINT> ids, CPPCTYPE coef = 1.0)
        : targets_(std::move(targets)), ids_(std::move(ids)), coef_(coef) {}
    CPPCTYPE get_coef() const { return coef_; }
    const std::vector<UINT>& get_index_list() const { return targets_; }
    const std::vector<UINT>& get_pauli_id_list() const { return ids_; }
    // coef * <P> (pauli_operator.cpp:132-183)
    CPPCTYPE get_expectation_value(const QuantumStateBase* state) const {
        double v = 0;
        if (state->is_state_vector())
            check(qs_expectation_value_multi_qubit_Pauli_operator_partial_list(targets_.data(), ids_.data(),
                      (UINT)targets_.size(), state->data(), state->dim, state->get_cuda_stream(), &v),
                "get_expectation_value");
        else
            check(qs_dm_expectation_value_multi_qubit_Pauli_operator_partial_list(targets_.data(), ids_.data(),
                      (UINT)targets_.size(), state->data(), state->dim, state->get_cuda_stream(), &v),
                "get_expectation_value");
        return coef_ * v;
    }
    void masks(ITYPE* x, ITYPE* z, UINT* ny) const {  // csim/utility.cpp:12-43
        *x = *z = 0;
        *ny = 0;
        for (size_t i = 0; i < targets_.size(); ++i) {
            const ITYPE b = ITYPE(1) << targets_[i];
            if (ids_[i] == 1) *x ^= b;
            else if (ids_[i] == 2) { *x ^= b; *z ^= b; ++*ny; }
            else if (ids_[i] == 3) *z ^= b;
        }
    }

private:
    std::vector<UINT> targets_, ids_;
    CPPCTYPE coef_;
};

class Observable {
public:
    explicit Observable(UINT qubit_count) : qubit_count_(qubit_count) {}
    void add_operator(const PauliOperator& op) { terms_.push_back(op); }
    void add_operator(CPPCTYPE coef, const std::string& s) { terms_.emplace_back(s, coef); }
    UINT get_term_count() const { return (UINT)terms_.size(); }
    // sum_k coef_k <P_k>, all terms in one batched device call for a state vector
    // (general_quantum_operator.cpp:105-141)
    double get_expectation_value(const QuantumStateBase* state) const {
        const UINT k = (UINT)terms_.size();
        if (k == 0) return 0.;
        if (!state->is_state_vector()) {
            CPPCTYPE s = 0;
            for (const auto& t : terms_) s += t.get_expectation_value(state);
            return s.real();
        }
        std::vector<ITYPE> xm(k), zm(k);
        std::vector<UINT> ny(k);
        for (UINT i = 0; i < k; ++i) terms_[i].masks(&xm[i], &zm[i], &ny[i]);
        std::vector<double> coefs(2 * (size_t)k);
        for (UINT i = 0; i < k; ++i) {
            coefs[2 * i] = terms_[i].get_coef().real();
            coefs[2 * i + 1] = terms_[i].get_coef().imag();
        }
        double out[2];
        check(qs_expectation_value_pauli_weighted(xm.data(), zm.data(), ny.data(), coefs.data(), k, state->data(),
                  state->dim, state->get_cuda_stream(), out),
            "get_expectation_value");
        return out[0];
    }

private:
    UINT qubit_count_;
    std::vector<PauliOperator> terms_;
};

}  // namespace qulacs_b200
