// C++ surface test: cppsim-style classes over libqulacs_b200 (run by tests/test_cpp_api.py).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <random>

#include "qulacs_b200/cppsim.hpp"

using namespace qulacs_b200;

static int failures = 0;
#define EXPECT(cond)                                                         \
    do {                                                                     \
        if (!(cond)) {                                                       \
            std::fprintf(stderr, "FAILED %s:%d %s\n", __FILE__, __LINE__, #cond); \
            ++failures;                                                      \
        }                                                                    \
    } while (0)

int main() {
    // Bell state through gate objects (reference ownership: caller deletes factory gates)
    {
        QuantumState s(3);
        QuantumGateBase* h = gate::H(0);
        QuantumGateBase* cx = gate::CNOT(0, 1);
        h->update_quantum_state(&s);
        cx->update_quantum_state(&s);
        delete h;
        delete cx;
        const ComplexVector v = s.get_vector();
        const double r = 1.0 / std::sqrt(2.0);
        EXPECT(std::abs(v[0] - r) < 1e-15 && std::abs(v[3] - r) < 1e-15 && std::abs(v[1]) < 1e-15);
        Observable zz(3);
        zz.add_operator(1.0, "Z 0 Z 1");
        zz.add_operator(0.5, "X 0 X 1");
        EXPECT(std::abs(zz.get_expectation_value(&s) - 1.5) < 1e-12);
        EXPECT(std::abs(s.get_squared_norm() - 1.0) < 1e-14);
        EXPECT(std::abs(s.get_zero_probability(0) - 0.5) < 1e-14);
        EXPECT(s.get_device_name() == "gpu");
    }
    // a random 12-qubit circuit: staged == gate by gate, and circuit + inverse == identity
    {
        const UINT n = 12;
        std::mt19937_64 rng(5);
        std::uniform_real_distribution<double> ang(0, 6.283185307179586);
        QuantumCircuit c(n), inv(n);
        std::vector<std::pair<int, std::pair<UINT, double>>> ops;
        for (int layer = 0; layer < 4; ++layer) {
            for (UINT q = 0; q < n; ++q) {
                const double a = ang(rng), b = ang(rng);
                c.add_gate(gate::RX(q, a));
                c.add_gate(gate::RZ(q, b));
                ops.push_back({0, {q, a}});
                ops.push_back({2, {q, b}});
            }
            for (UINT q = 0; q + 1 < n; ++q) {
                c.add_gate(gate::CNOT(q, q + 1));
                ops.push_back({5, {q, 0}});
            }
        }
        for (auto it = ops.rbegin(); it != ops.rend(); ++it) {
            if (it->first == 0) inv.add_gate(gate::RX(it->second.first, -it->second.second));
            else if (it->first == 2) inv.add_gate(gate::RZ(it->second.first, -it->second.second));
            else inv.add_gate(gate::CNOT(it->second.first, it->second.first + 1));
        }
        QuantumState a(n), b(n);
        c.update_quantum_state(&a, QS_EXEC_STAGED);
        c.update_quantum_state(&b, QS_EXEC_GATE_BY_GATE);
        const ComplexVector va = a.get_vector(), vb = b.get_vector();
        double err = 0;
        for (size_t i = 0; i < va.size(); ++i) err = std::max(err, std::abs(va[i] - vb[i]));
        EXPECT(err <= 1e-12);
        EXPECT(std::abs(std::abs(inner_product(a, b)) - 1.0) < 1e-12);
        inv.update_quantum_state(&a);
        EXPECT(std::abs(a.get_zero_probability(0) - 1.0) < 1e-12);
        std::vector<UINT> all0(n, 0);
        EXPECT(std::abs(a.get_marginal_probability(all0) - 1.0) < 1e-12);
    }
    // every gate kind's direct update_quantum_state (one csim-named call) equals the same gate run through
    // a one-gate circuit, on a state vector and on a density matrix
    {
        const UINT n = 5;
        const double h = 1.0 / std::sqrt(2.0);
        auto make = [&](int i) -> QuantumGateBase* {
            switch (i) {
                case 0: return gate::RX(1, 0.7);
                case 1: return gate::RY(3, -1.1);
                case 2: return gate::RZ(0, 2.3);
                case 3: return gate::CNOT(4, 1);
                case 4: return gate::CZ(2, 0);
                case 5: return gate::SWAP(0, 3);
                case 6: return gate::H(2);
                case 7: return gate::T(4);
                case 8: return gate::DenseMatrix({1, 3}, {h, 0, 0, h, 0, h, h, 0, 0, h, -h, 0, h, 0, 0, -h});
                case 9: return gate::Pauli({0, 2, 4}, {1, 2, 3});
                case 10: return gate::PauliRotation({1, 3}, {2, 1}, 0.4);
                case 11: {
                    QuantumGateBase* g = gate::DenseMatrix(2, {0, CPPCTYPE(0, 1), CPPCTYPE(0, 1), 0});
                    g->add_control_qubit(4, 1);
                    return g;
                }
                case 12: return gate::DiagonalMatrix({0, 3}, {1, CPPCTYPE(0, 1), -1, CPPCTYPE(0, -1)});
                default: return nullptr;
            }
        };
        QuantumState a(n), b(n);
        DensityMatrix ra(n), rb(n);
        QuantumGateBase* prep = gate::H(0);
        prep->update_quantum_state(&a);
        prep->update_quantum_state(&b);
        prep->update_quantum_state(&ra);
        prep->update_quantum_state(&rb);
        delete prep;
        for (int i = 0; i <= 12; ++i) {
            std::unique_ptr<QuantumGateBase> g(make(i));
            g->update_quantum_state(&a);
            g->update_quantum_state(&ra);
            QuantumCircuit c(n);
            c.add_gate(make(i));
            c.update_quantum_state(&b, QS_EXEC_GATE_BY_GATE);
            c.update_quantum_state(&rb, QS_EXEC_GATE_BY_GATE);
            const ComplexVector va = a.get_vector(), vb = b.get_vector();
            double err = 0;
            for (size_t k = 0; k < va.size(); ++k) err = std::max(err, std::abs(va[k] - vb[k]));
            EXPECT(err <= 1e-14);
            const ComplexVector ma = ra.get_matrix(), mb = rb.get_matrix();
            err = 0;
            for (size_t k = 0; k < ma.size(); ++k) err = std::max(err, std::abs(ma[k] - mb[k]));
            EXPECT(err <= 1e-14);
        }
    }
    // sampling a basis state (test/cppsim/test_state.cpp:38-47)
    {
        QuantumState s(10);
        s.set_computational_basis(100);
        for (ITYPE x : s.sampling(1024, 3)) EXPECT(x == 100);
    }
    // depolarizing identity on a density matrix (test/cppsim/test_noise_dm.cpp:274-309)
    {
        DensityMatrix rho(1);
        const double p = 0.2;
        QuantumGateBase* g = gate::DepolarizingNoise(0, 3 * p / 4);
        g->update_quantum_state(&rho);
        delete g;
        const ComplexVector m = rho.get_matrix();
        EXPECT(std::abs(m[0] - (1 - p / 2)) < 1e-15 && std::abs(m[3] - p / 2) < 1e-15);
        EXPECT(std::abs(rho.get_squared_norm() - 1.0) < 1e-15);
    }
    // FP64-fused staged mode equals gate by gate; NoiseSimulator draws and merges trajectories
    {
        const UINT n = 10;
        QuantumCircuit c(n);
        for (int layer = 0; layer < 3; ++layer) {
            for (UINT q = 0; q < n; ++q) c.add_noise_gate(gate::RY(q, 0.3 + 0.1 * q + layer), "Depolarizing", 0.01);
            for (UINT q = 0; q + 1 < n; ++q) c.add_noise_gate(gate::CZ(q, q + 1), "Depolarizing", 0.01);
        }
        NoiseSimulator sim(&c, nullptr, 11);
        const std::vector<ITYPE> s = sim.execute(200);
        EXPECT(s.size() == 200);
        for (ITYPE x : s) EXPECT(x < (ITYPE(1) << n));
        NoiseSimulator::Result* r = sim.execute_and_get_result(200);
        UINT total = 0;
        for (const auto& p : r->result) {
            total += p.second;
            EXPECT(std::abs(p.first->get_squared_norm() - 1.0) < 1e-12);
        }
        EXPECT(total == 200 && !r->result.empty());
        delete r;
        QuantumCircuit u(n);
        for (UINT q = 0; q < n; ++q) {
            u.add_gate(gate::RX(q, 0.2 * q));
            u.add_gate(gate::RZ(q, 0.7));
        }
        for (UINT q = 0; q + 1 < n; ++q) u.add_gate(gate::CNOT(q, q + 1));
        QuantumState a(n), b(n);
        u.update_quantum_state(&a, QS_EXEC_STAGED_FUSED);
        u.update_quantum_state(&b, QS_EXEC_GATE_BY_GATE);
        const ComplexVector va = a.get_vector(), vb = b.get_vector();
        double err = 0;
        for (size_t i = 0; i < va.size(); ++i) err = std::max(err, std::abs(va[i] - vb[i]));
        EXPECT(err <= 1e-12);
    }
    // errors become exceptions
    {
        bool threw = false;
        try {
            gate::CNOT(1, 1);
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        EXPECT(threw);
        threw = false;
        try {
            QuantumCircuit c(3);
            c.add_gate(gate::RX(5, 0.1));
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        EXPECT(threw);
    }
    {
        // state::tensor_product / permutate_qubit / drop_qubit: |1> (x) |0>|1>, right state on the low qubits
        QuantumState left(1), right(2);
        left.set_computational_basis(1);
        right.set_computational_basis(2);  // qubit 1 set
        std::unique_ptr<QuantumState> t(state::tensor_product(left, right));
        EXPECT(t->qubit_count == 3 && std::abs(t->get_vector()[0b110] - CPPCTYPE(1.0)) < 1e-15);
        // dst[i] = src[sum over set bits q of i of 2^order[q]]: src 0b110 comes from i = 0b101
        std::unique_ptr<QuantumState> p(state::permutate_qubit(*t, {2, 0, 1}));
        EXPECT(std::abs(p->get_vector()[0b101] - CPPCTYPE(1.0)) < 1e-15);
        std::unique_ptr<QuantumState> d(state::drop_qubit(*t, {2}, {1}));
        EXPECT(d->qubit_count == 2 && std::abs(d->get_vector()[0b10] - CPPCTYPE(1.0)) < 1e-15);
        // rejected before any allocation (cppsim/state.cpp:70): every qubit dropped, a short order
        bool threw = false;
        try {
            delete state::drop_qubit(*t, {0, 1, 2}, {0, 0, 0});
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        EXPECT(threw);
        threw = false;
        try {
            delete state::permutate_qubit(*t, {1, 0});
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        EXPECT(threw);
        // a bad projection value is rejected by the C ABI and the new state is freed, not leaked
        threw = false;
        try {
            delete state::drop_qubit(*t, {2}, {3});
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        EXPECT(threw);
    }
    if (failures == 0) std::printf("OK\n");
    return failures == 0 ? 0 : 1;
}
