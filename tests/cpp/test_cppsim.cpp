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
    }
    if (failures == 0) std::printf("OK\n");
    return failures == 0 ? 0 : 1;
}
