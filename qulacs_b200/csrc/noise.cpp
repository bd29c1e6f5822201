// cppsim NoiseSimulator (noisesimulator.cpp:18-198) on device-resident states.
//
// Each sample is one trajectory: every depolarizing channel of the circuit is replaced by one of its
// Kraus operators, drawn as the reference draws it -- the channel's operators reordered by descending
// (probability, index) (QuantumGate_Probabilistic::optimize_ProbablisticGate, gate_general.hpp:350-372),
// one uniform u per channel and sample, operator lower_bound(cumulative, u) - 1
// (randomly_select_which_gate_pos_to_apply, noisesimulator.cpp:167-185).  Identical trajectories
// are merged and visited in descending lexicographic order of their choices; a shared device state
// advances through the all-identity prefix common to the remaining trajectories, and each trajectory
// copies it and applies its own suffix (noisesimulator.cpp:85-165).  Circuits run through the
// FP64-fused staged executor at a fixed block size.  The reference draws from a Random seeded by
// std::random_device; here one mt19937_64(seed) stream supplies first every selection uniform
// (sample-major, channels in circuit order) and then each trajectory's sampling uniforms, in
// trajectory order, so a run is reproducible.
#include <algorithm>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/qulacs_b200.h"
#include "circuit.hpp"

namespace qs {

int set_error(int code, const std::string& msg);

using cd = std::complex<double>;

namespace {

constexpr int kNoiseFusionK = 2;

struct Channel {
    std::vector<GateRec> kraus;  // in sampling order; kind -1 = identity (nothing to apply)
    std::vector<double> cum;     // 0, p0, p0 + p1, ...
};

// Pauli string on `targets` (ids 0..3 = I X Y Z) as a stageable gate: a 2x2 / 4x4 dense matrix, a
// diagonal for Z on one qubit, or kind -1 for the identity.
GateRec pauli_kraus(const std::vector<UINT>& targets, const std::vector<UINT>& ids) {
    GateRec g;
    bool identity = true;
    for (UINT id : ids) identity &= id == 0;
    if (identity) {
        g.kind = -1;
        return g;
    }
    g.targets = targets;
    g.pauli_ids = ids;
    g.kind = QS_GATE_PAULI;
    std::vector<cd> m = g.dense_matrix();
    g.pauli_ids.clear();
    if (targets.size() == 1 && ids[0] == 3) {
        g.kind = QS_GATE_DIAGONAL;
        g.matrix = {m[0], m[3]};
    } else {
        g.kind = QS_GATE_DENSE;
        g.matrix = m;
    }
    return g;
}

// gate_factory.cpp:451-500: one qubit {X, Z, Y, I} with {p/3, p/3, p/3, 1 - p}; two qubits
// {I, Pauli(i % 4 on t1, i / 4 on t2) for i = 1..15} with {1 - p, p/15, ...}.
Channel make_channel(const GateRec& g) {
    std::vector<GateRec> ops;
    std::vector<double> probs;
    const double p = g.prob;
    if (g.targets.size() == 1) {
        const UINT ids[4] = {1, 3, 2, 0};
        for (int i = 0; i < 4; ++i) {
            ops.push_back(pauli_kraus(g.targets, {ids[i]}));
            probs.push_back(i < 3 ? p / 3 : 1 - p);
        }
    } else {
        for (UINT i = 0; i < 16; ++i) {
            ops.push_back(pauli_kraus(g.targets, {i % 4, i / 4}));
            probs.push_back(i == 0 ? 1 - p : p / 15);
        }
    }
    std::vector<std::pair<double, int>> order;
    for (size_t i = 0; i < probs.size(); ++i) order.push_back({probs[i], (int)i});
    std::sort(order.rbegin(), order.rend());
    Channel ch;
    double sum = 0.;
    ch.cum.push_back(0.);
    for (const auto& o : order) {
        ch.kraus.push_back(ops[o.second]);
        sum += o.first;
        ch.cum.push_back(sum);
    }
    return ch;
}

// lower_bound - 1, clamped to a valid operator (the reference's result is out of range for u == 0 or
// u above the rounded total; both have probability ~2^-53).
UINT select_kraus(const Channel& ch, double u) {
    const long pos = (long)(std::lower_bound(ch.cum.begin(), ch.cum.end(), u) - ch.cum.begin()) - 1;
    return (UINT)std::min<long>(std::max<long>(pos, 0), (long)ch.kraus.size() - 1);
}

struct Request {
    std::vector<uint8_t> choice;  // per channel, in circuit order
    UINT count;
};

struct NoisePlan {
    std::vector<int> channel_of;  // per gate: channel index or -1
    std::vector<Channel> channels;
    std::vector<Request> requests;
    std::mt19937_64 mt;           // continues with the sampling uniforms
};

void make_plan(const Circuit& c, UINT samples, UINT seed, NoisePlan* P) {
    for (const GateRec& g : c.gates) {
        if (g.kind == QS_GATE_DEPOLARIZING) {
            P->channel_of.push_back((int)P->channels.size());
            P->channels.push_back(make_channel(g));
        } else {
            P->channel_of.push_back(-1);
        }
    }
    const size_t nch = P->channels.size();
    P->mt.seed(seed);
    std::uniform_real_distribution<double> dist(0, 1);
    std::vector<std::vector<uint8_t>> sel(samples, std::vector<uint8_t>(nch, 0));
    for (UINT i = 0; i < samples; ++i)
        for (size_t j = 0; j < nch; ++j) sel[i][j] = (uint8_t)select_kraus(P->channels[j], dist(P->mt));
    std::sort(sel.begin(), sel.end());
    std::reverse(sel.begin(), sel.end());
    UINT run = 0;
    for (UINT i = 0; i < samples; ++i) {
        ++run;
        if (i + 1 == samples || sel[i] != sel[i + 1]) {
            P->requests.push_back({sel[i], run});
            run = 0;
        }
    }
}

// Gates [from, to) of the circuit with the channels' chosen operators.
void trajectory_gates(const Circuit& c, const NoisePlan& P, const std::vector<uint8_t>& choice, size_t from, size_t to,
    Circuit* out) {
    out->n = c.n;
    out->gates.clear();
    out->fusion_k = kNoiseFusionK;
    out->invalidate();
    for (size_t gi = from; gi < to; ++gi) {
        const int ch = P.channel_of[gi];
        if (ch < 0) {
            out->gates.push_back(c.gates[gi]);
            continue;
        }
        const GateRec& k = P.channels[ch].kraus[choice[ch]];
        if (k.kind >= 0) out->gates.push_back(k);
    }
}

}  // namespace

int noise_trajectories(Circuit& c, UINT samples, UINT seed, UINT* count, UINT* shots) {
    NoisePlan P;
    make_plan(c, samples, seed, &P);
    *count = (UINT)P.requests.size();
    if (shots)
        for (size_t i = 0; i < P.requests.size(); ++i) shots[i] = P.requests[i].count;
    return QS_OK;
}

int noise_execute(Circuit& c, const void* init, ITYPE dim, UINT samples, UINT seed, ITYPE* out,
    void* const* states_out, cudaStream_t st) {
    if (dim != (1ULL << c.n)) return set_error(QS_ERR_INVALID_ARGUMENT, "state dimension does not match the circuit");
    NoisePlan P;
    make_plan(c, samples, seed, &P);
    std::uniform_real_distribution<double> dist(0, 1);
    void* common = nullptr;
    void* buffer = nullptr;
    int rc = qs_allocate_quantum_state(dim, &common);
    if (rc == QS_OK) rc = qs_allocate_quantum_state(dim, &buffer);
    if (rc == QS_OK) {
        if (init) rc = cudaMemcpyAsync(common, init, dim * 16, cudaMemcpyDeviceToDevice, st) == cudaSuccess
                           ? QS_OK
                           : set_error(QS_ERR_CUDA, "noise simulator: state copy failed");
        else rc = qs_initialize_quantum_state(common, dim, st);
    }
    const size_t G = c.gates.size();
    size_t done = 0;  // gates [0, done) are applied to `common`
    ITYPE* dst = out;
    Circuit part;
    std::vector<double> u;
    for (size_t r = 0; rc == QS_OK && r < P.requests.size(); ++r) {
        const Request& q = P.requests[r];
        // the prefix of gates whose channels all chose operator 0 is common to every later request
        size_t stop = done;
        while (stop < G && (P.channel_of[stop] < 0 || q.choice[P.channel_of[stop]] == 0)) ++stop;
        if (stop > done) {
            trajectory_gates(c, P, q.choice, done, stop, &part);
            rc = run_staged_fused(part, common, dim, st);
            done = stop;
            if (rc != QS_OK) break;
        }
        if (cudaMemcpyAsync(buffer, common, dim * 16, cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
            rc = set_error(QS_ERR_CUDA, "noise simulator: state copy failed");
            break;
        }
        if (done < G) {
            trajectory_gates(c, P, q.choice, done, G, &part);
            rc = run_staged_fused(part, buffer, dim, st);
            if (rc != QS_OK) break;
        }
        if (states_out && states_out[r] &&
            cudaMemcpyAsync(states_out[r], buffer, dim * 16, cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
            rc = set_error(QS_ERR_CUDA, "noise simulator: state copy failed");
            break;
        }
        if (out) {
            u.resize(q.count);
            for (UINT i = 0; i < q.count; ++i) u[i] = dist(P.mt);
            rc = qs_state_sampling_with_uniforms(buffer, dim, u.data(), q.count, dst, st);
            dst += q.count;
        }
    }
    if (buffer) qs_release_quantum_state(buffer);
    if (common) qs_release_quantum_state(common);
    return rc;
}

}  // namespace qs

extern "C" {

QS_API int qs_noise_simulator_trajectories(qs_circuit_t circuit, QS_UINT sample_count, QS_UINT seed,
    QS_UINT* trajectory_count, QS_UINT* shots) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c || !trajectory_count) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null argument");
    return qs::noise_trajectories(*c, sample_count, seed, trajectory_count, shots);
}

QS_API int qs_noise_simulator_execute(qs_circuit_t circuit, const void* initial_state, QS_ITYPE dim,
    QS_UINT sample_count, QS_UINT seed, QS_ITYPE* samples, void* const* trajectory_states, void* stream) {
    qs::Circuit* c = reinterpret_cast<qs::Circuit*>(circuit);
    if (!c) return qs::set_error(QS_ERR_INVALID_ARGUMENT, "null circuit");
    return qs::noise_execute(*c, initial_state, dim, sample_count, seed, samples, trajectory_states,
        (cudaStream_t)stream);
}

}  // extern "C"
