"""Benchmark: the 30-qubit complex128 layered circuit (plain method) on B200.

Workload (one step): |0...0> on 30 qubits (16 GiB complex128 state, larger than L2), then 10 layers
of RX, RY, RZ on every qubit (angles U[0, 2pi), seeded) followed by a CNOT ladder q -> q+1 -- 1190
gates.  The value is gates/s through the circuit (1190 / circuit time, summed over ranks); the line
also carries the circuit time, the physical HBM bandwidth of the staged passes (passes x 2 x 16 x 2^n
bytes / time) and, named as such, the effective figure gates x 2 x 16 x 2^n / time against the
reference's per-gate roofline bytes.  The end-to-end figure (``e2e``) runs the same circuit through the
public API with the observable (256 Pauli strings of weight <= 6) and 1024-shot sampling, reading
results back to the host, in the same unit.  The reference arm (``--impl reference``) runs the
reference csim on all host cores over whole layers of the same circuit, in gates/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--mode staged|gate_by_gate]

Multi-GPU: replicas only (each rank runs its own 30-qubit state; no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_QUBITS = 30
DEPTH = 10
N_TERMS = 256
N_SHOTS = 1024
GATE_SEED, TERM_SEED, SHOT_SEED = 2124, 2125, 2126
METRIC = ("30q circuit time & HBM GB/s (plain c128 layered RX/RY/RZ+CNOT, depth 10): gates/s through the circuit; "
          "circuit_s and the physical HBM GB/s beside it")


def bytes_per_gate(n: int) -> int:
    return 2 * 16 * (1 << n)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.lines = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# DRAM bytes per amplitude per staged pass measured by ncu (dram__bytes_read.sum + write.sum of
# k_staged_pass on the 26-qubit layered circuit: 1.074e9 + 1.014e9 B for 2^26 amplitudes), scaled to
# the benchmark's size by the number of amplitudes.
STAGED_TRAFFIC_PER_AMP = 2.088e9 / (1 << 26)


def kernel_table(state, n: int, stream, reps: int = 5):
    """Each gate-by-gate kernel alone at n qubits: ms per launch and GB/s against 2 x 16 x 2^n B
    (and against the bytes the kernel actually has to move, for CNOT/CZ)."""
    import ctypes as C

    import torch

    from qulacs_b200._lib import call
    rng = np.random.default_rng(7)

    def unitary(k):
        a = rng.normal(size=(1 << k, 1 << k)) + 1j * rng.normal(size=(1 << k, 1 << k))
        q, _ = np.linalg.qr(a)
        return np.ascontiguousarray(q, dtype=np.complex128)

    p = state.data_ptr()
    dim = state.dim
    h = stream.cuda_stream
    m1 = unitary(1)
    mats = {k: unitary(k) for k in range(2, 7)}
    tls = {k: np.ascontiguousarray(np.arange(n - k, n, dtype=np.uint32)) for k in range(2, 7)}
    mp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    cases = [
        ("dense1 t=0 (k_dense1_shfl)", 1.0, lambda: call("qs_single_qubit_dense_matrix_gate", 0, mp(m1), p, dim, h)),
        ("dense1 t=4 (k_dense1_shfl)", 1.0, lambda: call("qs_single_qubit_dense_matrix_gate", 4, mp(m1), p, dim, h)),
        ("dense1 t=5 (k_pair)", 1.0, lambda: call("qs_single_qubit_dense_matrix_gate", 5, mp(m1), p, dim, h)),
        (f"dense1 t={n // 2} (k_pair)", 1.0, lambda: call("qs_single_qubit_dense_matrix_gate", n // 2, mp(m1), p, dim, h)),
        (f"dense1 t={n - 1} (k_pair)", 1.0, lambda: call("qs_single_qubit_dense_matrix_gate", n - 1, mp(m1), p, dim, h)),
        ("RZ t=10 (k_diag1)", 1.0, lambda: call("qs_RZ_gate", 10, 0.3, p, dim, h)),
        (f"CNOT {n - 2}->{n - 1} (k_pair swap)", 0.5, lambda: call("qs_CNOT_gate", n - 2, n - 1, p, dim, h)),
        ("CNOT 0->1 (k_perm2_tile, full read + write)", 1.0, lambda: call("qs_CNOT_gate", 0, 1, p, dim, h)),
        (f"CNOT 2->{n - 1} (k_perm2_tile, full read + write)", 1.0, lambda: call("qs_CNOT_gate", 2, n - 1, p, dim, h)),
        ("CZ 3,17 (k_single negate)", 0.25, lambda: call("qs_CZ_gate", 3, 17, p, dim, h)),
        (f"dense2 {n - 2},{n - 1} (k_dense2)", 1.0, lambda: call("qs_double_qubit_dense_matrix_gate_c", n - 2, n - 1, mp(mats[2]), p, dim, h)),
    ]
    for k in range(3, 7):
        cases.append((f"dense{k} high targets ({'k_denseK_blk' if k == 6 else 'k_denseK_reg'})", 1.0,
                      lambda k=k: call("qs_multi_qubit_dense_matrix_gate", mp(tls[k]), k, mp(mats[k]), p, dim, h)))
    out = []
    alg = bytes_per_gate(n)
    for name, frac, fn in cases:
        fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        out.append({"kernel": name, "ms": round(ms, 4), "gbs_vs_2x16x2^n": round(alg / 1e9 / (ms / 1e3), 1),
                    "gbs_touched": round(frac * alg / 1e9 / (ms / 1e3), 1)})
    return out


def layer_gates(n: int) -> int:
    """Gates in one layer of the layered circuit: RX, RY, RZ on every qubit, then n - 1 CNOTs."""
    return 3 * n + (n - 1)


def cpu_reference_layers(n: int, gates, layers: int, threads: int, state=None, first_layer: int = 0):
    """Time the reference csim (oracle/_ref, else the oracle port) gate by gate on host cores over
    `layers` WHOLE layers of the layered circuit (every gate kind in its circuit proportion)."""
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    os.environ.setdefault("QULACS_NUM_THREADS", str(threads))
    from oracle import oracle as O
    from oracle import replay as R
    sim = O.reference()
    kind = "reference"
    if sim is None:
        sim, kind = O.port(), "port"
        threads = 1
    from qulacs_b200 import workloads as W
    s = state
    if s is None:
        s = np.zeros(1 << n, dtype=np.complex128)
        s[0] = 1.0
        R.run_on_cpu(gates[:2], s, sim)  # first touch of every page, untimed
    per = layer_gates(n)
    lo = (first_layer % DEPTH) * per
    work = [gates[(lo + i) % len(gates)] for i in range(layers * per)]
    t0 = time.perf_counter()
    R.run_on_cpu(work, s, sim)
    dt = time.perf_counter() - t0
    return {"value": len(work) / dt, "unit": "gates/s", "gbs_per_gate": len(work) * bytes_per_gate(n) / dt / 1e9,
            "seconds": dt, "cores": threads, "kind": kind,
            "sample": f"{layers} whole layer(s) of the {n}-qubit layered circuit ({len(work)} gates: "
                      f"{3 * n * layers} rotations, {(n - 1) * layers} CNOTs), gate by gate, {dt:.1f} s"}


def run_reference(args, rank: int, world: int):
    """The reference arm: the reference csim, compiled from its own sources (oracle/_ref), on all host
    cores, gate by gate.  One step = one whole layer of the benchmark circuit (119 gates at 30 qubits,
    every gate kind in proportion); value = gates/s over the timed steps, the same unit as this
    library's arm.  Rank 0 only (the other ranks exit without work)."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    os.environ.setdefault("QULACS_NUM_THREADS", str(threads))
    from oracle import oracle as O
    from oracle import replay as R
    from qulacs_b200 import workloads as W
    n = args.qubits
    gates = W.layered_rotation_circuit(n, DEPTH, GATE_SEED)
    s = np.zeros(1 << n, dtype=np.complex128)
    s[0] = 1.0
    R.run_on_cpu(gates[:2], s, O.reference() or O.port())  # first touch of every page, untimed
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_reference_layers(n, gates, 1, threads, state=s, first_layer=i)
        if i >= args.warmup:
            vals.append(r)
    secs = sum(v["seconds"] for v in vals)
    value = len(vals) * layer_gates(n) / secs
    cb = dict(vals[-1])
    cb["value"] = value
    cb["sample"] = f"{len(vals)} timed steps of one whole layer each ({layer_gates(n)} gates), after " \
                   f"{args.warmup} warm-up layers"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "gates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / len(vals),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128 (f64)",
            "data": "synthetic (seeded)",
            "config": {"workload": f"layered RX/RY/RZ+CNOT n={n} depth={DEPTH}: one whole layer of {DEPTH} "
                                   f"({layer_gates(n)} gates) per step"},
            "circuit_s_from_layers": len(gates) / value,
            "gbs_per_gate": value * bytes_per_gate(n) / 1e9,
            "cpu_baseline": cb, "e2e": {"value": value, "unit": "gates/s", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def fused_comparison(n: int, layers: int, stream, with_gate_by_gate: bool, reps: int = 2):
    """Config 3: U3 + CZ(random matching) circuit; fused complex64 (tensor cores) vs plain complex128.

    Returns times (CUDA events), the infidelity 1 - |<psi_c128|psi_c64>|^2 and |d<H>| for 256 strings of
    weight <= 4 (coefficients N(0, 1)), both sides evaluated on the device with FP64 accumulation."""
    import torch

    import qulacs_b200 as Q
    from qulacs_b200 import workloads as W
    gates = W.u3_cz_circuit(n, layers, seed=3003)
    terms = W.random_pauli_terms(n, 256, 1, 4, seed=3004)
    circ = W.to_circuit(gates, n)
    obs = W.to_observable(terms, n)

    def timed(fn, reps=reps):
        fn()  # warm-up (plan build, first touch)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps / 1e3

    plain = Q.QuantumState(n)
    t_staged = timed(lambda: (plain.set_zero_state(), circ.update_quantum_state(plain, mode="staged")))
    t_gbg = None
    if with_gate_by_gate:
        t_gbg = timed(lambda: (plain.set_zero_state(), circ.update_quantum_state(plain, mode="gate_by_gate")), 1)
    plain.set_zero_state()
    circ.update_quantum_state(plain, mode="staged")
    fused = Q.QuantumStateC64(n)
    circ.set_c64_executor("fp64")  # the other complex64 executor: FP64 passes over the complex64 state
    t_c64_fp64 = timed(lambda: (fused.set_zero_state(), circ.update_quantum_state(fused)))
    circ.set_c64_executor("tensor")
    t_fused = timed(lambda: (fused.set_zero_state(), circ.update_quantum_state(fused)))
    fused.set_zero_state()
    circ.update_quantum_state(fused)
    inf = fused.infidelity(plain)
    coefs = np.array([c for c, _, _ in terms])
    ev_plain = obs.term_values(plain)
    ev_fused = obs.term_values(fused)
    passes, blocks = circ.fused_stats()
    out = {"workload": f"U3 + CZ(random matching) n={n} layers={layers} ({len(gates)} gates)",
           "plain_c128_staged_s": t_staged, "plain_c128_gate_by_gate_s": t_gbg, "fused_c64_tc_s": t_fused,
           "c64_fp64_passes_s": t_c64_fp64,
           "speedup_vs_staged": t_staged / t_fused,
           "speedup_vs_gate_by_gate": (t_gbg / t_fused) if t_gbg else None,
           "infidelity": inf, "abs_dH": abs(float(np.dot(coefs, ev_plain - ev_fused))),
           "max_abs_dP": float(np.max(np.abs(ev_plain - ev_fused))),
           "fused_passes": passes, "fused_blocks": blocks, "staged_passes": circ.pass_count()}
    del plain, fused
    return out


def batched_throughput(instances: int, budget_gb: float, seed: int = 4004,
                       precisions=("c128", "c64", "c64_tensor")):
    """Config 4: hardware-efficient-ansatz instances, n ~ U{10..24}, depth ~ U{4..16}, RY RZ + CZ ring,
    200 strings of weight <= 4 each.  Circuits are built once (outside the timed region, as a variational
    loop reuses them); the timed region is admission + circuit application + <H> for all instances."""
    from qulacs_b200 import workloads as W
    from qulacs_b200.batch import BatchRunner
    rng = np.random.default_rng(seed)
    jobs = []
    t_build = time.perf_counter()
    for i in range(instances):
        n = int(rng.integers(10, 25))
        d = int(rng.integers(4, 17))
        jobs.append((W.to_circuit(W.hea_circuit(n, d, seed * 10000 + i), n),
                     W.to_observable(W.random_pauli_terms(n, 200, 1, 4, seed * 10000 + 5000 + i), n)))
    t_build = time.perf_counter() - t_build
    out = {"workload": f"{instances} HEA instances, n~U{{10..24}}, depth~U{{4..16}}, 200 strings each",
           "host_build_s": t_build, "memory_budget_gb": budget_gb}
    for prec in precisions:
        # "c64": the default complex64 batch executor (FP64 passes over complex64 tiles when every gate
        # is stageable); "c64_tensor": the tensor-core blocks forced
        kw = {"precision": "c64", "c64_executor": "tensor"} if prec == "c64_tensor" else {"precision": prec}
        runner = BatchRunner(int(budget_gb * (1 << 30)), **kw)
        runner.run(jobs[: min(len(jobs), 64)])  # warm-up: plan building and first launches
        runner = BatchRunner(int(budget_gb * (1 << 30)), **kw)
        t0 = time.perf_counter()
        e = runner.run(jobs)
        dt = time.perf_counter() - t0
        out[prec] = {"circuits_per_s": instances / dt, "seconds": dt, "waves": runner.stats.waves,
                     "kernel_launches": runner.stats.kernel_launches, "energy_checksum": float(np.sum(e))}
    return out


def graph_replay(reps: int = 20):
    """Captured CUDA graphs against direct calls (wall time per call, host launch overhead included,
    since that is what a graph removes): a 16-qubit layered circuit gate by gate (454 launches) and
    staged, and a batch of 64 HEA circuits (n 10..16) in one persistent launch."""
    import ctypes as C

    import torch

    import qulacs_b200 as Q
    from qulacs_b200 import workloads as W
    from qulacs_b200._lib import call
    from qulacs_b200.graph import capture_batch, capture_circuit

    def wall(fn):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / reps * 1e3

    out = {"workload": "16q layered depth 10 (454 gates); 64 HEA circuits n~U{10..16} depth 6", "reps": reps}
    n = 16
    circ = W.to_circuit(W.layered_rotation_circuit(n, 10, 7), n)
    s = Q.QuantumState(n)
    for mode in ("gate_by_gate", "staged"):
        direct = wall(lambda: (s.set_zero_state(), circ.update_quantum_state(s, mode=mode)))
        g = capture_circuit(circ, s, mode=mode)
        replay = wall(g.launch)
        out[mode] = {"direct_ms": direct, "graph_ms": replay, "kernels": g.kernel_count()}
        g.close()
    rng = np.random.default_rng(8)
    sizes = [int(rng.integers(10, 17)) for _ in range(64)]
    circs = [W.to_circuit(W.hea_circuit(m, 6, seed=8000 + i), m) for i, m in enumerate(sizes)]
    states = [Q.QuantumState(m) for m in sizes]
    k = len(circs)
    ch = (C.c_void_p * k)(*[c._h for c in circs])
    sp = (C.c_void_p * k)(*[x.data_ptr() for x in states])

    def batch_direct():
        for x in states:
            x.set_zero_state()
        call("qs_batch_update_quantum_states", ch, sp, k, None)
    direct = wall(batch_direct)
    g = capture_batch(circs, states)
    out["batch64"] = {"direct_ms": direct, "graph_ms": wall(g.launch), "kernels": g.kernel_count()}
    g.close()
    return out


def noise_sampling(n: int = 20, depth: int = 4, p: float = 1e-3, shots: int = 1000, seed: int = 6006):
    """NoiseSimulator: HEA circuit with depolarizing noise after every gate (cppsim add_noise_gate rule),
    `shots` trajectories sampled on the device; the oracle port's time for a few trajectories on the
    host cores is the CPU comparison (extrapolated to all distinct trajectories)."""
    import torch

    import qulacs_b200 as Q
    from qulacs_b200 import workloads as W
    gates = W.noisy_circuit(W.hea_circuit(n, depth, seed), p)
    circ = W.to_circuit(gates, n)
    sim = Q.NoiseSimulator(circ, seed=seed)
    traj = sim.trajectories(shots)
    sim.execute(min(shots, 16))  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = sim.execute(shots)
    torch.cuda.synchronize()
    gpu_s = time.perf_counter() - t0
    res = {"workload": f"HEA n={n} depth={depth} + depolarizing p={p} after every gate ({len(gates)} ops), "
                       f"{shots} shots", "distinct_trajectories": int(traj.size), "gpu_s": gpu_s,
           "shots_per_s": shots / gpu_s, "checksum": int(out.sum() % (1 << 31))}
    try:
        from oracle import oracle as O
        from oracle import replay as R
        port = O.port()
        sample = 1
        t0 = time.perf_counter()
        for _ in range(sample):
            st = np.zeros(1 << n, dtype=np.complex128)
            st[0] = 1
            R.run_on_cpu([g for g in gates if g[0] != "DEPOL"], st, port)
        cpu_per = (time.perf_counter() - t0) / sample
        res["cpu_port_s_per_trajectory"] = cpu_per
        res["cpu_port_s_estimate"] = cpu_per * traj.size
        res["cpu_sample"] = f"{sample} full trajectory (noise-free gates) with the oracle port, 1 core"
    except Exception as e:  # noqa: BLE001
        res["cpu_port"] = f"unavailable: {type(e).__name__}: {e}"
    return res


def dm_noisy_circuit(n: int = 13, depth: int = 8, p: float = 1e-3, seed: int = 7007, reps: int = 3):
    """Density matrix (rows a16-a18): HEA circuit with depolarizing noise after every gate on an n-qubit
    density matrix (4^n entries, 1 GiB at 13 qubits), the exact channel, through the FP64-fused staged
    executor and through the gate-by-gate DM kernels.  Effective bandwidth counts 2 x 16 x 4^n bytes per
    gate or channel.  CPU: the reference csim's DM functions on a bounded sample of the ops."""
    import torch

    import qulacs_b200 as Q
    from qulacs_b200 import workloads as W
    gates = W.noisy_circuit(W.hea_circuit(n, depth, seed), p)
    circ = W.to_circuit(gates, n)
    rho = Q.DensityMatrix(n)
    per_op = 2.0 * 16.0 * float(4 ** n)
    res = {"workload": f"HEA n={n} depth={depth} + depolarizing p={p} after every gate, density matrix "
                       f"({len(gates)} gates and channels, {16 * 4 ** n / 2 ** 30:.2f} GiB)"}
    for mode in ("staged_fused", "gate_by_gate"):
        for _ in range(2):
            rho.set_zero_state()
            circ.update_quantum_state(rho, mode=mode)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            rho.set_zero_state()
            circ.update_quantum_state(rho, mode=mode)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        res[mode] = {"ms": ms, "effective_gbs": len(gates) * per_op / (ms / 1e3) / 1e9}
    res["trace"] = rho.get_squared_norm()  # DensityMatrix squared norm = trace (cppsim state_dm.hpp:142)
    try:
        from oracle import oracle as O
        from oracle import replay as R
        ref = O.reference()
        if ref is None:
            raise RuntimeError("reference csim not built")
        r = np.zeros((1 << n, 1 << n), dtype=np.complex128)
        r[0, 0] = 1
        t0 = time.perf_counter()
        done = 0
        for g in gates:
            R.run_on_cpu_dm([g], r, ref)
            done += 1
            if time.perf_counter() - t0 > 10.0:
                break
        dt = time.perf_counter() - t0
        res["cpu_reference"] = {"effective_gbs": done * per_op / dt / 1e9, "ops_timed": done, "seconds": dt,
                                "cores": os.cpu_count() or 1}
    except Exception as e:  # noqa: BLE001
        res["cpu_reference"] = f"unavailable: {type(e).__name__}: {e}"
    return res


GPUSIM_SO = os.path.join(ROOT, "baseline", "_ref", "libgpusim_ref.so")


def gpusim_baseline(n: int, gates, ours_s: float, reps: int = 2):
    """The reference's own GPU backend (src/gpusim, compiled for sm_100a by baseline/Makefile) running the
    same circuit gate by gate through its host wrappers on this B200: one kernel plus one stream
    synchronise per gate, as the reference's QuantumStateGpu path does.  Timed by the host clock around
    whole circuits (every wrapper synchronises).  Its amplitudes at the fixture's indices are checked
    against the reference csim's 30-qubit result when that fixture applies."""
    import ctypes as C
    if not os.path.exists(GPUSIM_SO):
        return {"unavailable": "baseline/_ref/libgpusim_ref.so not built (make -C baseline needs the reference "
                               "sources)"}
    lib = C.CDLL(GPUSIM_SO)
    lib.gs_allocate.restype = C.c_void_p
    lib.gs_allocate.argtypes = [C.c_ulonglong]
    lib.gs_norm.restype = C.c_double
    for f in ("gs_initialize", "gs_release", "gs_norm"):
        getattr(lib, f).argtypes = [C.c_void_p] + ([C.c_ulonglong] if f != "gs_release" else [])
    for f in ("gs_RX", "gs_RY", "gs_RZ"):
        getattr(lib, f).argtypes = [C.c_uint, C.c_double, C.c_void_p, C.c_ulonglong]
    lib.gs_CNOT.argtypes = [C.c_uint, C.c_uint, C.c_void_p, C.c_ulonglong]
    if not lib.gs_init():
        return {"unavailable": "gpusim stream allocation failed"}
    dim = 1 << n
    s = lib.gs_allocate(dim)
    fns = {"RX": lib.gs_RX, "RY": lib.gs_RY, "RZ": lib.gs_RZ}

    def run():
        lib.gs_initialize(s, dim)
        for g in gates:
            if g[0] == "CNOT":
                lib.gs_CNOT(g[1], g[2], s, dim)
            else:
                fns[g[0]](g[1], g[2], s, dim)

    run()  # warm-up
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        run()
        times.append(time.perf_counter() - t0)
    sec = min(times)
    out = {"workload": f"layered RX/RY/RZ+CNOT n={n} depth={DEPTH} ({len(gates)} gates), gate by gate through "
                       "gpusim's *_host wrappers (one kernel + one stream synchronise per gate)",
           "circuit_s": sec, "gates_per_s": len(gates) / sec,
           "gbs_per_gate": len(gates) * bytes_per_gate(n) / 1e9 / sec,
           "speedup_of_this_library": sec / ours_s, "norm": lib.gs_norm(s, dim), "reps": reps}
    fx = os.path.join(ROOT, "tests", "golden", "config2_n30.npz")
    if n == 30 and os.path.exists(fx):
        from qulacs_b200._lib import call
        g = np.load(fx)
        amp = (C.c_double * 2)()
        err = 0.0
        for i, want in zip(g["amp_index"][:512], g["amps"][:512]):
            call("qs_get_amplitude", C.c_void_p(s), dim, int(i), amp, None)
            err = max(err, abs(complex(amp[0], amp[1]) - complex(want)))
        out["max_abs_d_amp_vs_reference_csim"] = err
    lib.gs_release(s)
    return out


def timed_region(step, steps: int, warmup: int, dist=None, sync=None, make_timer=None, device: str = "cpu") -> float:
    """The timing contract: `warmup` untimed steps, then a barrier with a device synchronize on both
    sides, exactly `steps` timed steps, a synchronize, and the per-step time in ms as the MAX over
    ranks (`dist` = torch.distributed or None).  `make_timer()` returns (start, stop) where stop()
    returns elapsed ms (CUDA events on the launching stream in the bench; a host clock in CPU tests)."""
    import torch
    sync = sync or (lambda: None)
    if make_timer is None:
        def make_timer():
            t = [0.0]

            def start():
                t[0] = time.perf_counter()

            def stop():
                return (time.perf_counter() - t[0]) * 1e3
            return start, stop
    for _ in range(warmup):
        step()
    sync()
    if dist:
        dist.barrier()
    sync()
    start, stop = make_timer()
    start()
    for _ in range(steps):
        step()
    sync()
    ms = stop() / steps
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms


def fp64_per_amplitude(qubits, m) -> int:
    """FP64 instructions per amplitude of a gate in the staged register code: a rotation, or any 1-qubit
    matrix whose entries are each real or imaginary, and a 1-qubit diagonal cost 4; a general 1-qubit
    matrix 8; a k-qubit permutation or +-1 diagonal (CNOT, CZ, SWAP) 0; any other k-qubit matrix
    4 x 2^k (2^k complex multiply-adds)."""
    e = m.ravel()
    if len(qubits) == 1:
        if m[0, 1] == 0 and m[1, 0] == 0:
            return 4
        if all(x.real == 0 or x.imag == 0 for x in e):
            return 4
        return 8
    if np.all((e == 0) | (e == 1) | (e == -1)):
        return 0
    return 4 * (1 << len(qubits))


def serving_latency(requests: int, rate: float, budget_gb: float, workers: int, seed: int = 5005,
                    precisions=("c128", "c64")):
    """Config 5: Poisson arrivals of the request mix; p50/p99 latency and jobs/s per precision."""
    from qulacs_b200.serving import ServingLoop, make_request_mix
    out = {"workload": f"{requests} requests, Poisson rate {rate}/s, mix 70% <H> (n 12-28) / 20% sampling "
                       f"(n 16-30, 1024 shots) / 10% noisy DM (n 8-13)", "workers": workers,
           "memory_budget_gb": budget_gb}
    for prec in precisions:
        reqs = make_request_mix(requests, rate, seed)
        loop = ServingLoop(int(budget_gb * (1 << 30)), workers=workers, precision=prec)
        try:
            out[prec] = loop.run(reqs)
        finally:
            loop.close()
    return out


def serving_sweep(requests: int, rates, budget_gb: float, workers: int, seed: int = 5005,
                  precisions=("c128", "c64")):
    """Config 5 at several arrival rates up to saturation: per rate and precision, achieved jobs/s,
    p50/p99 latency, the mean and largest expectation batch and the mean number of worker batches on the
    device at once (continuous batching shows as batches > 1 and several in flight as the rate rises)."""
    from qulacs_b200.serving import ServingLoop, make_request_mix
    curve = []
    for rate in rates:
        row = {"rate_per_s": rate}
        for prec in precisions:
            reqs = make_request_mix(requests, rate, seed)
            loop = ServingLoop(int(budget_gb * (1 << 30)), workers=workers, precision=prec)
            try:
                st = loop.run(reqs)
            finally:
                loop.close()
            row[prec] = {k: st[k] for k in ("jobs_per_s", "p50_ms", "p99_ms", "mean_batch", "max_batch",
                                              "mean_batches_in_flight")}
        curve.append(row)
    return {"workload": f"{requests} requests per rate, Poisson arrivals, mix 70% <H> (n 12-28) / 20% sampling "
                        f"(n 16-30, 1024 shots) / 10% noisy DM (n 8-13)", "workers": workers,
            "memory_budget_gb": budget_gb, "curve": curve}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="staged_fused", choices=["staged_fused", "staged", "gate_by_gate"])
    ap.add_argument("--fusion-k", type=int, default=-1,
                    help="staged_fused block size (-1: autotuned; pin the autotuner's choice for profiler runs, "
                         "whose instrumented launches distort its timings)")
    ap.add_argument("--specialize", type=int, default=-1, choices=[-1, 0, 1],
                    help="specialised pass kernels for the staged modes: 1 on, 0 off (generic pass kernel), "
                         "-1 by state size (default: on from 22 qubits)")
    ap.add_argument("--no-mode-compare", action="store_true",
                    help="skip timing the other complex128 execution modes beside the headline one")
    ap.add_argument("--qubits", type=int, default=N_QUBITS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-kernel-table", action="store_true")
    ap.add_argument("--no-gpusim", action="store_true", help="skip the reference GPU backend leg")
    ap.add_argument("--workload", default="plain",
                    choices=["plain", "fused", "batched", "serving", "noise", "dm", "graphs"],
                    help="fused / batched / serving / noise / dm: only that measurement (configs 3 / 4 / 5, "
                         "NoiseSimulator, noisy density matrix)")
    ap.add_argument("--instances", type=int, default=4096)
    ap.add_argument("--budget-gb", type=float, default=96.0)
    ap.add_argument("--requests", type=int, default=120)
    ap.add_argument("--rate", type=float, default=8.0)
    ap.add_argument("--workers", type=int, default=4)
    ap.add_argument("--fused-qubits", type=int, default=32)
    ap.add_argument("--fused-layers", type=int, default=20)
    ap.add_argument("--with-gate-by-gate", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the fused / batched / serving measurements of the default line")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3  # timing rule: at least 3 untimed warm-up steps

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    import qulacs_b200 as Q
    from qulacs_b200 import _lib
    from qulacs_b200 import workloads as W

    n = args.qubits
    stream = torch.cuda.current_stream()
    Q.set_default_stream(stream.cuda_stream)
    lib = _lib.load()
    if args.workload == "fused":
        r = fused_comparison(args.fused_qubits, args.fused_layers, stream, args.with_gate_by_gate)
        if rank == 0:
            print(json.dumps({"metric": "fused vs plain at infidelity<=1e-6", **r}), flush=True)
        return
    if args.workload == "batched":
        r = batched_throughput(args.instances, args.budget_gb)
        if rank == 0:
            print(json.dumps({"metric": "batched uneven circuits: circuits/s", **r}), flush=True)
        return
    if args.workload == "graphs":
        r = graph_replay()
        if rank == 0:
            print(json.dumps({"metric": "captured graph replay vs direct call: ms per call", **r}), flush=True)
        return
    if args.workload == "dm":
        r = dm_noisy_circuit()
        if rank == 0:
            print(json.dumps({"metric": "noisy density matrix: effective GB/s", **r}), flush=True)
        return
    if args.workload == "noise":
        r = noise_sampling()
        if rank == 0:
            print(json.dumps({"metric": "noisy trajectory sampling: shots/s", **r}), flush=True)
        return
    if args.workload == "serving":
        r = serving_sweep(args.requests, (5.0, 20.0, 50.0, 100.0), args.budget_gb, args.workers)
        if rank == 0:
            print(json.dumps({"metric": "serve p99 ms", **r}), flush=True)
        return
    gates = W.layered_rotation_circuit(n, DEPTH, GATE_SEED)
    terms = W.random_pauli_terms(n, N_TERMS, 1, 6, TERM_SEED)
    circ = W.to_circuit(gates, n)
    if args.fusion_k >= 0:
        circ.set_fusion(args.fusion_k)
    circ.set_specialized(args.specialize)
    obs = W.to_observable(terms, n)
    state = Q.QuantumState(n)
    mode = args.mode

    def step():
        state.set_zero_state()
        circ.update_quantum_state(state, mode=mode)

    launch0 = [0]

    def cuda_timer():
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

        def start():
            launch0[0] = lib.qs_launch_count()
            ev0.record(stream)

        def stop():
            ev1.record(stream)
            torch.cuda.synchronize()
            return ev0.elapsed_time(ev1)
        return start, stop

    with ClockSampler(local) as clk:
        ms = timed_region(step, args.steps, args.warmup, dist, torch.cuda.synchronize, cuda_timer, "cuda")
    launches = lib.qs_launch_count() - launch0[0]
    gb_per_step = len(gates) * bytes_per_gate(n) / 1e9
    value = world * len(gates) / (ms / 1e3)  # gates/s, whole job

    # dominant kernel roofline: one HBM pass = 2 x 16 x 2^n algorithmic bytes
    staged_kernel = mode in ("staged", "staged_fused")
    fusion = None
    if mode == "staged_fused":
        fk, fcount, passes, fest = circ.fusion_info()
        _, spec, compile_ms = circ.specialized_info()
        fusion = {"k": fk, "gates_after_fusion": fcount, "autotuner_estimates_ms": fest,
                  "specialized_passes": spec, "specialize_compile_ms": compile_ms}
    elif mode == "staged":
        passes = circ.pass_count()
    else:
        passes = len(gates)
    per_launch_ms = ms / max(1, passes)
    hbm_peak, peak_kind = peaks()
    achieved = bytes_per_gate(n) / 1e9 / (per_launch_ms / 1e3)
    # FP64 view of the same work: specialised RX/RY/RZ code issues 4 FP64 instructions per amplitude
    # per rotation gate (CNOTs move data only); B200 FP64 CUDA-core peak = 148 SMs x 64 FMA/clk.
    rot = sum(1 for g in gates if g[0] in ("RX", "RY", "RZ"))
    fp64_instr = 4.0 * rot * (1 << n)
    if fusion is not None and fusion["k"] > 0:
        fl = circ.fuse(fusion["k"])
        fp64_instr = float(sum(fp64_per_amplitude(*fl[i]) for i in range(len(fl)))) * (1 << n)
    fp64_peak = 148 * 64 * 1.965e9
    kernels = kernel_table(state, n, stream) if not args.no_kernel_table else None

    # end to end through the public API: host gate list already built into the circuit, observable
    # masks, coefficients and uniforms from host, results (energy + samples) back to the host
    e2e_steps = max(1, min(args.steps, 3))
    # warm-up outside the timed region: the observable's pass plan, and its per-pass kernels, which the
    # library generates when the same terms are evaluated a second time (cached for the process)
    from qulacs_b200.observable import expectation_specialized_info
    spec0 = expectation_specialized_info()[0]
    for _ in range(2):
        obs.get_expectation_value(state)
    ev_generated = expectation_specialized_info()[0] > spec0
    ev_compile_ms = expectation_specialized_info()[1] if ev_generated else 0.0
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(3):
        obs.get_expectation_value(state)
    e1.record(stream)
    torch.cuda.synchronize()
    ev_ms = e0.elapsed_time(e1) / 3
    ev_plan = obs.weighted_plan(n)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    energy = None
    for i in range(e2e_steps):
        state.set_zero_state()
        circ.update_quantum_state(state, mode=mode)
        energy = obs.get_expectation_value(state)
        samples = state.sampling(N_SHOTS, SHOT_SEED + i)
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / e2e_steps
    if dist:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    h2d = N_TERMS * (8 + 8 + 4 + 16) + N_SHOTS * 8 + len(gates) * 64  # masks, Y counts, coefficients
    d2h = 16 + N_SHOTS * 8  # the complex energy and the samples
    # draws of the last e2e sampling call within 1e-12 of a cumulative boundary (outside the timed region)
    boundary_draws = state.sampling_boundary_draws(N_SHOTS, SHOT_SEED + e2e_steps - 1, 1e-12)

    # the other complex128 execution modes on the same circuit and state (outside the timed region)
    modes_ms = {mode: ms}
    if not args.no_mode_compare:
        for other in ("staged_fused", "staged", "gate_by_gate"):
            if other == mode:
                continue
            reps = 1 if other == "gate_by_gate" else 2
            state.set_zero_state()
            circ.update_quantum_state(state, mode=other)  # warm-up (plan build, autotuning)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                state.set_zero_state()
                circ.update_quantum_state(state, mode=other)
            e1.record(stream)
            torch.cuda.synchronize()
            modes_ms[other] = e0.elapsed_time(e1) / reps

    # the reference's own GPU backend on the same circuit and device (N = 1 only)
    gpusim = None
    if world == 1 and not args.no_gpusim:
        try:
            gpusim = gpusim_baseline(n, gates, ms / 1e3)
        except Exception as e:  # noqa: BLE001
            gpusim = {"error": f"{type(e).__name__}: {e}"}

    # the CPU baseline and the other configurations run at N = 1 only: with N > 1 ranks they would
    # keep the other ranks waiting at the closing barrier
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_layers(n, gates, 1, os.cpu_count() or 1)

    # configs 3-5 beside the headline (each guarded: a failure is reported, not fatal)
    extras = {}
    if world == 1 and not args.no_extras:
        del state
        torch.cuda.synchronize()
        for key, fn in (("fused", lambda: fused_comparison(args.fused_qubits, args.fused_layers, stream, True)),
                        ("batched", lambda: batched_throughput(args.instances, args.budget_gb)),
                        ("serving", lambda: serving_sweep(60, (5.0, 20.0, 50.0, 100.0), 96.0, 4)),
                        ("noise", lambda: noise_sampling()),
                        ("graphs", lambda: graph_replay()),
                        ("density_matrix", lambda: dm_noisy_circuit())):
            try:
                extras[key] = fn()
            except Exception as e:  # noqa: BLE001
                extras[key] = {"error": f"{type(e).__name__}: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "gates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128 (f64)", "data": "synthetic (seeded)",
            "config": {"workload": f"layered RX/RY/RZ+CNOT n={n} depth={DEPTH} ({len(gates)} gates), c128",
                       "exec_mode": mode, "hbm_passes": passes,
                       "l2": f"state {(16 << n) / 2**30:g} GiB > L2 (no flush needed)",
                       "parallelism": f"replicas x{world}"},
            "circuit_s": ms / 1e3,
            "hbm_gbs_physical": passes * bytes_per_gate(n) / 1e9 / (ms / 1e3),
            "effective_gbs": gb_per_step / (ms / 1e3),
            "effective_gbs_note": "gates x 2 x 16 x 2^n B (the reference's per-gate roofline bytes) / circuit "
                                  "time; not a bandwidth: a staged pass applies many gates per HBM read+write",
            "fusion": fusion,
            "modes_ms": modes_ms,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "peak_kind": peak_kind,
                         "traffic": (STAGED_TRAFFIC_PER_AMP * (1 << n)) if staged_kernel else None,
                         "kernel": (("k_pass_spec (specialised" if (fusion or {}).get("specialized_passes") else
                                     "k_staged_pass (generic") +
                                    " pass kernel): one HBM pass (2 x 16 x 2^n B) applying ~"
                                    f"{len(gates) / max(1, passes):.0f} circuit gates" if staged_kernel
                                    else "gate kernels: one HBM pass (2 x 16 x 2^n B) per gate"),
                         "traffic_note": "scaled from the 26-qubit ncu capture by amplitudes" if staged_kernel else None},
            "roofline_fp64": {"achieved_tinstr_s": fp64_instr / (ms / 1e3) / 1e12,
                              "peak_tinstr_s": fp64_peak / 1e12,
                              "frac": fp64_instr / (ms / 1e3) / fp64_peak,
                              "note": "FP64 instr/amplitude: rotation or 1q diagonal 4, 1q dense 8, k-qubit dense "
                                      "4 x 2^k, CNOT/CZ/SWAP 0; nominal 64 FP64 FMA/clk/SM at 1965 MHz"},
            "kernels": kernels,
            "e2e": {"value": world * len(gates) / (e2e_ms / 1e3), "unit": "gates/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "includes": "set_zero_state + circuit + <H> (256 strings) + 1024-shot sampling",
                    "sampling_boundary_draws": boundary_draws,
                    "sampling_boundary_note": "of the 1024 draws, those within 1e-12 of a cumulative boundary "
                                              "of the FP64 prefix (the draws parity with the reference excepts)"},
            "energy": energy,
            "expectation": {"ms": ev_ms, "passes": ev_plan["passes"], "plan": ev_plan,
                            "generated_kernels": ev_generated, "compile_ms": ev_compile_ms,
                            "note": "sum_k c_k <P_k> of the 256 strings on the final state, through "
                                    "Observable.get_expectation_value (host masks in, energy out), after "
                                    "warm-up; compile_ms = NVRTC time of the per-pass kernels, summed over "
                                    "parallel compiles, once per term list"},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "gpusim_baseline": gpusim,
            **extras,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
