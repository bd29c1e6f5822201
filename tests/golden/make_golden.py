"""Generate the golden fixtures in tests/golden/ by running the REFERENCE csim itself.

The reference csim is compiled from its own sources (oracle/Makefile -> oracle/_ref/libcsim_ref.so)
and driven here through oracle/csim_ref_shim.cpp.  Inputs come from qulacs_b200.workloads with the
seeds below.  Run from the repo root:  python tests/golden/make_golden.py
(``--config2`` makes the 30-qubit fixture of the benchmark circuit instead: minutes on all host cores.)
The fixtures are small .npz files; tests compare the oracle port and the CUDA library against them.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from oracle import replay as R  # noqa: E402
from qulacs_b200 import workloads as W  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def config1(ref):
    """16 qubits, depth 10 RX/RY/RZ + CNOT ladder, 64 Pauli strings (weight 1-4), 1024 shots."""
    n, depth = 16, 10
    gates = W.layered_rotation_circuit(n, depth, seed=2025)
    terms = W.random_pauli_terms(n, 64, 1, 4, seed=2026)
    u = W.uniforms(1024, seed=2027)
    s = np.zeros(1 << n, dtype=np.complex128)
    s[0] = 1.0
    R.run_on_cpu(gates, s, ref)
    ev = np.array([ref.expectation_value(tl, ids, s) for _, tl, ids in terms])
    coefs = np.array([c for c, _, _ in terms])
    samples = ref.sampling_with_uniforms(s, u)
    pick = np.random.default_rng(2028).choice(1 << n, size=512, replace=False)
    np.savez_compressed(os.path.join(OUT, "config1_n16.npz"), n=n, depth=depth, gate_seed=2025, term_seed=2026,
                        uniform_seed=2027, term_values=ev, coefs=coefs, energy=float(np.dot(coefs, ev)),
                        samples=samples, amp_index=pick, amps=s[pick], norm=ref.state_norm_squared(s))


def small_full(ref):
    """10 qubits, U3 + CZ layers, full final state; plus a 5-qubit noisy density matrix."""
    n = 10
    gates = W.u3_cz_circuit(n, 6, seed=3031)
    s = np.zeros(1 << n, dtype=np.complex128)
    s[0] = 1.0
    R.run_on_cpu(gates, s, ref)
    terms = W.random_pauli_terms(n, 32, 1, 6, seed=3032)
    ev = np.array([ref.expectation_value(tl, ids, s) for _, tl, ids in terms])
    np.savez_compressed(os.path.join(OUT, "u3cz_n10.npz"), n=n, layers=6, gate_seed=3031, term_seed=3032,
                        state=s, term_values=ev)
    # noisy density matrix (serving-mix DM job shape, small): depth-2 HEA, depolarizing p=1e-3
    nd = 5
    dg = W.noisy_circuit(W.hea_circuit(nd, 2, seed=3033), 1e-3)
    rho = np.zeros((1 << nd, 1 << nd), dtype=np.complex128)
    rho[0, 0] = 1.0
    R.run_on_cpu_dm(dg, rho, ref)
    dterms = W.random_pauli_terms(nd, 16, 1, 3, seed=3034)
    dev = np.array([ref.dm_expectation_value(tl, ids, rho) for _, tl, ids in dterms])
    np.savez_compressed(os.path.join(OUT, "noisy_dm_n5.npz"), n=nd, depth=2, gate_seed=3033, p=1e-3,
                        term_seed=3034, rho=rho, term_values=dev)


def config2_30q(ref, port):
    """30 qubits, the benchmark's layered circuit (depth 10, gate seed 2124, 1190 gates), run gate by gate
    by the reference csim on all host cores (~16 GiB state, ~8 GiB sampling prefix).  Stored: 4096
    amplitudes at seeded indices, the 256 <P_k> (weight <= 6, seed 2125) and the energy, and the 1024
    indices the reference samples for the seed-2126 uniforms, each with the oracle port's flag for a
    draw within 1e-12 of a cumulative boundary (same serial FP64 prefix)."""
    n, depth = 30, 10
    gates = W.layered_rotation_circuit(n, depth, seed=2124)
    terms = W.random_pauli_terms(n, 256, 1, 6, seed=2125)
    u = W.uniforms(1024, seed=2126)
    s = np.zeros(1 << n, dtype=np.complex128)
    s[0] = 1.0
    R.run_on_cpu(gates, s, ref)
    ev = np.array([ref.expectation_value(tl, ids, s) for _, tl, ids in terms])
    coefs = np.array([c for c, _, _ in terms])
    samples = ref.sampling_with_uniforms(s, u)
    port_samples, near = port.sampling_with_uniforms(s, u, eps=1e-12)
    assert np.all((port_samples == samples) | near)
    pick = np.sort(np.random.default_rng(2127).choice(1 << n, size=4096, replace=False))
    np.savez_compressed(os.path.join(OUT, "config2_n30.npz"), n=n, depth=depth, gate_seed=2124, term_seed=2125,
                        uniform_seed=2126, term_values=ev, coefs=coefs, energy=float(np.dot(coefs, ev)),
                        samples=samples, near_boundary=near, amp_index=pick, amps=s[pick],
                        norm=ref.state_norm_squared(s))


def main():
    O.build_reference()
    ref = O.reference()
    if ref is None:
        raise SystemExit("reference csim not built")
    if "--config2" in sys.argv:  # minutes of CPU time and ~26 GiB of host memory
        config2_30q(ref, O.port())
        print("30-qubit fixture written to", OUT)
        return
    config1(ref)
    small_full(ref)
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main()
