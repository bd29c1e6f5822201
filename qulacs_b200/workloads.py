"""Seeded synthetic circuits and observables for the benchmark configurations.

All random draws use numpy's PCG64 (``numpy.random.default_rng(seed)``); the same gate list is
fed to this library and to the CPU implementations, so both sides see identical inputs.
A gate is a tuple: ("RX"|"RY"|"RZ", q, angle), ("U3", q, theta, phi, lam), ("CNOT"|"CZ", c, t), ("SWAP", a, b),
("DENSE", targets, matrix), ("DEPOL", (q,) or (q0, q1), p).
"""
from __future__ import annotations

import math

import numpy as np

TWO_PI = 2.0 * math.pi


def layered_rotation_circuit(n: int, depth: int, seed: int):
    """Layers of RX, RY, RZ on every qubit (angles U[0, 2pi)), then a CNOT ladder q -> q+1."""
    rng = np.random.default_rng(seed)
    gates = []
    for _ in range(depth):
        for q in range(n):
            for kind in ("RX", "RY", "RZ"):
                gates.append((kind, q, float(rng.uniform(0.0, TWO_PI))))
        for q in range(n - 1):
            gates.append(("CNOT", q, q + 1))
    return gates


def u3_cz_circuit(n: int, layers: int, seed: int):
    """Layers of U3(theta, phi, lam ~ U[0, 2pi)) on every qubit, then CZ on a random perfect matching."""
    rng = np.random.default_rng(seed)
    gates = []
    for _ in range(layers):
        for q in range(n):
            th, ph, la = (float(x) for x in rng.uniform(0.0, TWO_PI, size=3))
            gates.append(("U3", q, th, ph, la))
        perm = rng.permutation(n)
        for i in range(0, n - 1, 2):
            gates.append(("CZ", int(perm[i]), int(perm[i + 1])))
    return gates


def hea_circuit(n: int, depth: int, seed: int):
    """Hardware-efficient ansatz: RY(theta) RZ(phi) on every qubit, then a CZ ring."""
    rng = np.random.default_rng(seed)
    gates = []
    for _ in range(depth):
        for q in range(n):
            gates.append(("RY", q, float(rng.uniform(0.0, TWO_PI))))
            gates.append(("RZ", q, float(rng.uniform(0.0, TWO_PI))))
        for q in range(n):
            if n > 1 and not (n == 2 and q == 1):
                gates.append(("CZ", q, (q + 1) % n))
    return gates


def random_pauli_terms(n: int, count: int, wmin: int, wmax: int, seed: int):
    """Terms (coef ~ N(0, 1), targets, pauli ids in {1, 2, 3}), weight ~ U{wmin..wmax} on distinct qubits."""
    rng = np.random.default_rng(seed)
    terms = []
    for _ in range(count):
        w = int(rng.integers(wmin, min(wmax, n) + 1))
        qs = [int(x) for x in rng.choice(n, size=w, replace=False)]
        ids = [int(x) for x in rng.integers(1, 4, size=w)]
        terms.append((float(rng.normal()), qs, ids))
    return terms


def uniforms(count: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).random(count)


def u3_matrix(theta, phi, lam) -> np.ndarray:
    """cppsim get_IBMQ_matrix (gate_factory.cpp:165-179)."""
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    e1, e2 = np.exp(1j * phi), np.exp(1j * lam)
    return np.array([[c, -e2 * s], [e1 * s, e1 * e2 * c]], dtype=np.complex128)


def count_gates(gates) -> int:
    return len(gates)


def to_circuit(gates, n: int):
    """Build a qulacs_b200.QuantumCircuit from a gate list."""
    from . import gate as G
    from .circuit import QuantumCircuit

    c = QuantumCircuit(n)
    for g in gates:
        k = g[0]
        if k in ("RX", "RY", "RZ"):
            c.add_gate(getattr(G, k)(g[1], g[2]))
        elif k == "U3":
            c.add_gate(G.DenseMatrix(g[1], u3_matrix(*g[2:5])))
        elif k == "CNOT":
            c.add_gate(G.CNOT(g[1], g[2]))
        elif k == "CZ":
            c.add_gate(G.CZ(g[1], g[2]))
        elif k == "SWAP":
            c.add_gate(G.SWAP(g[1], g[2]))
        elif k == "DENSE":
            c.add_gate(G.DenseMatrix(list(g[1]), g[2]))
        elif k == "DEPOL":
            qs = list(g[1])
            c.add_gate(G.DepolarizingNoise(qs[0], g[2]) if len(qs) == 1
                       else G.TwoQubitDepolarizingNoise(qs[0], qs[1], g[2]))
        else:
            raise ValueError(k)
    return c


def to_observable(terms, n: int):
    from .observable import Observable, PauliOperator

    obs = Observable(n)
    for coef, tl, ids in terms:
        obs.add_operator(PauliOperator(coef=coef, targets=tl, pauli_ids=ids))
    return obs


def rotation_matrix(kind: str, a: float) -> np.ndarray:
    """csim RX/RY/RZ matrices (update_ops_pauli_single.cpp:54-120): exp(+i a P / 2)."""
    c, s = math.cos(a / 2), math.sin(a / 2)
    if kind == "RX":
        return np.array([[c, 1j * s], [1j * s, c]])
    if kind == "RY":
        return np.array([[c, s], [-s, c]], dtype=np.complex128)
    return np.array([[c + 1j * s, 0], [0, c - 1j * s]])


def noisy_circuit(gates, p: float):
    """cppsim QuantumCircuit::add_noise_gate rule (circuit.cpp:167-190): depolarizing after every gate
    on its targets + controls (CNOT/CZ: (target, control))."""
    out = []
    for g in gates:
        out.append(g)
        k = g[0]
        if k in ("CNOT", "CZ"):
            out.append(("DEPOL", (g[2], g[1]), p))
        elif k == "DENSE":
            out.append(("DEPOL", tuple(g[1]), p))
        else:
            out.append(("DEPOL", (g[1],), p))
    return out
