"""Gate-list replay on a CPU implementation (test infrastructure only).

``run_on_cpu`` / ``run_on_cpu_dm`` apply a workload gate list (``qulacs_b200.workloads`` tuples) with
the oracle port or the compiled reference csim, gate by gate in csim's calling convention.  Only
tests, ``__graft_entry__.smoke()``, the fixture script and the CPU legs of ``bench.py`` use them.
"""
from __future__ import annotations

import numpy as np

from qulacs_b200.workloads import rotation_matrix, u3_matrix


def run_on_cpu(gates, state: np.ndarray, sim) -> None:
    """Apply a gate list with a CPU implementation (oracle port or reference csim) in place."""
    for g in gates:
        k = g[0]
        if k == "RX":
            sim.RX_gate(g[1], g[2], state)
        elif k == "RY":
            sim.RY_gate(g[1], g[2], state)
        elif k == "RZ":
            sim.RZ_gate(g[1], g[2], state)
        elif k == "U3":
            sim.single_qubit_dense_matrix_gate(g[1], u3_matrix(*g[2:5]), state)
        elif k == "CNOT":
            sim.CNOT_gate(g[1], g[2], state)
        elif k == "CZ":
            sim.CZ_gate(g[1], g[2], state)
        elif k == "SWAP":
            sim.SWAP_gate(g[1], g[2], state)
        elif k == "DENSE":
            sim.multi_qubit_dense_matrix_gate(list(g[1]), g[2], state)
        else:
            raise ValueError(k)


def run_on_cpu_dm(gates, rho: np.ndarray, sim) -> None:
    """Apply a gate list to a density matrix with a CPU implementation in place."""
    for g in gates:
        k = g[0]
        if k in ("RX", "RY", "RZ"):
            sim.dm_single_qubit_dense_matrix_gate(g[1], rotation_matrix(k, g[2]), rho)
        elif k == "U3":
            sim.dm_single_qubit_dense_matrix_gate(g[1], u3_matrix(*g[2:5]), rho)
        elif k == "CNOT":
            sim.dm_CNOT_gate(g[1], g[2], rho)
        elif k == "CZ":
            sim.dm_CZ_gate(g[1], g[2], rho)
        elif k == "DENSE":
            sim.dm_multi_qubit_dense_matrix_gate(list(g[1]), g[2], rho)
        elif k == "DEPOL":
            qs = list(g[1])
            if len(qs) == 1:
                sim.dm_depolarizing_noise(qs[0], g[2], rho)
            else:
                sim.dm_two_qubit_depolarizing_noise(qs[0], qs[1], g[2], rho)
        else:
            raise ValueError(k)
