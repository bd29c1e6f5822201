"""The oracle port against the golden fixtures that the reference csim produced (CPU only)."""
import os

import numpy as np

from conftest import GOLDEN
from qulacs_b200 import workloads as W
from oracle import replay as R


def test_config1_golden(port):
    g = np.load(os.path.join(GOLDEN, "config1_n16.npz"))
    n = int(g["n"])
    gates = W.layered_rotation_circuit(n, int(g["depth"]), int(g["gate_seed"]))
    assert len(gates) == 630
    s = np.zeros(1 << n, dtype=np.complex128)
    s[0] = 1
    R.run_on_cpu(gates, s, port)
    assert np.max(np.abs(s[g["amp_index"]] - g["amps"])) <= 1e-13
    terms = W.random_pauli_terms(n, 64, 1, 4, int(g["term_seed"]))
    ev = np.array([port.expectation_value(tl, ids, s) for _, tl, ids in terms])
    assert np.max(np.abs(ev - g["term_values"])) <= 1e-13
    u = W.uniforms(1024, int(g["uniform_seed"]))
    assert np.array_equal(port.sampling_with_uniforms(s, u), g["samples"])


def test_u3cz_golden(port):
    g = np.load(os.path.join(GOLDEN, "u3cz_n10.npz"))
    n = int(g["n"])
    s = np.zeros(1 << n, dtype=np.complex128)
    s[0] = 1
    R.run_on_cpu(W.u3_cz_circuit(n, int(g["layers"]), int(g["gate_seed"])), s, port)
    assert np.max(np.abs(s - g["state"])) <= 1e-13


def test_noisy_dm_golden(port):
    g = np.load(os.path.join(GOLDEN, "noisy_dm_n5.npz"))
    n = int(g["n"])
    rho = np.zeros((1 << n, 1 << n), dtype=np.complex128)
    rho[0, 0] = 1
    R.run_on_cpu_dm(W.noisy_circuit(W.hea_circuit(n, int(g["depth"]), int(g["gate_seed"])), float(g["p"])), rho, port)
    assert np.max(np.abs(rho - g["rho"])) <= 1e-13
