"""Specialised pass kernels, host side: the generated CUDA C of staged passes (plain gates, FP64-fused
dense blocks, CNOT-folded ops, CZ, SWAP, HBM-direct first/last phases and tile round trips) compiles for
sm_100a at the pass kernel's occupancy (128 threads, 3 CTAs per SM) with at most a few bytes of spill,
and gate parameters passed as a kernel-parameter block, so circuits that differ only in angles share a
kernel."""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from qulacs_b200 import gate as G
from qulacs_b200 import workloads as W
from qulacs_b200.circuit import QuantumCircuit

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _compile(src: str, tmp_path, name: str) -> str:
    cu = tmp_path / f"{name}.cu"
    cu.write_text(src)
    r = subprocess.run([NVCC, "-cubin", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-Xptxas", "-v",
                        "-o", str(tmp_path / f"{name}.cubin"), str(cu)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return r.stderr


def _mixed_circuit(n: int, seed: int) -> QuantumCircuit:
    rng = np.random.default_rng(seed)
    c = W.to_circuit(W.layered_rotation_circuit(n, 2, seed) + W.u3_cz_circuit(n, 2, seed + 1), n)
    for _ in range(30):
        a, b = (int(x) for x in rng.choice(n, size=2, replace=False))
        r = rng.random()
        if r < 0.3:
            c.add_gate(G.SWAP(a, b))
        elif r < 0.6:
            m = np.linalg.qr(rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4)))[0]
            c.add_gate(G.DenseMatrix([a, b], m))
        else:
            c.add_gate(G.CNOT(a, b))
            c.add_gate(G.H(b))
    return c


@pytest.mark.skipif(not os.path.exists(NVCC) and shutil.which("nvcc") is None, reason="nvcc not available")
def test_generated_pass_sources_compile_without_spills(tmp_path):
    n = 20
    c = _mixed_circuit(n, 3)
    passes = 0
    for p in range(64):
        try:
            src = c.specialized_source(p)
        except ValueError:  # past the last pass
            break
        log = _compile(src, tmp_path, f"p{p}")
        assert "k_pass_spec" in log
        spills = [int(x) for x in re.findall(r"(\d+) bytes spill stores", log)]
        assert spills and max(spills) <= 64, log
        regs = [int(x) for x in re.findall(r"Used (\d+) registers", log)]
        assert regs and max(regs) <= 168  # 3 CTAs x 128 threads per SM
        passes += 1
    assert passes >= 2


def test_kernels_depend_on_structure_not_angles():
    """Two circuits with the same gates on the same qubits but different angles give the same kernel
    source (their parameters travel in the kernel's parameter block)."""
    n = 9
    srcs = []
    for a in (0.1, 2.7):
        c = QuantumCircuit(n)
        c.add_gate(G.RX(3, a))
        c.add_gate(G.CNOT(0, 5))
        c.add_gate(G.RZ(7, -a))
        srcs.append(c.specialized_source(0))
    assert srcs[0] == srcs[1]
    assert "__grid_constant__ PassParams P" in srcs[0]
