"""Fused-path planning on the host (CPU only): the FP64 block matrices, replayed in order on the
tile qubits, reproduce the gate-by-gate oracle; the bf16 hi/lo operand image in the UMMA K-major
core-matrix layout reconstructs the real-ified block matrix."""
import ctypes as C

import numpy as np

from conftest import random_state
from qulacs_b200 import workloads as W
from qulacs_b200._lib import call


def kmajor_off(r, k):
    return (r >> 3) * 2048 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2


def bf16_to_f32(h):
    return (np.asarray(h, dtype=np.uint32) << 16).view(np.float32)


def export_blocks(circ):
    passes, blocks = C.c_uint(), C.c_uint()
    call("qs_circuit_fused_stats", circ._h, C.byref(passes), C.byref(blocks))
    out = []
    for b in range(blocks.value):
        tq = np.zeros(13, dtype=np.uint32)
        m = C.c_int()
        bits = np.zeros(6, dtype=np.uint32)
        U = np.zeros(64 * 64, dtype=np.complex128)
        img = np.zeros(2 * 128 * 128, dtype=np.uint16)
        call("qs_circuit_fused_block_export", circ._h, b, tq.ctypes.data_as(C.c_void_p), C.byref(m),
             bits.ctypes.data_as(C.c_void_p), U.ctypes.data_as(C.c_void_p), img.ctypes.data_as(C.c_void_p))
        qubits = [int(tq[int(j)]) for j in bits]
        out.append((qubits, U.reshape(64, 64), img, tq[:m.value].copy()))
    return passes.value, out


def test_fused_blocks_reproduce_circuit(port):
    n = 12
    gates = W.u3_cz_circuit(n, 5, seed=5) + W.layered_rotation_circuit(n, 2, seed=6)
    circ = W.to_circuit(gates, n)
    npasses, blocks = export_blocks(circ)
    assert 1 <= npasses <= len(gates)
    assert len(blocks) < len(gates)
    s0 = random_state(n, np.random.default_rng(1))
    want = s0.copy()
    W.run_on_cpu(gates, want, port)
    got = s0.copy()
    for qubits, U, _, tile in blocks:
        assert set(qubits) <= set(int(t) for t in tile)
        assert len(set(qubits)) == 6
        assert np.allclose(U @ U.conj().T, np.eye(64), atol=1e-12)
        port.multi_qubit_dense_matrix_gate(qubits, U, got)
    assert np.max(np.abs(got - want)) <= 1e-12


def test_operand_image_layout_and_split():
    n = 10
    circ = W.to_circuit(W.u3_cz_circuit(n, 2, seed=9), n)
    _, blocks = export_blocks(circ)
    qubits, U, img, _ = blocks[0]
    A = np.block([[U.real, -U.imag], [U.imag, U.real]])
    r, k = np.meshgrid(np.arange(128), np.arange(128), indexing="ij")
    off = kmajor_off(r, k) // 2
    hi = bf16_to_f32(img[:128 * 128][off])
    lo = bf16_to_f32(img[128 * 128:][off])
    assert np.max(np.abs(hi - A)) <= 2.0 ** -8 * np.max(np.abs(A)) + 1e-30
    assert np.max(np.abs(hi.astype(np.float64) + lo - A)) <= 2.0 ** -16 * np.max(np.abs(A))
    # every byte offset is used exactly once (the layout is a bijection)
    assert np.unique(off).size == 128 * 128
