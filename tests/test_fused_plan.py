"""Fused-path planning on the host (CPU only): the FP64 block matrices, replayed in order on the
tile qubits, reproduce the gate-by-gate oracle; the bf16 hi/lo operand image in the UMMA K-major
core-matrix layout reconstructs the real-ified block matrix."""
import ctypes as C

import numpy as np
import pytest

from conftest import random_state
from qulacs_b200 import workloads as W
from qulacs_b200._lib import call
from oracle import replay as R


def kmajor_off(r, k):
    """K-major, 128-byte swizzle (8-row x 128 B atoms, 16-byte chunk index XOR row % 8)."""
    return ((r >> 3) * 2 + (k >> 6)) * 1024 + (r & 7) * 128 + ((((k >> 3) & 7) ^ (r & 7)) << 4) + (k & 7) * 2


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
    R.run_on_cpu(gates, want, port)
    got = s0.copy()
    for qubits, U, _, tile in blocks:
        assert set(qubits) <= set(int(t) for t in tile)
        assert len(set(qubits)) == 6
        assert np.allclose(U @ U.conj().T, np.eye(64), atol=1e-12)
        port.multi_qubit_dense_matrix_gate(qubits, U, got)
    assert np.max(np.abs(got - want)) <= 1e-12


def block_layout(circ, index):
    rows = np.zeros(7, dtype=np.int32)
    ks = np.zeros(6, dtype=np.int32)
    cos = np.zeros(7, dtype=np.uint32)
    tabs = np.zeros(640, dtype=np.uint32)
    call("qs_circuit_fused_block_layout", circ._h, index, rows.ctypes.data_as(C.c_void_p),
         ks.ctypes.data_as(C.c_void_p), cos.ctypes.data_as(C.c_void_p), tabs.ctypes.data_as(C.c_void_p))
    return rows, ks, cos, tabs


def realified(U, rows, ks):
    """A[y][k] of the block operand in the exported orders: row y = (part, output index) by `rows`,
    column K = part (bit 0) | input index bits (by `ks`) << 1."""
    y = np.arange(128)
    xo = np.zeros(128, dtype=np.int64)
    po = np.zeros(128, dtype=np.int64)
    for i, src in enumerate(rows):
        bit = (y >> i) & 1
        if src == 6:
            po = bit
        else:
            xo |= bit << int(src)
    k = np.arange(128)
    pi = k & 1
    xi = np.zeros(128, dtype=np.int64)
    for i, src in enumerate(ks):
        xi |= ((k >> (1 + i)) & 1) << int(src)
    u = U[xo[:, None], xi[None, :]]
    return np.where(po[:, None] == 0, np.where(pi[None, :] == 0, u.real, -u.imag),
                    np.where(pi[None, :] == 0, u.imag, u.real))


def test_operand_image_layout_and_split():
    n = 10
    circ = W.to_circuit(W.u3_cz_circuit(n, 2, seed=9), n)
    _, blocks = export_blocks(circ)
    for index in range(len(blocks)):
        qubits, U, img, _ = blocks[index]
        rows, ks, _, _ = block_layout(circ, index)
        assert sorted(rows.tolist()) == list(range(7))
        assert sorted(ks.tolist()) == list(range(6))
        A = realified(U, rows, ks)
        r, k = np.meshgrid(np.arange(128), np.arange(128), indexing="ij")
        off = kmajor_off(r, k) // 2
        hi = bf16_to_f32(img[:128 * 128][off])
        lo = bf16_to_f32(img[128 * 128:][off])
        assert np.max(np.abs(hi - A)) <= 2.0 ** -8 * np.max(np.abs(A)) + 1e-30
        assert np.max(np.abs(hi.astype(np.float64) + lo - A)) <= 2.0 ** -16 * np.max(np.abs(A))
        # every byte offset is used exactly once (the layout is a bijection)
        assert np.unique(off).size == 128 * 128


def tswz(u):
    return u ^ ((((u >> 5) ^ (u >> 9)) & 15) << 1)


def emulate_fused(circ, n, state):
    """Replays the fused kernel's data movement on the CPU from the exported operand images and index
    tables: state -> B gather (global offsets gn | gj), A (hi + lo) times B in FP64, accumulator -> next B
    operand or output tile through rowtab[y] ^ coltab[n]."""
    npasses, blocks = export_blocks(circ)
    groups = []
    for index, (_, _, img, tile) in enumerate(blocks):
        key = tuple(int(t) for t in tile)
        if not groups or groups[-1][0] != key:
            groups.append((key, []))
        groups[-1][1].append(index)
    assert len(groups) == npasses
    r, k = np.meshgrid(np.arange(128), np.arange(128), indexing="ij")
    koff = kmajor_off(r, k) // 2
    state = state.copy()
    for tile, idxs in groups:
        m = len(tile)
        N = 1 << (m - 6)
        u = np.arange(1 << m)
        local = np.zeros(1 << m, dtype=np.int64)
        for j, q in enumerate(tile):
            local |= ((u >> j) & 1) << q
        others = [q for q in range(n) if q not in tile]
        layouts = [block_layout(circ, i) for i in idxs]
        A = []
        for i in idxs:
            img = blocks[i][2]
            A.append(bf16_to_f32(img[:128 * 128][koff]).astype(np.float64)
                     + bf16_to_f32(img[128 * 128:][koff]))
        for T in range(1 << len(others)):
            base = 0
            for j, q in enumerate(others):
                base |= ((T >> j) & 1) << q
            tabs = layouts[0][3]
            gn = np.ascontiguousarray(tabs[256:512]).view(np.uint64)[:N].astype(np.int64)  # global offsets
            gj = np.ascontiguousarray(tabs[512:640]).view(np.uint64).astype(np.int64)
            v = state[base | gn[:, None] | gj[None, :]]             # (N, 64), read straight from the state
            B = np.empty((N, 128))
            B[:, 0::2], B[:, 1::2] = v.real, v.imag
            for b in range(len(idxs)):
                tabs = layouts[b][3]
                D = A[b] @ B.T                                        # (128, N)
                rt, ct = tabs[:128].astype(np.int64), tabs[128:128 + N].astype(np.int64)
                dst = rt[:, None] ^ ct[None, :]
                if b + 1 < len(idxs):
                    flat = np.full(N * 128, np.nan)
                    assert np.unique(dst).size == N * 128 and np.all(dst % 2 == 0)
                    flat[dst // 2] = D
                    B = flat[kmajor_off(np.arange(N)[:, None], np.arange(128)[None, :]) // 2]
                else:
                    out = np.full(2 << m, np.nan)
                    assert np.unique(dst).size == 2 << m
                    out[dst] = D
                    state[base | local] = out[2 * tswz(u)] + 1j * out[2 * tswz(u) + 1]
    return state


@pytest.mark.parametrize("n,layers,seed", [(13, 6, 21), (14, 8, 22), (11, 4, 23)])
def test_kernel_dataflow_emulation(port, n, layers, seed):
    gates = W.u3_cz_circuit(n, layers, seed=seed) + W.layered_rotation_circuit(n, 1, seed=seed + 100)
    circ = W.to_circuit(gates, n)
    s0 = random_state(n, np.random.default_rng(seed))
    want = s0.copy()
    R.run_on_cpu(gates, want, port)
    got = emulate_fused(circ, n, s0)
    assert not np.any(np.isnan(got))
    # bf16 hi + lo operands carry ~16 significant bits per factor (the B operand is exact here)
    assert np.max(np.abs(got - want)) <= 1e-4 * np.max(np.abs(want))
