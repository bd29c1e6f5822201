"""State manipulation on the B200 (tensor product, qubit permutation, dropped qubits, partial traces,
reflection, FusedSWAP) against numpy restatements of the reference loops: stat_ops.cpp:111-158,
stat_ops_dm.cpp:193-296, update_ops_reflection.cpp:14-27, update_ops_named_FusedSWAP.cpp:21-25."""
import ctypes as C

import numpy as np
import pytest

from conftest import AMP_TOL, random_density_matrix, random_state
from qulacs_b200 import DensityMatrix, QuantumState
from qulacs_b200 import state as S
from qulacs_b200._lib import call

pytestmark = pytest.mark.gpu


def dev(vec):
    s = QuantumState(int(np.log2(vec.size)))
    s.load(vec)
    return s


def dev_dm(rho):
    d = DensityMatrix(int(np.log2(rho.shape[0])))
    d.load(rho)
    return d


def _perm_index(i, order):
    return sum(1 << order[q] for q in range(len(order)) if (i >> q) & 1)


def test_tensor_products():
    rng = np.random.default_rng(1400)
    a, b = random_state(3, rng), random_state(5, rng)
    got = S.tensor_product(dev(a), dev(b))
    assert got.get_qubit_count() == 8
    assert np.max(np.abs(got.get_vector() - np.kron(a, b))) <= AMP_TOL
    ra, rb = random_density_matrix(2, rng), random_density_matrix(3, rng)
    got = S.tensor_product(dev_dm(ra), dev_dm(rb))
    assert np.max(np.abs(got.get_matrix() - np.kron(ra, rb))) <= AMP_TOL
    with pytest.raises(TypeError):
        S.tensor_product(dev(a), dev_dm(ra))


def test_permutate_qubit():
    rng = np.random.default_rng(1410)
    n = 8
    a = random_state(n, rng)
    order = [int(x) for x in rng.permutation(n)]
    got = S.permutate_qubit(dev(a), order).get_vector()
    want = np.array([a[_perm_index(i, order)] for i in range(1 << n)])
    assert np.array_equal(got, want)
    rho = random_density_matrix(4, rng)
    order = [2, 0, 3, 1]
    got = S.permutate_qubit(dev_dm(rho), order).get_matrix()
    p = [_perm_index(i, order) for i in range(16)]
    assert np.array_equal(got, rho[np.ix_(p, p)])
    with pytest.raises(ValueError):
        S.permutate_qubit(dev(a), [0, 1, 2])
    with pytest.raises(ValueError):
        S.permutate_qubit(dev(a), [0, 0, 1, 2, 3, 4, 5, 6])


def test_drop_qubit():
    rng = np.random.default_rng(1420)
    n = 9
    a = random_state(n, rng)
    target, proj = [6, 1, 3], [1, 0, 1]
    got = S.drop_qubit(dev(a), target, proj).get_vector()
    keep = [q for q in range(n) if q not in target]
    want = np.empty(1 << (n - 3), dtype=np.complex128)
    for i in range(want.size):
        src = sum(1 << keep[j] for j in range(len(keep)) if (i >> j) & 1)
        src |= sum(1 << t for t, v in zip(target, proj) if v)
        want[i] = a[src]
    assert np.array_equal(got, want)


@pytest.mark.parametrize("from_dm", [False, True])
def test_partial_trace(from_dm):
    rng = np.random.default_rng(1430 + from_dm)
    n = 6
    traced = [4, 1]
    keep = [q for q in range(n) if q not in traced]
    if from_dm:
        rho = random_density_matrix(n, rng)
        got = S.partial_trace(dev_dm(rho), traced).get_matrix()
    else:
        a = random_state(n, rng)
        rho = np.outer(a, a.conj())
        got = S.partial_trace(dev(a), traced).get_matrix()
    d = 1 << len(keep)
    want = np.zeros((d, d), dtype=np.complex128)
    for y in range(d):
        for x in range(d):
            by = sum(1 << keep[j] for j in range(len(keep)) if (y >> j) & 1)
            bx = sum(1 << keep[j] for j in range(len(keep)) if (x >> j) & 1)
            for t in range(1 << len(traced)):
                m = sum(1 << traced[j] for j in range(len(traced)) if (t >> j) & 1)
                want[y, x] += rho[by ^ m, bx ^ m]
    assert np.max(np.abs(got - want)) <= AMP_TOL
    assert abs(np.trace(got) - np.trace(rho)) <= 1e-12


def test_reflection_and_fused_swap(port):
    rng = np.random.default_rng(1440)
    n = 10
    r, a = random_state(n, rng), random_state(n, rng)
    s, rs = dev(a), dev(r)  # both held: a temporary's device buffer would be freed before the call
    call("qs_reflection_gate", rs.data_ptr(), s.data_ptr(), s.dim, None)
    want = 2 * np.vdot(r, a) * r - a
    assert np.max(np.abs(s.get_vector() - want)) <= AMP_TOL
    s = dev(a)
    call("qs_FusedSWAP_gate", 1, 6, 3, s.data_ptr(), s.dim, None)
    want = a.copy()
    for i in range(3):
        port.SWAP_gate(1 + i, 6 + i, want)
    assert np.array_equal(s.get_vector(), want)
    with pytest.raises(ValueError):
        call("qs_FusedSWAP_gate", 1, 3, 3, s.data_ptr(), s.dim, None)  # the blocks overlap
    with pytest.raises(ValueError):
        call("qs_FusedSWAP_gate", 0, 8, 3, s.data_ptr(), s.dim, None)  # past the last qubit
    h = QuantumState(n)
    call("qs_initialize_Haar_random_state", h.data_ptr(), h.dim, None)
    assert abs(h.get_squared_norm() - 1.0) <= 1e-12


def test_merged_and_fused_swap_gates_on_device(port):
    """gate.merge / to_matrix_gate / FusedSWAP (composed on the host) act like their parts."""
    from qulacs_b200 import gate as G
    rng = np.random.default_rng(1450)
    n = 9
    a = random_state(n, rng)
    parts = [G.H(2), G.CNOT(2, 7), G.RZ(7, 0.4), G.CZ(0, 2)]
    m = parts[0]
    for g in parts[1:]:
        m = G.merge(m, g)
    s, t = dev(a), dev(a)
    for g in parts:
        g.update_quantum_state(s)
    m.update_quantum_state(t)
    assert np.max(np.abs(s.get_vector() - t.get_vector())) <= AMP_TOL
    u = dev(a)
    G.to_matrix_gate(G.CNOT(4, 1)).update_quantum_state(u)
    want = a.copy()
    port.CNOT_gate(4, 1, want)
    assert np.max(np.abs(u.get_vector() - want)) <= AMP_TOL
    f = dev(a)
    G.FusedSWAP(0, 5, 3).update_quantum_state(f)
    want = a.copy()
    for i in range(3):
        port.SWAP_gate(i, 5 + i, want)
    assert np.max(np.abs(f.get_vector() - want)) <= AMP_TOL
