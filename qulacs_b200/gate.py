"""Gate factory with the cppsim ``gate::`` names (cppsim/gate_factory.cpp).

Every gate carries its kind, qubits and parameters; ``update_quantum_state(state)`` applies it to a
``QuantumState`` through the csim-named C-ABI entry point, or to a ``DensityMatrix`` as
U rho U^dagger (or the exact channel for the noise gates).  Rotation conventions follow the
reference: ``RX(t, a)`` is exp(+i a X / 2) (csim/update_ops_pauli_single.cpp:54-66,
cppsim/gate_named_one.hpp:404-417), ``RotX(t, a)`` is exp(-i a X / 2) (gate_factory.cpp:152-163).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import GATE_KINDS, call

_SQ2 = 1.0 / math.sqrt(2.0)


def _arr_u(seq):
    return np.ascontiguousarray(np.asarray(seq, dtype=np.uint32))


class QuantumGateBase:
    """A gate: kind (C-ABI gate kind), targets, optional controls, parameters."""

    def __init__(self, kind: str, targets, params=(), controls=(), control_values=(), name: str = ""):
        self.kind = kind
        self.targets = [int(t) for t in targets]
        self.controls = [int(c) for c in controls]
        self.control_values = [int(v) for v in control_values]
        self.params = np.ascontiguousarray(np.asarray(params, dtype=np.float64).ravel())
        self.name = name or kind

    # cppsim QuantumGateBase accessors (gate.hpp:83-310)
    def get_target_index_list(self):
        return list(self.targets)

    def get_control_index_list(self):
        return list(self.controls)

    def get_control_value_list(self):
        return list(self.control_values)

    def get_control_index_value_list(self):
        return [[c, v] for c, v in zip(self.controls, self.control_values)]

    def get_name(self) -> str:
        return self.name

    def is_diagonal(self) -> bool:
        return self.kind in ("DIAGONAL", "RZ", "CZ") or (
            self.kind in ("PAULI", "PAULI_ROTATION") and all(int(i) in (0, 3) for i in self._pauli_ids()))

    def is_Pauli(self) -> bool:
        return self.kind == "PAULI" or self.name in ("I", "X", "Y", "Z")

    def is_parametric(self) -> bool:
        return False

    def copy(self) -> "QuantumGateBase":
        g = QuantumGateBase(self.kind, self.targets, self.params.copy(), self.controls, self.control_values, self.name)
        return g

    def add_control_qubit(self, qubit: int, control_value: int) -> None:
        if self.kind != "DENSE":
            raise NotImplementedError("controls can be added to DenseMatrix gates")
        if int(qubit) in self.targets or int(qubit) in self.controls:
            raise ValueError("control qubit is already a target or control of this gate")
        self.controls.append(int(qubit))
        self.control_values.append(int(control_value))

    def multiply_scalar(self, value: complex) -> None:
        """QuantumGateMatrix::multiply_scalar: matrix *= value (DenseMatrix / DiagonalMatrix gates)."""
        if self.kind not in ("DENSE", "DIAGONAL"):
            raise NotImplementedError("multiply_scalar is defined for matrix gates")
        self.params = _cplx_params((self.params[0::2] + 1j * self.params[1::2]) * complex(value))

    def _pauli_ids(self):
        n = len(self.targets)
        return [int(x) for x in self.params[:n]]

    def get_matrix(self) -> np.ndarray:
        """The gate's matrix on its targets (bit j of the index <-> targets[j]); controlled gates give
        the target matrix, as cppsim's set_matrix does (CNOT -> X, CZ -> Z)."""
        k = len(self.targets)
        if self.kind == "DENSE":
            md = 1 << k
            return (self.params[0::2] + 1j * self.params[1::2]).reshape(md, md).copy()
        if self.kind == "DIAGONAL":
            return np.diag(self.params[0::2] + 1j * self.params[1::2])
        if self.kind in ("RX", "RY", "RZ"):
            c, s = math.cos(self.params[0] / 2), math.sin(self.params[0] / 2)
            return {"RX": np.array([[c, 1j * s], [1j * s, c]]), "RY": np.array([[c, s], [-s, c]]),
                    "RZ": np.diag([c + 1j * s, c - 1j * s])}[self.kind]
        if self.kind == "CNOT":
            return _PAULI[1].copy()
        if self.kind == "CZ":
            return _PAULI[3].copy()
        if self.kind == "SWAP":
            return np.eye(4, dtype=np.complex128)[[0, 2, 1, 3]]
        if self.kind in ("PAULI", "PAULI_ROTATION"):
            m = np.ones((1, 1), dtype=np.complex128)
            for pid in self._pauli_ids():  # targets[j] <-> bit j: later targets are the left factors
                m = np.kron(_PAULI[pid], m)
            if self.kind == "PAULI":
                return m
            a = self.params[k]
            return math.cos(a / 2) * np.eye(m.shape[0]) + 1j * math.sin(a / 2) * m
        raise NotImplementedError(f"get_matrix for {self.name}")

    def get_inverse(self) -> "QuantumGateBase":
        """cppsim get_inverse: named one-qubit gates map to their named inverses (gate_named_one.cpp:3-48),
        rotations negate the angle (:51-62, gate_named_pauli.hpp:305), matrix gates take the adjoint
        (gate_matrix.cpp:330), CNOT/CZ/SWAP/Pauli are their own inverses; projections and noise have none."""
        if self.name in _NAMED_INVERSE:
            return _NAMED_INVERSE[self.name](self.targets[0])
        if self.name in ("Projection-0", "Projection-1"):
            raise NotImplementedError("Projection gate hasn't inverse gate")
        if self.kind in ("RX", "RY", "RZ"):
            return QuantumGateBase(self.kind, self.targets, [-self.params[0]], name=self.name)
        if self.kind == "PAULI_ROTATION":
            p = self.params.copy()
            p[-1] = -p[-1]
            return QuantumGateBase(self.kind, self.targets, p, name=self.name)
        if self.kind in ("CNOT", "CZ", "SWAP", "PAULI"):
            return self.copy()
        if self.kind == "DENSE":
            g = self.copy()
            g.params = _cplx_params(self.get_matrix().conj().T)
            return g
        if self.kind == "DIAGONAL":
            g = self.copy()
            g.params = _cplx_params((self.params[0::2] + 1j * self.params[1::2]).conj())
            return g
        raise NotImplementedError(f"Inverse of {self.name} gate is not Implemented")

    def to_string(self) -> str:
        """Debug text in cppsim's layout (gate.cpp:101-128); commutation flags are not tracked."""
        yn = lambda b: "yes" if b else "no"  # noqa: E731
        lines = [" *** gate info *** ", f" * gate name : {self.name}", " * target    : "]
        lines += [f" {t} : commute       " for t in self.targets]
        lines.append(" * control   : ")
        lines += [f" {c} : value {v}" for c, v in zip(self.controls, self.control_values)]
        lines += [f" * Pauli     : {yn(self.is_Pauli())}", " * Clifford  : no", " * Gaussian  : no",
                  f" * Parametric: {yn(self.is_parametric())}", f" * Diagonal  : {yn(self.is_diagonal())}"]
        return "\n".join(lines) + "\n"

    def __str__(self) -> str:
        return self.to_string()

    def _add_to(self, circuit_handle) -> None:
        t = _arr_u(self.targets)
        c = _arr_u(self.controls) if self.controls else _arr_u([0])
        cv = _arr_u(self.control_values) if self.controls else _arr_u([0])
        p = self.params if self.params.size else np.zeros(1)
        call("qs_circuit_add_gate", circuit_handle, GATE_KINDS[self.kind], t.ctypes.data_as(C.c_void_p), t.size,
             c.ctypes.data_as(C.c_void_p), cv.ctypes.data_as(C.c_void_p), len(self.controls),
             p.ctypes.data_as(C.c_void_p), self.params.size)

    def update_quantum_state(self, state) -> None:
        lib = _lib.load()
        h = C.c_void_p()
        n = state.get_qubit_count()
        call("qs_circuit_create", n, C.byref(h))
        try:
            self._add_to(h)
            if state.is_state_vector():
                call("qs_circuit_update_quantum_state", h, state.data_ptr(), state.dim, _lib.EXEC_GATE_BY_GATE,
                     state.stream)
            else:
                call("qs_circuit_update_density_matrix", h, state.data_ptr(), state.dim, _lib.EXEC_GATE_BY_GATE,
                     state.stream)
        finally:
            lib.qs_circuit_destroy(h)

    def __repr__(self):
        return f"{self.name}(targets={self.targets}, controls={self.controls})"


def _cplx_params(m) -> np.ndarray:
    m = np.asarray(m, dtype=np.complex128)
    out = np.empty(m.size * 2)
    out[0::2] = m.real.ravel()
    out[1::2] = m.imag.ravel()
    return out


def DenseMatrix(targets, matrix) -> QuantumGateBase:
    """cppsim gate::DenseMatrix; bit j of the matrix index <-> targets[j]."""
    if isinstance(targets, (int, np.integer)):
        targets = [int(targets)]
    m = np.asarray(matrix, dtype=np.complex128)
    md = 1 << len(targets)
    if m.shape != (md, md):
        raise ValueError(f"matrix must be {md}x{md}")
    return QuantumGateBase("DENSE", targets, _cplx_params(m), name="DenseMatrix")


def DiagonalMatrix(targets, diagonal) -> QuantumGateBase:
    if isinstance(targets, (int, np.integer)):
        targets = [int(targets)]
    d = np.asarray(diagonal, dtype=np.complex128).ravel()
    if d.size != 1 << len(targets):
        raise ValueError("diagonal length must be 2^k")
    return QuantumGateBase("DIAGONAL", targets, _cplx_params(d), name="DiagonalMatrix")


def _named(gate: QuantumGateBase, name: str) -> QuantumGateBase:
    gate.name = name
    return gate


# csim/constant.cpp:4-30; names as cppsim gate_named_one.hpp:87-323
def X(t):
    return _named(DenseMatrix(t, [[0, 1], [1, 0]]), "X")


def Y(t):
    return _named(DenseMatrix(t, [[0, -1j], [1j, 0]]), "Y")


def Z(t):
    return _named(DiagonalMatrix(t, [1, -1]), "Z")


def H(t):
    return _named(DenseMatrix(t, [[_SQ2, _SQ2], [_SQ2, -_SQ2]]), "H")


def S(t):
    return _named(DiagonalMatrix(t, [1, 1j]), "S")


def Sdag(t):
    return _named(DiagonalMatrix(t, [1, -1j]), "Sdag")


def T(t):
    return _named(DiagonalMatrix(t, [1, (1 + 1j) * _SQ2]), "T")


def Tdag(t):
    return _named(DiagonalMatrix(t, [1, (1 - 1j) * _SQ2]), "Tdag")


def sqrtX(t):
    return _named(DenseMatrix(t, [[0.5 + 0.5j, 0.5 - 0.5j], [0.5 - 0.5j, 0.5 + 0.5j]]), "sqrtX")


def sqrtXdag(t):
    return _named(DenseMatrix(t, [[0.5 - 0.5j, 0.5 + 0.5j], [0.5 + 0.5j, 0.5 - 0.5j]]), "sqrtXdag")


def sqrtY(t):
    return _named(DenseMatrix(t, [[0.5 + 0.5j, -0.5 - 0.5j], [0.5 + 0.5j, 0.5 + 0.5j]]), "sqrtY")


def sqrtYdag(t):
    return _named(DenseMatrix(t, [[0.5 - 0.5j, 0.5 - 0.5j], [-0.5 + 0.5j, 0.5 - 0.5j]]), "sqrtYdag")


def P0(t):
    return _named(DiagonalMatrix(t, [1, 0]), "Projection-0")


def P1(t):
    return _named(DiagonalMatrix(t, [0, 1]), "Projection-1")


def Identity(t):
    return _named(DiagonalMatrix(t, [1, 1]), "I")


_PAULI = [np.eye(2, dtype=np.complex128), np.array([[0, 1], [1, 0]], dtype=np.complex128),
          np.array([[0, -1j], [1j, 0]]), np.diag([1.0 + 0j, -1.0])]

_NAMED_INVERSE = {"I": Identity, "X": X, "Y": Y, "Z": Z, "H": H, "S": Sdag, "Sdag": S, "T": Tdag, "Tdag": T,
                  "sqrtX": sqrtXdag, "sqrtXdag": sqrtX, "sqrtY": sqrtYdag, "sqrtYdag": sqrtY}


def RX(t, angle):
    return QuantumGateBase("RX", [t], [angle], name="X-rotation")


def RY(t, angle):
    return QuantumGateBase("RY", [t], [angle], name="Y-rotation")


def RZ(t, angle):
    return QuantumGateBase("RZ", [t], [angle], name="Z-rotation")


def RotX(t, angle):
    return RX(t, -angle)


def RotY(t, angle):
    return RY(t, -angle)


def RotZ(t, angle):
    return RZ(t, -angle)


RotInvX, RotInvY, RotInvZ = RX, RY, RZ


def get_IBMQ_matrix(theta, phi, lam) -> np.ndarray:
    """cppsim gate_factory.cpp:165-179."""
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    e1, e2 = np.exp(1j * phi), np.exp(1j * lam)
    return np.array([[c, -e2 * s], [e1 * s, e1 * e2 * c]], dtype=np.complex128)


def U1(t, lam):
    return DenseMatrix(t, get_IBMQ_matrix(0, 0, lam))


def U2(t, phi, lam):
    return DenseMatrix(t, get_IBMQ_matrix(math.pi / 2, phi, lam))


def U3(t, theta, phi, lam):
    return DenseMatrix(t, get_IBMQ_matrix(theta, phi, lam))


def CNOT(control, target):
    if control == target:
        raise ValueError("CNOT: control and target are the same qubit")
    return QuantumGateBase("CNOT", [control, target], name="CNOT")


def CZ(control, target):
    if control == target:
        raise ValueError("CZ: control and target are the same qubit")
    return QuantumGateBase("CZ", [control, target], name="CZ")


def SWAP(a, b):
    if a == b:
        raise ValueError("SWAP: duplicated qubit")
    return QuantumGateBase("SWAP", [a, b], name="SWAP")


def _check_pauli(targets, pauli_ids):
    if len(targets) != len(pauli_ids):
        raise ValueError("target list and Pauli id list differ in length")
    if len(set(int(t) for t in targets)) != len(targets):
        raise ValueError("target list contains duplicated values")
    if any(int(i) > 3 for i in pauli_ids):
        raise ValueError("Pauli ids must be 0..3 (I, X, Y, Z)")


def Pauli(targets, pauli_ids):
    """cppsim gate::Pauli (gate_factory.cpp:255-266): the product of pauli_ids[j] on targets[j]."""
    _check_pauli(targets, pauli_ids)
    return QuantumGateBase("PAULI", targets, list(pauli_ids), name="Pauli")


def PauliRotation(targets, pauli_ids, angle):
    """cppsim gate::PauliRotation (gate_factory.cpp:267-280): exp(+i angle P / 2)."""
    _check_pauli(targets, pauli_ids)
    return QuantumGateBase("PAULI_ROTATION", targets, list(pauli_ids) + [angle], name="Pauli-rotation")


def RandomUnitary(targets, seed: int | None = None) -> QuantumGateBase:
    """cppsim gate::RandomUnitary (gate_factory.cpp:322-380): a Haar-random dense matrix on ``targets``;
    with a seed, the reference's matrix for that seed (same mt19937_64 normal draws, same QR phase
    convention)."""
    if isinstance(targets, (int, np.integer)):
        targets = [int(targets)]
    targets = [int(t) for t in targets]
    if len(set(targets)) != len(targets):
        raise ValueError("RandomUnitary: target list contains duplicated values")
    if seed is None:
        seed = int(np.random.SeedSequence().entropy & 0xFFFFFFFF)
    k = len(targets)
    m = np.zeros(2 * 4 ** k)
    _lib.load()
    call("qs_random_unitary_matrix", k, int(seed) & 0xFFFFFFFF, m.ctypes.data_as(C.c_void_p))
    return DenseMatrix(targets, m.view(np.complex128).reshape(1 << k, 1 << k))


def DepolarizingNoise(t, prob):
    """cppsim gate_factory.cpp:456-466 (exact channel on a DensityMatrix; sampled by NoiseSimulator).
    Named "Probabilistic" like the reference's QuantumGate_Probabilistic."""
    return QuantumGateBase("DEPOLARIZING", [t], [prob], name="Probabilistic")


def TwoQubitDepolarizingNoise(t1, t2, prob):
    """cppsim gate_factory.cpp:471-500 (exact channel on a DensityMatrix; sampled by NoiseSimulator)."""
    if t1 == t2:
        raise ValueError("TwoQubitDepolarizingNoise: duplicated qubit")
    return QuantumGateBase("DEPOLARIZING", [t1, t2], [prob], name="Probabilistic")


# ---- matrix utilities (cppsim gate_merge.cpp:19-356, python/cppsim_wrapper.cpp gate.merge / add /
# to_matrix_gate) and FusedSWAP (update_ops_named_FusedSWAP.cpp:19-60), composed on the host ----
def _action(g: QuantumGateBase):
    """(qubits, matrix): the gate's full action on its qubits, controls included (bit j <-> qubits[j])."""
    if g.kind == "DEPOLARIZING":
        raise NotImplementedError("a noise channel has no matrix")
    if g.kind == "CNOT":
        return list(g.targets), np.eye(4, dtype=np.complex128)[:, [0, 3, 2, 1]]
    if g.kind == "CZ":
        return list(g.targets), np.diag([1, 1, 1, -1]).astype(np.complex128)
    m = g.get_matrix()
    if not g.controls:
        return list(g.targets), m
    k, nc = len(g.targets), len(g.controls)
    full = np.eye(1 << (k + nc), dtype=np.complex128)
    c = sum(v << j for j, v in enumerate(g.control_values)) << k
    full[c:c + (1 << k), c:c + (1 << k)] = m
    return list(g.targets) + list(g.controls), full


def _embed(qubits, m, union):
    """m over `qubits` as a matrix over `union` (identity on the other qubits)."""
    pos = [union.index(q) for q in qubits]
    u, k = len(union), len(pos)
    xs = np.arange(1 << u)
    local = np.zeros_like(xs)
    for j, p in enumerate(pos):
        local |= ((xs >> p) & 1) << j
    rest = xs & ~sum(1 << p for p in pos)
    scat = np.array([sum(((yl >> j) & 1) << p for j, p in enumerate(pos)) for yl in range(1 << k)])
    full = np.zeros((1 << u, 1 << u), dtype=np.complex128)
    full[rest[None, :] | scat[:, None], xs[None, :]] = m[:, local]
    return full


def _union(*gates):
    out = []
    for g in gates:
        for q in _action(g)[0]:
            if q not in out:
                out.append(q)
    return out


def to_matrix_gate(g: QuantumGateBase) -> QuantumGateBase:
    """gate::to_matrix_gate: a DenseMatrix gate with the same action (controls folded in)."""
    q, m = _action(g)
    return DenseMatrix(q, m)


def merge(first: QuantumGateBase, then: QuantumGateBase) -> QuantumGateBase:
    """gate::merge(first, then): the product `then` x `first` over the union of their qubits."""
    u = _union(first, then)
    return DenseMatrix(u, _embed(*_action(then), u) @ _embed(*_action(first), u))


def add(a: QuantumGateBase, b: QuantumGateBase) -> QuantumGateBase:
    """gate::add(a, b): the sum of the two matrices over the union of their qubits."""
    u = _union(a, b)
    return DenseMatrix(u, _embed(*_action(a), u) + _embed(*_action(b), u))


def FusedSWAP(t0: int, t1: int, block_size: int) -> QuantumGateBase:
    """gate::FusedSWAP: qubits t0 + i and t1 + i exchanged for i < block_size, as one permutation
    matrix over the 2 x block_size qubits (block_size <= 6)."""
    lo, hi = min(t0, t1), max(t0, t1)
    if block_size < 1 or hi <= lo + block_size - 1:
        raise ValueError("FusedSWAP: the blocks overlap")
    if block_size > 6:
        raise NotImplementedError("FusedSWAP: at most 6 qubits a block")
    b = block_size
    qs = [t0 + i for i in range(b)] + [t1 + i for i in range(b)]
    x = np.arange(1 << (2 * b))
    y = (x >> b) | ((x & ((1 << b) - 1)) << b)
    m = np.zeros((1 << (2 * b), 1 << (2 * b)), dtype=np.complex128)
    m[y, x] = 1.0
    g = DenseMatrix(qs, m)
    g.name = "FusedSWAP"
    return g
