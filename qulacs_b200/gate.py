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

    def get_name(self) -> str:
        return self.name

    def copy(self) -> "QuantumGateBase":
        g = QuantumGateBase(self.kind, self.targets, self.params.copy(), self.controls, self.control_values, self.name)
        return g

    def add_control_qubit(self, qubit: int, control_value: int) -> None:
        if self.kind != "DENSE":
            raise NotImplementedError("controls can be added to DenseMatrix gates")
        self.controls.append(int(qubit))
        self.control_values.append(int(control_value))

    def get_matrix(self) -> np.ndarray:
        k = len(self.targets)
        if self.kind == "DENSE":
            md = 1 << k
            return (self.params[0::2] + 1j * self.params[1::2]).reshape(md, md)
        if self.kind == "DIAGONAL":
            return np.diag(self.params[0::2] + 1j * self.params[1::2])
        raise NotImplementedError(f"get_matrix for {self.kind}")

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


# csim/constant.cpp:4-30
def X(t):
    return DenseMatrix(t, [[0, 1], [1, 0]])


def Y(t):
    return DenseMatrix(t, [[0, -1j], [1j, 0]])


def Z(t):
    return DiagonalMatrix(t, [1, -1])


def H(t):
    return DenseMatrix(t, [[_SQ2, _SQ2], [_SQ2, -_SQ2]])


def S(t):
    return DiagonalMatrix(t, [1, 1j])


def Sdag(t):
    return DiagonalMatrix(t, [1, -1j])


def T(t):
    return DiagonalMatrix(t, [1, (1 + 1j) * _SQ2])


def Tdag(t):
    return DiagonalMatrix(t, [1, (1 - 1j) * _SQ2])


def sqrtX(t):
    return DenseMatrix(t, [[0.5 + 0.5j, 0.5 - 0.5j], [0.5 - 0.5j, 0.5 + 0.5j]])


def sqrtXdag(t):
    return DenseMatrix(t, [[0.5 - 0.5j, 0.5 + 0.5j], [0.5 + 0.5j, 0.5 - 0.5j]])


def sqrtY(t):
    return DenseMatrix(t, [[0.5 + 0.5j, -0.5 - 0.5j], [0.5 + 0.5j, 0.5 + 0.5j]])


def sqrtYdag(t):
    return DenseMatrix(t, [[0.5 - 0.5j, 0.5 - 0.5j], [-0.5 + 0.5j, 0.5 - 0.5j]])


def P0(t):
    return DiagonalMatrix(t, [1, 0])


def P1(t):
    return DiagonalMatrix(t, [0, 1])


def Identity(t):
    return DiagonalMatrix(t, [1, 1])


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


def Pauli(targets, pauli_ids):
    return QuantumGateBase("PAULI", targets, list(pauli_ids), name="Pauli")


def PauliRotation(targets, pauli_ids, angle):
    return QuantumGateBase("PAULI_ROTATION", targets, list(pauli_ids) + [angle], name="PauliRotation")


def DepolarizingNoise(t, prob):
    """cppsim gate_factory.cpp:456-466 (exact channel on a DensityMatrix)."""
    return QuantumGateBase("DEPOLARIZING", [t], [prob], name="DepolarizingNoise")


def TwoQubitDepolarizingNoise(t1, t2, prob):
    """cppsim gate_factory.cpp:471-500 (exact channel on a DensityMatrix)."""
    if t1 == t2:
        raise ValueError("TwoQubitDepolarizingNoise: duplicated qubit")
    return QuantumGateBase("DEPOLARIZING", [t1, t2], [prob], name="TwoQubitDepolarizingNoise")
