"""Python loader for the oracle (test infrastructure only).

Two CPU implementations share one calling convention (numpy complex128 arrays, csim argument order):

* ``port()``: the C restatement in ``oracle/qs_oracle.c`` (always buildable with gcc).
* ``reference()``: the reference csim itself, compiled from its own sources by ``oracle/Makefile``
  into ``oracle/_ref/libcsim_ref.so``; ``None`` when it was not built.

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libcsim_ref.so")

_U = C.c_uint
_IT = C.c_ulonglong
_D = C.c_double
_P = C.c_void_p
_lock = threading.Lock()


def build_port() -> str:
    """Compile the C restatement with gcc if its shared object is missing or stale."""
    src = os.path.join(HERE, "qs_oracle.c")
    with _lock:
        if not os.path.exists(PORT_SO) or os.path.getmtime(PORT_SO) < os.path.getmtime(src):
            subprocess.check_call(["make", "-s", "-C", HERE, "_build/liboracle.so"])
    return PORT_SO


def build_reference(ref_root: str = "/root/reference") -> str | None:
    """Compile the reference csim when its sources are present (never on a machine without them)."""
    if not os.path.isdir(os.path.join(ref_root, "src", "csim")):
        return REF_SO if os.path.exists(REF_SO) else None
    subprocess.check_call(["make", "-s", "-j8", "-C", HERE, "ref", f"REF={ref_root}"])
    return REF_SO


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_P)


def _u32(seq) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(seq, dtype=np.uint32))


def _c128(m) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(m, dtype=np.complex128))


class CpuSim:
    """numpy front end over one of the two CPU libraries; every call updates ``state`` in place."""

    def __init__(self, path: str, prefix: str):
        self.path = path
        self.prefix = prefix
        self.lib = C.CDLL(path)

    def _f(self, name, restype=None):
        fn = getattr(self.lib, self.prefix + name)
        fn.restype = restype
        return fn

    # ---- state-vector gates ----
    def single_qubit_dense_matrix_gate(self, t, m, s):
        m = _c128(m)
        self._f("single_qubit_dense_matrix_gate")(_U(t), _ptr(m), _ptr(s), _IT(s.size))

    def single_qubit_diagonal_matrix_gate(self, t, d, s):
        d = _c128(d)
        self._f("single_qubit_diagonal_matrix_gate")(_U(t), _ptr(d), _ptr(s), _IT(s.size))

    def single_qubit_phase_gate(self, t, phase, s):
        p = _c128([phase])
        self._f("single_qubit_phase_gate")(_U(t), _ptr(p), _ptr(s), _IT(s.size))

    def RX_gate(self, t, a, s):
        self._f("RX_gate")(_U(t), _D(a), _ptr(s), _IT(s.size))

    def RY_gate(self, t, a, s):
        self._f("RY_gate")(_U(t), _D(a), _ptr(s), _IT(s.size))

    def RZ_gate(self, t, a, s):
        self._f("RZ_gate")(_U(t), _D(a), _ptr(s), _IT(s.size))

    def CNOT_gate(self, c, t, s):
        self._f("CNOT_gate")(_U(c), _U(t), _ptr(s), _IT(s.size))

    def CZ_gate(self, c, t, s):
        self._f("CZ_gate")(_U(c), _U(t), _ptr(s), _IT(s.size))

    def SWAP_gate(self, a, b, s):
        self._f("SWAP_gate")(_U(a), _U(b), _ptr(s), _IT(s.size))

    def double_qubit_dense_matrix_gate_c(self, t1, t2, m, s):
        m = _c128(m)
        self._f("double_qubit_dense_matrix_gate_c")(_U(t1), _U(t2), _ptr(m), _ptr(s), _IT(s.size))

    def multi_qubit_dense_matrix_gate(self, tl, m, s):
        tl, m = _u32(tl), _c128(m)
        self._f("multi_qubit_dense_matrix_gate")(_ptr(tl), _U(tl.size), _ptr(m), _ptr(s), _IT(s.size))

    def multi_qubit_diagonal_matrix_gate(self, tl, d, s):
        tl, d = _u32(tl), _c128(d)
        self._f("multi_qubit_diagonal_matrix_gate")(_ptr(tl), _U(tl.size), _ptr(d), _ptr(s), _IT(s.size))

    def multi_qubit_control_single_qubit_dense_matrix_gate(self, cl, cv, t, m, s):
        cl, cv, m = _u32(cl), _u32(cv), _c128(m)
        self._f("multi_qubit_control_single_qubit_dense_matrix_gate")(
            _ptr(cl), _ptr(cv), _U(cl.size), _U(t), _ptr(m), _ptr(s), _IT(s.size))

    def multi_qubit_Pauli_gate_partial_list(self, tl, ids, s):
        tl, ids = _u32(tl), _u32(ids)
        self._f("multi_qubit_Pauli_gate_partial_list")(_ptr(tl), _ptr(ids), _U(tl.size), _ptr(s), _IT(s.size))

    def multi_qubit_Pauli_rotation_gate_partial_list(self, tl, ids, angle, s):
        tl, ids = _u32(tl), _u32(ids)
        self._f("multi_qubit_Pauli_rotation_gate_partial_list")(
            _ptr(tl), _ptr(ids), _U(tl.size), _D(angle), _ptr(s), _IT(s.size))

    # ---- statistics ----
    def state_norm_squared(self, s) -> float:
        return self._f("state_norm_squared", _D)(_ptr(s), _IT(s.size))

    def state_inner_product(self, a, b) -> complex:
        out = np.zeros(2)
        self._f("state_inner_product")(_ptr(a), _ptr(b), _IT(a.size), _ptr(out))
        return complex(out[0], out[1])

    def expectation_value(self, tl, ids, s) -> float:
        tl, ids = _u32(tl), _u32(ids)
        return self._f("expectation_value_multi_qubit_Pauli_operator_partial_list", _D)(
            _ptr(tl), _ptr(ids), _U(tl.size), _ptr(s), _IT(s.size))

    def M0_prob(self, t, s):
        return self._f("M0_prob", _D)(_U(t), _ptr(s), _IT(s.size))

    def M1_prob(self, t, s):
        return self._f("M1_prob", _D)(_U(t), _ptr(s), _IT(s.size))

    def marginal_prob(self, tl, vals, s):
        tl, vals = _u32(tl), _u32(vals)
        return self._f("marginal_prob", _D)(_ptr(tl), _ptr(vals), _U(tl.size), _ptr(s), _IT(s.size))

    def sampling_with_uniforms(self, s, uniforms, eps=None):
        """Indices for the supplied uniforms; with ``eps`` also a near-boundary flag per draw (port)."""
        u = np.ascontiguousarray(np.asarray(uniforms, dtype=np.float64))
        out = np.zeros(u.size, dtype=np.uint64)
        if self.prefix == "or_":
            flags = np.zeros(u.size, dtype=np.uint8)
            self._f("sampling_with_uniforms")(_ptr(s), _IT(s.size), _ptr(u), _U(u.size), _ptr(out),
                                              _D(eps or 0.0), _ptr(flags))
            return (out, flags.astype(bool)) if eps is not None else out
        self._f("sampling_with_uniforms")(_ptr(s), _IT(s.size), _ptr(u), _U(u.size), _ptr(out))
        return out

    # ---- density matrix (rho is a dim x dim complex128 array, row-major) ----
    def dm_single_qubit_dense_matrix_gate(self, t, m, r):
        m = _c128(m)
        self._f("dm_single_qubit_dense_matrix_gate")(_U(t), _ptr(m), _ptr(r), _IT(r.shape[0]))

    def dm_multi_qubit_dense_matrix_gate(self, tl, m, r):
        tl, m = _u32(tl), _c128(m)
        self._f("dm_multi_qubit_dense_matrix_gate")(_ptr(tl), _U(tl.size), _ptr(m), _ptr(r), _IT(r.shape[0]))

    def dm_CNOT_gate(self, c, t, r):
        self._f("dm_CNOT_gate")(_U(c), _U(t), _ptr(r), _IT(r.shape[0]))

    def dm_CZ_gate(self, c, t, r):
        self._f("dm_CZ_gate")(_U(c), _U(t), _ptr(r), _IT(r.shape[0]))

    def dm_depolarizing_noise(self, t, p, r):
        self._f("dm_depolarizing_noise")(_U(t), _D(p), _ptr(r), _IT(r.shape[0]))

    def dm_two_qubit_depolarizing_noise(self, t1, t2, p, r):
        self._f("dm_two_qubit_depolarizing_noise")(_U(t1), _U(t2), _D(p), _ptr(r), _IT(r.shape[0]))

    def dm_expectation_value(self, tl, ids, r) -> float:
        tl, ids = _u32(tl), _u32(ids)
        return self._f("dm_expectation_value_multi_qubit_Pauli_operator_partial_list", _D)(
            _ptr(tl), _ptr(ids), _U(tl.size), _ptr(r), _IT(r.shape[0]))

    def dm_sampling_with_uniforms(self, r, uniforms):
        u = np.ascontiguousarray(np.asarray(uniforms, dtype=np.float64))
        out = np.zeros(u.size, dtype=np.uint64)
        self._f("dm_sampling_with_uniforms")(_ptr(r), _IT(r.shape[0]), _ptr(u), _U(u.size), _ptr(out))
        return out


_port = None
_ref = None


def port() -> CpuSim:
    global _port
    if _port is None:
        _port = CpuSim(build_port(), "or_")
    return _port


def reference() -> CpuSim | None:
    global _ref
    if _ref is None and os.path.exists(REF_SO):
        _ref = CpuSim(REF_SO, "ref_")
    return _ref
