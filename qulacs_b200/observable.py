"""PauliOperator / Observable (cppsim/pauli_operator.cpp, general_quantum_operator.cpp).

``Observable.get_expectation_value`` evaluates all terms with one batched C-ABI call
(``qs_expectation_value_pauli_batch``) and sums coef_k <P_k> in FP64 on the host, the sum the
reference forms in GeneralQuantumOperator::get_expectation_value (general_quantum_operator.cpp:105-141).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import call

_PAULI = {"I": 0, "X": 1, "Y": 2, "Z": 3}


def _parse(pauli_string: str):
    toks = pauli_string.split()
    if len(toks) % 2:
        raise ValueError(f"bad Pauli string {pauli_string!r}")
    tl, ids = [], []
    for i in range(0, len(toks), 2):
        p = toks[i].upper()
        if p not in _PAULI:
            raise ValueError(f"bad Pauli symbol {toks[i]!r}")
        tl.append(int(toks[i + 1]))
        ids.append(_PAULI[p])
    return tl, ids


def masks(targets, ids):
    """(bit-flip mask, phase-flip mask, Y count) as csim get_Pauli_masks_partial_list (utility.cpp:12-43)."""
    x = z = 0
    ny = 0
    for t, p in zip(targets, ids):
        b = 1 << int(t)
        if p == 1:
            x ^= b
        elif p == 2:
            x ^= b
            z ^= b
            ny += 1
        elif p == 3:
            z ^= b
        elif p != 0:
            raise ValueError("Pauli id must be 0..3")
    return x, z, ny


class PauliOperator:
    def __init__(self, pauli_string: str = "", coef: complex = 1.0, *, targets=None, pauli_ids=None):
        if targets is not None:
            self.targets, self.ids = [int(t) for t in targets], [int(p) for p in pauli_ids]
        else:
            self.targets, self.ids = _parse(pauli_string)
        if len(set(self.targets)) != len(self.targets):
            raise ValueError("duplicated qubit in Pauli operator")
        self.coef = complex(coef)

    def get_coef(self) -> complex:
        return self.coef

    def get_index_list(self):
        return list(self.targets)

    def get_pauli_id_list(self):
        return list(self.ids)

    def get_expectation_value(self, state) -> complex:
        """coef * <P> (pauli_operator.cpp:132-183)."""
        tl = np.ascontiguousarray(np.asarray(self.targets, dtype=np.uint32))
        ids = np.ascontiguousarray(np.asarray(self.ids, dtype=np.uint32))
        out = C.c_double()
        fn = ("qs_expectation_value_multi_qubit_Pauli_operator_partial_list" if state.is_state_vector()
              else "qs_dm_expectation_value_multi_qubit_Pauli_operator_partial_list")
        call(fn, tl.ctypes.data_as(C.c_void_p), ids.ctypes.data_as(C.c_void_p), tl.size, state.data_ptr(),
             state.dim, state.stream, C.byref(out))
        return self.coef * out.value


class Observable:
    def __init__(self, qubit_count: int):
        self.qubit_count = int(qubit_count)
        self.terms: list[PauliOperator] = []

    def add_operator(self, coef_or_op, pauli_string: str | None = None) -> None:
        op = coef_or_op if isinstance(coef_or_op, PauliOperator) else PauliOperator(pauli_string, coef_or_op)
        if any(t >= self.qubit_count for t in op.targets):
            raise ValueError("Pauli operator acts on a qubit beyond the observable's qubit count")
        self.terms.append(op)

    def get_term_count(self) -> int:
        return len(self.terms)

    def get_qubit_count(self) -> int:
        return self.qubit_count

    def term_values(self, state) -> np.ndarray:
        """<P_k> for every term (real), one batched device call for a state vector."""
        k = len(self.terms)
        vals = np.zeros(k)
        if k == 0:
            return vals
        if not state.is_state_vector():
            for i, t in enumerate(self.terms):
                vals[i] = (PauliOperator(targets=t.targets, pauli_ids=t.ids).get_expectation_value(state)).real
            return vals
        xm = np.zeros(k, dtype=np.uint64)
        zm = np.zeros(k, dtype=np.uint64)
        ny = np.zeros(k, dtype=np.uint32)
        for i, t in enumerate(self.terms):
            xm[i], zm[i], ny[i] = masks(t.targets, t.ids)
        fn = "qs_expectation_value_pauli_batch_c64" if type(state).__name__ == "QuantumStateC64" else \
            "qs_expectation_value_pauli_batch"
        call(fn, xm.ctypes.data_as(C.c_void_p), zm.ctypes.data_as(C.c_void_p),
             ny.ctypes.data_as(C.c_void_p), k, state.data_ptr(), state.dim, state.stream,
             vals.ctypes.data_as(C.c_void_p))
        return vals

    def get_expectation_value(self, state) -> float:
        vals = self.term_values(state)
        coefs = np.array([t.coef for t in self.terms], dtype=np.complex128)
        return float(np.real(np.sum(coefs * vals)))
