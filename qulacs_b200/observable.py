"""PauliOperator / Observable (cppsim/pauli_operator.cpp, general_quantum_operator.cpp).

``Observable.get_expectation_value`` evaluates sum_k coef_k <P_k> with one weighted C-ABI call
(``qs_expectation_value_pauli_weighted``), the sum the reference forms term by term in
GeneralQuantumOperator::get_expectation_value (general_quantum_operator.cpp:105-141);
``Observable.term_values`` returns every <P_k> (``qs_expectation_value_pauli_batch``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import call

_PAULI = {"I": 0, "X": 1, "Y": 2, "Z": 3}


def _parse(pauli_string: str):
    """"X 0 Y 3 ..." -> (targets, ids); identity factors are dropped, as pauli_operator.cpp:17-47 does."""
    toks = pauli_string.split()
    if len(toks) % 2:
        raise ValueError(f"Detected pauli_str without indices: {pauli_string!r}")
    tl, ids = [], []
    for i in range(0, len(toks), 2):
        p = toks[i].upper()
        if p not in _PAULI:
            raise ValueError(f"invalid Pauli string is given : {toks[i]!r}")
        if _PAULI[p]:
            tl.append(int(toks[i + 1]))
            ids.append(_PAULI[p])
    return tl, ids


def _u32(seq) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(seq, dtype=np.uint32))


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

    def change_coef(self, coef: complex) -> None:
        self.coef = complex(coef)

    def get_index_list(self):
        return list(self.targets)

    def get_pauli_id_list(self):
        return list(self.ids)

    def get_qubit_count(self) -> int:
        return max(self.targets, default=-1) + 1

    def add_single_Pauli(self, index: int, pauli_id: int) -> None:
        """pauli_operator.cpp:116-130."""
        if not 0 <= int(pauli_id) <= 3:
            raise ValueError("Pauli id must be 0..3")
        if int(index) in self.targets:
            raise ValueError("duplicated qubit in Pauli operator")
        self.targets.append(int(index))
        self.ids.append(int(pauli_id))

    def get_pauli_string(self) -> str:
        """"X 0 Y 3" (pauli_operator.cpp:264-286); identity factors are left out."""
        return " ".join(f"{'IXYZ'[p]} {t}" for t, p in zip(self.targets, self.ids) if p)

    def copy(self) -> "PauliOperator":
        return PauliOperator(coef=self.coef, targets=self.targets, pauli_ids=self.ids)

    def get_transition_amplitude(self, state_bra, state_ket) -> complex:
        """coef * <bra|P|ket> (pauli_operator.cpp:225-262)."""
        if not (state_bra.is_state_vector() and state_ket.is_state_vector()):
            raise NotImplementedError("get_transition_amplitude for density matrix is not implemented")
        if state_bra.dim != state_ket.dim:
            raise ValueError("bra and ket differ in qubit count")
        tl, ids = _u32(self.targets), _u32(self.ids)
        out = np.zeros(2)
        call("qs_transition_amplitude_multi_qubit_Pauli_operator_partial_list", tl.ctypes.data_as(C.c_void_p),
             ids.ctypes.data_as(C.c_void_p), tl.size, state_bra.data_ptr(), state_ket.data_ptr(), state_ket.dim,
             state_ket.stream, out.ctypes.data_as(C.c_void_p))
        return self.coef * complex(out[0], out[1])

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

    def get_expectation_value_single_thread(self, state) -> complex:
        """The reference's single-thread variant; the device reduction has one form."""
        return self.get_expectation_value(state)


class Observable:
    def __init__(self, qubit_count: int):
        self.qubit_count = int(qubit_count)
        self.terms: list[PauliOperator] = []

    def add_operator(self, coef_or_op, pauli_string: str | None = None) -> None:
        op = coef_or_op if isinstance(coef_or_op, PauliOperator) else PauliOperator(pauli_string, coef_or_op)
        if any(t >= self.qubit_count for t in op.targets):
            raise ValueError("Pauli operator acts on a qubit beyond the observable's qubit count")
        self.terms.append(op)

    add_operator_copy = add_operator
    add_operator_move = add_operator

    def add_random_operator(self, operator_count: int, seed: int | None = None) -> None:
        """general_quantum_operator.cpp:179-202: terms with a Pauli on every qubit and a real coefficient
        in [-1, 1); with a seed, the reference's terms for that seed."""
        if seed is None:
            seed = int(np.random.SeedSequence().entropy & 0xFFFFFFFF)
        n, k = self.qubit_count, int(operator_count)
        ids = np.zeros(max(n * k, 1), dtype=np.uint32)
        coefs = np.zeros(max(k, 1))
        call("qs_random_operator_terms", n, k, int(seed) & 0xFFFFFFFF, ids.ctypes.data_as(C.c_void_p),
             coefs.ctypes.data_as(C.c_void_p))
        for t in range(k):
            row = [int(x) for x in ids[t * n:(t + 1) * n]]
            self.terms.append(PauliOperator(coef=coefs[t], targets=[q for q in range(n) if row[q]],
                                            pauli_ids=[p for p in row if p]))

    def get_term_count(self) -> int:
        return len(self.terms)

    def get_term(self, index: int) -> PauliOperator:
        if not 0 <= index < len(self.terms):
            raise IndexError("index out of range")
        return self.terms[index].copy()

    def get_qubit_count(self) -> int:
        return self.qubit_count

    def copy(self) -> "Observable":
        o = Observable(self.qubit_count)
        o.terms = [t.copy() for t in self.terms]
        return o

    def is_hermitian(self) -> bool:
        """Every coefficient real (general_quantum_operator.cpp: HermitianQuantumOperator's check)."""
        return all(complex(t.get_coef()).imag == 0.0 for t in self.terms)

    def get_matrix(self) -> np.ndarray:
        """The dense 2^n x 2^n matrix sum_k c_k P_k (bit j of the index <-> qubit j), on the host."""
        n = self.qubit_count
        if n > 14:
            raise NotImplementedError("get_matrix: at most 14 qubits")
        pm = [np.eye(2), np.array([[0, 1], [1, 0]]), np.array([[0, -1j], [1j, 0]]), np.diag([1, -1])]
        out = np.zeros((1 << n, 1 << n), dtype=np.complex128)
        for t in self.terms:
            ids = dict(zip(t.get_index_list(), t.get_pauli_id_list()))
            m = np.ones((1, 1), dtype=np.complex128)
            for q in range(n):
                m = np.kron(pm[ids.get(q, 0)], m)
            out += t.get_coef() * m
        return out

    def get_state_dim(self) -> int:
        return 1 << self.qubit_count

    def get_transition_amplitude(self, state_bra, state_ket) -> complex:
        """sum_k coef_k <bra|P_k|ket> (general_quantum_operator.cpp:160-177)."""
        if self.qubit_count > state_bra.get_qubit_count() or state_bra.dim != state_ket.dim:
            raise ValueError("invalid qubit count")
        return sum((t.get_transition_amplitude(state_bra, state_ket) for t in self.terms), 0j)

    def apply_to_state(self, work_state, state_to_be_multiplied, dst_state) -> None:
        """dst = sum_k coef_k P_k |state> (general_quantum_operator.cpp:330-348), through a work state."""
        if state_to_be_multiplied.get_qubit_count() != dst_state.get_qubit_count():
            raise ValueError("Qubit count of state_to_be_multiplied and dst_state must be the same")
        dst_state.set_zero_norm_state()
        for t in self.terms:
            work_state.load(state_to_be_multiplied)
            if t.targets:
                tl, ids = _u32(t.targets), _u32(t.ids)
                call("qs_multi_qubit_Pauli_gate_partial_list", tl.ctypes.data_as(C.c_void_p),
                     ids.ctypes.data_as(C.c_void_p), tl.size, work_state.data_ptr(), work_state.dim,
                     work_state.stream)
            dst_state.add_state_with_coef(t.coef, work_state)

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

    def _masks(self):
        k = len(self.terms)
        xm = np.zeros(k, dtype=np.uint64)
        zm = np.zeros(k, dtype=np.uint64)
        ny = np.zeros(k, dtype=np.uint32)
        for i, t in enumerate(self.terms):
            xm[i], zm[i], ny[i] = masks(t.targets, t.ids)
        return xm, zm, ny

    def weighted_plan(self, qubit_count: int | None = None) -> dict:
        """How get_expectation_value evaluates these terms on a state of `qubit_count` qubits (host
        only): passes over the state and terms per kind of evaluation."""
        n = self.qubit_count if qubit_count is None else int(qubit_count)
        xm, zm, ny = self._masks()
        passes = C.c_uint()
        kinds = (C.c_uint * 5)()
        call("qs_expectation_value_pauli_weighted_plan", xm.ctypes.data_as(C.c_void_p),
             zm.ctypes.data_as(C.c_void_p), ny.ctypes.data_as(C.c_void_p), len(self.terms), 1 << n,
             C.byref(passes), kinds)
        return {"passes": passes.value, "z_only": kinds[0], "in_registers": kinds[1], "shared_partner": kinds[2],
                "selected_rows": kinds[3], "one_value_each": kinds[4]}

    def pass_source(self, index: int, qubit_count: int | None = None, c64: bool = False) -> str:
        """CUDA C of the generated kernel for pass `index` of the weighted plan."""
        n = self.qubit_count if qubit_count is None else int(qubit_count)
        xm, zm, ny = self._masks()
        need = C.c_ulonglong()
        args = (xm.ctypes.data_as(C.c_void_p), zm.ctypes.data_as(C.c_void_p), ny.ctypes.data_as(C.c_void_p),
                len(self.terms), 1 << n, index, int(c64))
        call("qs_expectation_pass_source", *args, None, 0, C.byref(need))
        buf = C.create_string_buffer(need.value)
        call("qs_expectation_pass_source", *args, buf, need.value, C.byref(need))
        return buf.value.decode()

    def get_expectation_value_complex(self, state) -> complex:
        """sum_k coef_k <P_k> with complex coefficients kept (GeneralQuantumOperator's return)."""
        if not self.terms:
            return 0j
        if not state.is_state_vector():
            vals = self.term_values(state)
            return complex(np.sum(np.array([t.coef for t in self.terms], dtype=np.complex128) * vals))
        xm, zm, ny = self._masks()
        cf = np.zeros(2 * len(self.terms))
        for i, t in enumerate(self.terms):
            c = complex(t.coef)
            cf[2 * i], cf[2 * i + 1] = c.real, c.imag
        out = np.zeros(2)
        fn = "qs_expectation_value_pauli_weighted_c64" if type(state).__name__ == "QuantumStateC64" else \
            "qs_expectation_value_pauli_weighted"
        call(fn, xm.ctypes.data_as(C.c_void_p), zm.ctypes.data_as(C.c_void_p), ny.ctypes.data_as(C.c_void_p),
             cf.ctypes.data_as(C.c_void_p), len(self.terms), state.data_ptr(), state.dim, state.stream,
             out.ctypes.data_as(C.c_void_p))
        return complex(out[0], out[1])

    def get_expectation_value(self, state) -> float:
        """Re sum_k coef_k <P_k>.  For a state vector one weighted device call folds every term's
        contribution into a single FP64 sum (no per-term values); a density matrix sums term_values."""
        if not self.terms:
            return 0.0
        return self.get_expectation_value_complex(state).real

    get_expectation_value_single_thread = get_expectation_value


def set_expectation_specialized(mode: int) -> None:
    """0: generic expectation kernel only; 1 (default): per-pass kernels generated when the same terms
    are evaluated a second time on >= 20 qubits; 2: generated at the first evaluation, any size."""
    call("qs_set_expectation_specialized", int(mode))


def expectation_specialized_info() -> tuple[int, float]:
    """(launches of generated expectation kernels so far, compile ms of the last generated plan)."""
    n = C.c_ulonglong()
    ms = C.c_double()
    call("qs_expectation_specialized_info", C.byref(n), C.byref(ms))
    return n.value, ms.value
