"""QuantumCircuit over the C-ABI circuit object (cppsim/circuit.hpp, circuit.cpp)."""
from __future__ import annotations

import ctypes as C

from . import _lib
from . import gate as G
from ._lib import call


class QuantumCircuit:
    """Gate list applied in order by ``update_quantum_state`` (cppsim circuit.cpp:46-57).

    ``mode="gate_by_gate"`` launches one kernel per gate (the reference's method);
    ``mode="staged"`` applies several gates per HBM pass with the same per-gate arithmetic;
    ``mode="staged_fused"`` first composes runs of gates into k-qubit dense blocks in FP64 (k chosen
    per circuit by timing, or forced with ``set_fusion``), then stages them.
    """

    def __init__(self, qubit_count: int):
        _lib.load()
        self.qubit_count = int(qubit_count)
        h = C.c_void_p()
        call("qs_circuit_create", self.qubit_count, C.byref(h))
        self._h = h.value
        self.gate_list = []
        self._fusion_k = None
        self._specialize = None

    def get_qubit_count(self) -> int:
        return self.qubit_count

    def get_gate_count(self) -> int:
        return len(self.gate_list)

    def _check_qubits(self, gate: G.QuantumGateBase) -> None:
        # cppsim check_gate_index (circuit.cpp:119-131)
        for q in gate.get_target_index_list() + gate.get_control_index_list():
            if not 0 <= q < self.qubit_count:
                raise ValueError("gate must be applied to qubits of which the indices are smaller than qubit_count")

    def _rebuild(self) -> None:
        """Re-create the native circuit from gate_list (after an insertion or removal)."""
        h = C.c_void_p()
        call("qs_circuit_create", self.qubit_count, C.byref(h))
        old, self._h = self._h, h.value
        _lib.load().qs_circuit_destroy(old)
        for g in self.gate_list:
            g._add_to(self._h)
        if self._fusion_k is not None:
            call("qs_circuit_set_fusion", self._h, self._fusion_k)
        if self._specialize is not None:
            call("qs_circuit_set_specialized", self._h, self._specialize)

    def add_gate(self, gate: G.QuantumGateBase, position: int | None = None) -> None:
        """Append (or insert before ``position``) a copy of ``gate`` (cppsim circuit.cpp:133-165)."""
        self._check_qubits(gate)
        g = gate.copy()
        if position is None:
            g._add_to(self._h)
            self.gate_list.append(g)
            return
        if not 0 <= position <= len(self.gate_list):
            raise IndexError("insert index must be smaller than or equal to gate_count")
        self.gate_list.insert(position, g)
        self._rebuild()

    add_gate_copy = add_gate
    add_gate_consume = add_gate

    def remove_gate(self, index: int) -> None:
        """cppsim circuit.cpp:250-258."""
        if not 0 <= index < len(self.gate_list):
            raise IndexError("index must be smaller than gate_count")
        del self.gate_list[index]
        self._rebuild()

    def get_gate(self, index: int) -> G.QuantumGateBase:
        if not 0 <= index < len(self.gate_list):
            raise IndexError("index must be smaller than gate_count")
        return self.gate_list[index].copy()

    def copy(self) -> "QuantumCircuit":
        """cppsim circuit.cpp:111-117."""
        c = QuantumCircuit(self.qubit_count)
        c.merge_circuit(self)
        return c

    def merge_circuit(self, circuit: "QuantumCircuit") -> None:
        """Append copies of ``circuit``'s gates (cppsim circuit.hpp:150-155)."""
        for g in circuit.gate_list:
            self.add_gate(g)

    def get_inverse(self) -> "QuantumCircuit":
        """The inverses of the gates in reverse order (cppsim circuit.cpp:571-578)."""
        c = QuantumCircuit(self.qubit_count)
        for g in reversed(self.gate_list):
            c.add_gate(g.get_inverse())
        return c

    def calculate_depth(self) -> int:
        """Greedy layering over each gate's targets and controls (cppsim circuit.cpp:295-322)."""
        filled = [0] * self.qubit_count
        depth = 0
        for g in self.gate_list:
            qubits = g.get_target_index_list() + g.get_control_index_list()
            step = max((filled[q] for q in qubits), default=0) + 1
            for q in qubits:
                filled[q] = step
            depth = max(depth, step)
        return depth

    def to_string(self) -> str:
        """cppsim circuit.cpp:324-349."""
        sizes = [len(g.get_target_index_list()) + len(g.get_control_index_list()) for g in self.gate_list]
        top = max(sizes, default=0)
        lines = ["*** Quantum Circuit Info ***", f"# of qubit: {self.qubit_count}",
                 f"# of step : {self.calculate_depth()}", f"# of gate : {len(self.gate_list)}"]
        lines += [f"# of {i + 1} qubit gate: {sizes.count(i + 1)}" for i in range(top)]
        lines += ["Clifford  : no", "Gaussian  : no", ""]
        return "\n".join(lines) + "\n"

    def __str__(self) -> str:
        return self.to_string()

    # convenience adders (cppsim circuit.cpp:361-557)
    def add_X_gate(self, t): self.add_gate(G.X(t))
    def add_Y_gate(self, t): self.add_gate(G.Y(t))
    def add_Z_gate(self, t): self.add_gate(G.Z(t))
    def add_H_gate(self, t): self.add_gate(G.H(t))
    def add_S_gate(self, t): self.add_gate(G.S(t))
    def add_Sdag_gate(self, t): self.add_gate(G.Sdag(t))
    def add_T_gate(self, t): self.add_gate(G.T(t))
    def add_Tdag_gate(self, t): self.add_gate(G.Tdag(t))
    def add_sqrtX_gate(self, t): self.add_gate(G.sqrtX(t))
    def add_sqrtXdag_gate(self, t): self.add_gate(G.sqrtXdag(t))
    def add_sqrtY_gate(self, t): self.add_gate(G.sqrtY(t))
    def add_sqrtYdag_gate(self, t): self.add_gate(G.sqrtYdag(t))
    def add_P0_gate(self, t): self.add_gate(G.P0(t))
    def add_P1_gate(self, t): self.add_gate(G.P1(t))
    def add_RX_gate(self, t, a): self.add_gate(G.RX(t, a))
    def add_RY_gate(self, t, a): self.add_gate(G.RY(t, a))
    def add_RZ_gate(self, t, a): self.add_gate(G.RZ(t, a))
    def add_FusedSWAP_gate(self, t0, t1, block_size): self.add_gate(G.FusedSWAP(t0, t1, block_size))
    def add_RotInvX_gate(self, t, a): self.add_gate(G.RotInvX(t, a))
    def add_RotInvY_gate(self, t, a): self.add_gate(G.RotInvY(t, a))
    def add_RotInvZ_gate(self, t, a): self.add_gate(G.RotInvZ(t, a))
    def add_RotX_gate(self, t, a): self.add_gate(G.RotX(t, a))
    def add_RotY_gate(self, t, a): self.add_gate(G.RotY(t, a))
    def add_RotZ_gate(self, t, a): self.add_gate(G.RotZ(t, a))
    def add_U1_gate(self, t, l): self.add_gate(G.U1(t, l))
    def add_U2_gate(self, t, p, l): self.add_gate(G.U2(t, p, l))
    def add_U3_gate(self, t, th, p, l): self.add_gate(G.U3(t, th, p, l))
    def add_CNOT_gate(self, c, t): self.add_gate(G.CNOT(c, t))
    def add_CZ_gate(self, c, t): self.add_gate(G.CZ(c, t))
    def add_SWAP_gate(self, a, b): self.add_gate(G.SWAP(a, b))
    def add_dense_matrix_gate(self, targets, m): self.add_gate(G.DenseMatrix(targets, m))

    def add_random_unitary_gate(self, targets, seed: int | None = None) -> None:
        self.add_gate(G.RandomUnitary(targets, seed))

    def add_multi_Pauli_gate(self, targets_or_pauli, pauli_ids=None) -> None:
        """(targets, pauli_ids) or a PauliOperator (cppsim circuit.cpp:454-461)."""
        if pauli_ids is None:
            p = targets_or_pauli
            self.add_gate(G.Pauli(p.get_index_list(), p.get_pauli_id_list()))
        else:
            self.add_gate(G.Pauli(targets_or_pauli, pauli_ids))

    def add_multi_Pauli_rotation_gate(self, targets_or_pauli, pauli_ids=None, angle=None) -> None:
        """(targets, pauli_ids, angle), or a PauliOperator whose real coefficient is the angle
        (cppsim circuit.cpp:462-480)."""
        if pauli_ids is None:
            p = targets_or_pauli
            c = complex(p.get_coef())
            if abs(c.imag) > 1e-14:
                raise ValueError("add_multi_Pauli_rotation_gate: not implemented for non hermitian")
            self.add_gate(G.PauliRotation(p.get_index_list(), p.get_pauli_id_list(), c.real))
        else:
            self.add_gate(G.PauliRotation(targets_or_pauli, pauli_ids, angle))

    def add_noise_gate(self, gate: G.QuantumGateBase, noise_type: str, prob: float) -> None:
        """cppsim circuit.cpp:167-190: the gate, then depolarizing noise on its targets + controls."""
        self.add_gate(gate)
        qubits = gate.get_target_index_list() + gate.get_control_index_list()
        if noise_type != "Depolarizing":
            raise NotImplementedError(noise_type)
        if len(qubits) == 1:
            self.add_gate(G.DepolarizingNoise(qubits[0], prob))
        elif len(qubits) == 2:
            self.add_gate(G.TwoQubitDepolarizingNoise(qubits[0], qubits[1], prob))
        else:
            raise ValueError("depolarizing noise can be used up to 2 qubits")

    def update_quantum_state(self, state, mode: str = "staged") -> None:
        """Apply the circuit.  A QuantumStateC64 takes the circuit's complex64 executor (set_c64_executor:
        6-qubit blocks on the tensor cores, or FP64 passes over the complex64 state)."""
        if state.get_qubit_count() != self.qubit_count:
            raise ValueError("state qubit count differs from the circuit's")
        if type(state).__name__ == "QuantumStateC64":
            call("qs_circuit_update_quantum_state_c64", self._h, state.data_ptr(), state.dim, state.stream)
            return
        m = {"gate_by_gate": _lib.EXEC_GATE_BY_GATE, "staged": _lib.EXEC_STAGED,
             "staged_fused": _lib.EXEC_STAGED_FUSED}[mode]
        if state.is_state_vector():
            call("qs_circuit_update_quantum_state", self._h, state.data_ptr(), state.dim, m, state.stream)
        else:
            call("qs_circuit_update_density_matrix", self._h, state.data_ptr(), state.dim, m, state.stream)

    _C64_EXEC = {"auto": -1, "tensor": 0, "fp64": 1}

    def set_c64_executor(self, mode) -> None:
        """Executor for complex64 states: "tensor" (6-qubit blocks on the tensor cores, >= 10 qubits, gates
        of <= 6 qubits), "fp64" (FP64 passes over the complex64 state, gates of <= 2 qubits) or "auto"
        (default: the tensor cores when they take the circuit, else the FP64 passes)."""
        call("qs_circuit_set_c64_executor", self._h, self._C64_EXEC[mode] if isinstance(mode, str) else int(mode))

    def c64_executor_info(self):
        """Executor of the last complex64 run: "tensor", "fp64" or None."""
        ch = C.c_int()
        call("qs_circuit_c64_executor_info", self._h, C.byref(ch))
        return {0: "tensor", 1: "fp64"}.get(ch.value)

    def set_fusion(self, k: int) -> None:
        """Block size of mode="staged_fused": 0..6, or -1 to let the autotuner choose (default)."""
        call("qs_circuit_set_fusion", self._h, int(k))
        self._fusion_k = int(k)

    def set_specialized(self, mode: int) -> None:
        """Specialised pass kernels for the "staged" / "staged_fused" modes (each HBM pass compiled with
        its schedule and gate matrices as constants): 1 always, 0 never, -1 for states of at least 2^22
        amplitudes (default)."""
        call("qs_circuit_set_specialized", self._h, int(mode))
        self._specialize = int(mode)

    def specialized_info(self):
        """(staged schedule specialised, staged_fused schedule specialised, compile ms)."""
        a, b, ms = C.c_int(), C.c_int(), C.c_double()
        call("qs_circuit_specialized_info", self._h, C.byref(a), C.byref(b), C.byref(ms))
        return bool(a.value), bool(b.value), ms.value

    def specialized_source(self, pass_index: int) -> str:
        """CUDA C of the specialised kernel of one pass of the "staged" schedule (host only)."""
        size = C.c_ulonglong(0)
        call("qs_circuit_specialized_source", self._h, 1 << self.qubit_count, int(pass_index), None, C.byref(size))
        buf = C.create_string_buffer(size.value)
        call("qs_circuit_specialized_source", self._h, 1 << self.qubit_count, int(pass_index), buf, C.byref(size))
        return buf.value.decode()

    def fusion_info(self):
        """(k, gates after fusion, HBM passes, autotuner estimates in ms) of the last "staged_fused"
        schedule; k = -1 before the first run.  Estimates: [k] for k = 0..6 with 2^12-amplitude tiles,
        [7] for the best k with 2^11-amplitude tiles (< 0 where not tried)."""
        k, g, p = C.c_int(), C.c_uint(), C.c_uint()
        est = (C.c_double * 8)()
        call("qs_circuit_fusion_info", self._h, C.byref(k), C.byref(g), C.byref(p), est)
        return k.value, g.value, p.value, list(est)

    def fuse(self, k: int) -> "FusedGateList":
        """The greedy k-qubit FP64 fusion of this circuit (host only; cppsim QuantumCircuitOptimizer
        semantics): a read-only list of (qubits, dense matrix) pairs."""
        h = C.c_void_p()
        call("qs_circuit_fuse", self._h, int(k), C.byref(h))
        return FusedGateList(h.value, self.qubit_count)

    def density_matrix_as_vector(self) -> "FusedGateList":
        """This circuit acting on a density matrix as gates on the 2n-qubit vector rho[row * 2^n + col]
        (host only): (qubits, matrix) pairs, noise channels as superoperators."""
        h = C.c_void_p()
        call("qs_circuit_density_matrix_as_vector", self._h, C.byref(h))
        return FusedGateList(h.value, 2 * self.qubit_count)

    def fused_stats(self):
        """(tile passes, 6-qubit blocks) of the fused complex64 schedule."""
        p, b = C.c_uint(), C.c_uint()
        call("qs_circuit_fused_stats", self._h, C.byref(p), C.byref(b))
        return p.value, b.value

    def staged_stats(self):
        """(HBM passes, register phases, ops in phases, gates run singly) of the staged schedule."""
        v = [C.c_uint() for _ in range(4)]
        call("qs_circuit_staged_stats", self._h, *[C.byref(x) for x in v])
        return tuple(x.value for x in v)

    def pass_count(self) -> int:
        out = C.c_uint()
        call("qs_circuit_pass_count", self._h, 1 << self.qubit_count, C.byref(out))
        return out.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                _lib.load().qs_circuit_destroy(h)
            except Exception:
                pass
            self._h = None


class FusedGateList:
    """Gates of a fused circuit as (qubits, matrix) with matrix index bit j <-> qubits[j]."""

    def __init__(self, handle, qubit_count: int):
        self._h = handle
        self.qubit_count = qubit_count
        out = C.c_uint()
        call("qs_circuit_gate_count", self._h, C.byref(out))
        self._count = out.value

    def __len__(self):
        return self._count

    def __getitem__(self, i):
        import numpy as np
        if not 0 <= i < self._count:
            raise IndexError(i)
        qs = (C.c_uint * 6)()
        cnt = C.c_uint()
        m = np.zeros(2 * 4096, dtype=np.float64)
        call("qs_circuit_gate_matrix", self._h, i, qs, C.byref(cnt), m.ctypes.data_as(C.c_void_p))
        k = cnt.value
        mat = m[:2 * 4 ** k].view(np.complex128).reshape(1 << k, 1 << k).copy()
        return [int(qs[j]) for j in range(k)], mat

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                _lib.load().qs_circuit_destroy(h)
            except Exception:
                pass
            self._h = None
