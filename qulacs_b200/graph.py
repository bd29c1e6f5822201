"""Circuits and batches recorded as CUDA graphs (``qs_circuit_graph_create``, ``qs_batch_graph_create``).

A graph replays the exact kernel sequence of one call -- optionally preceded by setting the states to
|0...0> -- with a single ``cudaGraphLaunch``: the host planning, parameter uploads and per-pass or
per-gate launches are paid once, at capture.  It is bound to the state buffers and to the circuits'
gates as they were when captured.
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from ._lib import call

_MODES = {"gate_by_gate": _lib.EXEC_GATE_BY_GATE, "staged": _lib.EXEC_STAGED, "staged_fused": _lib.EXEC_STAGED_FUSED}


class CapturedGraph:
    def __init__(self, handle: int, stream, keep):
        self._h = handle
        self.stream = stream
        self._keep = keep  # the circuits and states the graph reads and writes stay alive with it

    def launch(self, stream=None) -> None:
        """Replay (asynchronous on the stream for a circuit graph; a batch graph synchronises)."""
        call("qs_graph_launch", self._h, self.stream if stream is None else stream)

    def kernel_count(self) -> int:
        n = C.c_ulonglong()
        call("qs_graph_kernel_count", self._h, C.byref(n))
        return n.value

    def close(self) -> None:
        if self._h:
            _lib.load().qs_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001  (interpreter shutdown)
            pass


def capture_circuit(circuit, state, mode: str = "staged", reset_state: bool = True) -> CapturedGraph:
    """Record `circuit` applied to `state` (complex128 state vector) in `mode`."""
    if state.get_qubit_count() != circuit.qubit_count:
        raise ValueError("state qubit count differs from the circuit's")
    h = C.c_void_p()
    call("qs_circuit_graph_create", circuit._h, state.data_ptr(), state.dim, _MODES[mode], int(reset_state),
         state.stream, C.byref(h))
    return CapturedGraph(h.value, state.stream, (circuit, state))


def capture_batch(circuits, states, reset_states: bool = True, stream=None) -> CapturedGraph:
    """Record every circuit applied to its state in one persistent launch; complex64 states (all or
    none) run the FP64 passes over complex64 tiles."""
    if len(circuits) != len(states) or not circuits:
        raise ValueError("one state per circuit, at least one")
    c64 = {type(s).__name__ == "QuantumStateC64" for s in states}
    if len(c64) != 1:
        raise ValueError("states must be all complex128 or all complex64")
    k = len(circuits)
    h = C.c_void_p()
    call("qs_batch_graph_create", (C.c_void_p * k)(*[c._h for c in circuits]),
         (C.c_void_p * k)(*[s.data_ptr() for s in states]), k, int(c64.pop()), int(reset_states), stream,
         C.byref(h))
    return CapturedGraph(h.value, stream, (list(circuits), list(states)))
