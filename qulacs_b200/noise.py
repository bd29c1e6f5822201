"""cppsim NoiseSimulator (noisesimulator.hpp / noisesimulator.cpp) over device-resident states.

Trajectories are drawn exactly as the reference draws them (see ``qs_noise_simulator_execute`` in
``include/qulacs_b200.h``); distinct trajectories are simulated once each on the device through the
FP64-fused staged executor, from a shared prefix state.  The reference seeds its generator from
``std::random_device``; here the seed is an argument, so results are reproducible.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import call
from .state import QuantumState


class NoiseSimulator:
    def __init__(self, circuit, init_state: QuantumState | None = None, seed: int = 0):
        self.circuit = circuit
        self.init_state = init_state
        self.seed = int(seed)
        self._stream = init_state.stream if init_state is not None else None

    def _args(self, seed):
        return self.seed if seed is None else int(seed)

    def trajectories(self, sample_count: int, seed: int | None = None) -> np.ndarray:
        """Sample count of each distinct trajectory, in the order they are simulated (host only)."""
        cnt = C.c_uint()
        call("qs_noise_simulator_trajectories", self.circuit._h, int(sample_count), self._args(seed), C.byref(cnt),
             None)
        shots = np.zeros(max(1, cnt.value), dtype=np.uint32)
        call("qs_noise_simulator_trajectories", self.circuit._h, int(sample_count), self._args(seed), C.byref(cnt),
             shots.ctypes.data_as(C.c_void_p))
        return shots[:cnt.value]

    def execute(self, sample_count: int, seed: int | None = None) -> np.ndarray:
        """NoiseSimulator::execute: sample_count basis indices, grouped by trajectory."""
        n = self.circuit.get_qubit_count()
        out = np.zeros(max(1, sample_count), dtype=np.uint64)
        init = self.init_state.data_ptr() if self.init_state is not None else None
        call("qs_noise_simulator_execute", self.circuit._h, init, 1 << n, int(sample_count), self._args(seed),
             out.ctypes.data_as(C.c_void_p), None, self._stream)
        return out[:sample_count]

    def execute_and_get_result(self, execution_count: int, seed: int | None = None) -> "Result":
        """NoiseSimulator::execute_and_get_result: each distinct trajectory's final state and count
        (one device state per trajectory)."""
        n = self.circuit.get_qubit_count()
        shots = self.trajectories(execution_count, seed)
        states = [QuantumState(n) for _ in shots]
        ptrs = (C.c_void_p * max(1, len(states)))(*[s.data_ptr() for s in states])
        init = self.init_state.data_ptr() if self.init_state is not None else None
        call("qs_noise_simulator_execute", self.circuit._h, init, 1 << n, int(execution_count), self._args(seed),
             None, ptrs, self._stream)
        return Result(list(zip(states, (int(s) for s in shots))))


class Result:
    """NoiseSimulator::Result: (state, count) pairs; sampling() samples each state count times."""

    def __init__(self, result):
        self.result = result

    def sampling(self, seed: int = 0) -> np.ndarray:
        out = [s.sampling(c, seed + i) for i, (s, c) in enumerate(self.result)]
        return np.concatenate(out) if out else np.zeros(0, dtype=np.uint64)
