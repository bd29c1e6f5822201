"""Batched execution of many circuits with their observables (the batched-ansatz configuration).

``BatchRunner.run(jobs)`` takes (circuit, observable) pairs of any qubit counts, admits them into
waves whose states fit an HBM budget (footprint 16 B x 2^n each, carved from one arena per wave),
and for each wave applies every circuit in ONE persistent kernel launch
(``qs_batch_update_quantum_states``; circuits of >= 21 qubits, which fill the device alone, run their
own passes in the same call) and evaluates every energy with ``qs_batch_expectation_weighted`` (the
small states' terms in one launch, each state of >= 18 qubits through the weighted passes).
``precision="c64"`` keeps the states in complex64 and runs the wave
in one persistent launch of the chosen executor (``qs_batch_update_quantum_states_c64``): FP64 passes
over complex64 tiles (``c64_executor="fp64"``; "auto" takes it whenever every gate is stageable) or
6-qubit blocks on the tensor cores ("tensor"); reductions are FP64 either way.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import call
from .observable import masks
from .state import QuantumState

ALIGN = 256


def footprint(n: int, precision: str = "c128") -> int:
    return (16 if precision == "c128" else 8) << n


@dataclass
class BatchStats:
    waves: int = 0
    circuits: int = 0
    kernel_launches: int = 0


class BatchRunner:
    def __init__(self, memory_budget_bytes: int, precision: str = "c128", stream: int | None = None,
                 c64_executor: str = "auto"):
        if precision not in ("c128", "c64"):
            raise ValueError("precision must be c128 or c64")
        if c64_executor not in ("auto", "tensor", "fp64"):
            raise ValueError("c64_executor must be auto, tensor or fp64")
        self.budget = int(memory_budget_bytes)
        self.precision = precision
        self.c64_executor = {"auto": -1, "tensor": 0, "fp64": 1}[c64_executor]
        self.stream = stream
        self.stats = BatchStats()

    def waves(self, jobs):
        """Greedy admission in submission order: a wave closes when the next state would exceed the budget."""
        wave, used = [], 0
        for idx, (circ, _) in enumerate(jobs):
            fp = (footprint(circ.qubit_count, self.precision) + ALIGN - 1) // ALIGN * ALIGN
            if fp > self.budget:
                raise MemoryError(f"job {idx}: a {circ.qubit_count}-qubit state exceeds the memory budget")
            if wave and used + fp > self.budget:
                yield wave
                wave, used = [], 0
            wave.append(idx)
            used += fp
        if wave:
            yield wave

    def run(self, jobs) -> np.ndarray:
        """Energies <H_i> (real) for jobs = [(QuantumCircuit, Observable), ...]."""
        out = np.zeros(len(jobs))
        lib = _lib.load()
        for wave in self.waves(jobs):
            l0 = lib.qs_launch_count()
            if self.precision == "c128":
                self._run_wave_c128(jobs, wave, out)
            else:
                self._run_wave_c64(jobs, wave, out)
            self.stats.waves += 1
            self.stats.circuits += len(wave)
            self.stats.kernel_launches += lib.qs_launch_count() - l0
        return out

    def _run_wave_c128(self, jobs, wave, out):
        self._run_wave(jobs, wave, out, c64=False)

    def _run_wave_c64(self, jobs, wave, out):
        self._run_wave(jobs, wave, out, c64=True)

    def _run_wave(self, jobs, wave, out, c64: bool):
        prec = "c64" if c64 else "c128"
        sizes = [(footprint(jobs[i][0].qubit_count, prec) + ALIGN - 1) // ALIGN * ALIGN for i in wave]
        arena = C.c_void_p()
        call("qs_allocate_bytes", sum(sizes), C.byref(arena))
        try:
            ptrs, off = [], 0
            for i, sz in zip(wave, sizes):
                n = jobs[i][0].qubit_count
                p = arena.value + off
                call("qs_initialize_quantum_state_c64" if c64 else "qs_initialize_quantum_state", p, 1 << n,
                     self.stream)
                ptrs.append(p)
                off += sz
            k = len(wave)
            states = (C.c_void_p * k)(*ptrs)
            circs = (C.c_void_p * k)(*[jobs[i][0]._h for i in wave])
            if c64:  # one persistent launch: FP64 passes over complex64 tiles, or tensor-core blocks
                call("qs_batch_update_quantum_states_c64", circs, states, k, self.c64_executor, self.stream)
            else:  # every circuit in one persistent launch
                call("qs_batch_update_quantum_states", circs, states, k, self.stream)
            # all terms of all observables in one launch
            xm, zm, ny, offs, coefs, nq = [], [], [], [0], [], []
            for i in wave:
                obs = jobs[i][1]
                for t in obs.terms:
                    x, z, y = masks(t.targets, t.ids)
                    xm.append(x)
                    zm.append(z)
                    ny.append(y)
                    coefs.append(t.coef)
                offs.append(len(xm))
                nq.append(jobs[i][0].qubit_count)
            xa = np.ascontiguousarray(np.array(xm, dtype=np.uint64))
            za = np.ascontiguousarray(np.array(zm, dtype=np.uint64))
            ya = np.ascontiguousarray(np.array(ny, dtype=np.uint32))
            oa = np.ascontiguousarray(np.array(offs, dtype=np.uint32))
            qa = np.ascontiguousarray(np.array(nq, dtype=np.uint32))
            ca = np.ascontiguousarray(np.array(coefs, dtype=np.complex128)).view(np.float64)
            energies = np.zeros(2 * k)
            vp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
            call("qs_batch_expectation_weighted", states, vp(qa), k, vp(oa), vp(xa), vp(za), vp(ya), vp(ca),
                 int(c64), vp(energies), self.stream)
            for j, i in enumerate(wave):
                out[i] = float(energies[2 * j])
        finally:
            _lib.load().qs_release_quantum_state(arena.value)


def run_alone(circ, obs, mode: str = "staged") -> float:
    """Reference point for tests: the same job on its own state through the single-circuit API."""
    s = QuantumState(circ.qubit_count)
    circ.update_quantum_state(s, mode=mode)
    return obs.get_expectation_value(s)
