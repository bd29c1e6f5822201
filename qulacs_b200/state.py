"""Device-resident states with the cppsim QuantumState / DensityMatrix surface.

Mirrors ``QuantumStateBase`` / ``QuantumStateGpu`` (cppsim/state.hpp:18-417, cppsim/state_gpu.hpp) and
``DensityMatrixCpu`` (cppsim/state_dm.hpp): the amplitudes live in HBM as csim's complex128 layout,
every operation is a C-ABI call into the CUDA library, and ``get_device_name()`` is ``"gpu"``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import call

_default_stream = None


def set_default_stream(stream_handle: int | None) -> None:
    """Stream (a cudaStream_t as an int, e.g. ``torch.cuda.current_stream().cuda_stream``) for new states."""
    global _default_stream
    _default_stream = stream_handle


def _u(seq) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(seq, dtype=np.uint32))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class QuantumState:
    """n-qubit complex128 state vector in HBM (cppsim QuantumStateGpu semantics)."""

    def __init__(self, qubit_count: int, stream: int | None = None):
        _lib.load()
        if qubit_count < 1:
            raise ValueError("qubit_count must be >= 1")
        self.qubit_count = int(qubit_count)
        self.dim = 1 << self.qubit_count
        self.stream = _default_stream if stream is None else stream
        p = C.c_void_p()
        call("qs_allocate_quantum_state", self.dim, C.byref(p))
        self._ptr = p.value
        self.set_zero_state()

    # --- identity ---
    def get_qubit_count(self) -> int:
        return self.qubit_count

    def get_device_name(self) -> str:
        return "gpu"

    def is_state_vector(self) -> bool:
        return True

    def data_ptr(self) -> int:
        return self._ptr

    # --- initialisation (cppsim/state.hpp set_zero_state / set_computational_basis / load) ---
    def set_zero_state(self) -> None:
        call("qs_initialize_quantum_state", self._ptr, self.dim, self.stream)

    def set_computational_basis(self, basis: int) -> None:
        call("qs_set_computational_basis", int(basis), self._ptr, self.dim, self.stream)

    def load(self, src) -> None:
        if isinstance(src, QuantumState):
            if src.dim != self.dim:
                raise ValueError("dimension mismatch")
            src = src.get_vector()
        v = np.ascontiguousarray(np.asarray(src, dtype=np.complex128))
        if v.size != self.dim:
            raise ValueError(f"expected {self.dim} amplitudes, got {v.size}")
        call("qs_load_state", _ptr(v), self._ptr, self.dim, self.stream)
        call("qs_stream_synchronize", self.stream)

    def get_vector(self) -> np.ndarray:
        out = np.empty(self.dim, dtype=np.complex128)
        call("qs_get_state", self._ptr, _ptr(out), self.dim, self.stream)
        return out

    def copy(self) -> "QuantumState":
        s = QuantumState(self.qubit_count, self.stream)
        s.load(self)
        return s

    # --- statistics (csim stat_ops) ---
    def get_squared_norm(self) -> float:
        out = C.c_double()
        call("qs_state_norm_squared", self._ptr, self.dim, self.stream, C.byref(out))
        return out.value

    def get_zero_probability(self, target: int) -> float:
        out = C.c_double()
        call("qs_M0_prob", int(target), self._ptr, self.dim, self.stream, C.byref(out))
        return out.value

    def get_marginal_probability(self, measured_values) -> float:
        """Qulacs convention: a list of length n with 0, 1 or 2 (2 = not measured)."""
        tl = [i for i, v in enumerate(measured_values) if v in (0, 1)]
        vals = [measured_values[i] for i in tl]
        out = C.c_double()
        t, v = _u(tl), _u(vals)
        call("qs_marginal_prob", _ptr(t), _ptr(v), len(tl), self._ptr, self.dim, self.stream, C.byref(out))
        return out.value

    def sampling(self, sampling_count: int, random_seed: int | None = None) -> list:
        """cppsim QuantumStateCpu::sampling (cppsim/state.hpp:899-992): mt19937_64 draws."""
        if random_seed is None:
            random_seed = int(np.random.SeedSequence().entropy & 0xFFFFFFFF)
        out = np.empty(sampling_count, dtype=np.uint64)
        call("qs_state_sampling", self._ptr, self.dim, int(sampling_count), int(random_seed) & 0xFFFFFFFF,
             _ptr(out), self.stream)
        return [int(x) for x in out]

    def sampling_with_uniforms(self, uniforms) -> np.ndarray:
        u = np.ascontiguousarray(np.asarray(uniforms, dtype=np.float64))
        out = np.empty(u.size, dtype=np.uint64)
        call("qs_state_sampling_with_uniforms", self._ptr, self.dim, _ptr(u), u.size, _ptr(out), self.stream)
        return out

    def __del__(self):
        p = getattr(self, "_ptr", None)
        if p:
            try:
                _lib.load().qs_release_quantum_state(p)
            except Exception:
                pass
            self._ptr = None


class QuantumStateC64:
    """n-qubit complex64 state vector in HBM for the fused reduced-precision path.

    Reductions on it (norm, <P>, inner product with a complex128 state, sampling prefix sums) read
    the single-precision amplitudes and accumulate in FP64.
    """

    def __init__(self, qubit_count: int, stream: int | None = None):
        _lib.load()
        self.qubit_count = int(qubit_count)
        self.dim = 1 << self.qubit_count
        self.stream = _default_stream if stream is None else stream
        p = C.c_void_p()
        call("qs_allocate_quantum_state_c64", self.dim, C.byref(p))
        self._ptr = p.value
        self.set_zero_state()

    def get_qubit_count(self) -> int:
        return self.qubit_count

    def get_device_name(self) -> str:
        return "gpu"

    def is_state_vector(self) -> bool:
        return True

    def data_ptr(self) -> int:
        return self._ptr

    def set_zero_state(self) -> None:
        call("qs_initialize_quantum_state_c64", self._ptr, self.dim, self.stream)

    def load(self, src) -> None:
        """From a complex128 QuantumState (rounded on the device) or a host vector."""
        if isinstance(src, QuantumState):
            call("qs_state_to_c64", src.data_ptr(), self._ptr, self.dim, self.stream)
            return
        v = np.ascontiguousarray(np.asarray(src, dtype=np.complex128))
        tmp = QuantumState(self.qubit_count, self.stream)
        tmp.load(v)
        call("qs_state_to_c64", tmp.data_ptr(), self._ptr, self.dim, self.stream)
        call("qs_stream_synchronize", self.stream)

    def to_c128(self, out: QuantumState | None = None) -> QuantumState:
        out = out or QuantumState(self.qubit_count, self.stream)
        call("qs_state_to_c128", self._ptr, out.data_ptr(), self.dim, self.stream)
        return out

    def get_vector(self) -> np.ndarray:
        return self.to_c128().get_vector()

    def get_squared_norm(self) -> float:
        out = C.c_double()
        call("qs_state_norm_squared_c64", self._ptr, self.dim, self.stream, C.byref(out))
        return out.value

    def inner_product_with(self, bra: QuantumState) -> complex:
        """<bra|self> with a complex128 bra, FP64 accumulation."""
        out = np.zeros(2)
        call("qs_state_inner_product_c128_c64", bra.data_ptr(), self._ptr, self.dim, self.stream, _ptr(out))
        return complex(out[0], out[1])

    def infidelity(self, reference: QuantumState) -> float:
        """1 - |<reference|self>|^2 / (<self|self> <reference|reference>)."""
        ip = self.inner_product_with(reference)
        return 1.0 - abs(ip) ** 2 / (self.get_squared_norm() * reference.get_squared_norm())

    def sampling_with_uniforms(self, uniforms) -> np.ndarray:
        u = np.ascontiguousarray(np.asarray(uniforms, dtype=np.float64))
        out = np.empty(u.size, dtype=np.uint64)
        call("qs_state_sampling_with_uniforms_c64", self._ptr, self.dim, _ptr(u), u.size, _ptr(out), self.stream)
        return out

    def __del__(self):
        p = getattr(self, "_ptr", None)
        if p:
            try:
                _lib.load().qs_release_quantum_state(p)
            except Exception:
                pass
            self._ptr = None


def inner_product(bra: QuantumState, ket: QuantumState) -> complex:
    """csim state_inner_product (stat_ops.cpp:65-86): sum conj(bra_i) ket_i."""
    if bra.dim != ket.dim:
        raise ValueError("dimension mismatch")
    out = np.zeros(2)
    call("qs_state_inner_product", bra.data_ptr(), ket.data_ptr(), bra.dim, bra.stream, _ptr(out))
    return complex(out[0], out[1])


class DensityMatrix:
    """n-qubit density matrix (dim x dim, row-major, complex128) in HBM (cppsim/state_dm.hpp)."""

    def __init__(self, qubit_count: int, stream: int | None = None):
        _lib.load()
        self.qubit_count = int(qubit_count)
        self.dim = 1 << self.qubit_count
        self.stream = _default_stream if stream is None else stream
        p = C.c_void_p()
        call("qs_dm_allocate", self.dim, C.byref(p))
        self._ptr = p.value
        self.set_zero_state()

    def get_qubit_count(self) -> int:
        return self.qubit_count

    def get_device_name(self) -> str:
        return "gpu"

    def is_state_vector(self) -> bool:
        return False

    def data_ptr(self) -> int:
        return self._ptr

    def set_zero_state(self) -> None:
        call("qs_dm_initialize_quantum_state", self._ptr, self.dim, self.stream)

    def load(self, src) -> None:
        if isinstance(src, QuantumState):
            call("qs_dm_initialize_with_pure_state", self._ptr, src.data_ptr(), self.dim, self.stream)
            return
        m = np.ascontiguousarray(np.asarray(src, dtype=np.complex128))
        if m.ndim == 1:
            m = np.ascontiguousarray(np.outer(m, m.conj()))
        if m.shape != (self.dim, self.dim):
            raise ValueError("shape mismatch")
        call("qs_load_state", _ptr(m), self._ptr, self.dim * self.dim, self.stream)
        call("qs_stream_synchronize", self.stream)

    def get_matrix(self) -> np.ndarray:
        out = np.empty((self.dim, self.dim), dtype=np.complex128)
        call("qs_get_state", self._ptr, _ptr(out), self.dim * self.dim, self.stream)
        return out

    def get_squared_norm(self) -> float:
        out = C.c_double()
        call("qs_dm_state_norm_squared", self._ptr, self.dim, self.stream, C.byref(out))
        return out.value

    def sampling_with_uniforms(self, uniforms) -> np.ndarray:
        u = np.ascontiguousarray(np.asarray(uniforms, dtype=np.float64))
        out = np.empty(u.size, dtype=np.uint64)
        call("qs_dm_sampling_with_uniforms", self._ptr, self.dim, _ptr(u), u.size, _ptr(out), self.stream)
        return out

    def __del__(self):
        p = getattr(self, "_ptr", None)
        if p:
            try:
                _lib.load().qs_release_quantum_state(p)
            except Exception:
                pass
            self._ptr = None
