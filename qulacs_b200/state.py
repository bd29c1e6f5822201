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


def _coef(c) -> np.ndarray:
    c = complex(c)
    return np.array([c.real, c.imag])


def _random_seed() -> int:
    """A fresh 32-bit seed, for calls that take an optional one (the reference draws it from its Random)."""
    return int(np.random.SeedSequence().entropy & 0xFFFFFFFF)


def _marginal_lists(measured_values, qubit_count: int):
    """Qulacs convention: a list of length n with 0, 1 or 2 (2 = not measured)."""
    if len(measured_values) != qubit_count:
        raise ValueError("the length of measured_values must be equal to qubit_count")
    tl = [i for i, v in enumerate(measured_values) if v in (0, 1)]
    return _u(tl), _u([measured_values[i] for i in tl])


class QuantumState:
    """n-qubit complex128 state vector in HBM (cppsim QuantumStateGpu semantics)."""

    def __init__(self, qubit_count: int, stream: int | None = None):
        _lib.load()
        if qubit_count < 1:
            raise ValueError("qubit_count must be >= 1")
        self.classical_register: list = []
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

    def set_zero_norm_state(self) -> None:
        """All amplitudes 0 (cppsim/state.hpp:484-487)."""
        self.set_zero_state()
        self.multiply_coef(0.0)

    def set_Haar_random_state(self, seed: int | None = None) -> None:
        """Haar-random pure state (cppsim/state.hpp:520-540): independent complex Gaussian amplitudes,
        normalised.  A seed gives the same state on every run; the values are not the reference's (its
        Gaussians come from its own Random), only the distribution is."""
        if seed is None:
            seed = _random_seed()
        call("qs_initialize_Haar_random_state_with_seed", self._ptr, self.dim, int(seed) & 0xFFFFFFFF, self.stream)

    def load(self, src) -> None:
        """From another state vector (device copy, classical register included) or host amplitudes
        (cppsim/state.hpp:700-760)."""
        if isinstance(src, DensityMatrix):
            raise TypeError("cannot load DensityMatrix to StateVector")
        if isinstance(src, QuantumState):
            if src.qubit_count != self.qubit_count:
                raise ValueError("invalid qubit count")
            call("qs_copy_state", src._ptr, self._ptr, self.dim, self.stream)
            self.classical_register = list(src.classical_register)
            return
        v = np.ascontiguousarray(np.asarray(src, dtype=np.complex128))
        if v.size != self.dim:
            raise ValueError(f"expected {self.dim} amplitudes, got {v.size}")
        call("qs_load_state", _ptr(v), self._ptr, self.dim, self.stream)
        call("qs_stream_synchronize", self.stream)

    def get_vector(self) -> np.ndarray:
        out = np.empty(self.dim, dtype=np.complex128)
        call("qs_get_state", self._ptr, _ptr(out), self.dim, self.stream)
        return out

    def get_amplitude(self, index: int) -> complex:
        out = np.zeros(2)
        call("qs_get_amplitude", self._ptr, self.dim, int(index), _ptr(out), self.stream)
        return complex(out[0], out[1])

    def allocate_buffer(self) -> "QuantumState":
        """A new |0...0> state of the same size (cppsim/state.hpp:670-682)."""
        return QuantumState(self.qubit_count, self.stream)

    def copy(self) -> "QuantumState":
        """Deep copy on the device, classical register included (cppsim/state.hpp:688-697)."""
        s = self.allocate_buffer()
        s.load(self)
        return s

    # --- whole-state arithmetic (csim update_ops_named_state.cpp) ---
    def _other(self, state, what) -> "QuantumState":
        if not isinstance(state, QuantumState):
            raise TypeError(f"{what}: cannot add DensityMatrix to StateVector")
        if state.dim != self.dim:
            raise ValueError(f"{what}: invalid qubit count")
        return state

    def add_state(self, state: "QuantumState") -> None:
        """self += state (cppsim/state.hpp:825-836)."""
        call("qs_state_add", self._other(state, "add_state")._ptr, self._ptr, self.dim, self.stream)

    def add_state_with_coef(self, coef: complex, state: "QuantumState") -> None:
        """self += coef * state (cppsim/state.hpp:841-856)."""
        c = _coef(coef)
        call("qs_state_add_with_coef", _ptr(c), self._other(state, "add_state_with_coef")._ptr, self._ptr,
             self.dim, self.stream)

    def multiply_coef(self, coef: complex) -> None:
        c = _coef(coef)
        call("qs_state_multiply", _ptr(c), self._ptr, self.dim, self.stream)

    def normalize(self, squared_norm: float) -> None:
        """Amplitudes *= 1 / sqrt(squared_norm) (csim update_ops_named_state.cpp:21-30)."""
        call("qs_normalize", float(squared_norm), self._ptr, self.dim, self.stream)

    def multiply_elementwise_function(self, func) -> None:
        """amplitude[i] *= func(i): the values are tabulated on the host, then multiplied in on the
        device (cppsim/state.hpp:885-891)."""
        f = np.fromiter((complex(func(i)) for i in range(self.dim)), dtype=np.complex128, count=self.dim)
        tmp = QuantumState(self.qubit_count, self.stream)
        tmp.load(f)
        call("qs_state_multiply_elementwise", tmp._ptr, self._ptr, self.dim, self.stream)
        call("qs_stream_synchronize", self.stream)

    # --- classical register (cppsim/state.hpp:313-340) ---
    def get_classical_value(self, index: int) -> int:
        if len(self.classical_register) <= index:
            self.classical_register.extend([0] * (index + 1 - len(self.classical_register)))
        return self.classical_register[index]

    def set_classical_value(self, index: int, value: int) -> None:
        if len(self.classical_register) <= index:
            self.classical_register.extend([0] * (index + 1 - len(self.classical_register)))
        self.classical_register[index] = int(value)

    def get_classical_register(self) -> list:
        return list(self.classical_register)

    def to_string(self) -> str:
        """Debug text in cppsim's layout (cppsim/state.hpp:365-392)."""
        body = "\n".join(f"({a.real:g},{a.imag:g})" for a in self.get_vector())
        return (f" *** Quantum State ***\n * Qubit Count : {self.qubit_count}\n * Dimension   : {self.dim}\n"
                f" * State vector : \n{body}\n")

    def __str__(self) -> str:
        return self.to_string()

    # --- statistics (csim stat_ops) ---
    def get_squared_norm(self) -> float:
        out = C.c_double()
        call("qs_state_norm_squared", self._ptr, self.dim, self.stream, C.byref(out))
        return out.value

    def get_zero_probability(self, target: int) -> float:
        out = C.c_double()
        call("qs_M0_prob", int(target), self._ptr, self.dim, self.stream, C.byref(out))
        return out.value

    def get_entropy(self) -> float:
        """Shannon entropy of the computational-basis distribution (csim stat_ops_probability.cpp:83-99)."""
        out = C.c_double()
        call("qs_measurement_distribution_entropy", self._ptr, self.dim, self.stream, C.byref(out))
        return out.value

    def get_marginal_probability(self, measured_values) -> float:
        """Qulacs convention: a list of length n with 0, 1 or 2 (2 = not measured)."""
        t, v = _marginal_lists(measured_values, self.qubit_count)
        out = C.c_double()
        call("qs_marginal_prob", _ptr(t), _ptr(v), t.size, self._ptr, self.dim, self.stream, C.byref(out))
        return out.value

    def sampling(self, sampling_count: int, random_seed: int | None = None) -> list:
        """cppsim QuantumStateCpu::sampling (cppsim/state.hpp:899-992): mt19937_64 draws."""
        if random_seed is None:
            random_seed = _random_seed()
        out = np.empty(sampling_count, dtype=np.uint64)
        call("qs_state_sampling", self._ptr, self.dim, int(sampling_count), int(random_seed) & 0xFFFFFFFF,
             _ptr(out), self.stream)
        return [int(x) for x in out]

    def sampling_with_uniforms(self, uniforms) -> np.ndarray:
        u = np.ascontiguousarray(np.asarray(uniforms, dtype=np.float64))
        out = np.empty(u.size, dtype=np.uint64)
        call("qs_state_sampling_with_uniforms", self._ptr, self.dim, _ptr(u), u.size, _ptr(out), self.stream)
        return out

    def sampling_with_uniforms_flagged(self, uniforms, eps: float = 1e-12):
        """Indices for the supplied uniforms and, per draw, whether it lies within `eps` of a cumulative
        boundary of the FP64 prefix sums (the draws whose index may differ from the reference's serial
        prefix by rounding).  Returns (indices, flags)."""
        u = np.ascontiguousarray(np.asarray(uniforms, dtype=np.float64))
        out = np.empty(u.size, dtype=np.uint64)
        flags = np.zeros(u.size, dtype=np.uint8)
        cnt = C.c_uint()
        call("qs_state_sampling_with_uniforms_flagged", self._ptr, self.dim, _ptr(u), u.size, float(eps), _ptr(out),
             _ptr(flags), C.byref(cnt), self.stream)
        return out, flags.astype(bool)

    def sampling_boundary_draws(self, sampling_count: int, random_seed: int, eps: float = 1e-12) -> int:
        """How many of the draws `sampling(sampling_count, random_seed)` makes lie within `eps` of a
        cumulative boundary."""
        u = np.empty(int(sampling_count), dtype=np.float64)
        call("qs_reference_uniforms", int(random_seed) & 0xFFFFFFFF, int(sampling_count), _ptr(u))
        return int(self.sampling_with_uniforms_flagged(u, eps)[1].sum())

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
        self.classical_register: list = []
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

    def set_zero_norm_state(self) -> None:
        """The zero matrix (cppsim/state_dm.hpp:41-44)."""
        self.set_zero_state()
        self.multiply_coef(0.0)

    def set_computational_basis(self, basis: int) -> None:
        """|basis><basis| (cppsim/state_dm.hpp:51-61): entry basis * dim + basis of the dim^2 vector."""
        if not 0 <= int(basis) < self.dim:
            raise IndexError("index of computational basis must be smaller than 2^qubit_count")
        b = int(basis)
        call("qs_set_computational_basis", b * self.dim + b, self._ptr, self.dim * self.dim, self.stream)

    def set_Haar_random_state(self, seed: int | None = None) -> None:
        """|psi><psi| of a Haar-random pure state (cppsim/state_dm.hpp:66-80)."""
        pure = QuantumState(self.qubit_count, self.stream)
        pure.set_Haar_random_state(seed)
        call("qs_dm_initialize_with_pure_state", self._ptr, pure.data_ptr(), self.dim, self.stream)
        call("qs_stream_synchronize", self.stream)

    def allocate_buffer(self) -> "DensityMatrix":
        return DensityMatrix(self.qubit_count, self.stream)

    def copy(self) -> "DensityMatrix":
        d = self.allocate_buffer()
        d.load(self)
        return d

    def load(self, src) -> None:
        """From a state vector (|psi><psi|), another density matrix (device copy), a host vector or a
        host dim x dim matrix (cppsim/state_dm.hpp:199-281)."""
        if isinstance(src, DensityMatrix):
            if src.qubit_count != self.qubit_count:
                raise ValueError("invalid qubit count")
            call("qs_copy_state", src._ptr, self._ptr, self.dim * self.dim, self.stream)
            self.classical_register = list(src.classical_register)
            return
        if isinstance(src, QuantumState):
            if src.qubit_count != self.qubit_count:
                raise ValueError("invalid qubit count")
            call("qs_dm_initialize_with_pure_state", self._ptr, src.data_ptr(), self.dim, self.stream)
            self.classical_register = list(src.classical_register)
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

    def get_zero_probability(self, target: int) -> float:
        if not 0 <= int(target) < self.qubit_count:
            raise IndexError("index of target qubit must be smaller than qubit_count")
        out = C.c_double()
        call("qs_dm_M0_prob", int(target), self._ptr, self.dim, self.stream, C.byref(out))
        return out.value

    def get_marginal_probability(self, measured_values) -> float:
        t, v = _marginal_lists(measured_values, self.qubit_count)
        out = C.c_double()
        call("qs_dm_marginal_prob", _ptr(t), _ptr(v), t.size, self._ptr, self.dim, self.stream, C.byref(out))
        return out.value

    def get_entropy(self) -> float:
        out = C.c_double()
        call("qs_dm_measurement_distribution_entropy", self._ptr, self.dim, self.stream, C.byref(out))
        return out.value

    def normalize(self, squared_norm: float) -> None:
        """rho *= 1 / squared_norm (csim update_ops_dm.cpp:14-28)."""
        call("qs_dm_normalize", float(squared_norm), self._ptr, self.dim, self.stream)

    def _other(self, state, what) -> "DensityMatrix":
        if not isinstance(state, DensityMatrix):
            raise TypeError(f"{what}: a state vector cannot be added to a DensityMatrix")
        if state.dim != self.dim:
            raise ValueError(f"{what}: invalid qubit count")
        return state

    def add_state(self, state: "DensityMatrix") -> None:
        call("qs_dm_state_add", self._other(state, "add_state")._ptr, self._ptr, self.dim, self.stream)

    def add_state_with_coef(self, coef: complex, state: "DensityMatrix") -> None:
        c = _coef(coef)
        call("qs_dm_state_add_with_coef", _ptr(c), self._other(state, "add_state_with_coef")._ptr, self._ptr,
             self.dim, self.stream)

    def multiply_coef(self, coef: complex) -> None:
        c = _coef(coef)
        call("qs_dm_state_multiply", _ptr(c), self._ptr, self.dim, self.stream)

    def multiply_elementwise_function(self, func) -> None:
        raise NotImplementedError("multiply_elementwise_function is not defined for DensityMatrix")

    def sampling(self, sampling_count: int, random_seed: int | None = None) -> list:
        """DensityMatrixCpu::sampling (cppsim/state_dm.hpp:383-407): mt19937_64(seed) uniforms over the
        diagonal's prefix sums."""
        if random_seed is None:
            random_seed = _random_seed()
        u = np.empty(int(sampling_count), dtype=np.float64)
        call("qs_reference_uniforms", int(random_seed) & 0xFFFFFFFF, u.size, _ptr(u))
        return [int(x) for x in self.sampling_with_uniforms(u)]

    def sampling_with_uniforms(self, uniforms) -> np.ndarray:
        u = np.ascontiguousarray(np.asarray(uniforms, dtype=np.float64))
        out = np.empty(u.size, dtype=np.uint64)
        call("qs_dm_sampling_with_uniforms", self._ptr, self.dim, _ptr(u), u.size, _ptr(out), self.stream)
        return out

    def get_classical_value(self, index: int) -> int:
        return QuantumState.get_classical_value(self, index)

    def set_classical_value(self, index: int, value: int) -> None:
        QuantumState.set_classical_value(self, index, value)

    def get_classical_register(self) -> list:
        return list(self.classical_register)

    def to_string(self) -> str:
        """Debug text in cppsim's layout (cppsim/state_dm.hpp:409-422)."""
        m = self.get_matrix()
        body = "\n".join(" ".join(f"({a.real:g},{a.imag:g})" for a in row) for row in m)
        return (f" *** Density Matrix ***\n * Qubit Count : {self.qubit_count}\n * Dimension   : {self.dim}\n"
                f" * Density matrix : \n{body}\n")

    def __str__(self) -> str:
        return self.to_string()

    def __del__(self):
        p = getattr(self, "_ptr", None)
        if p:
            try:
                _lib.load().qs_release_quantum_state(p)
            except Exception:
                pass
            self._ptr = None


# ---- qulacs.state helpers (python/cppsim_wrapper.cpp:650-680; cppsim/state.cpp) ----
def _u32(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.uint32))


def tensor_product(state_left, state_right):
    """state::tensor_product: the right state on the low qubits (stat_ops.cpp:111-121,
    stat_ops_dm.cpp:193-211); both state vectors or both density matrices."""
    n = state_left.qubit_count + state_right.qubit_count
    if isinstance(state_left, DensityMatrix) and isinstance(state_right, DensityMatrix):
        out, fn = DensityMatrix(n, state_left.stream), "qs_dm_state_tensor_product"
    elif isinstance(state_left, QuantumState) and isinstance(state_right, QuantumState):
        out, fn = QuantumState(n, state_left.stream), "qs_state_tensor_product"
    else:
        raise TypeError("tensor_product needs two QuantumStates or two DensityMatrices")
    if state_right.stream != state_left.stream:  # the right state's pending writes finish first
        call("qs_stream_synchronize", state_right.stream)
    call(fn, state_left.data_ptr(), state_left.dim, state_right.data_ptr(), state_right.dim, out.data_ptr(),
         out.stream)
    return out


def permutate_qubit(state, qubit_order):
    """state::permutate_qubit: new qubit q is old qubit qubit_order[q] (stat_ops.cpp:122-134,
    stat_ops_dm.cpp:213-231)."""
    order = _u32(qubit_order)
    if isinstance(state, DensityMatrix):
        out, fn = DensityMatrix(state.qubit_count, state.stream), "qs_dm_state_permutate_qubit"
    else:
        out, fn = QuantumState(state.qubit_count, state.stream), "qs_state_permutate_qubit"
    call(fn, _ptr(order), state.data_ptr(), out.data_ptr(), order.size, state.dim, state.stream)
    return out


def drop_qubit(state: QuantumState, target, projection) -> QuantumState:
    """state::drop_qubit: the amplitudes with target[j] = projection[j], on the remaining qubits
    (stat_ops.cpp:136-158; not renormalised)."""
    t, p = _u32(target), _u32(projection)
    if t.size != p.size:
        raise ValueError("target and projection differ in length")
    out = QuantumState(state.qubit_count - t.size, state.stream)
    call("qs_state_drop_qubits", _ptr(t), _ptr(p), t.size, state.data_ptr(), out.data_ptr(), state.dim, state.stream)
    return out


def partial_trace(state, target_traceout) -> DensityMatrix:
    """state::partial_trace: trace the listed qubits out of a state vector or a density matrix
    (stat_ops_dm.cpp:233-296)."""
    t = _u32(target_traceout)
    out = DensityMatrix(state.qubit_count - t.size, state.stream)
    fn = ("qs_dm_state_partial_trace_from_density_matrix" if isinstance(state, DensityMatrix)
          else "qs_dm_state_partial_trace_from_state_vector")
    call(fn, _ptr(t), t.size, state.data_ptr(), out.data_ptr(), state.dim, state.stream)
    return out
