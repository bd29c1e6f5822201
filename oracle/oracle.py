"""Python loader for the oracle (test infrastructure only).

Two CPU implementations share one calling convention (numpy complex128 arrays, csim argument order):

* ``port()``: the C restatement in ``oracle/qs_oracle.c`` (always buildable with gcc).
* ``reference()``: the reference csim itself, compiled from its own sources by ``oracle/Makefile``
  into ``oracle/_ref/libcsim_ref.so``; ``None`` when it was not built.

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import this module.
"""
from __future__ import annotations

import ctypes as C
import math
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


def reference_root() -> str:
    """The reference checkout: $QULACS_REFERENCE_ROOT, else a ``reference`` directory beside the repository."""
    env = os.environ.get("QULACS_REFERENCE_ROOT")
    if env:
        return env
    return os.path.abspath(os.path.join(HERE, "..", "..", "reference"))


def build_reference(ref_root: str | None = None) -> str | None:
    """Compile the reference csim when its sources are present (never on a machine without them)."""
    ref_root = ref_root or reference_root()
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

    # ---- whole-state arithmetic ----
    def state_add_with_coef(self, coef, added, s):
        c = np.array([complex(coef).real, complex(coef).imag])
        self._f("state_add_with_coef")(_ptr(c), _ptr(added), _ptr(s), _IT(s.size))

    def state_multiply(self, coef, s):
        c = np.array([complex(coef).real, complex(coef).imag])
        self._f("state_multiply")(_ptr(c), _ptr(s), _IT(s.size))

    def normalize(self, squared_norm, s):
        self._f("normalize")(_D(squared_norm), _ptr(s), _IT(s.size))

    def measurement_distribution_entropy(self, s) -> float:
        return self._f("measurement_distribution_entropy", _D)(_ptr(s), _IT(s.size))

    def dm_measurement_distribution_entropy(self, r) -> float:
        return self._f("dm_measurement_distribution_entropy", _D)(_ptr(r), _IT(r.shape[0]))

    def dm_normalize(self, squared_norm, r):
        self._f("dm_normalize")(_D(squared_norm), _ptr(r), _IT(r.shape[0]))

    def dm_M0_prob(self, t, r):
        return self._f("dm_M0_prob", _D)(_U(t), _ptr(r), _IT(r.shape[0]))

    def dm_M1_prob(self, t, r):
        return self._f("dm_M1_prob", _D)(_U(t), _ptr(r), _IT(r.shape[0]))

    def dm_marginal_prob(self, tl, vals, r):
        tl, vals = _u32(tl), _u32(vals)
        return self._f("dm_marginal_prob", _D)(_ptr(tl), _ptr(vals), _U(tl.size), _ptr(r), _IT(r.shape[0]))

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


# ---------------------------------------------------------------- reference RNG and NoiseSimulator

def std_normals(seed, count):
    """cppsim Random::normal (utility.hpp:86): libstdc++ std::normal_distribution<double>(0, 1) over
    mt19937_64(seed) -- the Marsaglia polar method: x, y = 2u - 1 until 0 < r2 = x^2 + y^2 <= 1, then
    y * m is returned and x * m kept for the next call, m = sqrt(-2 log(r2) / r2)."""
    u = mt19937_64_uniforms(seed, 4 * count + 64)
    k, out = 0, []
    while len(out) < count:
        x = 2.0 * u[k] - 1.0
        y = 2.0 * u[k + 1] - 1.0
        k += 2
        r2 = x * x + y * y
        if r2 > 1.0 or r2 == 0.0:
            continue
        m = math.sqrt(-2.0 * math.log(r2) / r2)
        out += [y * m, x * m]
    return np.array(out[:count])


def random_unitary(qubit_count, seed):
    """cppsim gate::RandomUnitary(targets, seed) (gate_factory.cpp:351-380): entries (normal() + i normal())
    / sqrt(2) row by row -- with g++ the imaginary draw comes first -- then Householder QR and column c of
    Q times R_cc / |R_cc|."""
    d = 1 << qubit_count
    g = std_normals(seed, 2 * d * d)
    a = ((g[1::2] + 1j * g[0::2]) / math.sqrt(2.0)).reshape(d, d)
    q, r = np.linalg.qr(a)
    ph = np.diag(r) / np.abs(np.diag(r))
    return q * ph[None, :]


def random_operator_terms(qubit_count, operator_count, seed):
    """GeneralQuantumOperator::add_random_operator(count, seed) (general_quantum_operator.cpp:179-202): per
    term, Random::int32() % 4 for qubits 0..n-1 (int32 = mt() % ULONG_MAX, utility.hpp:100), then
    uniform() * 2 - 1.  Returns [(pauli ids per qubit, coefficient)]."""
    raw = mt19937_64_raw(seed, operator_count * (qubit_count + 1))
    out, k = [], 0
    for _ in range(operator_count):
        ids = [int(raw[k + q] % 0xFFFFFFFFFFFFFFFF % 4) for q in range(qubit_count)]
        k += qubit_count
        u = float(raw[k]) / 18446744073709551616.0
        k += 1
        out.append((ids, (u if u < 1.0 else np.nextafter(1.0, 0.0)) * 2 - 1.0))
    return out


def mt19937_64_uniforms(seed, count):
    """cppsim Random (utility.hpp:54-80): libstdc++'s generate_canonical<double, 53> over mt19937_64 for a
    64-bit engine: x / 2^64, clamped below 1."""
    out = []
    for y in mt19937_64_raw(seed, count):
        r = float(y) / 18446744073709551616.0
        if r >= 1.0:
            r = np.nextafter(1.0, 0.0)
        out.append(r)
    return np.array(out)


def mt19937_64_raw(seed, count):
    """mt19937_64 (Matsumoto & Nishimura 2000, 64-bit parameters): the first `count` outputs for `seed`."""
    n, m = 312, 156
    mt = [0] * n
    mt[0] = seed & 0xFFFFFFFFFFFFFFFF
    for i in range(1, n):
        mt[i] = (6364136223846793005 * (mt[i - 1] ^ (mt[i - 1] >> 62)) + i) & 0xFFFFFFFFFFFFFFFF
    idx = n
    out = []
    upper, lower = 0xFFFFFFFF80000000, 0x7FFFFFFF
    for _ in range(count):
        if idx >= n:
            for i in range(n):
                y = (mt[i] & upper) | (mt[(i + 1) % n] & lower)
                v = mt[(i + m) % n] ^ (y >> 1)
                if y & 1:
                    v ^= 0xB5026F5AA96619E9
                mt[i] = v
            idx = 0
        y = mt[idx]
        idx += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        out.append(y)
    return out


def _pauli(ids):
    """Pauli string matrix, index bit j <-> ids[j] (ids 0..3 = I X Y Z)."""
    P = [np.eye(2), np.array([[0, 1], [1, 0]]), np.array([[0, -1j], [1j, 0]]), np.diag([1.0, -1.0])]
    m = np.array([[1.0 + 0j]])
    for i in ids:
        m = np.kron(P[i], m)
    return m


def depolarizing_channel(targets, p):
    """(Kraus operators, cumulative distribution) in the order NoiseSimulator samples them:
    gate_factory.cpp:451-500 lists ({X, Z, Y, I} with {p/3, p/3, p/3, 1-p}; {I, Pauli(i%4, i//4)
    for i = 1..15} with {1-p, p/15, ...}) reordered by descending (probability, index)
    (QuantumGate_Probabilistic::optimize_ProbablisticGate, gate_general.hpp:350-372)."""
    if len(targets) == 1:
        ops = [[1], [3], [2], [0]]
        probs = [p / 3, p / 3, p / 3, 1 - p]
    else:
        ops = [[i % 4, i // 4] for i in range(16)]
        probs = [1 - p] + [p / 15] * 15
    order = sorted(((probs[i], i) for i in range(len(ops))), reverse=True)
    kraus = [ops[i] for _, i in order]
    cum = [0.0]
    for w, _ in order:
        cum.append(cum[-1] + w)
    return kraus, cum


def noise_simulator_execute(gates, n, sample_count, seed, sim, apply_gate, init=None, eps=1e-12):
    """cppsim NoiseSimulator::execute (noisesimulator.cpp:18-198) restated for small n.

    `gates`: list of ("DEPOL", targets, p) channels and other gates that `apply_gate(g, state)` applies.
    One mt19937_64(seed) stream gives the selection uniforms (sample-major, channels in circuit
    order; operator = lower_bound(cumulative, u) - 1, noisesimulator.cpp:167-185), then each
    distinct trajectory's sampling uniforms in the order the trajectories are visited (descending
    lexicographic order of the choices, noisesimulator.cpp:85-120).  Each trajectory is simulated
    from the initial state.  Returns (samples, near_boundary flags, [(choices, count), ...])."""
    import bisect
    chans = [(j, depolarizing_channel(list(g[1]), g[2])) for j, g in enumerate(gates) if g[0] == "DEPOL"]
    u = mt19937_64_uniforms(seed, sample_count * len(chans) + sample_count)
    k = 0
    sel = []
    for _ in range(sample_count):
        row = []
        for _, (kraus, cum) in chans:
            pos = bisect.bisect_left(cum, u[k]) - 1
            row.append(min(max(pos, 0), len(kraus) - 1))
            k += 1
        sel.append(tuple(row))
    sel.sort(reverse=True)
    requests = []
    for s in sel:
        if requests and requests[-1][0] == s:
            requests[-1][1] += 1
        else:
            requests.append([s, 1])
    samples, near = [], []
    for choice, count in requests:
        state = np.zeros(1 << n, dtype=np.complex128)
        if init is None:
            state[0] = 1
        else:
            state[:] = init
        ci = 0
        for g in gates:
            if g[0] == "DEPOL":
                kraus, _ = chans[ci][1]
                ids = kraus[choice[ci]]
                ci += 1
                if any(ids):
                    sim.multi_qubit_dense_matrix_gate(list(g[1]), _pauli(ids), state)
            else:
                apply_gate(g, state)
        s, nb = sim.sampling_with_uniforms(state, u[k:k + count], eps=eps)
        k += count
        samples.extend(int(x) for x in s)
        near.extend(bool(x) for x in nb)
    return np.array(samples, dtype=np.uint64), np.array(near), [(c, m) for c, m in requests]
