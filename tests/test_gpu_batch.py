"""Batched uneven circuits in one persistent launch: each result equals the single-circuit result
(same kernels, same order) and the oracle; fused complex64 batches meet the infidelity bar."""
import numpy as np
import pytest

from conftest import EV_TOL
from qulacs_b200 import QuantumState
from qulacs_b200 import workloads as W
from qulacs_b200.batch import BatchRunner, run_alone
from oracle import replay as R

pytestmark = pytest.mark.gpu


def make_jobs(seed, count, nmin, nmax):
    rng = np.random.default_rng(seed)
    jobs, specs = [], []
    for i in range(count):
        n = int(rng.integers(nmin, nmax + 1))
        d = int(rng.integers(4, 17))
        gates = W.hea_circuit(n, d, seed=seed * 1000 + i)
        terms = W.random_pauli_terms(n, 40, 1, 4, seed=seed * 1000 + 500 + i)
        jobs.append((W.to_circuit(gates, n), W.to_observable(terms, n)))
        specs.append((n, gates, terms))
    return jobs, specs


def test_batch_matches_alone_and_oracle(port):
    jobs, specs = make_jobs(7, 24, 4, 15)
    runner = BatchRunner(memory_budget_bytes=1 << 20)  # forces several waves
    got = runner.run(jobs)
    assert runner.stats.waves >= 2
    for (circ, obs), (n, gates, terms), e in zip(jobs, specs, got):
        alone = run_alone(circ, obs)
        assert abs(e - alone) <= 1e-12  # same states; the reductions chunk the sums differently
        psi = np.zeros(1 << n, dtype=np.complex128)
        psi[0] = 1
        R.run_on_cpu(gates, psi, port)
        want = sum(c * port.expectation_value(tl, ids, psi) for c, tl, ids in terms)
        assert abs(e - want) <= EV_TOL


def test_batch_states_match_gate_by_gate(port):
    """The states after the persistent batch equal each circuit's gate-by-gate result (1e-12)."""
    import ctypes as C

    from qulacs_b200._lib import call
    jobs, specs = make_jobs(11, 6, 6, 13)
    states = [QuantumState(n) for n, _, _ in specs]
    circs = (C.c_void_p * len(jobs))(*[j[0]._h for j in jobs])
    ptrs = (C.c_void_p * len(jobs))(*[s.data_ptr() for s in states])
    call("qs_batch_update_quantum_states", circs, ptrs, len(jobs), None)
    for (circ, _), s, (n, gates, _) in zip(jobs, states, specs):
        psi = np.zeros(1 << n, dtype=np.complex128)
        psi[0] = 1
        R.run_on_cpu(gates, psi, port)
        v = s.get_vector()
        assert np.max(np.abs(v - psi)) <= 1e-12
        alone = QuantumState(n)
        circ.set_fusion(2)  # the batch's block size
        circ.update_quantum_state(alone, mode="staged_fused")
        if n <= 11:  # same tiles (the multi-circuit kernel's are 2^11, the single-circuit kernel's 2^12)
            assert np.array_equal(v, alone.get_vector())  # bit-identical alone and in the batch
        else:  # same gates per amplitude in another pass order: rounding-level differences only
            assert np.max(np.abs(v - alone.get_vector())) <= 1e-14


@pytest.mark.parametrize("executor", ["auto", "tensor", "fp64"])
def test_batch_fused_c64(port, executor):
    jobs, specs = make_jobs(13, 6, 10, 14)
    got = BatchRunner(1 << 30, precision="c64", c64_executor=executor).run(jobs)
    for (n, gates, terms), e in zip(specs, got):
        psi = np.zeros(1 << n, dtype=np.complex128)
        psi[0] = 1
        R.run_on_cpu(gates, psi, port)
        want = sum(c * port.expectation_value(tl, ids, psi) for c, tl, ids in terms)
        assert abs(e - want) <= 1e-4


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_batch_mixed_sizes_across_the_single_state_threshold(port, precision):
    """States of 12 and 19-20 qubits in one batch: the large ones take the single-state span-tile
    evaluation, the small ones the shared job launch; every energy matches its state alone."""
    jobs, specs = [], []
    for i, n in enumerate([12, 19, 13, 20, 12]):
        gates = W.hea_circuit(n, 3, seed=7700 + i)
        terms = W.random_pauli_terms(n, 60, 1, 5, seed=7800 + i)
        jobs.append((W.to_circuit(gates, n), W.to_observable(terms, n)))
        specs.append((n, gates, terms))
    got = BatchRunner(memory_budget_bytes=1 << 34, precision=precision).run(jobs)
    for (circ, obs), (n, gates, terms), e in zip(jobs, specs, got):
        psi = np.zeros(1 << n, dtype=np.complex128)
        psi[0] = 1
        R.run_on_cpu(gates, psi, port)
        want = sum(c * port.expectation_value(tl, ids, psi) for c, tl, ids in terms)
        assert abs(e - want) <= (EV_TOL if precision == "c128" else 1e-5), (n, e, want)


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_batch_repeats_a_circuit_and_reuses_plans(precision):
    """The same circuit object twice in one batch (its plan built once), then the batch again with the
    plans cached: every copy of a job gives the same energy."""
    jobs, _ = make_jobs(23, 5, 10, 13)
    jobs = jobs + [jobs[1], jobs[3]]
    first = BatchRunner(1 << 30, precision=precision).run(jobs)
    again = BatchRunner(1 << 30, precision=precision).run(jobs)
    assert first[5] == first[1] and first[6] == first[3]
    assert np.array_equal(first, again)


def test_dependency_wait_expires_and_context_stays_usable(port):
    """The batch kernel's bounded dependency wait, made to run out: the last pass of a one-circuit batch
    waits on its own completion counter (which nothing can complete) with a 1 ms limit.  The call must
    return QS_ERR_TIMEOUT, not hang or fault; the passes before it are applied; and a normal batch on
    the same context afterwards gives the oracle's state."""
    from qulacs_b200._lib import load
    lib = load()
    n = 12
    gates = W.hea_circuit(n, 8, seed=77)
    circ = W.to_circuit(gates, n)
    s = QuantumState(n)
    rc = lib.qs_debug_batch_wait_expiry(circ._h, s.data_ptr(), 1000, None)
    assert rc == 4, lib.qs_get_last_error()  # QS_ERR_TIMEOUT
    assert b"dependency wait expired" in lib.qs_get_last_error()
    # the context still works: the same circuit as a normal batch matches the oracle
    psi = np.zeros(1 << n, dtype=np.complex128)
    psi[0] = 1
    R.run_on_cpu(gates, psi, port)
    ok = QuantumState(n)
    import ctypes as C
    from qulacs_b200._lib import call
    call("qs_batch_update_quantum_states", (C.c_void_p * 1)(circ._h), (C.c_void_p * 1)(ok.data_ptr()), 1, None)
    assert np.max(np.abs(ok.get_vector() - psi)) <= 1e-12


def test_fused_c64_dependency_wait_expires_and_context_stays_usable(port):
    """The persistent complex64 batch kernel's bounded dependency wait, made to run out (last pass waits on
    its own counter, 1 ms limit): QS_ERR_TIMEOUT, no hang or fault, TMEM released; then a normal fused
    batch on the same context meets the infidelity bar."""
    from qulacs_b200 import QuantumStateC64
    from qulacs_b200._lib import load
    lib = load()
    n = 14
    gates = W.hea_circuit(n, 10, seed=78)
    circ = W.to_circuit(gates, n)
    s = QuantumStateC64(n)
    rc = lib.qs_debug_batch_wait_expiry_fused_c64(circ._h, s.data_ptr(), 1000, None)
    assert rc == 4, lib.qs_get_last_error()  # QS_ERR_TIMEOUT
    psi = np.zeros(1 << n, dtype=np.complex128)
    psi[0] = 1
    R.run_on_cpu(gates, psi, port)
    ok = QuantumStateC64(n)
    import ctypes as C
    from qulacs_b200._lib import call
    call("qs_batch_update_quantum_states_fused_c64", (C.c_void_p * 1)(circ._h), (C.c_void_p * 1)(ok.data_ptr()),
         1, None)
    ref = QuantumState(n)
    ref.load(psi)
    assert ok.infidelity(ref) <= 1e-6


def test_fused_c64_persistent_batch_equals_each_circuit_alone():
    """The persistent complex64 batch kernel applies each circuit's passes to its own state exactly as the
    single-circuit fused kernel does (same block records, same per-tile arithmetic): uneven sizes 10..20,
    several passes each, bit-identical states."""
    import ctypes as C
    from qulacs_b200 import QuantumStateC64
    from qulacs_b200._lib import call
    sizes = [10, 14, 11, 20, 13, 16, 10, 18]
    circs = [W.to_circuit(W.hea_circuit(n, 6 + i % 5, seed=8800 + i), n) for i, n in enumerate(sizes)]
    batch = [QuantumStateC64(n) for n in sizes]
    call("qs_batch_update_quantum_states_fused_c64", (C.c_void_p * len(circs))(*[c._h for c in circs]),
         (C.c_void_p * len(batch))(*[s.data_ptr() for s in batch]), len(circs), None)
    for c, n, b in zip(circs, sizes, batch):
        alone = QuantumStateC64(n)
        c.set_c64_executor("tensor")
        c.update_quantum_state(alone)
        assert np.array_equal(b.get_vector(), alone.get_vector()), n


def test_c64_fp64_batch_equals_each_circuit_alone():
    """The persistent batch kernel over complex64 tiles applies each circuit's FP64 passes to its own state
    as the single-circuit FP64 passes do, up to the tile shape (2^11 in the batch, 2^12 alone): states
    agree to complex64 rounding."""
    import ctypes as C
    from qulacs_b200 import QuantumStateC64
    from qulacs_b200._lib import call
    sizes = [6, 14, 11, 20, 13, 16, 9, 18]
    circs = [W.to_circuit(W.hea_circuit(n, 4 + i % 5, seed=9900 + i), n) for i, n in enumerate(sizes)]
    batch = [QuantumStateC64(n) for n in sizes]
    call("qs_batch_update_quantum_states_c64", (C.c_void_p * len(circs))(*[c._h for c in circs]),
         (C.c_void_p * len(batch))(*[s.data_ptr() for s in batch]), len(circs), 1, None)
    for c, n, b in zip(circs, sizes, batch):
        alone = QuantumStateC64(n)
        c.set_c64_executor("fp64")
        c.update_quantum_state(alone)
        assert np.max(np.abs(b.get_vector() - alone.get_vector())) <= 1e-5, n


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_large_circuits_of_a_batch_run_their_own_passes(precision):
    """Circuits of >= 21 qubits leave the persistent launch and run their own staged passes (blocks of
    <= 2 qubits, 2^12-amplitude tiles) in the same call: each such state equals its circuit run alone
    with that schedule bit for bit, and the small ones still equal theirs to rounding."""
    import ctypes as C
    from qulacs_b200 import QuantumStateC64
    from qulacs_b200._lib import call
    sizes = [12, 21, 14, 22]
    circs = [W.to_circuit(W.hea_circuit(n, 3 + i, seed=9950 + i), n) for i, n in enumerate(sizes)]
    State = QuantumStateC64 if precision == "c64" else QuantumState
    batch = [State(n) for n in sizes]
    k = len(circs)
    ch = (C.c_void_p * k)(*[c._h for c in circs])
    sp = (C.c_void_p * k)(*[s.data_ptr() for s in batch])
    if precision == "c64":
        call("qs_batch_update_quantum_states_c64", ch, sp, k, 1, None)
    else:
        call("qs_batch_update_quantum_states", ch, sp, k, None)
    for c, n, b in zip(circs, sizes, batch):
        alone = State(n)
        if precision == "c64":
            c.set_c64_executor("fp64")
            c.update_quantum_state(alone)
        else:
            c.set_fusion(2)
            c.update_quantum_state(alone, mode="staged_fused")
        if n >= 21:
            assert np.array_equal(b.get_vector(), alone.get_vector()), n
        else:
            tol = 1e-5 if precision == "c64" else 1e-14
            assert np.max(np.abs(b.get_vector() - alone.get_vector())) <= tol, n
