"""Serving loop: continuous batching of simulation requests with admission by HBM footprint.

Requests of three kinds arrive over time (Poisson arrivals in the benchmark):

* ``expectation``: a circuit and an observable -> <H> (FP64),
* ``sampling``: a circuit and supplied uniforms -> sampled basis indices,
* ``dm``: a noisy circuit on a density matrix and an observable -> Tr(H rho).

A dispatcher admits arrived requests in arrival order while their states fit the free part of one
device arena (first fit; a request that does not fit waits, and at most ``max_bypass`` later
requests may overtake it, which bounds starvation).  Admitted states stay resident in HBM until
their request completes.  ``workers`` threads, each owning a CUDA stream, take ready work
continuously: all ready expectation requests at once (up to ``max_batch``) go through ONE persistent
multi-circuit launch plus ONE batched <P> launch; sampling and density-matrix requests run one each.
Work of different workers overlaps on the device.  Latency = completion - arrival, per request.

``precision="c64"`` keeps expectation and sampling requests' states in complex64 (reductions in FP64):
a batch of expectation requests is one persistent launch of FP64 passes over complex64 tiles (the
tensor-core blocks when some gate cannot be staged) plus one batched <P> launch; a sampling request
takes its circuit's complex64 executor; density-matrix requests stay complex128.

Served circuits run the generic staged pass kernel, not specialised per-pass kernels: every request
brings new gate parameters, and compiling a kernel for each would add its compile time to the
request's latency.
"""
from __future__ import annotations

import ctypes as C
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from . import workloads as W
from ._lib import EXEC_STAGED_FUSED, call

# FP64 fusion block size for every served circuit: fixed (not autotuned per request) so that a
# request's result does not depend on timing noise, and equal to the batch executor's.
SERVE_FUSION_K = 2
# requests whose device footprint is at most this run on high-priority streams (24-qubit complex128)
SMALL_REQUEST_BYTES = 16 << 24
from .observable import masks

ALIGN = 256


@dataclass
class Request:
    rid: int
    kind: str               # "expectation" | "sampling" | "dm"
    n: int
    gates: list
    terms: list = field(default_factory=list)
    uniforms: np.ndarray | None = None
    arrival: float = 0.0    # seconds after the start of the run
    result: object = None
    t_admit: float = 0.0
    t_start: float = 0.0    # a worker began its device work
    batch_id: int = -1      # the worker batch that ran it
    t_done: float = 0.0

    def footprint(self, precision: str) -> int:
        if self.kind == "dm":
            b = 16 << (2 * self.n)
        elif precision == "c64":
            b = 8 << self.n
        else:
            b = 16 << self.n
        return (b + ALIGN - 1) // ALIGN * ALIGN


class FirstFit:
    """First-fit allocator over [0, size) with coalescing of freed ranges (host bookkeeping only)."""

    def __init__(self, size: int):
        self.size = size
        self.free = [(0, size)]  # sorted (offset, length)
        self.lock = threading.Lock()

    def alloc(self, nbytes: int):
        with self.lock:
            for i, (off, ln) in enumerate(self.free):
                if ln >= nbytes:
                    if ln == nbytes:
                        self.free.pop(i)
                    else:
                        self.free[i] = (off + nbytes, ln - nbytes)
                    return off
        return None

    def release(self, off: int, nbytes: int) -> None:
        with self.lock:
            self.free.append((off, nbytes))
            self.free.sort()
            merged = []
            for o, ln in self.free:
                if merged and merged[-1][0] + merged[-1][1] == o:
                    merged[-1] = (merged[-1][0], merged[-1][1] + ln)
                else:
                    merged.append((o, ln))
            self.free = merged

    def free_bytes(self) -> int:
        with self.lock:
            return sum(ln for _, ln in self.free)


class DeviceArena:
    """One device buffer carved by a FirstFit allocator: admitting a request allocates nothing on the
    device."""

    def __init__(self, nbytes: int):
        p = C.c_void_p()
        call("qs_allocate_bytes", nbytes, C.byref(p))
        self.base = p.value
        self.size = nbytes
        self.fit = FirstFit(nbytes)

    def alloc(self, nbytes: int):
        off = self.fit.alloc(nbytes)
        return None if off is None else self.base + off

    def release(self, ptr: int, nbytes: int) -> None:
        self.fit.release(ptr - self.base, nbytes)

    def close(self):
        if self.base:
            _lib.load().qs_release_quantum_state(self.base)
            self.base = 0


def make_request_mix(count: int, rate: float, seed: int, ranges=None):
    """The serving mix: 70% expectation (HEA ansatz, n ~ U{12..28}, depth ~ U{4..16}, 200 strings of
    weight <= 4), 20% sampling (layered circuit, n ~ U{16..30}, 1024 shots), 10% density-matrix jobs
    (n ~ U{8..13}, depth-8 HEA, depolarizing p = 1e-3 after every gate, 64 strings), Poisson arrivals."""
    r = {"exp": (12, 28), "samp": (16, 30), "dm": (8, 13)}
    r.update(ranges or {})
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += float(rng.exponential(1.0 / rate))
        u = float(rng.random())
        s = seed * 100000 + i
        if u < 0.7:
            n = int(rng.integers(r["exp"][0], r["exp"][1] + 1))
            d = int(rng.integers(4, 17))
            out.append(Request(i, "expectation", n, W.hea_circuit(n, d, s), W.random_pauli_terms(n, 200, 1, 4, s),
                               arrival=t))
        elif u < 0.9:
            n = int(rng.integers(r["samp"][0], r["samp"][1] + 1))
            out.append(Request(i, "sampling", n, W.layered_rotation_circuit(n, 10, s), arrival=t,
                               uniforms=W.uniforms(1024, s)))
        else:
            n = int(rng.integers(r["dm"][0], r["dm"][1] + 1))
            out.append(Request(i, "dm", n, W.noisy_circuit(W.hea_circuit(n, 8, s), 1e-3),
                               W.random_pauli_terms(n, 64, 1, 4, s), arrival=t))
    return out


def _vp(a):
    return a.ctypes.data_as(C.c_void_p)


class ServingLoop:
    def __init__(self, memory_budget_bytes: int, workers: int = 4, precision: str = "c128", max_batch: int = 64,
                 max_bypass: int = 16):
        _lib.load()
        self.arena = DeviceArena(memory_budget_bytes)
        self.workers = workers
        self.precision = precision
        self.max_batch = max_batch
        self.max_bypass = max_bypass
        self.cv = threading.Condition()
        self.ready = []          # admitted, not yet started (arrival order)
        self.outstanding = 0
        self.error = None
        self.batches = []        # sizes of the expectation batches that ran
        self.nbatches = 0        # worker batches of any kind started

    # ---- work execution (worker threads; each has its own stream) ----
    def _run_expectation_batch(self, reqs, stream):
        circs = [W.to_circuit(r.gates, r.n) for r in reqs]
        k = len(reqs)
        c64 = self.precision == "c64"
        for r in reqs:
            call("qs_initialize_quantum_state_c64" if c64 else "qs_initialize_quantum_state", r.ptr, 1 << r.n, stream)
        ch = (C.c_void_p * k)(*[c._h for c in circs])
        st = (C.c_void_p * k)(*[r.ptr for r in reqs])
        if c64:  # FP64 passes over complex64 tiles when every gate is stageable, else tensor-core blocks
            call("qs_batch_update_quantum_states_c64", ch, st, k, -1, stream)
        else:
            call("qs_batch_update_quantum_states", ch, st, k, stream)
        xm, zm, ny, offs, coefs = [], [], [], [0], []
        for r in reqs:
            for c, tl, ids in r.terms:
                x, z, y = masks(tl, ids)
                xm.append(x)
                zm.append(z)
                ny.append(y)
                coefs.append(c)
            offs.append(len(xm))
        xa, za = np.array(xm, dtype=np.uint64), np.array(zm, dtype=np.uint64)
        ya, oa = np.array(ny, dtype=np.uint32), np.array(offs, dtype=np.uint32)
        qa = np.array([r.n for r in reqs], dtype=np.uint32)
        ca = np.ascontiguousarray(np.array(coefs, dtype=np.complex128)).view(np.float64)
        energies = np.zeros(2 * k)
        call("qs_batch_expectation_weighted", st, _vp(qa), k, _vp(oa), _vp(xa), _vp(za), _vp(ya), _vp(ca), int(c64),
             _vp(energies), stream)
        for j, r in enumerate(reqs):
            r.result = float(energies[2 * j])

    def _run_sampling(self, r, stream):
        c = W.to_circuit(r.gates, r.n)
        out = np.zeros(r.uniforms.size, dtype=np.uint64)
        u = np.ascontiguousarray(r.uniforms)
        if self.precision == "c64":
            call("qs_initialize_quantum_state_c64", r.ptr, 1 << r.n, stream)
            call("qs_circuit_update_quantum_state_c64", c._h, r.ptr, 1 << r.n, stream)
            call("qs_state_sampling_with_uniforms_c64", r.ptr, 1 << r.n, _vp(u), u.size, _vp(out), stream)
        else:
            call("qs_initialize_quantum_state", r.ptr, 1 << r.n, stream)
            c.set_fusion(SERVE_FUSION_K)
            c.set_specialized(0)
            call("qs_circuit_update_quantum_state", c._h, r.ptr, 1 << r.n, EXEC_STAGED_FUSED, stream)
            call("qs_state_sampling_with_uniforms", r.ptr, 1 << r.n, _vp(u), u.size, _vp(out), stream)
        r.result = out

    def _run_dm(self, r, stream):
        c = W.to_circuit(r.gates, r.n)
        dim = 1 << r.n
        call("qs_dm_initialize_quantum_state", r.ptr, dim, stream)
        c.set_fusion(SERVE_FUSION_K)
        c.set_specialized(0)
        call("qs_circuit_update_density_matrix", c._h, r.ptr, dim, EXEC_STAGED_FUSED, stream)
        e = 0.0
        for coef, tl, ids in r.terms:
            t = np.array(tl, dtype=np.uint32)
            p = np.array(ids, dtype=np.uint32)
            v = C.c_double()
            call("qs_dm_expectation_value_multi_qubit_Pauli_operator_partial_list", _vp(t), _vp(p), t.size,
                 r.ptr, dim, stream, C.byref(v))
            e += coef * v.value
        r.result = e

    def _worker(self, t0):
        # two streams: requests whose state is small run on the high-priority one, so their kernels'
        # CTAs are scheduled ahead of a large request's remaining CTAs
        hi, lo = C.c_void_p(), C.c_void_p()
        call("qs_stream_create_with_priority", 1, C.byref(hi))
        call("qs_stream_create_with_priority", 0, C.byref(lo))
        try:
            while True:
                with self.cv:
                    while not self.ready and self.outstanding > 0 and self.error is None:
                        self.cv.wait(0.05)
                    if self.error is not None or (not self.ready and self.outstanding == 0):
                        return
                    head = self.ready[0]
                    if head.kind == "expectation":
                        batch = [r for r in self.ready if r.kind == "expectation"][: self.max_batch]
                    else:
                        batch = [head]
                    for r in batch:
                        self.ready.remove(r)
                start = time.perf_counter() - t0
                with self.cv:
                    bid = self.nbatches
                    self.nbatches += 1
                for r in batch:
                    r.t_start = start
                    r.batch_id = bid
                stream = hi.value if max(r.fp for r in batch) <= SMALL_REQUEST_BYTES else lo.value
                try:
                    if batch[0].kind == "expectation":
                        self._run_expectation_batch(batch, stream)
                        self.batches.append(len(batch))
                    elif batch[0].kind == "sampling":
                        self._run_sampling(batch[0], stream)
                    else:
                        self._run_dm(batch[0], stream)
                except Exception as e:  # report, stop the loop
                    with self.cv:
                        self.error = e
                        self.cv.notify_all()
                    return
                now = time.perf_counter() - t0
                with self.cv:
                    for r in batch:
                        r.t_done = now
                        self.arena.release(r.ptr, r.fp)
                        self.outstanding -= 1
                    self.cv.notify_all()
        finally:
            _lib.load().qs_stream_destroy(hi.value)
            _lib.load().qs_stream_destroy(lo.value)

    def run(self, requests):
        """Serve `requests` (their `arrival` offsets are honoured in wall-clock time); returns stats."""
        pending = sorted(requests, key=lambda r: r.arrival)
        for r in pending:
            r.fp = r.footprint(self.precision)
            if r.fp > self.arena.size:
                raise MemoryError(f"request {r.rid} needs {r.fp} bytes, more than the arena")
        waiting = []  # arrived, not admitted (arrival order)
        self.outstanding = len(pending)
        t0 = time.perf_counter()
        threads = [threading.Thread(target=self._worker, args=(t0,), daemon=True) for _ in range(self.workers)]
        for th in threads:
            th.start()
        i = 0
        while True:
            now = time.perf_counter() - t0
            while i < len(pending) and pending[i].arrival <= now:
                waiting.append(pending[i])
                i += 1
            admitted = []
            bypassed = 0
            for r in list(waiting):
                ptr = self.arena.alloc(r.fp)
                if ptr is None:
                    bypassed += 1
                    if bypassed > self.max_bypass:
                        break
                    continue
                r.ptr = ptr
                r.t_admit = now
                waiting.remove(r)
                admitted.append(r)
            if admitted:
                with self.cv:
                    self.ready.extend(admitted)
                    self.cv.notify_all()
            with self.cv:
                if self.error is not None:
                    break
                if i >= len(pending) and not waiting and self.outstanding == 0:
                    break
            nxt = pending[i].arrival - (time.perf_counter() - t0) if i < len(pending) else 0.002
            time.sleep(min(max(nxt, 0.0005), 0.002))
        with self.cv:
            self.cv.notify_all()
        for th in threads:
            th.join()
        if self.error is not None:
            raise self.error
        wall = max(r.t_done for r in requests) if requests else 0.0
        lat = np.array([r.t_done - r.arrival for r in requests])
        by_kind = {}
        for k in ("expectation", "sampling", "dm"):
            lk = np.array([r.t_done - r.arrival for r in requests if r.kind == k])
            if lk.size:
                by_kind[k] = {"count": int(lk.size), "p50_ms": float(np.percentile(lk, 50) * 1e3),
                              "p99_ms": float(np.percentile(lk, 99) * 1e3)}
        # device work in flight: time-average number of worker batches between their start and completion
        spans = {}
        for r in requests:
            spans[r.batch_id] = (r.t_start, r.t_done)
        busy = sum(d - s for s, d in spans.values())
        return {"jobs": len(requests), "wall_s": wall, "jobs_per_s": len(requests) / wall if wall else 0.0,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "mean_batch": float(np.mean(self.batches)) if self.batches else 0.0,
                "max_batch": int(max(self.batches)) if self.batches else 0,
                "mean_batches_in_flight": busy / wall if wall else 0.0, "by_kind": by_kind}

    def close(self):
        self.arena.close()


def run_alone(r: Request, precision: str = "c128"):
    """One request on an otherwise idle device through the same code path (for the alone-vs-mix test)."""
    loop = ServingLoop(r.footprint(precision) + (1 << 20), workers=1, precision=precision)
    try:
        rr = Request(r.rid, r.kind, r.n, r.gates, r.terms, r.uniforms, 0.0)
        loop.run([rr])
        return rr.result
    finally:
        loop.close()
