"""Serving loop on the B200: requests overlapping on the device give the same result as alone
(expectation <= 1e-10, density matrix <= 1e-12, identical sampled indices), and match the oracle."""
import numpy as np
import pytest

from conftest import EV_TOL
from qulacs_b200 import workloads as W
from qulacs_b200.serving import ServingLoop, make_request_mix, run_alone
from oracle import replay as R

pytestmark = pytest.mark.gpu

SMALL = {"exp": (6, 14), "samp": (8, 16), "dm": (3, 6)}


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_mix_equals_alone(port, precision):
    # arrivals within ~15 ms, so requests overlap on the device; the fused path needs >= 10 qubits
    ranges = SMALL if precision == "c128" else {"exp": (10, 14), "samp": (10, 16), "dm": (3, 6)}
    reqs = make_request_mix(30, rate=2000.0, seed=17, ranges=ranges)
    loop = ServingLoop(4 << 20, workers=3, precision=precision, max_batch=8)  # small arena: admission waits
    try:
        stats = loop.run(reqs)
    finally:
        loop.close()
    assert stats["jobs"] == 30 and stats["p99_ms"] >= stats["p50_ms"] > 0
    # continuous batching happened: some expectation batch held several requests, and requests of
    # different worker batches were on the device at the same time
    assert stats["max_batch"] > 1, stats
    overlapping = [(a.rid, b.rid) for a in reqs for b in reqs
                   if a.batch_id != b.batch_id and a.t_start < b.t_done and b.t_start < a.t_done]
    assert overlapping, "no two worker batches overlapped in time"
    for r in reqs:
        alone = run_alone(r, precision)
        if r.kind == "sampling":
            assert np.array_equal(r.result, alone)
        elif r.kind == "dm":
            assert abs(r.result - alone) <= 1e-12
        else:
            assert abs(r.result - alone) <= (1e-10 if precision == "c128" else 1e-6)
    # oracle check of every expectation request (c128: 1e-10; c64: 1e-4)
    for r in reqs:
        if r.kind != "expectation":
            continue
        psi = np.zeros(1 << r.n, dtype=np.complex128)
        psi[0] = 1
        R.run_on_cpu(r.gates, psi, port)
        want = sum(c * port.expectation_value(tl, ids, psi) for c, tl, ids in r.terms)
        assert abs(r.result - want) <= (EV_TOL if precision == "c128" else 1e-4)
