"""Serving loop host logic on the CPU: the first-fit arena and the request mix."""
import numpy as np

from qulacs_b200.serving import FirstFit, Request, make_request_mix


def test_first_fit_alloc_release_coalesce():
    f = FirstFit(1000)
    a = f.alloc(300)
    b = f.alloc(300)
    c = f.alloc(300)
    assert (a, b, c) == (0, 300, 600)
    assert f.alloc(200) is None  # 100 left
    f.release(b, 300)
    assert f.alloc(250) == 300  # first fit into the hole
    f.release(a, 300)
    f.release(300, 250)
    f.release(c, 300)
    assert f.free == [(0, 1000)] and f.free_bytes() == 1000


def test_request_mix_shape():
    reqs = make_request_mix(400, rate=50.0, seed=3)
    kinds = [r.kind for r in reqs]
    frac = {k: kinds.count(k) / len(kinds) for k in ("expectation", "sampling", "dm")}
    assert abs(frac["expectation"] - 0.7) < 0.08 and abs(frac["sampling"] - 0.2) < 0.07
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0)
    assert abs(len(reqs) / arr[-1] - 50.0) < 10.0  # Poisson rate
    for r in reqs:
        if r.kind == "expectation":
            assert 12 <= r.n <= 28 and len(r.terms) == 200
        elif r.kind == "sampling":
            assert 16 <= r.n <= 30 and r.uniforms.size == 1024
        else:
            assert 8 <= r.n <= 13


def test_footprints():
    assert Request(0, "expectation", 20, []).footprint("c128") == 16 << 20
    assert Request(0, "expectation", 20, []).footprint("c64") == 8 << 20
    assert Request(0, "dm", 10, []).footprint("c128") == 16 << 20
