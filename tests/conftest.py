import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")

# Tolerances (complex128 path): max |delta amplitude| and |delta <H>| against the reference csim.
AMP_TOL = 1e-12
EV_TOL = 1e-10
BOUNDARY_EPS = 1e-12


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


@pytest.fixture(scope="session")
def port():
    from oracle import oracle as O
    return O.port()


@pytest.fixture(scope="session")
def ref():
    from oracle import oracle as O
    r = O.reference()
    if r is None:
        pytest.skip("reference csim not built (oracle/_ref)")
    return r


@pytest.fixture(scope="session")
def lib():
    from qulacs_b200 import _lib
    return _lib.load()


def random_state(n, rng):
    s = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return s / np.linalg.norm(s)


def random_unitary(k, rng):
    a = rng.normal(size=(1 << k, 1 << k)) + 1j * rng.normal(size=(1 << k, 1 << k))
    q, r = np.linalg.qr(a)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def random_density_matrix(n, rng):
    a = rng.normal(size=(1 << n, 1 << n)) + 1j * rng.normal(size=(1 << n, 1 << n))
    rho = a @ a.conj().T
    return rho / np.trace(rho)


def mt19937_64_uniforms(seed, count):
    """mt19937_64 (Matsumoto & Nishimura 2000, 64-bit parameters) and libstdc++'s
    generate_canonical<double, 53> for a 64-bit engine: x / 2^64, clamped below 1."""
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
        r = float(y) / 18446744073709551616.0
        if r >= 1.0:
            r = np.nextafter(1.0, 0.0)
        out.append(r)
    return np.array(out)
