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


from oracle.oracle import mt19937_64_uniforms  # noqa: E402,F401  (re-exported for the tests)


def random_density_matrix(n, rng):
    a = rng.normal(size=(1 << n, 1 << n)) + 1j * rng.normal(size=(1 << n, 1 << n))
    rho = a @ a.conj().T
    return rho / np.trace(rho)


