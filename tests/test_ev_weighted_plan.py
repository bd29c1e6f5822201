"""Host-side plan of the weighted expectation value (no GPU): every term is evaluated exactly once,
by one kind of evaluation, and the max-coverage tile bases need fewer passes than one per term."""
import numpy as np
import pytest

from qulacs_b200 import workloads as W


def plan(n, terms):
    return W.to_observable(terms, n).weighted_plan(n)


@pytest.mark.parametrize("n", [11, 14, 20, 30])
def test_every_term_once(n):
    terms = W.random_pauli_terms(n, 256, 1, 6, seed=2125)
    p = plan(n, terms)
    kinds = ("z_only", "in_registers", "shared_partner", "selected_rows", "one_value_each")
    assert sum(p[k] for k in kinds) == len(terms)
    nz = sum(1 for _, _, ids in terms if all(i == 3 for i in ids))
    assert p["z_only"] == nz  # every Z-only string rides in the first pass
    assert p["one_value_each"] == 0
    assert 1 <= p["passes"] < len(terms) - nz


def test_bench_hamiltonian_pass_count():
    """The 256-string weight-1..6 Hamiltonian on 30 qubits: the most-shared reduced mask first covers
    the 233 bit-flip strings in 17 passes (23 when the masks are taken in term order)."""
    p = plan(30, W.random_pauli_terms(30, 256, 1, 6, seed=2125))
    assert p["passes"] == 17
    assert p["in_registers"] > 0 and p["shared_partner"] > 0 and p["selected_rows"] > 0


def test_small_states_and_few_flips_take_one_value_each():
    terms = W.random_pauli_terms(10, 40, 1, 4, seed=5)
    p = plan(10, terms)  # below the 11-qubit tile
    assert p["passes"] == 0 and p["one_value_each"] == len(terms)
    few = [(1.0, [0], [1]), (0.5, [3, 5], [2, 2]), (0.2, [1], [3])]
    p = plan(16, few)  # fewer than four bit-flip strings
    assert p["passes"] == 0 and p["one_value_each"] == 3


def test_single_string_per_basis_falls_back():
    """Strings whose masks never share a span beyond one each leave the last ones to the per-term path."""
    n = 40
    terms = [(1.0, [q, q + 20], [1, 1]) for q in range(4, 20)]
    p = plan(n, terms)
    assert sum(v for k, v in p.items() if k != "passes") == len(terms)


def _nvrtc():
    import ctypes as C
    for name in ("libnvrtc.so.12", "/usr/local/cuda/lib64/libnvrtc.so.12"):
        try:
            return C.CDLL(name)
        except OSError:
            pass
    return None


@pytest.mark.parametrize("c64", [False, True])
def test_generated_pass_sources_compile_without_spills(c64):
    """The generated expectation kernels compile with NVRTC for sm_100a (the compiler the library uses at
    run time) at 128 threads x 3 CTAs per SM without spilling: the largest pass (the bench Hamiltonian's
    first, with every Z-only string) and small ones."""
    import ctypes as C
    lib = _nvrtc()
    if lib is None:
        pytest.skip("NVRTC not available")
    obs = W.to_observable(W.random_pauli_terms(30, 256, 1, 6, seed=2125), 30)
    npass = obs.weighted_plan(30)["passes"]
    for i in (0, 1, npass - 1):
        src = obs.pass_source(i, 30, c64)
        assert "k_ev_spec" in src
        prog = C.c_void_p()
        assert lib.nvrtcCreateProgram(C.byref(prog), src.encode(), b"k_ev_spec.cu", 0, None, None) == 0
        opts = (C.c_char_p * 3)(b"--gpu-architecture=sm_100a", b"--std=c++17", b"--ptxas-options=-v")
        rc = lib.nvrtcCompileProgram(prog, 3, opts)
        n = C.c_size_t()
        lib.nvrtcGetProgramLogSize(prog, C.byref(n))
        buf = C.create_string_buffer(n.value)
        lib.nvrtcGetProgramLog(prog, buf)
        lib.nvrtcDestroyProgram(C.byref(prog))
        log = buf.value.decode()
        assert rc == 0, log[-2000:]
        assert "0 bytes spill stores" in log, (i, log[-1500:])
