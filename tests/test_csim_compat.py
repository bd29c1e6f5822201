"""libcsim_b200.so, the csim-signature boundary: csim's operator functions (C++ linkage, csim's argument
lists, CTYPE = std::complex<double>) over device memory.

* CPU: a translation unit compiled against the REFERENCE's own csim headers, taking the address of every
  function include/qulacs_b200/csim_compat.hpp declares, links against libcsim_b200.so -- so a program
  built for csim resolves every such call here (skipped without the reference checkout).
* CPU: every declared function is exported.
* GPU: a program written against the csim API runs a gate sequence on device memory; its final state
  and statistics match the oracle replaying the same sequence."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import AMP_TOL, EV_TOL, ROOT

INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "qulacs_b200")
HDR = os.path.join(INC, "qulacs_b200", "csim_compat.hpp")


def declared_functions():
    txt = re.sub(r"//[^\n]*", "", open(HDR).read())
    return sorted(set(re.findall(r"^\s*[\w:<>\*\s]+?\b(\w+)\s*\(", txt, flags=re.M)) - {"if", "return"})


def reference_root():
    from oracle import oracle as O
    return O.reference_root()


def test_every_declared_function_is_exported(lib):
    names = declared_functions()
    assert len(names) > 100
    out = subprocess.run(["nm", "-DC", "--defined-only", os.path.join(LIBDIR, "libcsim_b200.so")],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (\w+)\(", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing


@pytest.mark.skipif(not os.path.isdir(os.path.join(reference_root(), "src", "csim")),
                    reason="reference checkout not present")
def test_program_built_against_reference_headers_links(tmp_path, lib):
    csim = os.path.join(reference_root(), "src", "csim")
    heads = [h for h in ("update_ops.hpp", "stat_ops.hpp", "init_ops.hpp", "memory_ops.hpp", "update_ops_dm.hpp",
                         "stat_ops_dm.hpp", "memory_ops_dm.hpp") if os.path.exists(os.path.join(csim, h))]
    names = declared_functions()
    src = "".join(f'#include "csim/{h}"\n' for h in heads)
    src += "#include <cstdio>\nint main() {\n  void* volatile p;\n"
    src += "".join(f"  p = (void*)&{n}; std::printf(\"%p\", p);\n" for n in names)
    src += "  return 0;\n}\n"
    cpp = tmp_path / "uses_csim.cpp"
    cpp.write_text(src)
    exe = tmp_path / "uses_csim"
    r = subprocess.run(["g++", "-std=c++17", "-w", f"-I{os.path.join(reference_root(), 'src')}", str(cpp),
                        f"-L{LIBDIR}", "-lcsim_b200", "-lqulacs_b200", f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]


@pytest.mark.gpu
def test_csim_api_program_matches_oracle(tmp_path, lib, port):
    src = os.path.join(ROOT, "tests", "cpp", "test_csim_compat.cpp")
    exe = str(tmp_path / "csim_prog")
    r = subprocess.run(["g++", "-std=c++17", "-O1", f"-I{INC}", src, f"-L{LIBDIR}", "-lcsim_b200", "-lqulacs_b200",
                        f"-Wl,-rpath,{LIBDIR}", "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = str(tmp_path / "out.bin")
    r = subprocess.run([exe, out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "OK" in r.stdout, r.stdout + r.stderr
    raw = np.fromfile(out, dtype=np.float64)
    ev, norm, p0, ip, threw = raw[:5]
    got = raw[5:].view(np.complex128)
    n = 10
    s = np.zeros(1 << n, dtype=np.complex128)
    s[0] = 1
    for q in range(n):
        port.RX_gate(q, 0.3 + 0.1 * q, s)
        port.RY_gate(q, -0.7 + 0.05 * q, s)
        port.RZ_gate(q, 1.1 - 0.2 * q, s)
    for q in range(n - 1):
        port.CNOT_gate(q, q + 1, s)
    h = 1 / np.sqrt(2)
    u = np.array([[h, 1j * h], [1j * h, h]])
    port.single_qubit_dense_matrix_gate(4, u, s)
    m2 = np.zeros(16, dtype=np.complex128)
    m2[::5] = np.exp(0.4j)
    port.double_qubit_dense_matrix_gate_c(2, 7, m2.reshape(4, 4), s)
    port.CZ_gate(1, 8, s)
    port.SWAP_gate(0, 9, s)
    port.single_qubit_dense_matrix_gate(3, np.array([[h, h], [h, -h]]), s)
    port.single_qubit_diagonal_matrix_gate(5, np.array([1, np.exp(0.25j * np.pi)]), s)
    m3 = np.zeros((8, 8), dtype=np.complex128)
    for i in range(8):
        m3[i, 7 - i] = 1j
    port.multi_qubit_dense_matrix_gate([6, 2, 8], m3, s)
    port.multi_qubit_Pauli_rotation_gate_partial_list([1, 4, 7], [1, 2, 3], 0.9, s)
    port.multi_qubit_control_single_qubit_dense_matrix_gate([3], [1], 6, u, s)
    assert np.max(np.abs(got - s)) <= AMP_TOL
    assert abs(ev - port.expectation_value([1, 4, 7], [1, 2, 3], s)) <= EV_TOL
    assert abs(norm - 1.0) <= 1e-12 and abs(ip - 1.0) <= 1e-12
    assert abs(p0 - port.M0_prob(2, s)) <= 1e-12
    assert threw == 1.0
