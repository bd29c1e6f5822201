"""The header-only C++ surface (include/qulacs_b200/cppsim.hpp): compiles on the CPU; on a GPU the
test program links against libqulacs_b200.so and checks Bell states, staged vs gate-by-gate,
circuit inverse, sampling, the depolarizing identity and error-to-exception mapping."""
import os
import subprocess

import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "test_cppsim.cpp")
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "qulacs_b200")


def test_header_compiles():
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wextra", f"-I{INC}", SRC],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_cpp_program_runs(tmp_path, lib):
    exe = str(tmp_path / "test_cppsim")
    r = subprocess.run(["g++", "-std=c++17", "-O1", f"-I{INC}", SRC, f"-L{LIBDIR}", "-lqulacs_b200",
                        f"-Wl,-rpath,{LIBDIR}", "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "OK" in r.stdout, r.stdout + r.stderr
