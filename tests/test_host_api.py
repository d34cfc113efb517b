"""The C++ host layer (paraphysicell_b200/host/ppc_solver.h): the
reference's unit tests written in C++ against it (tests/cpp/test_host_api.cpp)
compile here, and pass on the GPU."""
import os
import shutil
import subprocess

import pytest

from paraphysicell_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_host_api.cpp")
OUT = os.path.join(ROOT, "tests", "cpp", "_build", "test_host_api")


def compile_host_test():
    build.ensure_built()
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    libdir = os.path.dirname(build.LIB)
    cmd = [cxx, "-O2", "-std=c++17", "-fopenmp", "-Wall", "-o", OUT, SRC, f"-L{libdir}", "-lppc",
           f"-Wl,-rpath,{libdir}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return OUT


def test_host_layer_compiles():
    assert os.path.exists(compile_host_test())


@pytest.mark.gpu
def test_reference_unit_tests_pass_through_host_layer():
    exe = compile_host_test()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600, env=dict(os.environ, OMP_NUM_THREADS="4"))
    print(r.stdout)
    lines = [l for l in r.stdout.splitlines() if l.startswith(("PASS", "FAIL"))]
    assert len(lines) == 28, r.stdout + r.stderr
    assert r.returncode == 0, r.stdout + r.stderr
