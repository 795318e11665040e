"""The C++ drop-in header (include/clique_b200/clique.hpp): the flow of the
reference's tests/Solve.cpp, compiled with g++ against libcliqgpu.so and run
on the GPU (FP64 real and complex, FP32 real, and an indefinite FP64 case
with intra-front pivoting)."""
import os
import shutil
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_solve_driver(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no C++ compiler")
    exe = tmp_path / "solve_driver"
    lib = os.path.join(ROOT, "clique_b200", "_lib")
    subprocess.run([gxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "solve_driver.cpp"), "-L", lib, "-lcliqgpu",
                    f"-Wl,-rpath,{lib}", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), "24"], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "||X - X_hat||" in r.stdout
