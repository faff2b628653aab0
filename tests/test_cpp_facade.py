"""The C++ facade (include/sap/*.h: sap::Options, Solver, SpmvCusp,
MVBanded, BandedMatrix, system_error over the C ABI): a C++ program written
the way reference code is written (tests/cpp/facade_solve.cu) compiles with
nvcc and links against libsap_b200.so without a GPU; on a GPU it runs the
reference unit test's configuration and a generated banded system to their
tolerances and reports an illegal call order as sap::system_error."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
LIB = os.path.join(ROOT, "saplibrary_b200", "libsap_b200.so")


def build(tmpdir) -> str:
    exe = os.path.join(str(tmpdir), "facade_solve")
    cmd = [NVCC, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "facade_solve.cu"), LIB, "-Xlinker",
           "-rpath," + os.path.dirname(LIB), "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_facade_program_compiles_and_links(tmp_path):
    exe = build(tmp_path)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_facade_program_solves(tmp_path):
    exe = build(tmp_path)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    line = json.loads(out.stdout.strip().splitlines()[-1])
    print(line)
    assert out.returncode == 0, (out.stdout, out.stderr)
    assert line["unit_test_converged"] and line["code"] == 1 and line["message"] == "Converged"
    assert line["rel_residual"] <= 1e-13 and line["rel_error"] <= 1e-9
    assert line["banded_converged"] and line["banded_rel_residual"] <= 1e-6
    assert line["solve_before_setup_reason"] == -4  # system_error::Illegal_solve
