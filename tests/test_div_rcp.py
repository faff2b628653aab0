"""sapb::div_rcp_fast, the division of the narrow band factorisation's fast
path (one reciprocal per pivot, then Markstein's FMA correction per entry;
a panel with any operand outside the safe range is redone with the
division), must equal the division operator bit for bit wherever it reports
its result valid: tests/cpp/div_check.cu compares them on ~85 million pairs
per precision on the GPU (random bit patterns, matrix-like values, exponents
at the edges of the range) and counts the pairs outside the fast path."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def build(tmpdir) -> str:
    exe = os.path.join(str(tmpdir), "div_check")
    cmd = [NVCC, "-std=c++17", "-O3", "--expt-relaxed-constexpr", "-gencode", "arch=compute_100a,code=sm_100a",
           os.path.join(ROOT, "tests", "cpp", "div_check.cu"), "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_div_check_compiles(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_div_rcp_fast_equals_division_where_valid(tmp_path):
    out = subprocess.run([build(tmp_path)], capture_output=True, text=True, timeout=300)
    line = json.loads(out.stdout.strip().splitlines()[-1])
    print(line)
    assert out.returncode == 0, (out.stdout, out.stderr)
    assert line["double_pairs"] > 80_000_000 and line["float_pairs"] > 80_000_000
    assert line["double_mismatches"] == 0 and line["float_mismatches"] == 0
    # matrix-like operands stay on the fast path (only zero divisors leave it)
    assert line["double_typical_outside"] == 0 and line["float_typical_outside"] == 0
