"""The C++ example shown in INTEGRATION.md compiles against the sap:: headers
(include/sap/*.h over include/sap_b200.h; syntax and types only, no device
needed)."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_cpp_binding_snippet_compiles(tmp_path):
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", text, re.S)
    assert blocks, "no C++ block in INTEGRATION.md"
    src = tmp_path / "binding.cpp"
    src.write_text("\n".join(blocks) + "\nint main() { return 0; }\n")
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                        "-I", "/usr/local/cuda/include", str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
