"""The C++ binding shown in INTEGRATION.md compiles against include/irbc.h
(syntax and types only; nothing runs)."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_stub_compiles(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not found")
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", text, re.S)
    assert blocks, "no C++ block in INTEGRATION.md"
    src = tmp_path / "stub.cpp"
    src.write_text(blocks[0])
    subprocess.run([gxx, "-std=c++17", "-fsyntax-only", "-Wall", "-I", os.path.join(ROOT, "include"), str(src)],
                   check=True)
