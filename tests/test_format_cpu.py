"""The output files' number formatting (zedm-x_b200/csrc/zdx_format.h) against std::ostream, the
reference's own writer (src/main.cpp:1710-1870): a small C++ program is compiled with g++ and checks
several hundred thousand values, rounding boundaries and special values, plus sliced multi-thread
writing."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_to_chars_formatting_matches_ostream(tmp_path):
    exe = str(tmp_path / "format_check")
    src = os.path.join(ROOT, "tests", "cpp", "format_check.cpp")
    inc = os.path.join(ROOT, "zedm-x_b200", "csrc")
    subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", "-I", inc, "-o", exe, src], check=True, timeout=300)
    p = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert p.stdout.startswith("ok ")
