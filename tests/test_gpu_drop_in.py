"""The C++ drop-in: a reference-style program built against include/tree3d_b200.h."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_style_program(tmp_path):
    libdir = os.path.join(ROOT, "bit_b200", "lib")
    exe = str(tmp_path / "treecode_b200")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "drop_in", "treecode_b200.cpp"), "-o", exe,
                    "-L", libdir, "-ltree3d_b200", "-lbit_b200", f"-Wl,-rpath,{libdir}"],
                   check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Test PASSED" in r.stdout
