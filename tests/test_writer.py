"""output_potential (bit_write_potential) byte for byte against a file the reference's own
output_potential wrote (tests/golden/output_potential.txt).  Host code: no GPU."""
import os

from conftest import GOLDEN, ROOT, load_golden


def test_writer_matches_reference_output_byte_for_byte(tmp_path):
    import bit_b200 as B
    g = load_golden("output_potential")
    out = tmp_path / "pot.txt"
    B.write_potential(str(out), g["x"], g["y"], g["z"], g["pot"])
    ref = open(os.path.join(GOLDEN, "output_potential.txt"), "rb").read()
    assert out.read_bytes() == ref


def test_drop_in_output_potential_matches_reference_output(tmp_path):
    """A program calling output_potential(npart, part, pot, filename) through the drop-in
    header and libtree3d_b200.so writes the reference's file.  Host code: no GPU."""
    import subprocess
    import numpy as np
    libdir = os.path.join(ROOT, "bit_b200", "lib")
    exe = str(tmp_path / "output_b200")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "drop_in", "output_b200.cpp"), "-o", exe,
                    "-L", libdir, "-ltree3d_b200", "-lbit_b200", f"-Wl,-rpath,{libdir}"],
                   check=True)
    g = load_golden("output_potential")
    data = tmp_path / "in.bin"
    with open(data, "wb") as f:
        f.write(np.int64(len(g["x"])).tobytes())
        for k in ("x", "y", "z", "pot"):
            f.write(np.ascontiguousarray(g[k], dtype=np.float64).tobytes())
    out = tmp_path / "pot.txt"
    r = subprocess.run([exe, str(data), str(out)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert out.read_bytes() == open(os.path.join(GOLDEN, "output_potential.txt"), "rb").read()
