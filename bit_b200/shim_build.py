"""Build libtree3d_b200.so: the reference-named drop-in (include/tree3d_b200.h) over
libbit_b200.so.  ``python -m bit_b200.shim_build``."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc", "tree3d_shim.cpp")
OUT = os.path.join(HERE, "lib", "libtree3d_b200.so")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def build(force=False):
    deps = [SRC, os.path.join(ROOT, "include", "tree3d_b200.h"),
            os.path.join(ROOT, "include", "bit_b200.h"), os.path.join(HERE, "lib", "libbit_b200.so")]
    if not force and os.path.exists(OUT) and all(os.path.getmtime(d) <= os.path.getmtime(OUT) for d in deps):
        return OUT
    cmd = [CXX, "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall", "-I", os.path.join(ROOT, "include"),
           SRC, "-o", OUT, "-L", os.path.join(HERE, "lib"), "-lbit_b200", "-Wl,-rpath,$ORIGIN"]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force=True))
