"""bit_gmres_dense_static: the dense GMRES with no allocation at call time, through the C ABI.

Two calls in a row must each agree with the allocating entry point (bit_gmres_dense)
within the tolerance of the dense-GMRES tests; sizes over the static limit are refused
with a message.  Collected last so that it also runs after every other test.
"""
import ctypes as C

import numpy as np
import pytest

TOL = 1e-12  # relative, against bit_gmres_dense (same kernels, same order of operations)


def system(n, seed):
    rng = np.random.default_rng(seed)
    A = np.eye(n) * 3 + rng.uniform(-0.5, 0.5, (n, n)) / np.sqrt(n)
    b = rng.uniform(-1, 1, n)
    return np.ascontiguousarray(A), np.ascontiguousarray(b)


def static_solve(n, A, b):
    import bit_b200 as B
    L = B.lib()
    x = np.ones(n)
    it = C.c_int()
    err = C.create_string_buffer(256)
    dp = C.POINTER(C.c_double)
    st = L.bit_gmres_dense_static(None, n, A.ctypes.data_as(dp), b.ctypes.data_as(dp),
                                  x.ctypes.data_as(dp), C.byref(it), err, len(err))
    return st, x, it.value, err.value.decode()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [300, 512])
def test_static_matches_allocating_entry_point_twice(n):
    import bit_b200 as B
    systems = [system(n, seed) for seed in (11, 12)]
    # two calls in a row: the second starts from the scratch the first left behind
    static = [static_solve(n, A, b) for A, b in systems]
    ctx = B.Context()
    try:
        for call, ((A, b), (st, x, it, msg)) in enumerate(zip(systems, static)):
            assert st == 0, msg
            x_ref, it_ref, st_ref = ctx.gmres_dense(A, b)
            assert st_ref == 0
            assert it == it_ref, (call, it, it_ref)
            assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) < TOL, call
            exact = np.linalg.solve(A, b)
            assert np.linalg.norm(x - exact) / np.linalg.norm(exact) < 1e-5
    finally:
        ctx.close()


def test_static_refuses_sizes_over_the_limit():
    """Refused before any CUDA call, so this runs without a GPU too."""
    import bit_b200 as B
    n = 513
    A, b = system(n, 1)
    st, _, _, msg = static_solve(n, A, b)
    assert st == 4  # BIT_ERR_CAPACITY
    assert "512" in msg and "513" in msg


_SECOND_CONTEXT = r"""
import ctypes as C, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import bit_b200 as B
L = B.lib()
dp = C.POINTER(C.c_double)
rng = np.random.default_rng(7)
n = 256
A = np.ascontiguousarray(np.eye(n) * 3 + rng.uniform(-0.5, 0.5, (n, n)) / np.sqrt(n))
b = rng.uniform(-1, 1, n)
def solve():
    x = np.ones(n)
    it = C.c_int()
    err = C.create_string_buffer(256)
    st = L.bit_gmres_dense_static(None, n, A.ctypes.data_as(dp), b.ctypes.data_as(dp),
                                  x.ctypes.data_as(dp), C.byref(it), err, len(err))
    assert st == 0, err.value
    return x, it.value
x1, it1 = solve()  # in the device's primary context
cu = C.CDLL("libcuda.so.1")
assert cu.cuInit(0) == 0
dev, ctx = C.c_int(), C.c_void_p()
assert cu.cuDeviceGet(C.byref(dev), 0) == 0
assert cu.cuCtxCreate_v2(C.byref(ctx), 0, dev) == 0  # now current on this thread
x2, it2 = solve()  # the library's code and scratch are loaded anew in this context
assert cu.cuCtxDestroy_v2(ctx) == 0
assert it1 == it2 and (x1 == x2).all()
exact = np.linalg.solve(A, b)
assert np.linalg.norm(x2 - exact) / np.linalg.norm(exact) < 1e-5
print("second context ok")
"""


@pytest.mark.gpu
def test_static_in_a_second_context_of_the_same_device():
    """A second CUDA context on the same device (a driver-API caller, or the runtime after
    cudaDeviceReset) holds its own copy of the scratch array at another address.  The
    entry point looks the address up in the current context on every call, so a call made
    in the new context gives the same result as one made in the first.  Runs in a fresh
    process of its own."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _SECOND_CONTEXT, root], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "second context ok" in r.stdout
