"""The hand-written per-node reverse of the cavity step (node_ad.h) passes
the dot-product test against forward-mode dual numbers (CPU only)."""
import ctypes
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    out = tmp_path_factory.mktemp("nodead") / "libnodead.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", str(out),
                    os.path.join(HERE, "native", "node_ad_check.cpp")], check=True)
    L = ctypes.CDLL(str(out))
    L.node_ad_check.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
                                ctypes.POINTER(ctypes.c_double)]
    return L


@pytest.mark.parametrize("wall_mode,zero_pi", [(0, 0), (1, 0), (2, 0), (0, 1)])
def test_node_reverse_is_the_transpose_of_the_tangent(lib, wall_mode, zero_pi):
    worst = ctypes.c_double()
    lib.node_ad_check(2000, 1234 + wall_mode, wall_mode, zero_pi, ctypes.byref(worst))
    assert worst.value < 1e-10, worst.value
