"""The support estimate sums its terms with nan_pairwise::Feed, a one-term-at-
a-time form of numpy's float64 sum of a float32 array (buffers of 8192,
pairwise inside). The header is plain C++ as well as CUDA, so this test
compiles it on the host (no fused multiply-add, as the library is built)
and checks it against numpy bit for bit: every size to 600, sizes around the
buffer length and its multiples, and random sizes to 70,000, over values of
mixed magnitude."""

import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

HEADER_DIR = Path(__file__).resolve().parents[1] / "nan_b200" / "csrc"

SHIM = r"""
#include "nan_pairwise.h"
extern "C" double feed_sum(const float* v, unsigned n, unsigned* max_depth) {
    nan_pairwise::Feed s;
    s.begin(n);
    unsigned md = 0;
    for (unsigned i = 0; i < n; ++i) {
        s.push((double)v[i]);
        if (s.depth > md) md = s.depth;
    }
    *max_depth = md;
    return s.total;
}
"""


@pytest.fixture(scope="module")
def feed(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ is not installed")
    d = tmp_path_factory.mktemp("pairwise")
    (d / "shim.cpp").write_text(SHIM)
    lib = d / "libshim.so"
    subprocess.run([cxx, "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-I", str(HEADER_DIR), str(d / "shim.cpp"),
                    "-o", str(lib)], check=True)
    so = ctypes.CDLL(str(lib))
    so.feed_sum.restype = ctypes.c_double
    so.feed_sum.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.POINTER(ctypes.c_uint)]
    return so


def test_feed_equals_numpy_sum(feed):
    rng = np.random.default_rng(1)
    sizes = (list(range(0, 600)) + list(range(8000, 8400)) + list(range(16300, 16500)) +
             [int(x) for x in rng.integers(0, 70000, 200)])
    deepest = 0
    for n in sizes:
        v = (rng.random(n, dtype=np.float32) * rng.choice([1e-3, 1.0, 1e3], n)).astype(np.float32)
        depth = ctypes.c_uint()
        got = feed.feed_sum(v.ctypes.data, n, ctypes.byref(depth))
        assert got == np.sum(v, dtype=np.float64), n
        deepest = max(deepest, depth.value)
    assert deepest <= 8  # the frame arrays hold 8 levels
