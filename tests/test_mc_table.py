"""The marching-cubes triangle table, pinned to the reference.

tests/golden/mc_tri_table.json is the reference's triTable
(include/pb_class.h:245-502), extracted by oracle/make_mc_table.py.  The
oracle's own copy and the product's packed copy (csrc/mc_tables.h, expanded the
way the energy kernels expand it) must both equal it entry by entry, so a
transcription error in either table cannot pass both sides of a parity test."""
import ctypes
import json
import os
import subprocess
import tempfile

import numpy as np

import oracle_lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "mc_tri_table.json")


def _golden():
    return np.array(json.load(open(GOLDEN))["tri_table"], dtype=np.int32)


def test_oracle_table_equals_reference():
    L = oracle_lib.load()
    out = np.zeros(256 * 16, dtype=np.int32)
    assert L.oracle_tri_table(out.ctypes.data_as(ctypes.POINTER(ctypes.c_int))) == 0
    assert np.array_equal(out.reshape(256, 16), _golden())


def test_product_packed_table_equals_reference():
    src = r"""
#include <cstdio>
#include "mc_tables.h"
int main() {
  signed char t[256][16];
  pbmc::expand_tri_table(t);
  for (int k = 0; k < 256; ++k)
    for (int j = 0; j < 16; ++j) std::printf("%d\n", (int)t[k][j]);
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.cpp")
        exe = os.path.join(d, "t")
        open(c, "w").write(src)
        subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "cudanextgenpb_b200", "csrc"), c, "-o", exe],
                       check=True)
        vals = np.array(subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split(),
                        dtype=np.int32)
    assert np.array_equal(vals.reshape(256, 16), _golden())


def test_triangle_edges_are_cut_edges():
    """Every edge a case's triangles use is one whose end vertices differ
    (the reference's edgeTable property), under the corner order of
    src/pb_class.cpp:2579-2581 and edge2nodes of include/pb_class.h:190-207."""
    corner = [0, 1, 3, 2, 4, 5, 7, 6]
    vertex = {c: v for v, c in enumerate(corner)}
    e2n = [0, 1, 1, 3, 2, 3, 0, 2, 4, 5, 5, 7, 6, 7, 4, 6, 0, 4, 1, 5, 3, 7, 2, 6]
    t = _golden()
    for k in range(256):
        cut = {e for e in range(12) if ((k >> vertex[e2n[2 * e]]) ^ (k >> vertex[e2n[2 * e + 1]])) & 1}
        used = {int(e) for e in t[k] if e >= 0}
        assert used == cut, k
