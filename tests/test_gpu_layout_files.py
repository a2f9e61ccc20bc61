"""Layouts read from the reference's own layout files, on the device.

* frw_layout_from_file on each fixture file holds exactly the rects and
  bounds that the reference's Parser produced (golden fixtures), and its
  queries equal the complete-semantics oracle on the golden query points.
* The reference-side bridge (engineer-thesis_b200/bridge/frw_b200_bridge.cpp,
  compiled against the reference's Cuda/mainkernels.h and linked to
  libfrw.so) is what a reference caller of getAvgPathLenCUDA reaches: called
  through its C++ symbol it returns what frw_avg_path_len returns for the
  same seed, and writes the reference's "<ts>wyniki.txt" histogram.
"""
import glob
import os
import subprocess
import sys

import numpy as np
import pytest

import frw
import oracle as O
from conftest import FIXTURES, GOLDEN

pytestmark = pytest.mark.gpu
LAYOUTS = os.path.join(GOLDEN, "layouts")
BRIDGE = os.path.join(os.path.dirname(frw.LIB_PATH), "libfrw_bridge.so")


@pytest.mark.parametrize("name", FIXTURES)
def test_layout_from_file_holds_reference_rects_and_bounds(name, golden):
    g = golden(name)
    with frw.Layout.from_file(os.path.join(LAYOUTS, name)) as L:
        assert L.n == len(g["rects"])
        assert np.array_equal(L.rects(), g["rects"])
        assert np.array_equal(L.bounds, g["bounds"])
        sq, hit = L.query(g["pts"])
    sq_o, hit_o = O.Grid(g["rects"], g["bounds"]).query_batch(g["pts"])
    assert np.array_equal(sq, sq_o) and np.array_equal(hit, hit_o)


# getAvgPathLenCUDA(char*, int, int, bool, int) called as a reference caller
# would; in a child process, because the bridge ends the process with exit(0)
# on failure as the reference does
_CALL = """
import ctypes as C, sys
fn = getattr(C.CDLL(sys.argv[1]), "_Z17getAvgPathLenCUDAPciibi")
fn.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_bool, C.c_int]
fn.restype = C.c_double
print("fraction=%r" % fn(sys.argv[2].encode(), 50000, 10, False, 0))
"""


def test_reference_bridge_equals_avg_path_len(tmp_path):
    if not os.path.exists(BRIDGE):
        pytest.skip("the bridge is built only where the reference's header is present")
    path = os.path.join(LAYOUTS, "test2")
    env = dict(os.environ, FRW_SEED="4242")
    out = subprocess.run([sys.executable, "-c", _CALL, BRIDGE, path], cwd=tmp_path, env=env, capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    got = [ln for ln in out.stdout.splitlines() if ln.startswith("fraction=")]
    assert got, (out.stdout, out.stderr)
    got = float(got[0].split("=", 1)[1])
    want = frw.get_avg_path_len_cuda(path, 50_000, 10, layer=0, seed=4242)
    assert got == want and 0.0 < got < 1.0
    assert "wyniki.txt" in out.stdout
    hist = glob.glob(str(tmp_path / "*wyniki.txt"))
    assert len(hist) == 1 and open(hist[0], encoding="utf-8").readline().strip() == "[GPU]"
