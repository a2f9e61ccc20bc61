"""Generate tests/golden/cube_green.npz from the reference itself.

Run in a container that has the reference checkout (the GPU machine only
reads the committed .npz):

    python tests/golden/make_golden_cube.py

The reference ships a unit-cube Green's function (green/green.cpp:232-431)
that it never calls.  This records, from the unmodified reference compiled by
oracle/Makefile (oracle/_ref/librefcpu.so):

* precompute_unit_cube_green(g, dgdx, dgdy, dgdz, intg, n) for n in
  {1, 2, 3, 5, 8, 16}, in full;
* SHA-256 digests of the five arrays for n = 50 and n = 100 (the walk's
  default resolution and the largest accepted one);
* green_cube and deriv_green_cube at 64 seeded points of every face for cube
  sides 1, 0.37 and 12.5.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

FULL = (1, 2, 3, 5, 8, 16)
DIGEST = (50, 100)


def digest(arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def main():
    O.build(ref=True)
    L = O.ref()
    out = {}
    for n in FULL:
        for name, a in zip(("g", "dgdx", "dgdy", "dgdz", "intg"), O.ref_cube_green_table(n)):
            out[f"n{n}_{name}"] = a
    out["digest_n"] = np.array(DIGEST)
    out["digest"] = np.array([digest(O.ref_cube_green_table(n)) for n in DIGEST])
    rng = np.random.default_rng(0xC0BE)
    pts, g, dg = [], [], []
    for a in (1.0, 0.37, 12.5):
        for k in range(6):
            for _ in range(64):
                eta, dz = (k + rng.random()) * a, (k + rng.random()) * a
                d = np.zeros(3)
                L.ref_deriv_green_cube(O._p(d), a, eta, dz)
                pts.append((a, eta, dz))
                g.append(L.ref_green_cube(a, eta, dz))
                dg.append(d)
    out["pt"] = np.array(pts)
    out["pt_g"] = np.array(g)
    out["pt_dg"] = np.array(dg)
    path = os.path.join(HERE, "cube_green.npz")
    np.savez_compressed(path, **out)
    print(f"{os.path.relpath(path, ROOT)}: {os.path.getsize(path) / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
