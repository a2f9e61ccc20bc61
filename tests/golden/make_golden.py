"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run in a container that has the reference checkout (it is not needed on the
GPU machine, which only reads the committed .npz files):

    python tests/golden/make_golden.py

For every reference layout fixture (tests/test*, generatedtests/test{100,1000,
10000}.txt) it loads the layout with the reference's own Parser and builds the
reference CPU quadtree (oracle/_ref/librefcpu.so, compiled from the unmodified
reference sources), then records:

* the rects and layer bounds exactly as the reference parsed them;
* the reference's Green tables (g, dgdx, dgdy, intg);
* 2,000 seeded query points with the reference's drawBiggestSquareAtPoint
  square and checkCollisons hit (defect semantics, as shipped);
* the reference's Gaussian surfaces (creatGaussianSurfFrom, factor 1.5) for
  up to 16 targets;
* a few hundred reference walks (RandomWalk's body, JKISS seeded once) with
  the uniform stream they consumed, their end rect and hop count.

The fixture layout files themselves are copied, unchanged, to
tests/golden/layouts/ so that the product's own reader can be checked against
the rects and bounds above on machines without the reference checkout.  The
checkout is $REFERENCE, else the default of oracle/Makefile.
"""
from __future__ import annotations

import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

REF_ROOT = O.reference_root()
LAYOUTS = os.path.join(HERE, "layouts")
FIXTURES = [
    ("test", "tests/test", 10, 300),
    ("test1", "tests/test1", 5, 300),
    ("test2", "tests/test2", 10, 400),
    ("test100", "generatedtests/test100.txt", 7, 200),
    ("test1000", "generatedtests/test1000.txt", 500, 60),
    ("test10000", "generatedtests/test10000.txt", 1234, 20),
]


def query_points(rects, b, rng, n=2000):
    """Uniform, integer-snapped and near-edge points (ties are the hard cases)."""
    pts = np.stack([rng.uniform(b[0], b[2], n), rng.uniform(b[1], b[3], n)], 1)
    a = n // 4
    pts[:a] = np.floor(pts[:a])
    k = rng.integers(0, len(rects), a)
    pts[a:2 * a, 0] = rects[k, 0] - rng.integers(0, 4, a)
    pts[a:2 * a, 1] = rects[k, 1] + np.round(rng.uniform(-3, 3, a), 1)
    k = rng.integers(0, len(rects), a)
    pts[2 * a:3 * a, 0] = rects[k, 2] + rng.integers(0, 3, a) + 0.5 * rng.integers(0, 2, a)
    pts[2 * a:3 * a, 1] = rects[k, 3] + rng.integers(-2, 3, a)
    return pts


def copy_layouts():
    os.makedirs(LAYOUTS, exist_ok=True)
    for name, rel, _, _ in FIXTURES:
        shutil.copyfile(os.path.join(REF_ROOT, rel), os.path.join(LAYOUTS, name))


def main():
    O.build(ref=True)
    copy_layouts()
    for name, rel, target, nwalks in FIXTURES:
        path = os.path.join(REF_ROOT, rel)
        R = O.Ref(path=path)
        rng = np.random.default_rng(0xF4A7 + len(name))
        g, dgdx, dgdy, intg = R.green()
        pts = query_points(R.rects, R.bounds, rng)
        sq, hit = R.query_batch(pts)
        targets = np.unique(np.concatenate([[target], rng.integers(0, R.n, 15)]))[:16]
        gauss = np.array([R.gauss(t, 1.5) for t in targets])
        end, hops, rs, used = R.walks_seeded(target, nwalks, seed=(0x1234, 0x5678, 0x9ABC, 0xDEF0),
                                             r_cap=5_000_000)
        assert used == len(rs)
        out = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(
            out, rects=R.rects, bounds=R.bounds, g=g, dgdx=dgdx, dgdy=dgdy, intg=intg,
            pts=pts, ref_sq=sq, ref_hit=hit, gauss_targets=targets, ref_gauss=gauss,
            walk_target=np.int64(target), walk_r=rs, walk_end=end, walk_hops=hops)
        print(f"{name}: {R.n} rects, {len(pts)} points, {nwalks} walks "
              f"({len(rs)} uniforms) -> {os.path.relpath(out, ROOT)} "
              f"{os.path.getsize(out) / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
