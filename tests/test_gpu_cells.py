"""Cell lists: queries answered from a cell's rect list equal those from the
tree and the CPU oracle bit for bit -- on the fixtures, on points placed on
cell boundaries, rect edges and corners, with lists small enough that many
cells overflow to the tree, and through whole walks."""
import numpy as np
import pytest

import frw
import oracle as O

pytestmark = pytest.mark.gpu


def _points(rects, bounds, n, seed, side=None):
    rng = np.random.default_rng(seed)
    pts = [np.stack([rng.uniform(bounds[0], bounds[2], n), rng.uniform(bounds[1], bounds[3], n)], 1)]
    k = rng.integers(0, len(rects), n // 4)
    r = rects[k]
    # rect corners and edge points (closed intervals decide hits)
    pts.append(np.stack([r[:, 0], r[:, 1]], 1))
    pts.append(np.stack([r[:, 2], rng.uniform(r[:, 1], r[:, 3])], 1))
    pts.append(np.stack([rng.uniform(r[:, 0], r[:, 2]), r[:, 3] + rng.choice([0.0, 1.0, 0.5], len(k))], 1))
    if side:  # cell boundaries and corners
        ix = rng.integers(0, max(1, int((bounds[2] - bounds[0]) / side)), n // 4)
        iy = rng.integers(0, max(1, int((bounds[3] - bounds[1]) / side)), n // 4)
        gx, gy = bounds[0] + ix * side, bounds[1] + iy * side
        pts.append(np.stack([gx, rng.uniform(bounds[1], bounds[3], len(gx))], 1))
        pts.append(np.stack([gx, gy], 1))
        pts.append(np.stack([np.nextafter(gx, -np.inf), np.nextafter(gy, np.inf)], 1))
    p = np.concatenate(pts)
    inside = (p[:, 0] >= bounds[0]) & (p[:, 0] <= bounds[2]) & (p[:, 1] >= bounds[1]) & (p[:, 1] <= bounds[3])
    return p[inside]


@pytest.mark.parametrize("name", ["test", "test1", "test2", "test100", "test1000", "test10000"])
def test_cells_equal_tree_and_oracle_on_fixtures(golden, name):
    gd = golden(name)
    rects, bounds = gd["rects"], gd["bounds"]
    with frw.Layout.from_rects(rects, bounds) as L:
        ci = L.cells
        assert ci.cells > 0 and ci.entries > 0
        pts = _points(rects, bounds, 20_000, 7, ci.cell_side)
        sq_c, hit_c = L.query(pts)
        L.set_cells(0)
        assert L.cells.cells == 0
        sq_t, hit_t = L.query(pts)
    assert np.array_equal(sq_c, sq_t) and np.array_equal(hit_c, hit_t)
    G = O.Grid(rects, bounds)
    sq_o, hit_o = G.query_batch(pts[:5000])
    assert np.array_equal(sq_c[:5000], sq_o) and np.array_equal(hit_c[:5000], hit_o)


@pytest.mark.parametrize("cells_per_rect,max_per_cell", [(0.05, 32), (1.0, 2), (8.0, 1), (64.0, 32)])
def test_cells_any_resolution_and_overflow(cells_per_rect, max_per_cell):
    rects = frw.generate_layout(0xF4A7 + 2, 10_000, 1e4)
    with frw.Layout.from_rects(rects) as L:
        b = L.bounds
        L.set_cells(0)
        pts = _points(rects.astype(np.float64), b, 40_000, 11, 25.0)
        sq_t, hit_t = L.query(pts)
        L.set_cells(cells_per_rect, max_per_cell)
        ci = L.cells
        if max_per_cell <= 2:
            assert ci.overflow_cells > 0  # both paths are exercised
        sq_c, hit_c = L.query(_points(rects.astype(np.float64), b, 40_000, 11, 25.0))
        pts_c = _points(rects.astype(np.float64), b, 40_000, 11, ci.cell_side)
        sq_c2, hit_c2 = L.query(pts_c)
        L.set_cells(0)
        sq_t2, hit_t2 = L.query(pts_c)
    assert np.array_equal(sq_c, sq_t) and np.array_equal(hit_c, hit_t)
    assert np.array_equal(sq_c2, sq_t2) and np.array_equal(hit_c2, hit_t2)


def test_cells_c2_lists_are_short():
    """10^4 rects: 16 cells per rect, a handful of rects per list, no overflow."""
    rects = frw.generate_layout(0xF4A7 + 2, 10_000, 1e4)
    with frw.Layout.from_rects(rects) as L:
        ci = L.cells
    assert ci.cells >= 16 * 10_000 * 0.9
    assert ci.entries / ci.cells < 8
    assert ci.overflow_cells == 0


def test_walks_identical_with_and_without_cells(golden):
    gd = golden("test1000")
    o = frw.capacitance_opts(1.0)
    with frw.Layout.from_rects(gd["rects"], gd["bounds"]) as L:
        a = L.walk_trace(17, 0, 20_000, seed=5, o=o)
        L.set_cells(0)
        b = L.walk_trace(17, 0, 20_000, seed=5, o=o)
        L.set_cells(2.0, 4)
        c = L.walk_trace(17, 0, 20_000, seed=5, o=o)
    for x, y, z in zip(a, b, c):
        assert np.array_equal(x, y) and np.array_equal(x, z)


def test_cv_features_equal_with_and_without_cells():
    """The nearest-other-conductor lookup of the control-variate features
    answers from the cell list when the list settles it and from the tree
    otherwise; both give the oracle's features bit for bit."""
    rects = frw.generate_layout(0xF4A7 + 2, 10_000, 1e4)
    rng = np.random.default_rng(3)
    n = 30_000
    rec = np.zeros((n, 4))
    t = 0
    r = rects[t].astype(np.float64)
    rec[: n // 2, 0] = rng.uniform(r[0] - 60, r[2] + 60, n // 2)
    rec[: n // 2, 1] = rng.uniform(r[1] - 60, r[3] + 60, n // 2)
    with frw.Layout.from_rects(rects) as L:
        b = L.bounds
        rec[n // 2:, 0] = rng.uniform(b[0], b[2], n - n // 2)
        rec[n // 2:, 1] = rng.uniform(b[1], b[3], n - n // 2)
        rec[:, 2] = rng.choice([1.0, 2.5, 7.0], n)
        f_cells = L.cv_features(t, rec)
        L.set_cells(0)
        f_tree = L.cv_features(t, rec)
    assert np.array_equal(f_cells, f_tree)
    want = O.cv_features(rects.astype(np.float64), t, rec[::10])
    assert np.array_equal(f_cells[::10], want)
