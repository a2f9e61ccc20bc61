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


def test_two_level_build_with_overflowing_coarse_cells():
    """Large grids build their cells from coarse cells of 4 x 4 cells; a dense
    cluster of small rects in a sparse layout overflows its coarse cell (over
    64 rects), whose cells then enumerate the tree.  Queries from the cells
    equal the tree's on uniform points and on points in and around the
    cluster."""
    rng = np.random.default_rng(0x2C0)
    sparse = frw.generate_layout(0xF4A7 + 9, 70_000, 1e5)
    # 20 x 20 rects of side 1, two apart, in an empty patch
    gx, gy = np.meshgrid(np.arange(20) * 3.0, np.arange(20) * 3.0)
    x0, y0 = 50_000.0 + gx.ravel(), 50_000.0 + gy.ravel()
    cluster = np.stack([x0, y0, x0 + 1, y0 + 1], 1).astype(np.float32)
    keep = ~((sparse[:, 2] >= 49_900) & (sparse[:, 0] <= 50_200) & (sparse[:, 3] >= 49_900) & (sparse[:, 1] <= 50_200))
    rects = np.concatenate([sparse[keep], cluster]).astype(np.float32)
    with frw.Layout.from_rects(rects) as L:
        ci = L.cells
        assert ci.cells >= 1 << 16 and ci.overflow_cells > 0
        b = L.bounds
        near = np.stack([50_000 + rng.uniform(-200, 260, 20_000), 50_000 + rng.uniform(-200, 260, 20_000)], 1)
        pts = np.concatenate([_points(rects.astype(np.float64), b, 40_000, 13, ci.cell_side), near])
        sq_c, hit_c = L.query(pts)
        L.set_cells(0)
        sq_t, hit_t = L.query(pts)
    assert np.array_equal(sq_c, sq_t) and np.array_equal(hit_c, hit_t)
    assert np.any(hit_c[-20_000:] >= len(rects) - 400)  # some points hit the cluster


def _aligned_array(nx=30, ny=30, pitch=3.0):
    """nx x ny rects of side 1 on a pitch-3 grid: seen from beside a column
    (or a row), every rect of it within the L-inf cone ties exactly."""
    gx, gy = np.meshgrid(np.arange(nx) * pitch, np.arange(ny) * pitch)
    x0, y0 = 100.0 + gx.ravel(), 100.0 + gy.ravel()
    return np.stack([x0, y0, x0 + 1, y0 + 1], 1).astype(np.float32)


def test_tree_query_with_many_exact_ties_equals_oracle():
    """Points beside the array see up to ~25 rects at one exact gap, more than
    the tree's near-tie list holds: those points take the whole-tree replay.
    Squares and hits equal the oracle's, from the tree and from the cells."""
    rects = _aligned_array()
    b = np.array([0.0, 0.0, 300.0, 300.0])
    rng = np.random.default_rng(0x71E5)
    far = np.stack([rng.uniform(0, 300, 30_000), rng.uniform(0, 300, 30_000)], 1)
    side = np.stack([rng.uniform(20, 99, 10_000), rng.uniform(100, 190, 10_000)], 1)  # left of column 0
    below = np.stack([rng.uniform(100, 190, 10_000), rng.uniform(20, 99, 10_000)], 1)  # under row 0
    pts = np.concatenate([far, side, below])
    G = O.Grid(rects.astype(np.float64), b)
    sq_o, hit_o = G.query_batch(pts)
    with frw.Layout.from_rects(rects, b) as L:
        sq_c, hit_c = L.query(pts)
        L.set_cells(0)
        sq_t, hit_t = L.query(pts)
    assert np.array_equal(sq_t, sq_o) and np.array_equal(hit_t, hit_o)
    assert np.array_equal(sq_c, sq_o) and np.array_equal(hit_c, hit_o)


def test_tree_walks_with_many_exact_ties_equal_oracle():
    """The walk kernel answers tree points with many exact ties by the
    whole-tree replay (the layout has no cell lists): per-walk records equal
    the oracle's, and the estimator rows equal those of the cell-list walks
    (a kernel built without the whole-tree replay, the cells leaving no point
    to the tree)."""
    rects = _aligned_array()
    b = np.array([0.0, 0.0, 300.0, 300.0])
    target = 15 * 30 + 0  # a rect of column 0
    o = frw.opts(gauss_mode=frw.GAUSS_OFFSET, gauss_param=4.0, start_mode=frw.START_UNIFORM)
    G = O.Grid(rects.astype(np.float64), b)
    n = 4000
    end_o, hops_o, b1_o, w_o = G.walks(G.walk_cfg(target=target, gauss_mode=o.gauss_mode, gauss_param=o.gauss_param,
                                                  start_mode=o.start_mode, hop_cap=o.hop_cap, seed=77,
                                                  stream=o.stream_id), 0, n)
    with frw.Layout.from_rects(rects, b) as L:
        rows_c = L.walk(target, 200_000, seed=78, o=o)
        L.set_cells(0)
        end, hops, b1, w = L.walk_trace(target, 0, n, seed=77, o=o)
        rows_t = L.walk(target, 200_000, seed=78, o=o)
    assert np.array_equal(end, end_o) and np.array_equal(hops, hops_o)
    assert np.array_equal(b1, b1_o) and np.array_equal(w, w_o)
    # same walks: equal counts; the weight sums differ only in summation order
    assert np.array_equal(rows_c.conductor, rows_t.conductor) and np.array_equal(rows_c.hits, rows_t.hits)
    assert np.allclose(rows_c.sum_w, rows_t.sum_w, rtol=1e-12, atol=1e-300)


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
