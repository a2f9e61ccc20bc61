"""Collision queries on the device vs the CPU oracle (complete semantics):
bit-exact squares and hit ids."""
import numpy as np
import pytest

import frw
import oracle as O
from conftest import FIXTURES

pytestmark = pytest.mark.gpu


def edge_points(rects, b, rng, n):
    """Points on rect edges/corners, integer lattice points and bounds edges."""
    k = rng.integers(0, len(rects), n)
    r = rects[k]
    t = rng.integers(0, 6, n)
    x = np.where(t == 0, r[:, 0], np.where(t == 1, r[:, 2], rng.uniform(r[:, 0] - 3, r[:, 2] + 3)))
    y = np.where(t == 2, r[:, 1], np.where(t == 3, r[:, 3], rng.uniform(r[:, 1] - 3, r[:, 3] + 3)))
    x = np.where(t == 4, np.round(x), x)
    y = np.where(t == 5, np.round(y) + 0.5, y)
    pts = np.stack([x, y], 1)
    m = n // 10
    pts[:m, 0] = b[0] + rng.integers(0, 3, m)  # at / near the bounds
    pts[m:2 * m, 1] = b[3] - rng.integers(0, 3, m)
    return pts


@pytest.mark.parametrize("name", FIXTURES)
def test_query_golden_fixtures(golden, name):
    gd = golden(name)
    G = O.Grid(gd["rects"], gd["bounds"])
    with frw.Layout.from_rects(gd["rects"], gd["bounds"]) as L:
        rng = np.random.default_rng(11)
        pts = np.concatenate([gd["pts"], edge_points(gd["rects"], gd["bounds"], rng, 2000)])
        sq, hit = L.query(pts)
        sq_o, hit_o = G.query_batch(pts)
        bad = np.nonzero((sq != sq_o).any(1) | (hit != hit_o))[0]
        assert len(bad) == 0, (name, len(bad), pts[bad[:3]], sq[bad[:3]], sq_o[bad[:3]])


def test_query_config2_1e5_points():
    """10,000 rects on [0,1e4]^2 (sizes 5-50, gap >= 2), 1e5 seeded points."""
    rects = frw.generate_layout(0xF4A7 + 2, 10_000, 1e4)
    G = O.Grid(rects.astype(np.float64))
    rng = np.random.default_rng(0x0C2)
    b = G.bounds
    pts = np.stack([rng.uniform(b[0], b[2], 100_000), rng.uniform(b[1], b[3], 100_000)], 1)
    with frw.Layout.from_rects(rects) as L:
        assert np.array_equal(L.bounds, b)
        sq, hit = L.query(pts)
    sq_o, hit_o = G.query_batch(pts)
    assert np.array_equal(sq, sq_o)
    assert np.array_equal(hit, hit_o)
    assert (hit >= 0).sum() > 100  # some points do land inside conductors


def test_query_outside_and_degenerate():
    rects = np.array([[10, 10, 20, 20], [30, 10, 30, 40], [25, 25, 25, 25]], dtype=np.float32)
    G = O.Grid(rects.astype(np.float64))
    pts = np.array([[0, 0], [-50, 5], [1e6, 1e6], [30, 20], [25, 25], [20, 20], [15, 15], [24.5, 25.5]])
    with frw.Layout.from_rects(rects) as L:
        sq, hit = L.query(pts)
    sq_o, hit_o = G.query_batch(pts)
    assert np.array_equal(sq, sq_o) and np.array_equal(hit, hit_o)


def test_query_overlapping_rects_lowest_index():
    rects = np.array([[0, 0, 100, 100], [50, 50, 150, 150], [60, 60, 70, 70]], dtype=np.float32)
    with frw.Layout.from_rects(rects, bounds=np.array([-10.0, -10, 200, 200])) as L:
        _, hit = L.query(np.array([[65.0, 65.0], [120, 120], [10, 10], [180, 180]]))
    assert list(hit) == [0, 1, 0, -1]


@pytest.mark.parametrize("name", ["test", "test2", "test1000"])
def test_box_collisions_with_ignore(golden, name):
    gd = golden(name)
    rects, b = gd["rects"], gd["bounds"]
    G = O.Grid(rects, b)
    rng = np.random.default_rng(5)
    c = np.stack([rng.uniform(b[0], b[2], 3000), rng.uniform(b[1], b[3], 3000)], 1)
    s = rng.uniform(0, 60, (3000, 2))
    boxes = np.concatenate([c - s, c + s], 1)
    boxes[:300] = rects[rng.integers(0, len(rects), 300)]  # boxes equal to rects
    ign = rects[3]
    with frw.Layout.from_rects(rects, b) as L:
        got = L.check_collisions(boxes)
        got_i = L.check_collisions(boxes, ignore=ign)
    want = np.array([G.box_collides(x) for x in boxes])
    want_i = np.array([G.box_collides(x, ign) for x in boxes])
    assert np.array_equal(got, want) and np.array_equal(got_i, want_i)


@pytest.mark.parametrize("name", FIXTURES)
def test_gauss_surface_scale_mode(golden, name):
    gd = golden(name)
    G = O.Grid(gd["rects"], gd["bounds"])
    T = O.RefTree(gd["rects"], gd["bounds"])
    with frw.Layout.from_rects(gd["rects"], gd["bounds"]) as L:
        for t, gref in zip(gd["gauss_targets"], gd["ref_gauss"]):
            got = L.gauss_surface(int(t))
            assert np.array_equal(got, G.gauss_scale(gd["rects"][t], 1.5))
            # where the reference's incomplete query finds the same collisions,
            # it agrees with the reference itself
            if np.array_equal(T.gauss_scale(gd["rects"][t], 1.5, False), gref):
                assert np.array_equal(got, gref)


def test_layout_info_and_tree_shape():
    rects = frw.generate_layout(3, 50_000, 3e4)
    with frw.Layout.from_rects(rects) as L:
        info = L.info
        assert info.n_rects == 50_000 and 0 < info.n_nodes < 50_000 and info.depth >= 4
        assert np.array_equal(L.rects(), rects.astype(np.float64))


@pytest.mark.parametrize("n", [1, 2, 8, 9, 33, 65_536, 65_537])
def test_tiny_and_threshold_layouts_match_oracle(n):
    """Layouts around the tree builder's special sizes: a root leaf (n <= 8),
    the first split, and both sides of the one-block build's 65,536-rect
    limit; queries and walk records equal the oracle's."""
    dom = max(200.0, float(np.sqrt(n)) * 100.0)
    rects = frw.generate_layout(0xA11 + n, n, dom)
    G = O.Grid(rects.astype(np.float64))
    rng = np.random.default_rng(n)
    with frw.Layout.from_rects(rects) as L:
        b = L.bounds
        pts = np.stack([rng.uniform(b[0], b[2], 4000), rng.uniform(b[1], b[3], 4000)], 1)
        pts[:200] = rects[rng.integers(0, n, 200), :2]  # rect corners
        sq, hit = L.query(pts)
        o = frw.capacitance_opts(1.0)
        end, hops, b1, w = L.walk_trace(0, 0, 2000, seed=9, o=o)
        for cells in (0.0, 16.0):  # the tree alone, then with cell lists again
            L.set_cells(cells)
            sq2, hit2 = L.query(pts)
            assert np.array_equal(sq2, sq) and np.array_equal(hit2, hit)
    sq_o, hit_o = G.query_batch(pts)
    assert np.array_equal(sq, sq_o) and np.array_equal(hit, hit_o)
    cfg = G.walk_cfg(target=0, gauss_mode=o.gauss_mode, gauss_param=o.gauss_param, start_mode=o.start_mode, seed=9)
    end_o, hops_o, b1_o, w_o = G.walks(cfg, 0, 2000)
    assert np.array_equal(end, end_o) and np.array_equal(hops, hops_o)
    assert np.array_equal(b1, b1_o) and np.array_equal(w, w_o)


def test_degenerate_and_equal_key_layouts_match_oracle():
    """A layout of one point-sized rect (zero-area bounds), and 40 nested
    rects sharing one centre (equal Morton keys: the tree splits them by
    index); queries and walks equal the oracle's."""
    cases = [
        np.array([[50, 50, 50, 50]], dtype=np.float32),
        np.array([[100 - k, 100 - k, 100 + k, 100 + k] for k in range(1, 41)], dtype=np.float32),
    ]
    rng = np.random.default_rng(4)
    for rects in cases:
        G = O.Grid(rects.astype(np.float64))
        b = G.bounds
        pts = np.stack([rng.uniform(b[0] - 1, b[2] + 1, 3000), rng.uniform(b[1] - 1, b[3] + 1, 3000)], 1)
        pts[:40] = rects[: min(40, len(rects)), :2]
        with frw.Layout.from_rects(rects) as L:
            sq, hit = L.query(pts)
            o = frw.capacitance_opts(1.0)
            end, hops, b1, w = L.walk_trace(0, 0, 500, seed=3, o=o)
        sq_o, hit_o = G.query_batch(pts)
        assert np.array_equal(sq, sq_o) and np.array_equal(hit, hit_o)
        cfg = G.walk_cfg(target=0, gauss_mode=o.gauss_mode, gauss_param=o.gauss_param, start_mode=o.start_mode,
                         seed=3)
        end_o, hops_o, b1_o, w_o = G.walks(cfg, 0, 500)
        assert np.array_equal(end, end_o) and np.array_equal(hops, hops_o)
        assert np.array_equal(b1, b1_o) and np.array_equal(w, w_o)
