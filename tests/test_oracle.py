"""The CPU oracle against the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from the compiled reference), and -- when the
compiled reference library is present -- against it live."""
import numpy as np
import pytest

import oracle as O
from conftest import FIXTURES


def test_philox_known_answers():
    # Random123 known-answer vectors for philox4x32-10.
    assert list(O.philox([0, 0, 0, 0], [0, 0])) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert list(O.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6,
                                                                    0x6D5451FD]
    assert list(O.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                         [0xA4093822, 0x299F31D0])) == [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_green_table_bit_exact(golden):
    gd = golden("test2")
    g, intg = O.green_table()
    assert np.array_equal(g, gd["g"])
    assert np.array_equal(intg, gd["intg"])
    # values quoted from the reference run
    assert intg[1] == 0.00021881202738647482 and intg[200] == 1.0 and g[0] == 0.010942197558909085


def test_weight_table_properties():
    g, intg = O.green_table()
    wx, wy = O.weight_table(intg)
    # corner landings carry no gradient; each side's normal part is positive outward
    assert wx[0] == wy[0] == wx[50] == wy[50] == 0.0
    assert (wy[1:50] < 0).all() and (wx[51:100] > 0).all() and (wy[101:150] > 0).all() and (wx[151:200] < 0).all()
    # sum_i pi_i W_i over the four sides cancels by symmetry up to the index shift
    pi = np.diff(intg)
    assert abs((pi * wx).sum()) < 0.2 and abs((pi * wy).sum()) < 0.2


@pytest.mark.parametrize("name", FIXTURES)
def test_parser_and_bounds(golden, name):
    gd = golden(name)
    b = O.layer_bounds(gd["rects"])
    assert np.array_equal(b, gd["bounds"])


@pytest.mark.parametrize("name", FIXTURES)
def test_defect_mode_queries_match_reference(golden, name):
    gd = golden(name)
    T = O.RefTree(gd["rects"], gd["bounds"])
    sq = np.array([T.biggest_square(x, y, True) for x, y in gd["pts"]])
    hit = np.array([T.point_hit(x, y) for x, y in gd["pts"]])
    assert np.array_equal(sq, gd["ref_sq"])
    assert np.array_equal(hit, gd["ref_hit"])
    for t, gref in zip(gd["gauss_targets"], gd["ref_gauss"]):
        assert np.array_equal(T.gauss_scale(gd["rects"][t], 1.5, True), gref)


@pytest.mark.parametrize("name", FIXTURES)
def test_complete_mode_consistent(golden, name):
    """Grid (brute-force predicate) == the reference tree with a complete DFS."""
    gd = golden(name)
    T = O.RefTree(gd["rects"], gd["bounds"])
    G = O.Grid(gd["rects"], gd["bounds"])
    pts = gd["pts"][:600]
    sq, hit = G.query_batch(pts)
    sq2 = np.array([T.biggest_square(x, y, False) for x, y in pts])
    assert np.array_equal(sq, sq2)
    # complete hits equal the reference's wherever the reference found one
    found = gd["ref_hit"][:600] >= 0
    assert np.array_equal(hit[found], gd["ref_hit"][:600][found])


@pytest.mark.parametrize("name", FIXTURES)
def test_reference_walks_replay(golden, name):
    """Each seeded reference walk replays identically on the restated tree."""
    gd = golden(name)
    T = O.RefTree(gd["rects"], gd["bounds"])
    G = O.Grid(gd["rects"], gd["bounds"])
    gauss = gd["ref_gauss"][list(gd["gauss_targets"]).index(gd["walk_target"])]
    r = gd["walk_r"]
    k = 0
    for w in range(len(gd["walk_end"])):
        e, u, h = O.walk_stream(G, T, True, gauss, gd["intg"], r[k:])
        assert (e, h) == (gd["walk_end"][w], gd["walk_hops"][w]), (name, w)
        k += u
    assert k == len(r)


def test_point_from_index_matches_reference_cases(golden):
    """Corner and shifted-index landings on a square of side 2 and 4 (the p+-1,
    p+-2 squares) and a rectangle."""
    sq = np.array([10.0, 20.0, 12.0, 22.0])
    pts = np.array([O.point_from_index(sq, i) for i in range(200)])
    assert tuple(pts[0]) == (9.0, 20.0)          # (int)(x0 - v/2): outside the corner
    assert tuple(pts[50]) == (12.0, 20.0)        # top-right corner
    assert tuple(pts[100]) == (12.0, 22.0)       # bottom-right corner
    assert tuple(pts[150]) == (10.0, 22.0)       # bottom-left corner
    assert (pts[1:50, 1] == 20.0).all() and (pts[51:100, 0] == 12.0).all()


@pytest.mark.skipif(not O.ref_available(), reason="compiled reference not present")
def test_live_reference_point_from_index():
    R = O.Ref(path=None, rects=np.array([[0.0, 0, 5, 5]]), bounds=np.array([-10.0, -10, 15, 15]))
    rng = np.random.default_rng(3)
    for _ in range(2000):
        s = rng.uniform(0.3, 60)
        c = rng.uniform(-100, 100, 2)
        sq = np.array([c[0] - s, c[1] - s, c[0] + s, c[1] + s])
        if rng.random() < 0.3:
            sq[2] += rng.uniform(0, 30)
        i = int(rng.integers(0, 200))
        assert np.array_equal(R.point_from_index(sq, i), O.point_from_index(sq, i))


def test_oracle_walks_deterministic():
    rects = np.array([[100.0, 100, 130, 120], [140.0, 100, 160, 140], [90.0, 130, 120, 170]])
    G = O.Grid(rects, np.array([0.0, 0, 300, 300]))
    cfg = G.walk_cfg(target=0, seed=7)
    a = G.walks(cfg, 0, 300)
    b = G.walks(cfg, 100, 100)
    for x, y in zip(a, b):
        assert np.array_equal(x[100:200], y)
    end, hops, b1, w = a
    assert ((end >= -2) & (end < 3)).all() and (hops >= 0).all() and (end >= 0).mean() > 0.5
    # the weight factor is defined by the first hop; walks without one carry 0
    assert (w[b1 < 0] == 0).all() and (w[end >= 0] != 0).mean() > 0.5


@pytest.mark.skipif(not O.ref_available(), reason="compiled reference not present")
def test_aligned_ties_oracle_pinned_to_reference():
    """Points beside an aligned array of rects see up to ~30 rects at one
    exact L-inf gap.  On them the restated reference tree (defect mode)
    equals the compiled reference, and the brute-force complete predicate
    equals the restated tree with a complete traversal: the oracle the
    device's tie handling is checked against is pinned on such points."""
    gx, gy = np.meshgrid(np.arange(30) * 3.0, np.arange(30) * 3.0)
    x0, y0 = 100.0 + gx.ravel(), 100.0 + gy.ravel()
    rects = np.stack([x0, y0, x0 + 1, y0 + 1], 1)
    bounds = np.array([0.0, 0.0, 300.0, 300.0])
    rng = np.random.default_rng(0x71E6)
    pts = np.concatenate([np.stack([rng.uniform(20, 99, 1500), rng.uniform(100, 190, 1500)], 1),
                          np.stack([rng.uniform(100, 190, 1500), rng.uniform(20, 99, 1500)], 1),
                          np.stack([rng.uniform(0, 300, 1000), rng.uniform(0, 300, 1000)], 1)])
    R = O.Ref(rects=rects, bounds=bounds)
    sq_r, hit_r = R.query_batch(pts)
    T = O.RefTree(rects, bounds)
    sq_d = np.array([T.biggest_square(x, y, True) for x, y in pts])
    hit_d = np.array([T.point_hit(x, y) for x, y in pts])
    assert np.array_equal(sq_d, sq_r) and np.array_equal(hit_d, hit_r)
    G = O.Grid(rects, bounds)
    sq_g, _ = G.query_batch(pts)
    sq_c = np.array([T.biggest_square(x, y, False) for x, y in pts])
    assert np.array_equal(sq_g, sq_c)
    # the points beside the array do tie: many rects at the minimum gap
    px, py = pts[:1500, :1], pts[:1500, 1:]
    g = np.maximum(np.maximum(rects[:, 0] - px, px - rects[:, 2]), np.maximum(rects[:, 1] - py, py - rects[:, 3]))
    assert ((g == g.min(1, keepdims=True)).sum(1) > 8).mean() > 0.3
