"""3-D walk path on the device vs the CPU oracle (frwcpu3d.c): clearance
queries and walks bit-for-bit, the estimator's rows, and the physical
identities the capacitance row must satisfy."""
import numpy as np
import pytest

import frw
import oracle as O

pytestmark = pytest.mark.gpu


def _bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float64).view(np.uint64), np.asarray(b, np.float64).view(np.uint64))


def _layout(seed, n, domain, zdomain, zmin=5, zmax=50):
    return frw.generate_layout3(seed, n, domain, zdomain, 5, 50, zmin, zmax, 2)


def _hard_points(b, bounds, rng, n):
    """Uniform points plus points on box faces, edges and corners, inside
    boxes, half-way between neighbours (equal distances) and at the bounds."""
    lo, hi = bounds[:3], bounds[3:]
    pts = lo + rng.random((n, 3)) * (hi - lo)
    q = n // 6
    k = rng.integers(0, len(b), 5 * q)
    bl, bh = b[k, :3].astype(np.float64), b[k, 3:].astype(np.float64)
    pts[:q] = bl[:q] - rng.integers(0, 3, (q, 3))
    pts[q:2 * q] = bh[q:2 * q] + rng.integers(0, 3, (q, 3))
    pts[2 * q:3 * q] = (bl[2 * q:3 * q] + bh[2 * q:3 * q]) / 2
    j = rng.integers(0, len(b), q)
    pts[3 * q:4 * q] = (bh[3 * q:4 * q] + b[j, :3]) / 2  # between two boxes
    pts[4 * q:5 * q] = np.round(pts[4 * q:5 * q])
    pts[5 * q:5 * q + 10] = lo + 1e-9
    return pts


@pytest.mark.parametrize("n,cells", [(1, 0.0), (2, 0.0), (60, 0.5), (60, 64.0), (3000, 0.0), (3000, 2.0)])
def test_query3_bit_exact(n, cells):
    b = _layout(0xF4A7 + 40 + n, n, 400.0 + n, 200.0 + n / 10)
    B = O.Boxes3(b)
    rng = np.random.default_rng(n)
    pts = _hard_points(b, B.bounds, rng, 6000)
    with frw.Layout3.from_boxes(b, cells_per_box=cells) as L:
        assert np.array_equal(L.bounds, B.bounds)
        d, k = L.query(pts)
        info = L.info
    d_o, k_o = B.nearest(pts)
    bad = np.nonzero(~((d == d_o) & (k == k_o)))[0]
    assert len(bad) == 0, (len(bad), pts[bad[:3]], d[bad[:3]], d_o[bad[:3]], k[bad[:3]], k_o[bad[:3]])
    assert info.max_list >= 1 and info.list_entries >= info.grid[0] * info.grid[1] * info.grid[2]


@pytest.mark.parametrize("case", ["two_clusters", "wide_bounds"])
def test_query3_sparse_layouts_use_coarser_levels(case):
    """Layouts with large empty regions: cells far from every box defer to
    coarser grid levels (bounded build work); queries and walks still equal
    the oracle's everywhere, far points included."""
    a = frw.generate_layout3(0xF4A7 + 60, 1500, 400.0, 400.0, 5, 30, 5, 30, 2)
    if case == "two_clusters":
        c = frw.generate_layout3(0xF4A7 + 61, 1500, 400.0, 400.0, 5, 30, 5, 30, 2)
        b = np.vstack([a, c + np.float32(2600)])
        bounds = None
    else:
        b = a
        bounds = np.array([-5000.0, -5000.0, -5000.0, 5400.0, 5400.0, 5400.0])
    B = O.Boxes3(b, bounds, grid=True)
    rng = np.random.default_rng(17)
    pts = _hard_points(b, B.bounds, rng, 20000)
    with frw.Layout3.from_boxes(b, bounds) as L:
        info = L.info
        d, k = L.query(pts)
        e, h, bb, w = L.walk_trace(0, 0, 3000, 23)
    assert info.levels > 1 and info.deferred_cells > 0 and info.build_ms < 1000
    d_o, k_o = B.nearest(pts)
    assert np.array_equal(d, d_o) and np.array_equal(k, k_o)
    assert (d > 500).sum() > 100  # far points were exercised
    e_o, h_o, b_o, w_o = B.walks(B.cfg(target=0, seed=23), 0, 3000)
    assert np.array_equal(e, e_o) and np.array_equal(h, h_o) and np.array_equal(bb, b_o)
    assert _bits_equal(w, w_o)


def test_query3_touching_and_explicit_bounds():
    # two boxes sharing a face, a third far away; explicit bounds
    b = np.array([[0, 0, 0, 10, 10, 10], [10, 0, 0, 20, 10, 10], [100, 100, 100, 101, 103, 107]], np.float32)
    bounds = np.array([-50, -50, -50, 200, 200, 200.0])
    B = O.Boxes3(b, bounds)
    pts = np.array([[10, 5, 5], [15, 5, 5], [10, 20, 20], [50, 50, 50], [-49, -49, -49], [100.5, 101.5, 103.5]],
                   np.float64)
    with frw.Layout3.from_boxes(b, bounds) as L:
        d, k = L.query(pts)
    d_o, k_o = B.nearest(pts)
    assert _bits_equal(d, d_o) and np.array_equal(k, k_o)
    assert k[0] == 0 and d[0] == 0  # on the shared face: the lower index wins


@pytest.mark.parametrize("nsample,offset,first,stream", [(50, 1.0, 0, 0), (8, 2.5, 1 << 40, 3), (1, 1.0, 77, 1)])
def test_walk3_trace_bit_exact(nsample, offset, first, stream):
    b = _layout(0xF4A7 + 50, 300, 1000.0, 300.0)
    B = O.Boxes3(b)
    cfg = B.cfg(target=7, offset=offset, seed=0x5EED + nsample, stream=stream, nsample=nsample)
    e_o, h_o, b_o, w_o = B.walks(cfg, first, 4000)
    o = frw.opts3(gauss_offset=offset, nsample=nsample, stream_id=stream)
    with frw.Layout3.from_boxes(b) as L:
        e, h, b1, w = L.walk_trace(7, first, 4000, 0x5EED + nsample, o)
    assert np.array_equal(e, e_o)
    assert np.array_equal(h, h_o)
    assert np.array_equal(b1, b_o)
    assert _bits_equal(w, w_o)
    assert (e == 7).mean() > 0.5 and (e == frw.END_ABORTED).sum() == 0


def test_walk3_trace_max_table_and_launch_shapes():
    """The largest cube table (n = 100: 60,000 bins) and every launch shape
    give the same walks: results depend only on (seed, stream, walk index)."""
    b = _layout(0xF4A7 + 56, 250, 900.0, 300.0)
    B = O.Boxes3(b)
    e_o, h_o, b_o, w_o = B.walks(B.cfg(target=4, seed=31, nsample=100), 5, 3000)
    with frw.Layout3.from_boxes(b) as L:
        for bps, rm in ((0, 4), (1, 1), (2, 32), (4, 0)):
            o = frw.opts3(nsample=100, blocks_per_sm=bps, refill_min=rm)
            e, h, b1, w = L.walk_trace(4, 5, 3000, 31, o)
            assert np.array_equal(e, e_o) and np.array_equal(h, h_o) and np.array_equal(b1, b_o), (bps, rm)
            assert _bits_equal(w, w_o)
            r = L.walk(4, 3000, 31, frw.opts3(nsample=100, blocks_per_sm=bps, refill_min=rm, first_walk=5))
            ks, cnt = np.unique(e_o[e_o >= 0], return_counts=True)
            assert np.array_equal(r.conductor, ks) and np.array_equal(r.hits, cnt)
    assert b_o.max() >= 30_000  # bins of the later faces were drawn


def test_query3_device_memory():
    """frw3_query_batch on device arrays (torch tensors) equals the host call."""
    import torch

    b = _layout(0xF4A7 + 57, 800, 1200.0, 300.0)
    rng = np.random.default_rng(8)
    with frw.Layout3.from_boxes(b) as L:
        bd = L.bounds
        pts = bd[:3] + rng.random((50_000, 3)) * (bd[3:] - bd[:3])
        d_h, k_h = L.query(pts)
        pt = torch.as_tensor(pts, device="cuda")
        d = torch.empty(len(pts), dtype=torch.float64, device="cuda")
        k = torch.empty(len(pts), dtype=torch.int64, device="cuda")
        L.query_device(pt, d, k)
        torch.cuda.synchronize()
    assert _bits_equal(d.cpu().numpy(), d_h) and np.array_equal(k.cpu().numpy(), k_h)


def test_walk3_trace_hop_cap_and_shell():
    b = _layout(0xF4A7 + 51, 120, 500.0, 150.0)
    B = O.Boxes3(b)
    for shell, cap in ((0.5, 100000), (0.0, 3)):
        cfg = B.cfg(target=0, offset=1.0, shell=shell if shell > 0 else None, hop_cap=cap, seed=9)
        e_o, h_o, b_o, w_o = B.walks(cfg, 0, 3000)
        with frw.Layout3.from_boxes(b) as L:
            e, h, b1, w = L.walk_trace(0, 0, 3000, 9, frw.opts3(shell=shell, hop_cap=cap))
        assert np.array_equal(e, e_o) and np.array_equal(h, h_o) and np.array_equal(b1, b_o)
        assert _bits_equal(w, w_o)
    assert (e == frw.END_ABORTED).sum() > 0 and h.max() == 3


def test_walk3_rows_match_oracle():
    b = _layout(0xF4A7 + 52, 500, 1200.0, 300.0)
    B = O.Boxes3(b, grid=True)
    walks, seed = 60_000, 0xABCDEF
    e, h, b1, w = B.walks(B.cfg(target=11, offset=1.0, seed=seed), 0, walks)
    with frw.Layout3.from_boxes(b) as L:
        r = L.walk(11, walks, seed)
    ks, cnt = np.unique(e[e >= 0], return_counts=True)
    assert np.array_equal(r.conductor, ks) and np.array_equal(r.hits, cnt)
    sw = np.array([w[e == k].sum() for k in ks])
    sw2 = np.array([(w[e == k] ** 2).sum() for k in ks])
    np.testing.assert_allclose(r.sum_w, sw, rtol=1e-12, atol=1e-12 * np.abs(sw).max())
    np.testing.assert_allclose(r.sum_w2, sw2, rtol=1e-12)
    np.testing.assert_allclose(r.cap, sw / walks, rtol=1e-12, atol=1e-12 * np.abs(sw).max() / walks)
    assert r.escaped == (e == -1).sum() and r.aborted == 0 and r.hops_total == h.sum()
    assert r.fraction_other == pytest.approx(1 - (e == 11).mean())
    assert r.extra["shell"] == B.shell


def test_walk3_device_rows_match_host_rows():
    """frw3_walk_device accumulates into device arrays without a host sync;
    two calls over disjoint walk ranges equal one frw3_walk over their union."""
    import torch

    b = _layout(0xF4A7 + 58, 600, 1200.0, 300.0)
    n = len(b)
    with frw.Layout3.from_boxes(b) as L:
        ref = L.walk(9, 200_000, 0xD3)
        hits = torch.zeros(n, dtype=torch.int64, device="cuda")
        sw = torch.zeros(n, dtype=torch.float64, device="cuda")
        sw2 = torch.zeros(n, dtype=torch.float64, device="cuda")
        stats = torch.zeros(4, dtype=torch.int64, device="cuda")
        status = torch.zeros(1, dtype=torch.int32, device="cuda")
        L.walk_device(9, 120_000, 0xD3, frw.opts3(first_walk=0), hits, sw, sw2, stats, status)
        L.walk_device(9, 80_000, 0xD3, frw.opts3(first_walk=120_000), hits, sw, sw2, stats, status)
        L.walk_device(9, 0, 0xD3, None, hits, sw, sw2, stats, status)  # zero walks: nothing added
        torch.cuda.synchronize()
        with pytest.raises(frw.FrwError) as e:
            L.walk_device(n, 10, 1, None, hits, sw, sw2, stats, status)
        assert e.value.status == frw.E_ARG
    h = hits.cpu().numpy()
    k = np.nonzero(h)[0]
    assert np.array_equal(k, ref.conductor) and np.array_equal(h[k], ref.hits)
    np.testing.assert_allclose(sw.cpu().numpy()[k], ref.sum_w, rtol=1e-12, atol=1e-12 * np.abs(ref.sum_w).max())
    np.testing.assert_allclose(sw2.cpu().numpy()[k], ref.sum_w2, rtol=1e-12)
    st = stats.cpu().numpy()
    assert st[3] == 200_000 and st[0] == ref.escaped and st[1] == ref.aborted and st[2] == ref.hops_total
    assert int(status.cpu()[0]) == 0


def test_walk3_stratified_start_bit_exact_and_unbiased():
    """start_strata: walks equal the oracle's; C_00 agrees with unstratified
    runs within errors and its spread over seeds is no larger."""
    b = _layout(0xF4A7 + 59, 300, 900.0, 300.0)
    B = O.Boxes3(b)
    e_o, h_o, b_o, w_o = B.walks(B.cfg(target=2, seed=41, start_strata=64), 1 << 33, 3000)
    with frw.Layout3.from_boxes(b) as L:
        e, h, b1, w = L.walk_trace(2, 1 << 33, 3000, 41, frw.opts3(start_strata=64))
        assert np.array_equal(e, e_o) and np.array_equal(h, h_o) and np.array_equal(b1, b_o)
        assert _bits_equal(w, w_o)
        n, S = 1 << 16, 1024
        plain = np.array([L.walk(2, n, 100 + k).row(2)[1] for k in range(24)])
        strat = np.array([L.walk(2, n, 100 + k, frw.opts3(start_strata=S)).row(2)[1] for k in range(24)])
    assert abs(plain.mean() - strat.mean()) <= 4 * np.hypot(plain.std(ddof=1), strat.std(ddof=1)) / np.sqrt(24)
    assert strat.std(ddof=1) <= 1.25 * plain.std(ddof=1)


def test_walk3_batch_rows_equal_single_target_runs():
    """frw3_walk_batch: one launch over several targets (a duplicate
    included) gives each target the row of its own frw3_walk."""
    b = _layout(0xF4A7 + 62, 400, 1000.0, 300.0)
    targets = [3, 17, 250, 3, 399]
    o = frw.opts3(first_walk=1 << 20, stream_id=2)
    with frw.Layout3.from_boxes(b) as L:
        batch = L.walk_batch(targets, 40_000, 0xBA7C, o)
        singles = [L.walk(t, 40_000, 0xBA7C, o) for t in targets]
        empty = L.walk_batch([1, 2], 0, 5)
        with pytest.raises(frw.FrwError) as e:
            L.walk_batch([1, 400], 10, 5)
        assert e.value.status == frw.E_ARG
    for t, rb, rs in zip(targets, batch, singles):
        assert np.array_equal(rb.conductor, rs.conductor) and np.array_equal(rb.hits, rs.hits), t
        np.testing.assert_allclose(rb.sum_w, rs.sum_w, rtol=1e-12, atol=1e-12 * np.abs(rs.sum_w).max())
        np.testing.assert_allclose(rb.sum_w2, rs.sum_w2, rtol=1e-12)
        assert (rb.escaped, rb.aborted, rb.hops_total) == (rs.escaped, rs.aborted, rs.hops_total)
        assert rb.fraction_other == rs.fraction_other and np.array_equal(rb.gauss, rs.gauss)
        assert rb.row(t)[1] > 0
    assert all(r.walks == 0 and len(r.conductor) == 0 for r in empty)


def test_walk3_disjoint_ranges_add_up():
    b = _layout(0xF4A7 + 53, 200, 800.0, 250.0)
    with frw.Layout3.from_boxes(b) as L:
        full = L.walk(5, 30_000, 77)
        a = L.walk(5, 10_000, 77, frw.opts3(first_walk=0))
        c = L.walk(5, 20_000, 77, frw.opts3(first_walk=10_000))
    ha = dict(zip(a.conductor, a.hits))
    hc = dict(zip(c.conductor, c.hits))
    for k, n in zip(full.conductor, full.hits):
        assert ha.get(k, 0) + hc.get(k, 0) == n


def test_walk3_physical_identities():
    # weights of all walks sum to the charge of a constant potential (zero);
    # C_ij = C_ji (reciprocity) between two neighbours
    b = _layout(0xF4A7 + 54, 400, 900.0, 250.0)
    with frw.Layout3.from_boxes(b) as L:
        r = L.walk(0, 4_000_000, 1)
        s = L.walk(0, 2_000_000, 2)
        tot = r.cap.sum()
        e, h, b1, w = L.walk_trace(0, 0, 400_000, 3)
        assert abs(w.mean()) < 4.5 * w.std() / np.sqrt(len(w))
        # the target's most-hit neighbour, then walks from it
        others = [(n, k) for k, n in zip(r.conductor, r.hits) if k != 0]
        j = max(others)[1]
        rj = L.walk(int(j), 4_000_000, 4)
    c0j, se0j = r.row(j)[1:]
    cj0, sej0 = rj.row(0)[1:]
    assert c0j < 0 and cj0 < 0
    assert abs(c0j - cj0) < 4.5 * np.hypot(se0j, sej0)
    assert r.row(0)[1] > 0 and abs(s.row(0)[1] - r.row(0)[1]) < 4.5 * np.hypot(s.row(0)[2], r.row(0)[2])
    assert tot < r.row(0)[1]


def test_walk3_unit_cube_capacitance():
    # One cube of side a = 10 inside a grounded box 1000 units away on every
    # side.  The capacitance of an isolated cube is 0.6606781 x 4 pi eps0 a
    # (the known value of the unit cube); the enclosure (a cube of side L =
    # 2010, itself of capacitance ~0.6607 x 4 pi eps0 L) raises it by the
    # factor 1 / (1 - C/C_enclosure) ~ 1.005.  Checks the cube table, the
    # first-hop weights and the walk together, to 1%.
    eps0 = frw.PERMITTIVITY
    c_unit = 0.6606781 * 4 * np.pi * eps0
    a, R = 10.0, 1000.0
    box = np.array([[0, 0, 0, a, a, a]], np.float32)
    bounds = np.array([-R, -R, -R, a + R, a + R, a + R])
    with frw.Layout3.from_boxes(box, bounds) as L:
        r = L.walk(0, 50_000_000, 0xC0BE)
    c, se = r.row(0)[1:]
    c_enc = 0.6606781 * 4 * np.pi * eps0 * (a + 2 * R)
    isolated = c * (1 - c / c_enc)
    assert se < 0.003 * c
    assert abs(isolated / (c_unit * a) - 1) < 0.01, isolated / (c_unit * a)


def test_walk3_layout_from_file_extrudes_layers(tmp_path):
    a = frw.generate_layout(3, 40, 400.0)
    c = frw.generate_layout(4, 40, 400.0)
    p = str(tmp_path / "two.txt")
    with open(p, "w") as f:
        f.write("<< skipped >>\n")
        for r in a:
            f.write("rect %g %g %g %g\n" % tuple(r))
        f.write("<< m2 >>\n")
        for r in c:
            f.write("rect %g %g %g %g\n" % tuple(r))
        f.write("<< end >>\n")
    z0, z1 = [0.0, 20.0], [10.0, 30.0]
    with frw.Layout3.from_file(p, z0, z1) as L:
        boxes = L.boxes()
    first = O.parse_layout(p, 0)
    second = O.parse_layout(p, 1)
    exp = np.concatenate([
        np.column_stack([first[:, 0], first[:, 1], np.full(len(first), 0.0), first[:, 2], first[:, 3],
                         np.full(len(first), 10.0)]),
        np.column_stack([second[:, 0], second[:, 1], np.full(len(second), 20.0), second[:, 2], second[:, 3],
                         np.full(len(second), 30.0)])])
    assert np.array_equal(boxes.astype(np.float64), exp)
    with pytest.raises(frw.FrwError) as e:
        frw.Layout3.from_file(p, [0.0], [10.0])
    assert e.value.status == frw.E_ARG


def test_walk3_argument_errors():
    ok = np.array([[0, 0, 0, 10, 10, 10], [20, 0, 0, 30, 10, 10]], np.float32)
    bad = [
        np.array([[0, 0, 0, 10, 10, 10], [5, 5, 5, 15, 15, 15]], np.float32),  # overlap
        np.array([[0, 0, 0, 10, 10, 0]], np.float32),  # empty
        np.array([[0, 0, 0, 10, 10, np.nan]], np.float32),
        np.array([[0, 0, 0, 2 ** 25, 1, 1]], np.float32),
    ]
    for x in bad:
        with pytest.raises(frw.FrwError) as e:
            frw.Layout3.from_boxes(x)
        assert e.value.status == frw.E_ARG
    # one overlapping pair among thousands of disjoint boxes; touching faces are fine
    many = _layout(0xF4A7 + 55, 3000, 1500.0, 400.0)
    extra = many[1234].copy()
    extra[:3] += 1
    extra[3:] += 1
    with pytest.raises(frw.FrwError) as e:
        frw.Layout3.from_boxes(np.vstack([many, extra]))
    assert e.value.status == frw.E_ARG and "1234" in str(e.value)
    touch = many[77].copy()
    touch[0], touch[3] = many[77, 3], many[77, 3] + 1  # shares box 77's x1 face
    if not (np.maximum(many[:, :3], touch[:3]) < np.minimum(many[:, 3:], touch[3:])).all(1).any():
        frw.Layout3.from_boxes(np.vstack([many, touch])).close()
    with pytest.raises(frw.FrwError):
        frw.Layout3.from_boxes(ok, bounds=[1, 1, 1, 50, 50, 50])  # does not contain box 0
    with frw.Layout3.from_boxes(ok) as L:
        for kw in ({"gauss_offset": 0.0}, {"hop_cap": 0}, {"nsample": 0}, {"nsample": 101}):
            with pytest.raises(frw.FrwError) as e:
                L.walk(0, 10, 1, frw.opts3(**kw))
            assert e.value.status == frw.E_ARG
        with pytest.raises(frw.FrwError):
            L.walk(2, 10, 1)
        r = L.walk(0, 0, 1)
        assert r.walks == 0 and len(r.conductor) == 0


def test_walk3_full_size_workload():
    """The benchmark's 3-D workload: 10,000 boxes in [0,2000)^2 x [0,400),
    1e7 walks from box 0: every walk ends, none aborted, the row balances,
    and two disjoint halves of the walks add up to the full run's hits."""
    b = frw.generate_layout3(0xF4A7 + 6, 10_000, 2000.0, 400.0, 5, 50, 5, 20, 2)
    with frw.Layout3.from_boxes(b) as L:
        r = L.walk(0, 10_000_000, 0x3D)
        h1 = L.walk(0, 5_000_000, 0x3D)
        h2 = L.walk(0, 5_000_000, 0x3D, frw.opts3(first_walk=5_000_000))
    assert r.aborted == 0 and r.hits.sum() + r.escaped == 10_000_000
    c0, se0 = r.row(0)[1:]
    assert c0 > 0 and se0 < 0.01 * c0
    # the row sums to minus the charge at the bounds, which few walks reach
    # here: the conductors' charges cancel to within a per cent of the target's
    assert r.escaped < 1e-4 * r.walks
    assert abs(r.cap.sum()) < 0.01 * c0
    a = dict(zip(h1.conductor, h1.hits))
    for k, n in zip(h2.conductor, h2.hits):
        a[k] = a.get(k, 0) + n
    assert a == dict(zip(r.conductor, r.hits))


def test_walk3_million_boxes():
    """10^6 boxes in [0,20000)^2 x [0,2000): 2e5 clearance queries and 2e4
    walks from the middle of the walk index space equal the oracle's."""
    b = frw.generate_layout3(0xF4A7 + 8, 1_000_000, 20000.0, 2000.0, 5, 50, 5, 20, 2)
    B = O.Boxes3(b, grid=True, boxes_per_cell=2.0)
    rng = np.random.default_rng(3)
    pts = B.bounds[:3] + rng.random((200_000, 3)) * (B.bounds[3:] - B.bounds[:3])
    with frw.Layout3.from_boxes(b) as L:
        info = L.info
        d, k = L.query(pts)
        e, h, bb, w = L.walk_trace(0, 1 << 35, 20_000, 9)
    assert info.grid[0] * info.grid[1] * info.grid[2] > 8_000_000
    d_o, k_o = B.nearest(pts)
    assert np.array_equal(d, d_o) and np.array_equal(k, k_o)
    e_o, h_o, b_o, w_o = B.walks(B.cfg(target=0, seed=9), 1 << 35, 20_000)
    assert np.array_equal(e, e_o) and np.array_equal(h, h_o) and np.array_equal(bb, b_o)
    assert _bits_equal(w, w_o)


def test_cli_3d_mode(tmp_path):
    """lib/frw --3d: the layers of a reference layout file extruded to z
    ranges, the reference's two lines, the histogram and the JSON record of
    the 3-D run."""
    import json
    import os
    import subprocess

    a = frw.generate_layout(21, 40, 400.0)
    c = frw.generate_layout(22, 40, 400.0)
    p = str(tmp_path / "two.txt")
    with open(p, "w") as f:
        f.write("<< m1 >>\n")
        for r in a:
            f.write("rect %g %g %g %g\n" % tuple(r))
        f.write("<< m2 >>\n")
        for r in c:
            f.write("rect %g %g %g %g\n" % tuple(r))
        f.write("<< end >>\n")
    exe = os.path.join(frw.PKG, "lib", "frw")
    h = str(tmp_path / "hist3.txt")
    out = subprocess.run([exe, "-S", p, "-I", "50000", "-O", "3", "--3d", "0:8,12:20", "--seed", "5", "--hist", h,
                          "--json", "--cap"], capture_output=True, text=True, check=True).stdout.splitlines()
    assert out[1].startswith("[GPU] Ile sciezek trafi") and out[2].startswith("Czas wykonania:")
    rec = json.loads(out[-1])
    with frw.Layout3.from_file(p, [0.0, 12.0], [8.0, 20.0]) as L:
        r = L.walk(3, 50_000, 5)
    assert rec["dims"] == 3 and rec["boxes"] == 80 and rec["fraction_other"] == r.fraction_other
    assert [x["conductor"] for x in rec["rows"]] == list(r.conductor)
    assert open(h, encoding="utf-8").readline().strip() == "[GPU 3D]"
    bad = subprocess.run([exe, "-S", p, "--3d", "0:8"], capture_output=True, text=True)
    assert bad.returncode != 0 and "layers" in bad.stderr
