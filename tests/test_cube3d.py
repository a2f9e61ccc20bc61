"""3-D path, CPU side: the cube Green's function table (oracle restatement
and the library's host table, both pinned bit-for-bit against the
reference's precompute_unit_cube_green, green/green.cpp:392-431), the
physics the table must satisfy, and the 3-D oracle's own consistency."""
import ctypes as C
import hashlib

import numpy as np
import pytest

import frw
import oracle as O

FULL = (1, 2, 3, 5, 8, 16)
NAMES = ("g", "dgdx", "dgdy", "dgdz", "intg")


def _digest(arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def _bits_equal(a, b):
    return np.array_equal(np.asarray(a).view(np.uint64), np.asarray(b).view(np.uint64))


@pytest.mark.parametrize("table", ["oracle", "library"])
def test_cube_table_matches_reference_golden(golden, table):
    gd = golden("cube_green")
    fn = O.cube_green_table if table == "oracle" else frw.cube_green_table
    for n in FULL:
        got = fn(n)
        for name, a in zip(NAMES, got):
            assert _bits_equal(a, gd[f"n{n}_{name}"]), (table, n, name)
    for n, d in zip(gd["digest_n"], gd["digest"]):
        assert _digest(fn(int(n))) == str(d), (table, n)


def test_cube_point_functions_match_reference(golden):
    gd = golden("cube_green")
    L = O.lib()
    for (a, eta, dz), g, dg in zip(gd["pt"], gd["pt_g"], gd["pt_dg"]):
        assert _bits_equal(L.oc3_green_cube(a, eta, dz), g)
        assert _bits_equal(frw.green_cube(a, eta, dz), g)
        d = np.zeros(3)
        L.oc3_deriv_green_cube(O._p(d), a, eta, dz)
        assert _bits_equal(d, dg)
        assert _bits_equal(frw.deriv_green_cube(a, eta, dz), dg)


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
def test_cube_table_matches_reference_library_n50():
    for a, b in zip(O.cube_green_table(50), O.ref_cube_green_table(50)):
        assert _bits_equal(a, b)


def _face_points(n):
    """Cube-surface points of the table's bins, (k, i, j) order: face k at
    k n^2 + i n + j with u = (i+1/2)/n, v = (j+1/2)/n on faces
    0 (u,v,0) 1 (1,u,v) 2 (1-v,1,u) 3 (1-u,1-v,1) 4 (0,1-u,1-v) 5 (v,0,1-u)."""
    u = (np.arange(n) + 0.5) / n
    U, V = np.meshgrid(u, u, indexing="ij")
    U, V = U.ravel(), V.ravel()
    one, zero = np.ones_like(U), np.zeros_like(U)
    faces = [(U, V, zero), (one, U, V), (1 - V, one, U), (1 - U, 1 - V, one), (zero, 1 - U, 1 - V),
             (V, zero, 1 - U)]
    return np.concatenate([np.stack(f, 1) for f in faces])


def _poisson_kernel(x, q, terms=40):
    """Landing density at cube-surface point q from interior point x, unit
    cube, from the eigenfunction series of the face q lies on (all m, n)."""
    out = np.zeros(len(q))
    m = np.arange(1, terms + 1)
    M, N = np.meshgrid(m, m, indexing="ij")
    gam = np.pi * np.sqrt(M ** 2 + N ** 2)
    for idx, p in enumerate(q):
        c = int(np.argmax([min(p[a], 1 - p[a]) < 1e-12 for a in range(3)]))
        a1, a2 = [a for a in range(3) if a != c]
        xi = x[c] if p[c] < 0.5 else 1 - x[c]
        ratio = np.exp(-gam * xi) * (1 - np.exp(-2 * gam * (1 - xi))) / (1 - np.exp(-2 * gam))
        s = (np.sin(M * np.pi * x[a1]) * np.sin(N * np.pi * x[a2]) * np.sin(M * np.pi * p[a1]) *
             np.sin(N * np.pi * p[a2]))
        out[idx] = 4 * np.sum(s * ratio)
    return out


def test_cube_table_is_the_poisson_kernel_and_its_gradient():
    # g = K(centre; q) and dg = -grad_x K(x; q) at the centre, by central
    # differences of an independent series: checks the face parametrisation
    # the walk lands with.
    n = 6
    g, dx, dy, dz, _ = O.cube_green_table(n)
    q = _face_points(n)
    c = np.full(3, 0.5)
    K = _poisson_kernel(c, q)
    np.testing.assert_allclose(g, K, rtol=1e-10, atol=1e-12)
    h = 1e-5
    dg = np.stack([dx, dy, dz], 1)
    for a in range(3):
        e = np.zeros(3)
        e[a] = h
        fd = (_poisson_kernel(c + e, q) - _poisson_kernel(c - e, q)) / (2 * h)
        np.testing.assert_allclose(dg[:, a], -fd, rtol=0, atol=1e-6 * np.abs(dg).max())


def test_cube_table_normalisation_and_symmetry():
    g, dx, dy, dz, intg = O.cube_green_table(50)
    assert intg[0] == 0.0 and abs(intg[-1] - 1.0) < 1e-15 and np.all(np.diff(intg) > 0)
    assert abs(g.sum() / 50 ** 2 - 1.0) < 1e-3  # harmonic measure integrates to one
    for d in (dx, dy, dz):
        assert abs(d.sum()) < 1e-9 * np.abs(d).sum()  # the field of a constant is zero
    w = O.cube_weight_table(50)
    assert np.all(np.isfinite(w))


@pytest.mark.parametrize("lists", [True, False])
def test_oracle_grid_nearest_equals_brute_force(lists):
    b = frw.generate_layout3(0xF4A7 + 20, 400, 1200.0, 400.0)
    B = O.Boxes3(b, grid=True, boxes_per_cell=1.0, lists=lists)
    rng = np.random.default_rng(5)
    lo, hi = B.bounds[:3], B.bounds[3:]
    pts = lo + rng.random((3000, 3)) * (hi - lo)
    # points on faces, edges and corners of boxes, and inside them
    k = rng.integers(0, len(b), 1000)
    pts[:1000] = b[k, :3] - rng.integers(0, 3, (1000, 3))
    pts[1000:1500] = (b[k[:500], :3] + b[k[:500], 3:]) / 2
    pts[1500:1510] = B.bounds[3:] + 5.0  # outside the grid: the ring search
    d1, k1 = B.nearest(pts, use_grid=False)
    d2, k2 = B.nearest(pts, use_grid=True)
    assert np.array_equal(d1, d2) and np.array_equal(k1, k2)
    assert np.all(d1[1000:1500] == 0)


def test_oracle_grid_lists_exact_on_a_sparse_layout():
    # one cluster inside bounds ten times wider: coarse cells far from every box
    b = frw.generate_layout3(0xF4A7 + 22, 1500, 400.0, 400.0, 5, 30, 5, 20, 2)
    bounds = np.array([-5000.0] * 3 + [5400.0] * 3)
    G = O.Boxes3(b, bounds, grid=True)
    rng = np.random.default_rng(22)
    pts = bounds[:3] + rng.random((8000, 3)) * (bounds[3:] - bounds[:3])
    pts[:2000] = rng.random((2000, 3)) * 420 - 10  # in and around the cluster
    d1, k1 = G.nearest(pts, use_grid=False)
    d2, k2 = G.nearest(pts, use_grid=True)
    assert np.array_equal(d1, d2) and np.array_equal(k1, k2)


def test_oracle_walks_grid_equals_brute_force_and_weights_balance():
    b = frw.generate_layout3(0xF4A7 + 21, 150, 600.0, 200.0)
    G = O.Boxes3(b, grid=True)
    Bf = O.Boxes3(b, grid=False)
    cfg = G.cfg(target=3, offset=1.0, seed=11, stream=2)
    e1, h1, b1, w1 = G.walks(cfg, 1 << 33, 3000)
    e2, h2, b2, w2 = Bf.walks(cfg, 1 << 33, 3000)
    for x, y in ((e1, e2), (h1, h2), (b1, b2)):
        assert np.array_equal(x, y)
    assert _bits_equal(w1, w2)
    # the weights of all walks estimate the charge of a constant potential: 0
    e, h, bb, w = G.walks(G.cfg(target=3, offset=1.0, seed=12), 0, 20000)
    assert abs(w.mean()) < 4.5 * w.std() / np.sqrt(len(w))
    assert (e == 3).mean() > 0.5 and np.all(bb[h > 1] >= 0) and np.all(bb[h == 1] == -1)
    # charge on the target is positive; on the well-sampled neighbours and at
    # the bounds (escapes) it is negative
    assert w[e == 3].sum() > 0 and w[e == -1].sum() < 0
    ks, cnt = np.unique(e[e >= 0], return_counts=True)
    for k in ks[(ks != 3) & (cnt >= 200)]:
        assert w[e == k].sum() < 0, k


def test_generator3_deterministic_sizes_and_gap():
    a = frw.generate_layout3(0xF4A7 + 30, 300, 1000.0, 300.0, 5, 50, 4, 20, 2)
    b = frw.generate_layout3(0xF4A7 + 30, 300, 1000.0, 300.0, 5, 50, 4, 20, 2)
    assert np.array_equal(a, b) and np.array_equal(a, np.round(a))
    e = a[:, 3:] - a[:, :3]
    assert e[:, :2].min() >= 5 and e[:, :2].max() <= 50 and e[:, 2].min() >= 4 and e[:, 2].max() <= 20
    assert a[:, :2].min() >= 0 and a[:, 3:5].max() <= 1000 and a[:, 5].max() <= 300
    lo, hi = a[:, :3].astype(np.float64), a[:, 3:].astype(np.float64)
    gap = np.max(np.maximum(lo[None] - hi[:, None], lo[:, None] - hi[None]), axis=2)
    np.fill_diagonal(gap, np.inf)
    assert gap.min() >= 2


def test_cube_api_argument_errors_without_device():
    with pytest.raises(frw.FrwError) as e:
        frw.cube_green_table(0)
    assert e.value.status == frw.E_ARG
    with pytest.raises(frw.FrwError) as e:
        frw.green_cube(1.0, 0.5, 1.5)  # eta and dzeta on different faces
    assert e.value.status == frw.E_ARG
    with pytest.raises(frw.FrwError) as e:
        frw.Layout3.from_file("/nonexistent/layout", [0.0], [1.0])
    assert e.value.status == frw.E_IO


def test_opts3_builds_without_a_device():
    # frw3_opts_default is host-only; the Python mirror must fill every field
    o = frw.opts3(gauss_offset=2.0, nsample=8, start_strata=4)
    assert o.struct_size == C.sizeof(frw.Opts3) and o.gauss_offset == 2.0 and o.nsample == 8
