"""The learned control variate on the device: features equal the oracle's
bit-for-bit, the BF16 tensor-core forward and gradients agree with an FP64
reference, the estimate is unbiased against an independent plain run, and
the trained network reduces the variance."""
import numpy as np
import pytest

import frw
import mlp_ref as M
import oracle as O

pytestmark = pytest.mark.gpu


def config1():
    return frw.generate_layout(0xF4A7 + 1, 100, 1000.0)


def test_features_match_oracle(golden):
    gd = golden("test2")
    rects, t = gd["rects"], int(gd["walk_target"])
    rng = np.random.default_rng(2)
    r = rects[t]
    n = 4000
    rec = np.zeros((n, 4))
    rec[:, 0] = rng.uniform(r[0] - 40, r[2] + 40, n)
    rec[:, 1] = rng.uniform(r[1] - 40, r[3] + 40, n)
    rec[: n // 4, :2] = np.round(rec[: n // 4, :2])
    rec[:, 2] = rng.choice([0.0, 1.0, 2.0, 4.0, 7.5], n)
    with frw.Layout.from_rects(rects, gd["bounds"]) as L:
        got = L.cv_features(t, rec)
    want = O.cv_features(rects, t, rec)
    assert np.array_equal(got, want)


def _random_params(seed):
    rng = np.random.default_rng(seed)
    p = rng.normal(0, 0.3, M.NPARAM).astype(np.float32)
    return p


KERNELS = [pytest.param(frw.MLP_TCGEN05, id="tcgen05"), pytest.param(frw.MLP_MMA_SYNC, id="mma_sync")]


@pytest.fixture
def mlp_kernels(request):
    frw.set_mlp_kernels(request.param)
    yield request.param
    frw.set_mlp_kernels(frw.MLP_TCGEN05)


@pytest.mark.parametrize("mlp_kernels", KERNELS, indirect=True)
def test_mlp_forward_matches_fp64(mlp_kernels):
    p = _random_params(1)
    x = np.random.default_rng(3).uniform(-3, 3, (5000, 16)).astype(np.float32)
    got = frw.mlp_forward(p, x)
    want, _ = M.forward(p, x)
    err = np.abs(got - want)
    assert err.max() < 2e-2 * (1 + np.abs(want).max())
    assert np.corrcoef(got, want)[0, 1] > 0.9999


@pytest.mark.parametrize("mlp_kernels", KERNELS, indirect=True)
def test_mlp_gradients_match_fp64(mlp_kernels):
    p = _random_params(4)
    rng = np.random.default_rng(5)
    n = 4096 + 37  # a ragged last chunk
    x = rng.uniform(-3, 3, (n, 16)).astype(np.float32)
    y = (rng.random(n) < 0.4).astype(np.float32)
    wt = rng.exponential(1.0, n).astype(np.float32)
    wt[:50] = 0
    inv = 1.0 / float(wt.sum())
    loss, g = frw.mlp_grad(p, x, y, wt, inv)
    loss_r, g_r = M.loss_grad(p, x.astype(np.float64), y, wt, inv)
    assert loss == pytest.approx(loss_r, rel=1e-2)
    cos = float(g @ g_r / np.linalg.norm(g) / np.linalg.norm(g_r))
    assert cos > 0.999
    assert np.linalg.norm(g - g_r) / np.linalg.norm(g_r) < 3e-2
    # every parameter block gets its gradient
    for a, b in [(M.O_W1, M.O_B1), (M.O_B1, M.O_W2), (M.O_W2, M.O_B2), (M.O_B2, M.O_W3), (M.O_W3, M.O_B3)]:
        ga, gb = g[a:b], g_r[a:b]
        assert np.linalg.norm(ga - gb) <= 5e-2 * np.linalg.norm(gb) + 1e-7
    assert g[M.O_B3] == pytest.approx(g_r[M.O_B3], rel=1e-2)


def test_tcgen05_and_mma_sync_kernels_agree():
    # same BF16 operands and FP32 accumulation: only the order of the FP32
    # sums (and so an occasional BF16 rounding of an activation) differs
    p = _random_params(7)
    rng = np.random.default_rng(8)
    n = 3 * 128 + 5
    x = rng.uniform(-3, 3, (n, 16)).astype(np.float32)
    y = (rng.random(n) < 0.4).astype(np.float32)
    wt = rng.exponential(1.0, n).astype(np.float32)
    inv = 1.0 / float(wt.sum())
    out = {}
    try:
        for k in (frw.MLP_TCGEN05, frw.MLP_MMA_SYNC):
            frw.set_mlp_kernels(k)
            assert frw.mlp_kernels() == k
            out[k] = (frw.mlp_forward(p, x), *frw.mlp_grad(p, x, y, wt, inv))
    finally:
        frw.set_mlp_kernels(frw.MLP_TCGEN05)
    (f_a, l_a, g_a), (f_b, l_b, g_b) = out[frw.MLP_TCGEN05], out[frw.MLP_MMA_SYNC]
    assert np.abs(f_a - f_b).max() <= 1e-2 * (1 + np.abs(f_b).max())
    assert l_a == pytest.approx(l_b, rel=1e-3)
    assert np.linalg.norm(g_a - g_b) <= 2e-2 * np.linalg.norm(g_b)


def test_cv_unbiased_and_reduces_variance():
    rects = config1()
    o = frw.capacitance_opts(1.0, start_grid=4096)
    with frw.Layout.from_rects(rects) as L:
        cv = frw.ControlVariate(L, 0, o, frw.cv_opts(train_walks=200_000, epochs=6, batch=4096, lr=3e-3))
        info = cv.info
        r = cv.walk(2_000_000, seed=99)
        ref = L.walk(0, 20_000_000, seed=12345, o=o)  # independent plain run
        cv.close()
    c_ref, se_ref = ref.row(0)[1:]
    assert r.plain == pytest.approx(c_ref, abs=4 * np.hypot(r.plain_se, se_ref))
    assert abs(r.cv - c_ref) <= 3.5 * np.hypot(r.cv_se, se_ref), (r.cv, c_ref, r.cv_se, se_ref)
    assert r.variance_ratio > 1.5, r.variance_ratio
    assert info.quad_points == 4096 * 200 and info.train_loss > 0


def test_cv_walk_fused_equals_records_path():
    """The walk kernel's own control-variate sums give the estimates of the
    per-walk records summed by a second kernel (same walks, sums in another
    order)."""
    o = frw.capacitance_opts(1.0, start_grid=1024)
    with frw.Layout.from_rects(config1()) as L:
        cv = frw.ControlVariate(L, 0, o, frw.cv_opts(train_walks=200_000))
        assert frw.cv_walk_mode() == frw.CV_WALK_FUSED
        a = cv.walk(3_000_000, seed=5)
        try:
            frw.set_cv_walk_mode(frw.CV_WALK_RECORDS)
            b = cv.walk(3_000_000, seed=5)
        finally:
            frw.set_cv_walk_mode(frw.CV_WALK_FUSED)
        cv.close()
    for k in ("plain", "plain_se", "cv", "cv_se", "variance_ratio"):
        assert getattr(a, k) == pytest.approx(getattr(b, k), rel=1e-10), k
    assert a.walks == b.walks == 3_000_000
    with pytest.raises(frw.FrwError):
        frw.set_cv_walk_mode(7)


def test_cv_mean_term_is_the_mean_of_f():
    """Unbiasedness of the re-added term: over many walks, mean(f) = E[f]."""
    rects = config1()
    o = frw.capacitance_opts(1.0, start_grid=1024)
    with frw.Layout.from_rects(rects) as L:
        cv = frw.ControlVariate(L, 0, o, frw.cv_opts(train_walks=100_000, epochs=3, batch=4096, lr=3e-3))
        mu = cv.info.mean_term
        r = cv.walk(8_000_000, seed=7)
        cv.close()
    # mean(f) = plain - (cv - mu); its standard error is bounded by se_plain + se_cv
    mean_f = r.plain - (r.cv - mu)
    assert abs(mean_f - mu) <= 4 * (r.plain_se + r.cv_se)


def _perimeter_point(G, u):
    """Uniform point on the Gaussian perimeter, clockwise from the top-left
    corner (same IEEE double operations as the device)."""
    w, h = G[2] - G[0], G[3] - G[1]
    s = u * (2.0 * w + 2.0 * h)
    if s < w:
        return 0, G[0] + s, G[1]
    if s < w + h:
        return 1, G[2], G[1] + (s - w)
    if s < 2.0 * w + h:
        return 2, G[2] - ((s - w) - h), G[3]
    return 3, G[0], G[3] - ((s - 2.0 * w) - h)


def test_cv_exact_mean_equals_enumeration():
    """E[f] from the fused quadrature kernel equals the sum over every (grid
    start, first-hop bin) pair built on the host from the oracle's squares and
    weights, with phi from the device forward of the same network: the terms
    are identical, only the summation order differs."""
    rects = config1()
    Q = 256
    o = frw.capacitance_opts(1.0, start_grid=Q)
    with frw.Layout.from_rects(rects) as L:
        cv = frw.ControlVariate(L, 0, o, frw.cv_opts(train_walks=50_000, epochs=2, batch=4096, lr=3e-3))
        mu = cv.info.mean_term
        params = cv.params()
        cv.close()
        bounds = L.bounds
        G = O.Grid(rects.astype(np.float64), bounds)
        gs = G.gauss_surface(G.walk_cfg(target=0, gauss_mode=O.GAUSS_OFFSET, gauss_param=1.0))
        _, intg = O.green_table()
        wx, wy = O.weight_table(intg)
        pi = (np.ceil(np.ldexp(intg[1:], 32)) - np.ceil(np.ldexp(intg[:-1], 32))) / 2.0 ** 32
        perim = 2.0 * (gs[2] - gs[0]) + 2.0 * (gs[3] - gs[1])
        eps = o.permittivity
        recs, wts = [], []
        for q in range(Q):
            side, x, y = _perimeter_point(gs, (q + 0.5) / Q)
            if not (x > bounds[0] and y > bounds[1] and x < bounds[2] and y < bounds[3]):
                continue
            if G.point_hit(x, y) >= 0:
                continue
            sq = G.biggest_square(x, y)
            a0 = sq[2] - sq[0]
            nx = 1.0 if side == 1 else (-1.0 if side == 3 else 0.0)
            ny = 1.0 if side == 2 else (-1.0 if side == 0 else 0.0)
            for i in range(O.NSAMPLE):
                x1, y1 = O.point_from_index(sq, i)
                c = ((-eps * perim) * (wx[i] * nx + wy[i] * ny)) / a0
                recs.append((x1, y1, a0, 0.0))
                wts.append(c * pi[i] / Q)
        assert len(recs) > 100 * O.NSAMPLE
        phi = frw.mlp_forward(params, L.cv_features(0, np.array(recs)))
    want = float(np.dot(np.array(wts), phi.astype(np.float64)))
    assert mu == pytest.approx(want, rel=1e-11, abs=1e-11 * np.abs(np.array(wts)).sum())
