"""The large configurations under test, not only in the benchmark.

* Learned control variate on the 10^6-rect layout (0xF4A7+3 on [0,1e5]^2,
  grid start Q = 16384): each estimator run to 0.1% relative standard error
  of C_00 (pilot batch, then the walks the pilot says are needed); the two
  estimates agree within 3 combined standard errors, the variance reduction
  exceeds 3 and the control-variate run needs at least 3x less wall time with
  its training and exact mean included.
* Batched walks over 256 layouts of 100..1e5 rects (log-uniform, 1e8 walks in
  proportion to the rect counts, one graph-captured launch): eight jobs --
  the smallest, the largest and six others -- equal their solo runs.
"""
import time

import numpy as np
import pytest

import frw

pytestmark = pytest.mark.gpu


def _plain_to(L, o, target, rel):
    pilot = L.walk(target, 2_000_000, seed=11, o=o)
    c, se = pilot.row(target)[1:]
    need = int(pilot.walks * (se / abs(c) / rel) ** 2 * 1.05) + 1
    main = L.walk(target, need, seed=12, o=o)
    n = pilot.walks + main.walks
    i0, i1 = (np.searchsorted(r.conductor, target) for r in (pilot, main))
    s1 = pilot.sum_w[i0] + main.sum_w[i1]
    s2 = pilot.sum_w2[i0] + main.sum_w2[i1]
    mean = s1 / n
    return mean, np.sqrt(max(s2 / n - mean * mean, 0.0) / (n - 1))


def _cv_to(L, o, target, rel):
    cv = frw.ControlVariate(L, target, o, frw.cv_opts(train_walks=1_000_000, epochs=4))
    pilot = cv.walk(1_000_000, seed=21)
    need = int(pilot.walks * (pilot.cv_se / abs(pilot.cv) / rel) ** 2 * 1.05) + 1
    main = cv.walk(max(need, 2), seed=22)
    n = pilot.walks + main.walks
    c = (pilot.cv * pilot.walks + main.cv * main.walks) / n
    se = np.sqrt((pilot.cv_se * pilot.walks) ** 2 + (main.cv_se * main.walks) ** 2) / n
    ratio = main.variance_ratio
    cv.close()
    return c, se, ratio


def test_control_variate_on_1e6_rects_reaches_0p1pct_3x_faster():
    import torch

    rel = 1e-3
    rects = frw.generate_layout(0xF4A7 + 3, 1_000_000, 1e5)
    with frw.Layout.from_rects(rects) as L:
        o = frw.capacitance_opts(1.0, start_grid=16384)
        L.walk(0, 1_000_000, seed=1, o=o)  # warm-up: module loading, memory pool
        frw.ControlVariate(L, 0, o, frw.cv_opts(train_walks=100_000, epochs=1)).close()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cp, sp = _plain_to(L, o, 0, rel)
        t_plain = time.perf_counter() - t0
        t0 = time.perf_counter()
        cc, sc, ratio = _cv_to(L, o, 0, rel)
        t_cv = time.perf_counter() - t0
    assert sp / abs(cp) <= 1.1 * rel and sc / abs(cc) <= 1.1 * rel
    assert abs(cp - cc) <= 3.0 * np.hypot(sp, sc), (cp, sp, cc, sc)
    assert ratio > 3.0, ratio
    assert t_plain / t_cv >= 3.0, (t_plain, t_cv)


def test_256_layout_batch_jobs_equal_solo_runs():
    rng = np.random.default_rng(0x0C4)
    counts = np.exp(rng.uniform(np.log(100), np.log(100_000), 256)).astype(int)
    layouts = [frw.Layout.from_rects(frw.generate_layout(0x0C4 + i, int(n), float(np.sqrt(n) * 100.0)))
               for i, n in enumerate(counts)]
    walks = np.maximum(1, np.round(counts / counts.sum() * 100_000_000)).astype(np.uint64)
    o = frw.capacitance_opts(1.0)
    B = frw.Batch(layouts, np.zeros(256, dtype=np.int64), walks, o)
    got = B.run(seed=77, capacity=4096)
    picks = sorted({int(np.argmin(counts)), int(np.argmax(counts))} | set(rng.choice(256, 6, replace=False).tolist()))
    for j in picks:
        ref = layouts[j].walk(0, int(walks[j]), seed=77, o=frw.capacitance_opts(1.0, stream_id=j), capacity=4096)
        g = got[j]
        assert (g.walks, g.escaped, g.aborted, g.hops_total) == (ref.walks, ref.escaped, ref.aborted, ref.hops_total)
        assert np.array_equal(g.conductor, ref.conductor) and np.array_equal(g.hits, ref.hits)
        np.testing.assert_allclose(g.cap, ref.cap, rtol=1e-12, atol=0)
    B.close()
    for L in layouts:
        L.close()
