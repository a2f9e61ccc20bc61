"""Batched walks: one graph-captured persistent launch over many layouts
equals running each job alone (same Philox streams), before and after the
autotuner picks the launch parameters."""
import numpy as np
import pytest

import frw

pytestmark = pytest.mark.gpu


def _jobs():
    rng = np.random.default_rng(9)
    counts = [100, 300, 1000, 2500, 60]
    layouts = [frw.Layout.from_rects(frw.generate_layout(100 + i, n, float(np.sqrt(n) * 100 + 200)))
               for i, n in enumerate(counts)]
    targets = [int(rng.integers(0, n)) for n in counts]
    walks = [int(20 * n) for n in counts]
    return layouts, targets, walks


@pytest.mark.parametrize("mode", ["capacitance", "reference"])
def test_batch_equals_individual_runs(mode):
    o = frw.capacitance_opts(1.0) if mode == "capacitance" else frw.opts()
    layouts, targets, walks = _jobs()
    B = frw.Batch(layouts, targets, walks, o)
    got = B.run(seed=31, capacity=4096)
    for j, (L, t, w) in enumerate(zip(layouts, targets, walks)):
        oj = frw.capacitance_opts(1.0, stream_id=j) if mode == "capacitance" else frw.opts(stream_id=j)
        ref = L.walk(t, w, seed=31, o=oj)
        g = got[j]
        assert (g.walks, g.escaped, g.aborted, g.hops_total) == (ref.walks, ref.escaped, ref.aborted, ref.hops_total)
        assert np.array_equal(g.conductor, ref.conductor) and np.array_equal(g.hits, ref.hits)
        np.testing.assert_allclose(g.cap, ref.cap, rtol=1e-12, atol=0)
        assert np.array_equal(g.gauss, ref.gauss)
    B.close()


def test_tuning_changes_speed_not_results():
    layouts, targets, walks = _jobs()
    o = frw.capacitance_opts(1.0)
    B = frw.Batch(layouts, targets, walks, o)
    before = B.run(seed=5, capacity=4096)
    t = B.tune(trial_walks=200_000)
    assert t.blocks_per_sm >= 1 and t.refill_min >= 1 and t.chunk >= 32 and t.ms > 0
    after = B.run(seed=5, capacity=4096)
    for a, b in zip(before, after):
        assert np.array_equal(a.hits, b.hits) and np.array_equal(a.conductor, b.conductor)
        np.testing.assert_allclose(a.cap, b.cap, rtol=1e-12, atol=0)
    B.set_tuning(1, 32, 1024)
    again = B.run(seed=5, capacity=4096)
    for a, b in zip(before, again):
        assert np.array_equal(a.hits, b.hits)
    B.close()


def test_single_job_batch():
    L = frw.Layout.from_rects(frw.generate_layout(3, 200, 1500.0))
    o = frw.capacitance_opts(1.0)
    B = frw.Batch([L], [7], [50_000], o)
    g = B.run(seed=2, capacity=4096)[0]
    ref = L.walk(7, 50_000, seed=2, o=o)
    assert np.array_equal(g.hits, ref.hits)
    B.close()
