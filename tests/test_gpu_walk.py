"""Walks on the device vs the CPU oracle: every walk's end conductor, hop
count, first-hop bin and capacitance weight bit-identical on the same Philox
stream, and the estimator rows equal to the oracle's sums."""
import numpy as np
import pytest

import frw
import oracle as O

pytestmark = pytest.mark.gpu


def oracle_cfg(G, o: frw.Opts, target, seed):
    return G.walk_cfg(target=target, gauss_mode=o.gauss_mode, gauss_param=o.gauss_param,
                      start_mode=o.start_mode, exact_perimeter=bool(o.exact_perimeter), hop_cap=o.hop_cap,
                      seed=seed, stream=o.stream_id, start_grid=o.start_grid, start_strata=o.start_strata)


CASES = [
    ("test2", 10, dict()),  # reference start and surface
    ("test2", 10, dict(gauss_mode=frw.GAUSS_OFFSET, gauss_param=1.0, start_mode=frw.START_UNIFORM)),
    ("test", 3, dict(exact_perimeter=True)),
    ("test100", 7, dict(start_mode=frw.START_UNIFORM)),
    ("test1000", 500, dict()),
    ("test1000", 17, dict(gauss_mode=frw.GAUSS_OFFSET, gauss_param=1.0, start_mode=frw.START_UNIFORM,
                          stream_id=3)),
    ("test100", 5, dict(gauss_mode=frw.GAUSS_OFFSET, gauss_param=1.0, start_mode=frw.START_UNIFORM,
                        start_grid=4096)),
    ("test100", 7, dict(gauss_mode=frw.GAUSS_OFFSET, gauss_param=1.0, start_mode=frw.START_UNIFORM,
                        start_strata=64)),
    ("test2", 10, dict(start_strata=7)),  # Green-CDF start, stratified
    ("test100", 5, dict(gauss_mode=frw.GAUSS_OFFSET, gauss_param=1.0, start_mode=frw.START_UNIFORM,
                        start_grid=4096, start_strata=256)),
]


@pytest.mark.parametrize("name,target,kw", CASES)
def test_walk_records_bit_exact(golden, name, target, kw):
    gd = golden(name)
    o = frw.opts(**kw)
    G = O.Grid(gd["rects"], gd["bounds"])
    n = 3000 if len(gd["rects"]) < 1000 else 600
    with frw.Layout.from_rects(gd["rects"], gd["bounds"]) as L:
        end, hops, b1, w = L.walk_trace(target, 1000, n, seed=12345, o=o)
    end_o, hops_o, b1_o, w_o = G.walks(oracle_cfg(G, o, target, 12345), 1000, n)
    assert np.array_equal(end, end_o)
    assert np.array_equal(hops, hops_o)
    assert np.array_equal(b1, b1_o)
    assert np.array_equal(w, w_o)


def config1_layout():
    return frw.generate_layout(0xF4A7 + 1, 100, 1000.0)


def test_estimator_matches_oracle_sums_config1():
    """C1: 100 rects on [0,1000]^2, target 0, offset-1 surface, 1e5 walks."""
    rects = config1_layout()
    o = frw.capacitance_opts(1.0)
    G = O.Grid(rects.astype(np.float64))
    n = 100_000
    with frw.Layout.from_rects(rects) as L:
        res = L.walk(0, n, seed=99, o=o)
    end, hops, b1, w = G.walks(oracle_cfg(G, o, 0, 99), 0, n)
    assert res.walks == n and res.escaped == (end == -1).sum() and res.aborted == (end == -2).sum()
    assert res.hops_total == hops.sum()
    ks, counts = np.unique(end[end >= 0], return_counts=True)
    assert np.array_equal(res.conductor, ks) and np.array_equal(res.hits, counts)
    w = np.where(end >= 0, w, 0.0)  # the weight factor counts for the end conductor only
    for k, c, se in zip(res.conductor, res.cap, res.cap_se):
        wk = np.where(end == k, w, 0.0)
        assert c == pytest.approx(wk.mean(), rel=1e-12, abs=1e-30)
        assert se == pytest.approx(wk.std(ddof=1) / np.sqrt(n), rel=1e-6)
    # physics sanity: self-capacitance positive, couplings not significantly positive
    i0 = np.searchsorted(res.conductor, 0)
    assert res.cap[i0] > 0 and (np.delete(res.cap, i0) <= 3 * np.delete(res.cap_se, i0)).all()
    assert res.fraction_other == pytest.approx(1 - counts[ks == 0][0] / n)


@pytest.mark.parametrize("seed,n_rects,domain", [(0xF4A7 + 2, 10_000, 1e4), (0xF4A7 + 3, 10**6, 1e5)])
def test_estimator_matches_oracle_sums_c2_c3(seed, n_rects, domain):
    """C2 (10^4 rects) and C3 (10^6 rects): 2e5 walks taken from the middle of
    the walk index space; hits, hop total and every conductor's row equal the
    FP64 oracle's over the same walks."""
    rects = frw.generate_layout(seed, n_rects, domain)
    n, first = 200_000, 50_000_000
    o = frw.capacitance_opts(1.0, first_walk=first)
    G = O.Grid(rects.astype(np.float64))
    with frw.Layout.from_rects(rects) as L:
        res = L.walk(0, n, seed=2024, o=o)
    end, hops, b1, w = G.walks(oracle_cfg(G, o, 0, 2024), first, n)
    assert res.walks == n and res.hops_total == hops.sum() and res.escaped == (end == -1).sum()
    ks, counts = np.unique(end[end >= 0], return_counts=True)
    assert np.array_equal(res.conductor, ks) and np.array_equal(res.hits, counts)
    w = np.where(end >= 0, w, 0.0)
    s1 = np.array([w[end == k].sum() for k in ks])
    s2 = np.array([(w[end == k] ** 2).sum() for k in ks])
    assert np.allclose(res.sum_w, s1, rtol=1e-12, atol=1e-12 * np.abs(s1).max())
    assert np.allclose(res.sum_w2, s2, rtol=1e-12, atol=1e-12 * np.abs(s2).max())


def test_walks_independent_of_launch_shape():
    rects = config1_layout()
    o1 = frw.capacitance_opts(1.0)
    o2 = frw.capacitance_opts(1.0, blocks_per_sm=1, refill_min=8)
    with frw.Layout.from_rects(rects) as L:
        a = L.walk_trace(0, 0, 20_000, seed=5, o=o1)
        b = L.walk_trace(0, 0, 20_000, seed=5, o=o2)
        r1 = L.walk(0, 50_000, seed=5, o=o1)
        r2 = L.walk(0, 50_000, seed=5, o=o2)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert np.array_equal(r1.hits, r2.hits)
    np.testing.assert_allclose(r1.cap, r2.cap, rtol=1e-12)


def test_hop_cap_and_escapes():
    rects = config1_layout()
    o = frw.capacitance_opts(1.0, hop_cap=1)
    with frw.Layout.from_rects(rects) as L:
        end, hops, b1, w = L.walk_trace(0, 0, 5000, seed=1, o=o)
        res = L.walk(0, 5000, seed=1, o=o)
    assert hops.max() <= 1 and ((end == -2) | (end >= -1)).all()
    assert res.aborted == (end == -2).sum() > 0
    # a cap of one query ends every walk before its first hop: no weight anywhere
    assert (b1 == -1).all() and (w == 0).all()


def test_reference_mode_matches_reference_hit_distribution(golden):
    """test2 with the reference's own start and Gaussian surface: the device
    hit shares agree with the compiled reference's seeded walks within 3
    combined standard errors (the defect does not change test2's result)."""
    gd = golden("test2")
    t = int(gd["walk_target"])
    ref_end = gd["walk_end"]
    with frw.Layout.from_rects(gd["rects"], gd["bounds"]) as L:
        res = L.walk(t, 400_000, seed=2024, o=frw.opts())
    n_ref = len(ref_end)
    for k in np.unique(np.concatenate([ref_end[ref_end >= 0], res.conductor])):
        p_ref = (ref_end == k).mean()
        p_gpu = res.row(k)[0] / res.walks
        se = np.sqrt(p_ref * (1 - p_ref) / n_ref + p_gpu * (1 - p_gpu) / res.walks) + 1e-12
        assert abs(p_ref - p_gpu) <= 3 * se + 1.0 / n_ref, (k, p_ref, p_gpu)


def test_avg_path_len_entry_point(tmp_path):
    rects = config1_layout()
    p = str(tmp_path / "c1.txt")
    frw.write_layout(p, rects)
    h = str(tmp_path / "wyniki.txt")
    f = frw.get_avg_path_len_cuda(p, 20_000, 0, seed=3, hist_path=h)
    with frw.Layout.from_file(p) as L:
        r = L.walk(0, 20_000, seed=3, o=frw.opts())
    assert f == r.fraction_other and 0 < f < 1
    lines = open(h, encoding="utf-8").read().splitlines()
    assert lines[0] == "[GPU]" and len(lines) >= 2


def test_resume_from_checkpoint():
    """Two runs over disjoint walk ranges add up exactly to one run over both."""
    rects = config1_layout()
    with frw.Layout.from_rects(rects) as L:
        full = L.walk(0, 60_000, seed=8, o=frw.capacitance_opts(1.0))
        a = L.walk(0, 25_000, seed=8, o=frw.capacitance_opts(1.0))
        b = L.walk(0, 35_000, seed=8, o=frw.capacitance_opts(1.0, first_walk=25_000))
    ks = np.union1d(a.conductor, b.conductor)
    assert np.array_equal(ks, full.conductor)
    for k in ks:
        ha, _, _ = a.row(k)
        hb, _, _ = b.row(k)
        assert ha + hb == full.row(k)[0]
    ia, ib, i = (np.searchsorted(r.conductor, 0) for r in (a, b, full))
    assert a.sum_w[ia] + b.sum_w[ib] == pytest.approx(full.sum_w[i], rel=1e-12)
    assert a.hops_total + b.hops_total == full.hops_total


def test_cli_reference_flags(tmp_path):
    """The command-line front end with the reference's flags prints the
    reference's two lines, writes the histogram and a JSON record."""
    import json
    import os
    import subprocess

    rects = config1_layout()
    p = str(tmp_path / "c1.txt")
    frw.write_layout(p, rects)
    exe = os.path.join(frw.PKG, "lib", "frw")
    h = str(tmp_path / "hist.txt")
    out = subprocess.run([exe, "-S", p, "-I", "20000", "-O", "0", "-G", "-L", "0", "--seed", "3", "--hist", h,
                          "--json"], capture_output=True, text=True, check=True).stdout.splitlines()
    assert out[1].startswith("[GPU] Ile sciezek trafi") and out[2].startswith("Czas wykonania:")
    rec = json.loads(out[3])
    with frw.Layout.from_file(p) as L:
        r = L.walk(0, 20_000, seed=3, o=frw.opts())
    assert rec["fraction_other"] == r.fraction_other and rec["walks"] == 20_000
    assert open(h, encoding="utf-8").readline().strip() == "[GPU]"


def test_multilayer_file_and_layer_flag(tmp_path):
    a = frw.generate_layout(1, 30, 400.0)
    b = frw.generate_layout(2, 40, 500.0)
    p = str(tmp_path / "two.txt")
    with open(p, "w") as f:
        f.write("magic\n<< metal1 >>\n")
        for r in a:
            f.write("rect %d %d %d %d\n" % tuple(r))
        f.write("<< metal2 >>\n")
        for r in b:
            f.write("rect %d %d %d %d\n" % tuple(r))
        f.write("<< end >>\n")
    with frw.Layout.from_file(p, layer=1) as L:
        assert np.array_equal(L.rects(), b.astype(np.float64))
    with pytest.raises(frw.FrwError):
        frw.Layout.from_file(p, layer=2)


def test_stratified_start_unbiased_and_not_worse():
    """C1 with the start stratified into 1024 strata: the row agrees with an
    unstratified run within errors, and the spread of C_00 over independent
    seeds is no larger than without strata."""
    rects = config1_layout()
    n, S = 1 << 17, 1024
    o0 = frw.capacitance_opts(1.0)
    o1 = frw.capacitance_opts(1.0, start_strata=S)
    with frw.Layout.from_rects(rects) as L:
        plain = np.array([L.walk(0, n, seed=100 + k, o=o0).row(0)[1] for k in range(24)])
        strat = np.array([L.walk(0, n, seed=100 + k, o=o1).row(0)[1] for k in range(24)])
    assert abs(plain.mean() - strat.mean()) <= 4 * np.hypot(plain.std(ddof=1), strat.std(ddof=1)) / np.sqrt(24)
    assert strat.std(ddof=1) <= 1.25 * plain.std(ddof=1)


def test_start_grid_needs_uniform_start():
    with frw.Layout.from_rects(config1_layout()) as L:
        with pytest.raises(frw.FrwError, match="start_grid"):
            L.walk(0, 1000, seed=1, o=frw.opts(start_grid=64))


def test_full_size_c3_counts_and_signs():
    """C3 at its full size (10^6 rects, 1e8 walks): every walk is accounted
    for (hits + escapes + aborts), the self-capacitance is positive and no
    coupling is significantly positive; a second run over the next 1e8 walk
    indices agrees within the combined errors."""
    rects = frw.generate_layout(0xF4A7 + 3, 10**6, 1e5)
    n = 100_000_000
    with frw.Layout.from_rects(rects) as L:
        a = L.walk(0, n, seed=77, o=frw.capacitance_opts(1.0))
        b = L.walk(0, n, seed=77, o=frw.capacitance_opts(1.0, first_walk=n))
    for r in (a, b):
        assert r.walks == n and int(r.hits.sum()) + r.escaped + r.aborted == n
        i0 = np.searchsorted(r.conductor, 0)
        assert r.conductor[i0] == 0 and r.cap[i0] > 0
        others = np.delete(np.arange(len(r.conductor)), i0)
        assert (r.cap[others] <= 5 * r.cap_se[others]).all()
    ca, sa = a.row(0)[1:]
    cb, sb = b.row(0)[1:]
    assert abs(ca - cb) <= 5 * np.hypot(sa, sb)


def test_walk_argument_errors_and_empty_runs():
    """Bad targets and options are rejected with FRW_E_ARG and a message; a run
    of zero walks returns an empty row."""
    with frw.Layout.from_rects(config1_layout()) as L:
        for bad in (-1, L.n):
            with pytest.raises(frw.FrwError, match="target"):
                L.walk(bad, 1000, seed=1, o=frw.capacitance_opts(1.0))
        o = frw.capacitance_opts(1.0)
        o.struct_size = 8
        with pytest.raises(frw.FrwError, match="struct_size"):
            L.walk(0, 1000, seed=1, o=o)
        with pytest.raises(frw.FrwError, match="hop_cap"):
            L.walk(0, 1000, seed=1, o=frw.capacitance_opts(1.0, hop_cap=0))
        r = L.walk(0, 0, seed=1, o=frw.capacitance_opts(1.0))
        assert r.walks == 0 and len(r.conductor) == 0


@pytest.mark.parametrize("mode", ["reference", "capacitance", "capacitance-grid"])
def test_walks_with_and_without_records_agree(mode):
    """The walk kernel is compiled per launch configuration (per-walk records
    or none, start mode): the same walks traced with records and run without
    them give the same ends, hop totals and weight sums."""
    o = {"reference": frw.opts(), "capacitance": frw.capacitance_opts(1.0),
         "capacitance-grid": frw.capacitance_opts(1.0, start_grid=512)}[mode]
    n = 200_000
    with frw.Layout.from_rects(config1_layout()) as L:
        r = L.walk(0, n, seed=77, o=o, capacity=4096)
        end, hops, _, w = L.walk_trace(0, 0, n, 77, o)
    cond, cnt = np.unique(end[end >= 0], return_counts=True)
    assert np.array_equal(cond, r.conductor) and np.array_equal(cnt, r.hits)
    assert hops.sum() == r.hops_total and (end == -1).sum() == r.escaped and (end == -2).sum() == r.aborted
    sw = np.array([w[end == k].sum() for k in cond])
    np.testing.assert_allclose(r.sum_w, sw, rtol=1e-12, atol=1e-12 * max(np.abs(sw).max(), 1e-300))
    if mode == "reference":  # the Green-CDF start carries no weight
        assert not np.any(w) and not np.any(r.sum_w)


def test_walk_device_rows_match_frw_walk():
    """frw_walk_device accumulates the same rows into device arrays without a
    host sync: two runs over disjoint walk ranges equal one frw_walk run over
    their union (hits exactly, sums to 1e-12), and the stats add up."""
    import torch

    rects = config1_layout()
    n = 300_000
    dev = torch.device("cuda", 0)
    with frw.Layout.from_rects(rects) as L:
        ref = L.walk(0, 2 * n, seed=31, o=frw.capacitance_opts(1.0))
        hits = torch.zeros(L.n, dtype=torch.int64, device=dev)
        s1 = torch.zeros(L.n, dtype=torch.float64, device=dev)
        s2 = torch.zeros(L.n, dtype=torch.float64, device=dev)
        stats = torch.zeros(4, dtype=torch.int64, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        for first in (0, n):
            L.walk_device(0, n, 31, frw.capacitance_opts(1.0, first_walk=first), hits, s1, s2, stats, status)
        torch.cuda.synchronize()
    h, a, b, st = hits.cpu().numpy(), s1.cpu().numpy(), s2.cpu().numpy(), stats.cpu().numpy()
    assert int(status.item()) == 0
    assert st[3] == 2 * n and st[0] == ref.escaped and st[1] == ref.aborted and st[2] == ref.hops_total
    k = np.flatnonzero(h)
    assert np.array_equal(k, ref.conductor) and np.array_equal(h[k], ref.hits)
    np.testing.assert_allclose(a[k], ref.sum_w, rtol=1e-12, atol=1e-12 * np.abs(ref.sum_w).max())
    np.testing.assert_allclose(b[k], ref.sum_w2, rtol=1e-12, atol=1e-12 * np.abs(ref.sum_w2).max())
