"""Bounded host waits (FRW_E_TIMEOUT).

A legitimate, finite run -- 1e8 walks on the 100-rect layout, tens of
milliseconds of device work -- is given a 1 ms bound on its host wait: the
call returns FRW_E_TIMEOUT while the walks keep running, writes nothing into
the caller's host arrays, and a later call on the same layout and stream
(queued behind the running walks) succeeds with the same results as a run
that was never interrupted.  Nothing here faults or hangs the device: the
kernel always finishes on its own.
"""
import ctypes as C

import numpy as np
import pytest

import frw

pytestmark = pytest.mark.gpu

BIG = 100_000_000


def _layout():
    return frw.Layout.from_rects(frw.generate_layout(0xF4A7 + 1, 100, 1000.0))


def test_walk_timeout_then_next_call_succeeds():
    with _layout() as L:
        with pytest.raises(frw.FrwError) as e:
            L.walk(0, BIG, seed=3, o=frw.capacitance_opts(1.0, timeout_ms=1.0))
        assert e.value.status == frw.E_TIMEOUT and "wait limit" in str(e.value)
        a = L.walk(0, 200_000, seed=5, o=frw.capacitance_opts(1.0))
        b = L.walk(0, 200_000, seed=5, o=frw.capacitance_opts(1.0, timeout_ms=60_000.0))
        assert a.walks == b.walks == 200_000
        assert np.array_equal(a.conductor, b.conductor) and np.array_equal(a.hits, b.hits)
        np.testing.assert_allclose(a.cap, b.cap, rtol=1e-12, atol=0)


def test_timed_out_trace_leaves_host_arrays_untouched():
    n = 1 << 22
    with _layout() as L:
        end = np.full(n, -77, dtype=np.int64)
        hops = np.full(n, -77, dtype=np.int32)
        o = frw.capacitance_opts(1.0, timeout_ms=1.0)
        # occupy the stream first so the trace's own walks cannot finish within 1 ms
        with pytest.raises(frw.FrwError):
            L.walk(0, BIG, seed=9, o=o)
        st = frw.lib().frw_walk_trace(L._h, 0, 0, n, 11, C.byref(o), end.ctypes.data_as(C.c_void_p),
                                      hops.ctypes.data_as(C.c_void_p), None, None, frw.MEM_HOST, None)
        assert st == frw.E_TIMEOUT
        L.walk(0, 1000, seed=1)  # waits (no limit) until everything queued before it has run
        assert (end == -77).all() and (hops == -77).all()
        want_end, want_hops, _, _ = L.walk_trace(0, 0, n, seed=11, o=frw.capacitance_opts(1.0))
        assert (want_hops > 0).all()


def test_process_wide_limit():
    with _layout() as L:
        frw.set_wait_limit(1.0)
        try:
            assert frw.wait_limit() == 1.0
            with pytest.raises(frw.FrwError) as e:
                L.walk(0, BIG, seed=4, o=frw.capacitance_opts(1.0))
            assert e.value.status == frw.E_TIMEOUT
            # a call's own bound replaces the process-wide one
            r = L.walk(0, 100_000, seed=4, o=frw.capacitance_opts(1.0, timeout_ms=60_000.0))
            assert r.walks == 100_000
        finally:
            frw.set_wait_limit(0.0)
        assert frw.wait_limit() == 0.0
        pts = np.random.default_rng(1).uniform(0, 1000, (1000, 2))
        sq, hit = L.query(pts)
        assert len(sq) == 1000
