"""CPU-side checks of the C-ABI library: it loads, exports every symbol that
include/frw.h declares, its host-only helpers agree with the reference
(Green table) and it refuses compute without an sm_100 device (no CPU
fallback)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import frw
import oracle as O


def _have_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def test_library_exports_every_header_symbol():
    syms = frw.header_symbols()
    assert len(syms) >= 18
    L = ctypes.CDLL(frw.LIB_PATH)
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", frw.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert set(syms) <= exported


def test_version_and_opts_default():
    assert "sm_100a" in frw.version()
    o = frw.opts()
    assert o.struct_size == ctypes.sizeof(frw.Opts) and o.gauss_param == 1.5 and o.hop_cap == 100000


def test_green_table_matches_reference(golden):
    g, intg = frw.green_table()
    gd = golden("test2")
    assert np.array_equal(g, gd["g"]) and np.array_equal(intg, gd["intg"])


def test_weight_table_matches_oracle():
    # the product's weights are only visible on the device; the host table of
    # the oracle is the same mathematics -- check the CDF the two share
    _, intg = frw.green_table()
    _, intg_o = O.green_table()
    assert np.array_equal(intg, intg_o)


def test_generator_deterministic_and_gap():
    a = frw.generate_layout(0xF4A7 + 1, 100, 1000.0)
    b = frw.generate_layout(0xF4A7 + 1, 100, 1000.0)
    assert np.array_equal(a, b)
    w = a[:, 2] - a[:, 0]
    h = a[:, 3] - a[:, 1]
    assert w.min() >= 5 and w.max() <= 50 and h.min() >= 5 and h.max() <= 50
    assert a.min() >= 0 and a.max() <= 1000 and np.array_equal(a, np.round(a))
    # pairwise L-infinity gap >= 2
    x0, y0, x1, y1 = (a[:, k].astype(np.float64) for k in range(4))
    gap = np.maximum(np.maximum(x0[None] - x1[:, None], x0[:, None] - x1[None]),
                     np.maximum(y0[None] - y1[:, None], y0[:, None] - y1[None]))
    np.fill_diagonal(gap, np.inf)
    assert gap.min() >= 2


def test_layout_writer_roundtrip(tmp_path):
    a = frw.generate_layout(7, 50, 500.0)
    p = str(tmp_path / "l.txt")
    frw.write_layout(p, a, "metal1")
    back = O.parse_layout(p)
    assert np.array_equal(back, a.astype(np.float64))


@pytest.mark.skipif(_have_gpu(), reason="checks the no-GPU refusal")
def test_compute_refused_without_device():
    with pytest.raises(frw.FrwError) as e:
        frw.device_check(0)
    assert e.value.status == frw.E_DEVICE
    with pytest.raises(frw.FrwError) as e:
        frw.Layout.from_rects(np.array([[0, 0, 5, 5]], dtype=np.float32))
    assert e.value.status == frw.E_DEVICE


def test_bad_layout_arguments_rejected_before_device():
    # argument errors are reported without touching a device
    with pytest.raises(frw.FrwError) as e:
        frw.Layout.from_file("/nonexistent/layout")
    assert e.value.status == frw.E_IO
    import ctypes as C

    one = np.array([[0, 0, 5, 5]], dtype=np.float32)
    h = C.c_void_p()
    ptr = one.ctypes.data_as(C.POINTER(C.c_float))
    # empty layout; more than 2^26 - 1 rects (refused before the rects are read)
    assert frw.lib().frw_layout_create(ptr, 0, None, 0, None, C.byref(h)) == frw.E_ARG
    assert frw.lib().frw_layout_create(ptr, 1 << 26, None, 0, None, C.byref(h)) == frw.E_ARG
    assert "2^26" in frw.lib().frw_last_error().decode()
    # bounds that are not a box
    bad = np.array([10.0, 0.0, 0.0, 10.0])
    assert frw.lib().frw_layout_create(ptr, 1, bad.ctypes.data_as(C.POINTER(C.c_double)), 0, None,
                                       C.byref(h)) == frw.E_ARG
    assert "bounds invalid" in frw.lib().frw_last_error().decode()
    assert not h.value


@pytest.mark.parametrize("seed,n,domain", [(0xF4A7 + 1, 100, 1000.0), (0xF4A7 + 2, 10_000, 1e4),
                                           (0xF4A7 + 3, 1_000_000, 1e5), (5, 70_000, 2e4)])
def test_oracle_generator_equals_product_generator(seed, n, domain):
    # the CPU legs of the benchmark make their layouts with the oracle's
    # generator (no product library in those processes): it must give the
    # product's rects exactly, including the 10^6-rect layout
    a = O.generate_layout(seed, n, domain)
    b = frw.generate_layout(seed, n, domain)
    assert a.shape == (n, 4) and np.array_equal(a, b.astype(np.float64))
