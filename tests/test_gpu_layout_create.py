"""frw_layout_create: the rect checks (made on the device), the bounds rule
(reference Parser::getLayerSize, CPU/Parser.cpp:79-84) and the host copy of
the rects, against the oracle."""
import numpy as np
import pytest

import oracle as O

frw = pytest.importorskip("frw")
pytestmark = pytest.mark.gpu


def _layout(n=2000, seed=0x1C, domain=4000.0):
    return O.generate_layout(seed, n, domain).astype(np.float32)


@pytest.mark.parametrize("bad, why", [
    ((0, np.nan), "not finite"),
    ((2, np.inf), "not finite"),
    ((1, -np.inf), "not finite"),
    ((3, 16777216.0), "2\\^24"),
    ((0, -16777216.0), "2\\^24"),
    ("inverted-x", "inverted"),
    ("inverted-y", "inverted"),
])
def test_bad_rects_name_the_first_offender(bad, why):
    r = _layout()
    for i in (777, 1500):  # two offenders: the first is named
        if bad == "inverted-x":
            r[i, 0], r[i, 2] = r[i, 2] + 1, r[i, 0]
        elif bad == "inverted-y":
            r[i, 1], r[i, 3] = r[i, 3] + 1, r[i, 1]
        else:
            r[i, bad[0]] = bad[1]
    with pytest.raises(frw.FrwError, match=f"rect 777: .*{why}") as e:
        frw.Layout.from_rects(r)
    assert e.value.status == frw.E_ARG


def test_rects_outside_given_bounds():
    r = _layout()
    b = np.array([r[:, 0].min(), r[:, 1].min(), r[:, 2].max(), r[:, 3].max()], dtype=np.float64)
    with frw.Layout.from_rects(r, bounds=b) as L:  # the tight box is accepted as given
        assert np.array_equal(L.bounds, b)
    r[901, 2] = b[2] + 0.5
    r[1200, 1] = b[1] - 3
    with pytest.raises(frw.FrwError, match="rect 901 lies outside the bounds"):
        frw.Layout.from_rects(r, bounds=b)
    with pytest.raises(frw.FrwError, match="bounds invalid"):
        frw.Layout.from_rects(r, bounds=np.array([10.0, 0, 0, 10]))


@pytest.mark.parametrize("shift", [(0.0, 0.0), (-3000.5, -100.25), (-8000.0, 2500.0), (-4000.0, -4000.0)])
def test_bounds_rule_and_host_copy(shift):
    """Bounds equal the oracle's getLayerSize rule for negative, mixed-sign and
    zero-touching extents; the host copy returns the rects as given."""
    # 300,000 rects: the host copy is split over several threads
    r = _layout(n=300_000, seed=0x2C, domain=40_000.0) if shift == (0.0, 0.0) else _layout()
    r = (r + np.array([shift[0], shift[1], shift[0], shift[1]], dtype=np.float32)).astype(np.float32)
    with frw.Layout.from_rects(r) as L:
        assert np.array_equal(L.bounds, O.layer_bounds(r.astype(np.float64)))
        assert np.array_equal(L.rects(), r.astype(np.float64))


def test_negative_zero_extent():
    r = np.array([[-0.0, -0.0, 10, 10], [20, 0.0, 30, 10], [0.0, 20, 10, 30]], dtype=np.float32)
    with frw.Layout.from_rects(r) as L:
        b = L.bounds
        assert np.array_equal(b, O.layer_bounds(r.astype(np.float64)))
        assert not np.signbit(b[0]) and not np.signbit(b[1])  # -0 and +0 extents settle on +0
