"""The product's layout reader (frw_parse_layout, host only) on the
reference's own layout files: the rects and the bounds must equal what the
reference's Parser produced for the golden fixtures (Parser::parse,
getLayerAt and getLayerSize, CPU/Parser.cpp:15-87), and the malformed-file
cases behave as documented in include/frw.h -- an over-long line ends the
reading exactly where the reference's getline stops, other defects are
errors instead of undefined reads."""
import os

import numpy as np
import pytest

import frw
import oracle as O
from conftest import FIXTURES, GOLDEN

LAYOUTS = os.path.join(GOLDEN, "layouts")


@pytest.mark.parametrize("name", FIXTURES)
def test_reader_equals_reference_parser_on_fixture_files(name, golden):
    g = golden(name)
    rects, bounds, layers = frw.parse_layout(os.path.join(LAYOUTS, name), 0)
    assert layers >= 1
    assert rects.shape == g["rects"].shape and np.array_equal(rects, g["rects"])
    assert np.array_equal(bounds, g["bounds"])


def _write(tmp_path, text):
    p = tmp_path / "layout.txt"
    p.write_text(text)
    return str(p)


def _status(path, layer=0):
    with pytest.raises(frw.FrwError) as e:
        frw.parse_layout(path, layer)
    return e.value.status, str(e.value)


TWO_LAYERS = ("magic\n<< metal1 >>\nrect 0 0 10 10\nrect 20 0 30 12\n<< metal2 >>\n"
              "rect 5 5 9 9\n<< end >>\n")


def test_two_layers_and_trailing_rects_dropped(tmp_path):
    # rects after the last delimiter belong to no closed layer (reference rule)
    p = _write(tmp_path, TWO_LAYERS + "rect 100 100 110 110\n")
    r0, b0, n = frw.parse_layout(p, 0)
    r1, b1, _ = frw.parse_layout(p, 1)
    assert n == 2
    assert np.array_equal(r0, [[0, 0, 10, 10], [20, 0, 30, 12]]) and np.array_equal(r1, [[5, 5, 9, 9]])
    assert np.array_equal(b0, O.layer_bounds(r0)) and np.array_equal(b1, O.layer_bounds(r1))
    assert _status(p, 2)[0] == frw.E_ARG


def test_overlong_line_ends_reading_like_the_reference(tmp_path):
    long_line = "rect 1 1 2 2" + " " * 60 + "\n"
    p = _write(tmp_path, TWO_LAYERS.replace("<< metal2 >>\n", "<< metal2 >>\n" + long_line))
    r0, _, n = frw.parse_layout(p, 0)
    assert n == 1 and len(r0) == 2  # layer 1 is never closed: the reading stopped inside it
    assert _status(p, 1)[0] == frw.E_ARG
    if O.ref_available():  # the reference's own Parser on the same file
        R = O.Ref(path=p, layer=0)
        assert np.array_equal(R.rects, r0)
        with pytest.raises(ValueError):
            O.Ref(path=p, layer=1)


@pytest.mark.parametrize("line", ["rect 1 2 3", "rect 1 2 3 4 5", "rect a b c d"])
def test_rect_line_without_four_numbers_is_an_error(tmp_path, line):
    p = _write(tmp_path, f"<< m >>\nrect 0 0 4 4\n{line}\n<< end >>\n")
    st, msg = _status(p)
    assert st == frw.E_IO and ":3:" in msg


def test_missing_file_is_an_io_error():
    assert _status("/nonexistent/layout.txt")[0] == frw.E_IO


def test_capacity_too_small_reports_count(tmp_path):
    import ctypes as C

    p = _write(tmp_path, TWO_LAYERS)
    n = C.c_int64()
    out = np.zeros((1, 4))
    st = frw.lib().frw_parse_layout(p.encode(), 0, out.ctypes.data_as(C.POINTER(C.c_double)), 1, C.byref(n),
                                    None, None)
    assert st == frw.E_ARG and n.value == 2
