"""ctypes bindings for the CPU checkers -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the cpu_baseline / reference legs
of ``bench.py`` import this module.  It wraps

* ``liboracle.so``      -- the C restatement of the reference CPU path
                           (``frwcpu.c``) and of the 3-D walk with the cube
                           table (``frwcpu3d.c``), and
* ``_ref/librefcpu.so`` -- the unmodified reference CPU sources compiled in
                           place (``ref_driver.cpp``), when present.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_root() -> str:
    """The reference checkout: $REFERENCE, else the default of oracle/Makefile."""
    if os.environ.get("REFERENCE"):
        return os.environ["REFERENCE"]
    out = subprocess.run(["make", "-s", "--no-print-directory", "-C", HERE, "print-reference"],
                         capture_output=True, text=True)
    return out.stdout.strip()

NSAMPLE = 200
END_ESCAPED = -1
END_ABORTED = -2
GAUSS_SCALE, GAUSS_OFFSET = 0, 1
START_GREEN, START_UNIFORM = 0, 1
PERMITTIVITY = 8.854187817620e-12

_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)
_I32 = C.POINTER(C.c_int32)
_U32 = C.POINTER(C.c_uint32)


def _p(a, t=_D):
    return a.ctypes.data_as(t) if a is not None else None


def build(ref: bool = True) -> None:
    """Compile liboracle.so, and the reference library when its sources exist."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref-if-present"], check=True)


class WalkCfg(C.Structure):
    _fields_ = [
        ("target", C.c_int64),
        ("gauss_mode", C.c_int),
        ("gauss_param", C.c_double),
        ("start_mode", C.c_int),
        ("exact_perimeter", C.c_int),
        ("hop_cap", C.c_int64),
        ("permittivity", C.c_double),
        ("seed", C.c_uint64),
        ("stream", C.c_uint32),
        ("start_grid", C.c_uint32),
        ("start_strata", C.c_uint32),
    ]


class Cfg3(C.Structure):
    """oc3_cfg of frwcpu3d.h."""
    _fields_ = [
        ("target", C.c_int64),
        ("offset", C.c_double),
        ("shell", C.c_double),
        ("hop_cap", C.c_int64),
        ("permittivity", C.c_double),
        ("seed", C.c_uint64),
        ("stream", C.c_uint32),
        ("nsample", C.c_int),
        ("start_strata", C.c_uint32),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        L = C.CDLL(path)
        L.oc_parse_layout.argtypes = [C.c_char_p, C.c_int, C.POINTER(_D), _I64, C.POINTER(C.c_int)]
        L.oc_free.argtypes = [C.c_void_p]
        L.oc_layer_bounds.argtypes = [_D, C.c_int64, _D]
        L.oc_green_table.argtypes = [C.c_int, _D, _D]
        L.oc_weight_table.argtypes = [C.c_int, _D, _D, _D]
        L.oc_bin_index.argtypes = [_D, C.c_int, C.c_double]
        L.oc_philox4x32_10.argtypes = [_U32, _U32, _U32]
        L.oc_u01.argtypes = [C.c_uint32, C.c_uint32]
        L.oc_u01.restype = C.c_double
        L.oc_point_from_index.argtypes = [_D, C.c_int, C.c_int, C.c_int, _D]
        L.oc_scale_rect.argtypes = [_D, C.c_double, C.c_double, _D]
        L.oc_grid_create.argtypes = [_D, C.c_int64, _D]
        L.oc_grid_create.restype = C.c_void_p
        L.oc_grid_destroy.argtypes = [C.c_void_p]
        L.oc_grid_box_collides.argtypes = [C.c_void_p, _D, _D]
        L.oc_grid_point_hit.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.oc_grid_point_hit.restype = C.c_int64
        L.oc_grid_biggest_square.argtypes = [C.c_void_p, C.c_double, C.c_double, _D]
        L.oc_grid_query_batch.argtypes = [C.c_void_p, _D, C.c_int64, _D, _I64]
        L.oc_grid_gauss_scale.argtypes = [C.c_void_p, _D, C.c_double, _D]
        L.oc_rtree_create.argtypes = [_D, C.c_int64, _D]
        L.oc_rtree_create.restype = C.c_void_p
        L.oc_rtree_destroy.argtypes = [C.c_void_p]
        L.oc_rtree_box_collides.argtypes = [C.c_void_p, _D, _D, C.c_int]
        L.oc_rtree_point_hit.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.oc_rtree_point_hit.restype = C.c_int64
        L.oc_rtree_biggest_square.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, _D]
        L.oc_rtree_gauss_scale.argtypes = [C.c_void_p, _D, C.c_double, C.c_int, _D]
        L.oc_rtree_stats.argtypes = [C.c_void_p, _I64, _I64, C.POINTER(C.c_int)]
        L.oc_walk_gauss_surface.argtypes = [C.c_void_p, _D, C.POINTER(WalkCfg), _D]
        L.oc_walk_run.argtypes = [C.c_void_p, _D, C.POINTER(WalkCfg), C.c_uint64, C.c_uint64,
                                  _I64, _I32, _I32, _D, _D]
        L.oc_walk_stream.argtypes = [C.c_void_p, C.c_void_p, C.c_int, _D, _D, _D, C.c_int64,
                                     _I64, _I32]
        L.oc_walk_stream.restype = C.c_int64
        L.oc_cv_features.argtypes = [_D, C.c_int64, C.c_int64, _D, C.c_int64, C.POINTER(C.c_float)]
        L.oc_generate_layout.argtypes = [C.c_uint64, C.c_int64, C.c_double, C.c_int, C.c_int, C.c_double, _D]
        L.oc3_cube_green_table.argtypes = [C.c_int, _D, _D, _D, _D, _D]
        L.oc3_green_cube.argtypes = [C.c_double, C.c_double, C.c_double]
        L.oc3_green_cube.restype = C.c_double
        L.oc3_deriv_green_cube.argtypes = [_D, C.c_double, C.c_double, C.c_double]
        L.oc3_weight_table.argtypes = [C.c_int, _D, _D, _D, _D, _D]
        L.oc3_layout_bounds.argtypes = [_D, C.c_int64, _D]
        L.oc3_default_shell.argtypes = [_D, C.c_int64]
        L.oc3_default_shell.restype = C.c_double
        L.oc3_nearest.argtypes = [_D, C.c_int64, _D, _D, _I64]
        L.oc3_grid_create.argtypes = [_D, C.c_int64, _D, C.c_double, C.c_int]
        L.oc3_grid_create.restype = C.c_void_p
        L.oc3_grid_destroy.argtypes = [C.c_void_p]
        L.oc3_grid_nearest.argtypes = [C.c_void_p, _D, _D, _I64]
        L.oc3_query_batch.argtypes = [_D, C.c_int64, C.c_void_p, _D, C.c_int64, _D, _I64]
        L.oc3_walk_run.argtypes = [_D, C.c_int64, _D, C.c_void_p, C.POINTER(Cfg3), C.c_uint64, C.c_uint64,
                                   _I64, _I32, _I32, _D]
        _lib = L
    return _lib


# ---------------------------------------------------------------- helpers
def parse_layout(path: str, layer: int = 0) -> np.ndarray:
    L = lib()
    out = _D()
    n = C.c_int64()
    nl = C.c_int()
    st = L.oc_parse_layout(path.encode(), layer, C.byref(out), C.byref(n), C.byref(nl))
    if st != 0:
        raise ValueError(f"oc_parse_layout({path!r}, {layer}) -> {st} (layers={nl.value})")
    arr = np.ctypeslib.as_array(out, shape=(n.value, 4)).copy() if n.value else np.zeros((0, 4))
    L.oc_free(out)
    return arr


def layer_bounds(rects: np.ndarray) -> np.ndarray:
    rects = np.ascontiguousarray(rects, dtype=np.float64)
    b = np.zeros(4)
    lib().oc_layer_bounds(_p(rects), len(rects), _p(b))
    return b


def green_table(nsample: int = NSAMPLE):
    g = np.zeros(nsample)
    intg = np.zeros(nsample + 1)
    lib().oc_green_table(nsample, _p(g), _p(intg))
    return g, intg


def weight_table(intg: np.ndarray, nsample: int = NSAMPLE):
    wx = np.zeros(nsample)
    wy = np.zeros(nsample)
    intg = np.ascontiguousarray(intg, dtype=np.float64)
    lib().oc_weight_table(nsample, _p(intg), _p(wx), _p(wy))
    return wx, wy


def philox(ctr, key):
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    lib().oc_philox4x32_10(_p(c, _U32), _p(k, _U32), _p(o, _U32))
    return o


def point_from_index(sq, index: int, exact_perimeter: bool = False):
    s = np.ascontiguousarray(sq, dtype=np.float64)
    o = np.zeros(2)
    lib().oc_point_from_index(_p(s), int(index), NSAMPLE, int(exact_perimeter), _p(o))
    return o


def generate_layout(seed: int, n: int, domain: float, wmin: int = 5, wmax: int = 50,
                    gap: float = 2.0) -> np.ndarray:
    """The benchmark layout generator restated in C (n x 4 float64, integer
    corners); equal to the product's frw_generate_layout rect for rect."""
    out = np.zeros((int(n), 4))
    rc = lib().oc_generate_layout(int(seed), int(n), float(domain), int(wmin), int(wmax), float(gap), _p(out))
    if rc != 0:
        raise ValueError(f"oc_generate_layout -> {rc}")
    return out


class Grid:
    """Complete-semantics index (exact brute-force predicates)."""

    def __init__(self, rects: np.ndarray, bounds=None):
        self.rects = np.ascontiguousarray(rects, dtype=np.float64)
        self.bounds = np.ascontiguousarray(layer_bounds(self.rects) if bounds is None else bounds,
                                           dtype=np.float64)
        self.h = lib().oc_grid_create(_p(self.rects), len(self.rects), _p(self.bounds))
        if not self.h:
            raise MemoryError("oc_grid_create")

    def __del__(self):
        if getattr(self, "h", None):
            lib().oc_grid_destroy(self.h)
            self.h = None

    def box_collides(self, box, ignore=None) -> bool:
        b = np.ascontiguousarray(box, dtype=np.float64)
        ig = None if ignore is None else np.ascontiguousarray(ignore, dtype=np.float64)
        return bool(lib().oc_grid_box_collides(self.h, _p(b), _p(ig)))

    def point_hit(self, x, y) -> int:
        return int(lib().oc_grid_point_hit(self.h, float(x), float(y)))

    def biggest_square(self, x, y) -> np.ndarray:
        o = np.zeros(4)
        lib().oc_grid_biggest_square(self.h, float(x), float(y), _p(o))
        return o

    def query_batch(self, pts: np.ndarray):
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        sq = np.zeros((len(pts), 4))
        hit = np.zeros(len(pts), dtype=np.int64)
        lib().oc_grid_query_batch(self.h, _p(pts), len(pts), _p(sq), _p(hit, _I64))
        return sq, hit

    def gauss_scale(self, r, factor=1.5):
        rr = np.ascontiguousarray(r, dtype=np.float64)
        o = np.zeros(4)
        lib().oc_grid_gauss_scale(self.h, _p(rr), float(factor), _p(o))
        return o

    def walk_cfg(self, target=0, gauss_mode=GAUSS_OFFSET, gauss_param=1.0, start_mode=START_UNIFORM,
                 exact_perimeter=False, hop_cap=100000, seed=1, stream=0, start_grid=0, start_strata=0):
        return WalkCfg(target, gauss_mode, gauss_param, start_mode, int(exact_perimeter), hop_cap,
                       PERMITTIVITY, seed, stream, start_grid, start_strata)

    def gauss_surface(self, cfg: WalkCfg):
        o = np.zeros(4)
        lib().oc_walk_gauss_surface(self.h, _p(self.rects), C.byref(cfg), _p(o))
        return o

    def walks(self, cfg: WalkCfg, first: int, count: int, cv: bool = False):
        """Per-walk (end, hops, first bin, weight factor c[, (p1x, p1y, a0, c)])."""
        end = np.zeros(count, dtype=np.int64)
        hops = np.zeros(count, dtype=np.int32)
        b1 = np.zeros(count, dtype=np.int32)
        w = np.zeros(count)
        cvo = np.zeros((count, 4)) if cv else None
        lib().oc_walk_run(self.h, _p(self.rects), C.byref(cfg), first, count, _p(end, _I64),
                          _p(hops, _I32), _p(b1, _I32), _p(w), _p(cvo))
        return (end, hops, b1, w, cvo) if cv else (end, hops, b1, w)


class RefTree:
    """The reference CPU quadtree restated (insertion-order structure)."""

    def __init__(self, rects: np.ndarray, bounds=None):
        self.rects = np.ascontiguousarray(rects, dtype=np.float64)
        self.bounds = np.ascontiguousarray(layer_bounds(self.rects) if bounds is None else bounds,
                                           dtype=np.float64)
        self.h = lib().oc_rtree_create(_p(self.rects), len(self.rects), _p(self.bounds))
        if not self.h:
            raise MemoryError("oc_rtree_create")

    def __del__(self):
        if getattr(self, "h", None):
            lib().oc_rtree_destroy(self.h)
            self.h = None

    def box_collides(self, box, ignore=None, defect=True) -> bool:
        b = np.ascontiguousarray(box, dtype=np.float64)
        ig = None if ignore is None else np.ascontiguousarray(ignore, dtype=np.float64)
        return bool(lib().oc_rtree_box_collides(self.h, _p(b), _p(ig), int(defect)))

    def point_hit(self, x, y) -> int:
        return int(lib().oc_rtree_point_hit(self.h, float(x), float(y)))

    def biggest_square(self, x, y, defect=True) -> np.ndarray:
        o = np.zeros(4)
        lib().oc_rtree_biggest_square(self.h, float(x), float(y), int(defect), _p(o))
        return o

    def gauss_scale(self, r, factor=1.5, defect=True):
        rr = np.ascontiguousarray(r, dtype=np.float64)
        o = np.zeros(4)
        lib().oc_rtree_gauss_scale(self.h, _p(rr), float(factor), int(defect), _p(o))
        return o

    def stats(self):
        a, b, c = C.c_int64(), C.c_int64(), C.c_int()
        lib().oc_rtree_stats(self.h, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value


def cv_features(rects, target: int, rec4):
    """Control-variate features (16 floats per point) of points rec4 = (x, y, a0, _)."""
    r = np.ascontiguousarray(rects, dtype=np.float64)
    q = np.ascontiguousarray(rec4, dtype=np.float64).reshape(-1, 4)
    out = np.zeros((len(q), 16), dtype=np.float32)
    lib().oc_cv_features(_p(r), len(r), int(target), _p(q), len(q), out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


def walk_stream(grid: Grid | None, tree: RefTree | None, defect: bool, gauss, intg, r):
    """Replay one reference-style walk on an explicit uniform stream."""
    g = np.ascontiguousarray(gauss, dtype=np.float64)
    it = np.ascontiguousarray(intg, dtype=np.float64)
    rr = np.ascontiguousarray(r, dtype=np.float64)
    used = C.c_int64()
    hops = C.c_int32()
    end = lib().oc_walk_stream(grid.h if grid else None, tree.h if tree else None, int(defect),
                               _p(g), _p(it), _p(rr), len(rr), C.byref(used), C.byref(hops))
    return int(end), int(used.value), int(hops.value)


# ------------------------------------------------------- reference library
_ref = None


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "librefcpu.so"))


def ref():
    """The unmodified reference CPU code (single global layout)."""
    global _ref
    if _ref is None:
        L = C.CDLL(os.path.join(HERE, "_ref", "librefcpu.so"))
        L.ref_load.argtypes = [C.c_char_p, C.c_int]
        L.ref_load.restype = C.c_int64
        L.ref_load_rects.argtypes = [_D, C.c_int64, _D]
        L.ref_load_rects.restype = C.c_int64
        L.ref_rects.argtypes = [_D]
        L.ref_bounds.argtypes = [_D]
        L.ref_green.argtypes = [_D, _D, _D, _D]
        L.ref_get_index.argtypes = [C.c_double]
        L.ref_point_from_index.argtypes = [_D, C.c_int, _D]
        L.ref_box_collides.argtypes = [_D, _D]
        L.ref_biggest_square.argtypes = [C.c_double, C.c_double, _D]
        L.ref_point_hit.argtypes = [C.c_double, C.c_double, _D]
        L.ref_point_hit.restype = C.c_int64
        L.ref_query_batch.argtypes = [_D, C.c_int64, _D, _I64]
        L.ref_gauss.argtypes = [C.c_int64, C.c_double, _D]
        L.ref_walks_seeded.argtypes = [C.c_int64, C.c_int64, C.c_uint32, C.c_uint32, C.c_uint32,
                                       C.c_uint32, _I64, _I32, _D, C.c_int64, _I64]
        L.ref_walks_as_shipped.argtypes = [C.c_int64, C.c_int64, _I64, _I32]
        L.ref_unit_cube_green.argtypes = [C.c_int, _D, _D, _D, _D, _D]
        L.ref_green_cube.argtypes = [C.c_double, C.c_double, C.c_double]
        L.ref_green_cube.restype = C.c_double
        L.ref_deriv_green_cube.argtypes = [_D, C.c_double, C.c_double, C.c_double]
        _ref = L
    return _ref


class Ref:
    """Convenience wrapper over the reference library's global layout."""

    def __init__(self, path: str | None = None, layer: int = 0, rects=None, bounds=None):
        L = ref()
        if path is not None:
            n = L.ref_load(path.encode(), layer)
        else:
            r = np.ascontiguousarray(rects, dtype=np.float64)
            b = np.ascontiguousarray(bounds, dtype=np.float64)
            n = L.ref_load_rects(_p(r), len(r), _p(b))
        if n <= 0:
            raise ValueError("reference failed to load the layout")
        self.n = int(n)
        self.rects = np.zeros((self.n, 4))
        L.ref_rects(_p(self.rects))
        self.bounds = np.zeros(4)
        L.ref_bounds(_p(self.bounds))

    def green(self):
        g, dx, dy, it = np.zeros(NSAMPLE), np.zeros(NSAMPLE), np.zeros(NSAMPLE), np.zeros(NSAMPLE + 1)
        ref().ref_green(_p(g), _p(dx), _p(dy), _p(it))
        return g, dx, dy, it

    def get_index(self, r):
        return int(ref().ref_get_index(float(r)))

    def point_from_index(self, sq, index):
        s = np.ascontiguousarray(sq, dtype=np.float64)
        o = np.zeros(2)
        ref().ref_point_from_index(_p(s), int(index), _p(o))
        return o

    def box_collides(self, box, ignore=None):
        b = np.ascontiguousarray(box, dtype=np.float64)
        ig = None if ignore is None else np.ascontiguousarray(ignore, dtype=np.float64)
        return bool(ref().ref_box_collides(_p(b), _p(ig)))

    def biggest_square(self, x, y):
        o = np.zeros(4)
        ref().ref_biggest_square(float(x), float(y), _p(o))
        return o

    def point_hit(self, x, y):
        return int(ref().ref_point_hit(float(x), float(y), None))

    def query_batch(self, pts):
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        sq = np.zeros((len(pts), 4))
        hit = np.zeros(len(pts), dtype=np.int64)
        ref().ref_query_batch(_p(pts), len(pts), _p(sq), _p(hit, _I64))
        return sq, hit

    def gauss(self, target, factor=1.5):
        o = np.zeros(4)
        ref().ref_gauss(int(target), float(factor), _p(o))
        return o

    def walks_seeded(self, target, n, seed=(1, 2, 3, 4), r_cap=0):
        end = np.zeros(n, dtype=np.int64)
        hops = np.zeros(n, dtype=np.int32)
        r = np.zeros(max(r_cap, 1))
        used = C.c_int64()
        ref().ref_walks_seeded(int(target), int(n), *[int(s) & 0xFFFFFFFF for s in seed],
                               _p(end, _I64), _p(hops, _I32), _p(r) if r_cap else None, r_cap,
                               C.byref(used))
        return end, hops, (r[: min(used.value, r_cap)] if r_cap else None), used.value

    def walks_as_shipped(self, target, n):
        end = np.zeros(n, dtype=np.int64)
        hops = np.zeros(n, dtype=np.int32)
        ref().ref_walks_as_shipped(int(target), int(n), _p(end, _I64), _p(hops, _I32))
        return end, hops


# ---------------------------------------------------------------- 3-D path
NSAMPLE3 = 50


def cube_green_table(n: int = NSAMPLE3):
    """The restated precompute_unit_cube_green: (g, dgdx, dgdy, dgdz, intg)."""
    nb = 6 * n * n
    out = [np.zeros(nb) for _ in range(4)] + [np.zeros(nb + 1)]
    lib().oc3_cube_green_table(n, *[_p(a) for a in out])
    return tuple(out)


def ref_cube_green_table(n: int = NSAMPLE3):
    """The reference's own precompute_unit_cube_green (oracle/_ref)."""
    nb = 6 * n * n
    out = [np.zeros(nb) for _ in range(4)] + [np.zeros(nb + 1)]
    ref().ref_unit_cube_green(n, *[_p(a) for a in out])
    return tuple(out)


def cube_weight_table(n: int = NSAMPLE3) -> np.ndarray:
    g, dx, dy, dz, intg = cube_green_table(n)
    w = np.zeros((6 * n * n, 3))
    lib().oc3_weight_table(n, _p(intg), _p(dx), _p(dy), _p(dz), _p(w))
    return w


def layout_bounds3(boxes) -> np.ndarray:
    b = np.ascontiguousarray(boxes, dtype=np.float64)
    out = np.zeros(6)
    lib().oc3_layout_bounds(_p(b), len(b), _p(out))
    return out


class Boxes3:
    """A 3-D layout for the oracle: brute-force or cell-grid nearest box and walks."""

    def __init__(self, boxes, bounds=None, grid: bool = False, boxes_per_cell: float = 2.0, lists=None):
        """grid: answer through a cell grid (equal to the brute force);
        lists: per-cell candidate lists for speed (default: up to 2e5 boxes)."""
        self.boxes = np.ascontiguousarray(boxes, dtype=np.float64)
        self.n = len(self.boxes)
        self.bounds = layout_bounds3(self.boxes) if bounds is None else np.ascontiguousarray(bounds, np.float64)
        self.shell = float(lib().oc3_default_shell(_p(self.boxes), self.n))
        with_lists = int(self.n <= 200_000 if lists is None else bool(lists))
        self._g = (lib().oc3_grid_create(_p(self.boxes), self.n, _p(self.bounds), boxes_per_cell, with_lists)
                   if grid else None)

    def __del__(self):
        g, self._g = getattr(self, "_g", None), None
        if g:
            lib().oc3_grid_destroy(g)

    def nearest(self, pts, use_grid: bool | None = None):
        """(clearance, nearest box) per point; the grid when built unless use_grid is False."""
        p = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        d = np.zeros(len(p))
        k = np.zeros(len(p), dtype=np.int64)
        g = self._g if use_grid is None or use_grid else None
        lib().oc3_query_batch(_p(self.boxes), self.n, g, _p(p), len(p), _p(d), _p(k, _I64))
        return d, k

    def cfg(self, target=0, offset=1.0, shell=None, hop_cap=100000, seed=0, stream=0, nsample=NSAMPLE3,
            start_strata=0):
        return Cfg3(target, offset, self.shell if shell is None else shell, hop_cap, PERMITTIVITY, seed, stream,
                    nsample, start_strata)

    def walks(self, cfg: Cfg3, first: int, count: int):
        end = np.zeros(count, dtype=np.int64)
        hops = np.zeros(count, dtype=np.int32)
        b1 = np.zeros(count, dtype=np.int32)
        w = np.zeros(count)
        rc = lib().oc3_walk_run(_p(self.boxes), self.n, _p(self.bounds), self._g, C.byref(cfg), first, count,
                                _p(end, _I64), _p(hops, _I32), _p(b1, _I32), _p(w))
        if rc != 0:
            raise ValueError(f"oc3_walk_run failed: {rc}")
        return end, hops, b1, w
