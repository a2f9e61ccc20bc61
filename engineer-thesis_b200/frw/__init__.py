"""Python mirror of the FRW C ABI (include/frw.h) over lib/libfrw.so.

The compute path is the CUDA library only: importing this module loads
``lib/libfrw.so`` (built in-tree by ``make -C engineer-thesis_b200``) and every
compute call raises :class:`FrwError` when no sm_100 device is usable.  There
is no CPU fallback.

Names follow the reference (piogrzej/engineer-thesis, randomWalk/):

* :class:`Layout` -- ``createQuadTree`` / ``freeQuadTreeManager``
  (Cuda/mainkernels.h:10,13) plus the layout reader (CPU/Parser.cpp).
* :meth:`Layout.draw_biggest_square` / :meth:`Layout.check_collisions_point`
  -- ``drawBiggestSquareAtPoint`` / ``checkCollisons(point)``, batched.
* :meth:`Layout.check_collisions` -- ``checkCollisions(rect, ignore)``.
* :meth:`Layout.gauss_surface` -- ``creatGaussianSurfFrom``.
* :meth:`Layout.walk` -- the estimator of ``getAvgPathLen(CUDA)``.
* :meth:`Layout.walk_trace` -- ``randomWalkCudaWrapper``'s per-walk outputs.
* :func:`get_avg_path_len_cuda` -- ``getAvgPathLenCUDA``.
* :func:`cube_green_table`, :func:`green_cube`, :func:`deriv_green_cube` --
  ``precompute_unit_cube_green``, ``green_cube``, ``deriv_green_cube``
  (green/green.h:71-80), and :class:`Layout3`, the 3-D walk over box
  conductors that the reference's cube table was written for (include/frw3d.h).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG, "lib", "libfrw.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "frw.h")
HEADER3 = os.path.join(os.path.dirname(PKG), "include", "frw3d.h")

OK, E_ARG, E_IO, E_CUDA, E_OOM, E_HOPCAP, E_TIMEOUT, E_DEVICE, E_KERNEL = 0, -1, -2, -3, -4, -5, -6, -7, -8
NSAMPLE = 200
MEM_HOST, MEM_DEVICE = 0, 1
GAUSS_SCALE, GAUSS_OFFSET = 0, 1
START_GREEN, START_UNIFORM = 0, 1
END_ESCAPED, END_ABORTED = -1, -2
PERMITTIVITY = 8.854187817620e-12


class FrwError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"frw status {status}: {msg}")
        self.status = status


class Opts(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("gauss_mode", C.c_int32),
        ("gauss_param", C.c_double),
        ("start_mode", C.c_int32),
        ("exact_perimeter", C.c_int32),
        ("hop_cap", C.c_int64),
        ("permittivity", C.c_double),
        ("stream_id", C.c_uint32),
        ("threads_per_block", C.c_int32),
        ("blocks_per_sm", C.c_int32),
        ("refill_min", C.c_int32),
        ("start_grid", C.c_uint32),
        ("first_walk", C.c_uint64),
        ("start_strata", C.c_uint32),
        ("timeout_ms", C.c_double),
    ]


class Result(C.Structure):
    _fields_ = [
        ("walks", C.c_uint64),
        ("escaped", C.c_uint64),
        ("aborted", C.c_uint64),
        ("hops_total", C.c_uint64),
        ("gauss", C.c_double * 4),
        ("fraction_other", C.c_double),
        ("kernel_ms", C.c_double),
        ("capacity", C.c_int64),
        ("n_entries", C.c_int64),
        ("conductor", C.POINTER(C.c_int64)),
        ("hits", C.POINTER(C.c_uint64)),
        ("cap", C.POINTER(C.c_double)),
        ("cap_se", C.POINTER(C.c_double)),
        ("sum_w", C.POINTER(C.c_double)),
        ("sum_w2", C.POINTER(C.c_double)),
    ]


class CvOpts(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("train_walks", C.c_uint64),
        ("train_seed", C.c_uint64),
        ("epochs", C.c_int32),
        ("batch", C.c_int32),
        ("lr", C.c_float),
    ]


class CvInfo(C.Structure):
    _fields_ = [
        ("mean_term", C.c_double),
        ("train_loss", C.c_double),
        ("train_ms", C.c_double),
        ("quad_ms", C.c_double),
        ("train_walks", C.c_uint64),
        ("quad_points", C.c_uint32),
    ]


class CvResult(C.Structure):
    _fields_ = [
        ("walks", C.c_uint64),
        ("plain", C.c_double),
        ("plain_se", C.c_double),
        ("cv", C.c_double),
        ("cv_se", C.c_double),
        ("variance_ratio", C.c_double),
        ("kernel_ms", C.c_double),
    ]


class Tuning(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("blocks_per_sm", C.c_int32),
        ("refill_min", C.c_int32),
        ("chunk", C.c_int32),
        ("ms", C.c_double),
    ]

    def as_dict(self):
        return {"blocks_per_sm": self.blocks_per_sm, "refill_min": self.refill_min, "chunk": self.chunk,
                "trial_ms": self.ms}


class LayoutInfo(C.Structure):
    _fields_ = [
        ("n_rects", C.c_int64),
        ("n_nodes", C.c_int64),
        ("depth", C.c_int32),
        ("leaf_max", C.c_int32),
        ("bounds", C.c_double * 4),
        ("device_bytes", C.c_int64),
        ("device", C.c_int32),
        ("build_ms", C.c_double),
    ]


class CellsInfo(C.Structure):
    _fields_ = [
        ("cells", C.c_int64),
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("cell_side", C.c_double),
        ("entries", C.c_int64),
        ("overflow_cells", C.c_int64),
        ("device_bytes", C.c_int64),
        ("build_ms", C.c_double),
    ]


class Opts3(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("gauss_offset", C.c_double),
        ("shell", C.c_double),
        ("hop_cap", C.c_int64),
        ("permittivity", C.c_double),
        ("stream_id", C.c_uint32),
        ("nsample", C.c_int32),
        ("first_walk", C.c_uint64),
        ("blocks_per_sm", C.c_int32),
        ("refill_min", C.c_int32),
        ("start_strata", C.c_uint32),
    ]


class Result3(C.Structure):
    _fields_ = [
        ("walks", C.c_uint64),
        ("escaped", C.c_uint64),
        ("aborted", C.c_uint64),
        ("hops_total", C.c_uint64),
        ("gauss", C.c_double * 6),
        ("shell", C.c_double),
        ("fraction_other", C.c_double),
        ("kernel_ms", C.c_double),
        ("capacity", C.c_int64),
        ("n_entries", C.c_int64),
        ("conductor", C.POINTER(C.c_int64)),
        ("hits", C.POINTER(C.c_uint64)),
        ("cap", C.POINTER(C.c_double)),
        ("cap_se", C.POINTER(C.c_double)),
        ("sum_w", C.POINTER(C.c_double)),
        ("sum_w2", C.POINTER(C.c_double)),
    ]


class Layout3Info(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("device", C.c_int),
        ("grid", C.c_int32 * 3),
        ("bounds", C.c_double * 6),
        ("cell_side", C.c_double),
        ("min_edge", C.c_double),
        ("list_entries", C.c_int64),
        ("max_list", C.c_int32),
        ("mean_list", C.c_double),
        ("build_ms", C.c_float),
        ("levels", C.c_int32),
        ("deferred_cells", C.c_int64),
        ("upper_entries", C.c_int64),
    ]


_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
_I64 = C.POINTER(C.c_int64)
_I32 = C.POINTER(C.c_int32)
_U8 = C.POINTER(C.c_uint8)
_VP = C.c_void_p

_SIGS = {
    "frw_version": ([], C.c_char_p),
    "frw_last_error": ([], C.c_char_p),
    "frw_device_check": ([C.c_int], C.c_int),
    "frw_green_table": ([_D, _D], C.c_int),
    "frw_layout_from_file": ([C.c_char_p, C.c_int, C.c_int, C.POINTER(_VP)], C.c_int),
    "frw_rows_compact": ([_VP, _VP, _VP, _VP, C.c_int64, _VP, _VP, _VP, _VP, _VP, _VP], C.c_int),
    "frw_set_wait_limit": ([C.c_double], C.c_int),
    "frw_mlp_set_kernels": ([C.c_int], C.c_int),
    "frw_mlp_get_kernels": ([], C.c_int),
    "frw_cv_set_walk_mode": ([C.c_int], C.c_int),
    "frw_cv_get_walk_mode": ([], C.c_int),
    "frw_get_wait_limit": ([], C.c_double),
    "frw_parse_layout": ([C.c_char_p, C.c_int, _D, C.c_int64, _I64, _D, _I32], C.c_int),
    "frw_layout_create": ([_F, C.c_int64, _D, C.c_int, _VP, C.POINTER(_VP)], C.c_int),
    "frw_layout_destroy": ([_VP], C.c_int),
    "frw_layout_info_get": ([_VP, C.POINTER(LayoutInfo)], C.c_int),
    "frw_layout_rects": ([_VP, _D], C.c_int),
    "frw_layout_set_cells": ([_VP, C.c_double, C.c_int, _VP], C.c_int),
    "frw_layout_cells_info": ([_VP, C.POINTER(CellsInfo)], C.c_int),
    "frw_query_batch": ([_VP, _VP, C.c_int64, _VP, _VP, C.c_int, _VP], C.c_int),
    "frw_box_collides_batch": ([_VP, _VP, C.c_int64, _D, _VP, C.c_int, _VP], C.c_int),
    "frw_opts_default": ([C.POINTER(Opts)], None),
    "frw_walk": ([_VP, C.c_int64, C.c_uint64, C.c_uint64, C.POINTER(Opts), C.POINTER(Result), _VP], C.c_int),
    "frw_walk_device": ([_VP, C.c_int64, C.c_uint64, C.c_uint64, C.POINTER(Opts), _VP, _VP, _VP, _VP, _VP, _VP],
                        C.c_int),
    "frw_walk_trace": ([_VP, C.c_int64, C.c_uint64, C.c_uint64, C.c_uint64, C.POINTER(Opts), _VP, _VP, _VP,
                        _VP, C.c_int, _VP], C.c_int),
    "frw_gauss_surface": ([_VP, C.c_int64, C.POINTER(Opts), _D, _VP], C.c_int),
    "frw_avg_path_len": ([C.c_char_p, C.c_int64, C.c_int64, C.c_int, C.c_uint64, C.c_int, C.c_char_p, _D],
                         C.c_int),
    "frw_generate_layout": ([C.c_uint64, C.c_int64, C.c_double, C.c_int32, C.c_int32, C.c_double, _F], C.c_int),
    "frw_write_layout": ([C.c_char_p, _F, C.c_int64, C.c_char_p], C.c_int),
    "frw_batch_create": ([C.POINTER(_VP), _I64, C.POINTER(C.c_uint64), C.c_int32, C.POINTER(Opts), C.POINTER(_VP)],
                         C.c_int),
    "frw_batch_tune": ([_VP, C.c_uint64, C.POINTER(Tuning)], C.c_int),
    "frw_batch_set_tuning": ([_VP, C.POINTER(Tuning)], C.c_int),
    "frw_batch_get_tuning": ([_VP, C.POINTER(Tuning)], C.c_int),
    "frw_batch_run": ([_VP, C.c_uint64, C.POINTER(Result), _VP], C.c_int),
    "frw_batch_destroy": ([_VP], C.c_int),
    "frw_cv_opts_default": ([C.POINTER(CvOpts)], None),
    "frw_cv_train": ([_VP, C.c_int64, C.POINTER(Opts), C.POINTER(CvOpts), C.POINTER(_VP), _VP], C.c_int),
    "frw_cv_info_get": ([_VP, C.POINTER(CvInfo)], C.c_int),
    "frw_cv_walk": ([_VP, C.c_uint64, C.c_uint64, C.POINTER(CvResult), _VP], C.c_int),
    "frw_cv_destroy": ([_VP], C.c_int),
    "frw_cv_params": ([_VP, _F], C.c_int),
    "frw_mlp_forward": ([_F, _F, C.c_int64, _F, C.c_int], C.c_int),
    "frw_mlp_grad": ([_F, _F, _F, _F, C.c_int64, C.c_double, _F, _D, C.c_int], C.c_int),
    "frw_cv_features": ([_VP, C.c_int64, _D, C.c_int64, _F], C.c_int),
    "frw3_cube_green_table": ([C.c_int, _D, _D, _D, _D, _D], C.c_int),
    "frw3_green_cube": ([C.c_double, C.c_double, C.c_double, _D], C.c_int),
    "frw3_deriv_green_cube": ([C.c_double, C.c_double, C.c_double, _D], C.c_int),
    "frw3_layout_create": ([_F, C.c_int64, _D, C.c_double, C.c_int, C.POINTER(_VP)], C.c_int),
    "frw3_layout_from_file": ([C.c_char_p, _D, _D, C.c_int, _D, C.c_double, C.c_int, C.POINTER(_VP)], C.c_int),
    "frw3_layout_destroy": ([_VP], C.c_int),
    "frw3_layout_info_get": ([_VP, C.POINTER(Layout3Info)], C.c_int),
    "frw3_layout_boxes": ([_VP, _F], C.c_int),
    "frw3_query_batch": ([_VP, _VP, C.c_int64, _VP, _VP, C.c_int, _VP], C.c_int),
    "frw3_opts_default": ([C.POINTER(Opts3)], None),
    "frw3_walk": ([_VP, C.c_int64, C.c_uint64, C.c_uint64, C.POINTER(Opts3), C.POINTER(Result3), _VP], C.c_int),
    "frw3_walk_device": ([_VP, C.c_int64, C.c_uint64, C.c_uint64, C.POINTER(Opts3), _VP, _VP, _VP, _VP, _VP, _VP],
                         C.c_int),
    "frw3_walk_batch": ([_VP, _I64, C.c_int32, C.c_uint64, C.c_uint64, C.POINTER(Opts3), C.POINTER(Result3), _VP],
                        C.c_int),
    "frw3_walk_trace": ([_VP, C.c_int64, C.c_uint64, C.c_uint64, C.c_uint64, C.POINTER(Opts3), _VP, _VP, _VP,
                         _VP, C.c_int, _VP], C.c_int),
    "frw3_generate_layout": ([C.c_uint64, C.c_int64, C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_int32,
                              C.c_int32, C.c_int32, _F], C.c_int),
}
CV_PARAMS = 5313

_lib = None


def lib():
    """Load lib/libfrw.so; raises ImportError when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} missing: build it with `make -C {PKG}`")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _check(st: int):
    if st != OK:
        raise FrwError(st, lib().frw_last_error().decode(errors="replace"))


def _ptr(a, t=_VP):
    return None if a is None else C.cast(a.ctypes.data, t)


def version() -> str:
    return lib().frw_version().decode()


def device_check(device: int = 0) -> None:
    _check(lib().frw_device_check(device))


MLP_TCGEN05, MLP_MMA_SYNC = 0, 1


def set_mlp_kernels(which: int) -> None:
    """MLP_TCGEN05 (128-row tcgen05 / TMEM tiles, the default) or MLP_MMA_SYNC."""
    _check(lib().frw_mlp_set_kernels(int(which)))


def mlp_kernels() -> int:
    return int(lib().frw_mlp_get_kernels())


CV_WALK_FUSED, CV_WALK_RECORDS = 0, 1


def set_cv_walk_mode(mode: int) -> None:
    """CV_WALK_FUSED (phi looked up and z summed inside the walk kernel, the
    default) or CV_WALK_RECORDS (per-walk records, then a summing kernel)."""
    _check(lib().frw_cv_set_walk_mode(int(mode)))


def cv_walk_mode() -> int:
    return int(lib().frw_cv_get_walk_mode())


def set_wait_limit(ms: float) -> None:
    """Process-wide bound on the library's host waits (0: none); see frw.h."""
    _check(lib().frw_set_wait_limit(float(ms)))


def wait_limit() -> float:
    return float(lib().frw_get_wait_limit())


def green_table():
    """(g[200], intg[201]) -- precompute_unit_square_green's g and intg."""
    g = np.zeros(NSAMPLE)
    intg = np.zeros(NSAMPLE + 1)
    _check(lib().frw_green_table(_ptr(g, _D), _ptr(intg, _D)))
    return g, intg


def opts(gauss_mode=GAUSS_SCALE, gauss_param=1.5, start_mode=START_GREEN, exact_perimeter=False,
         hop_cap=100000, stream_id=0, blocks_per_sm=0, refill_min=1, permittivity=PERMITTIVITY,
         start_grid=0, first_walk=0, start_strata=0, timeout_ms=0.0) -> Opts:
    o = Opts()
    lib().frw_opts_default(C.byref(o))
    o.gauss_mode = gauss_mode
    o.gauss_param = gauss_param
    o.start_mode = start_mode
    o.exact_perimeter = int(exact_perimeter)
    o.hop_cap = hop_cap
    o.stream_id = stream_id
    o.blocks_per_sm = blocks_per_sm
    o.refill_min = refill_min
    o.permittivity = permittivity
    o.start_grid = start_grid
    o.first_walk = first_walk
    o.start_strata = start_strata
    o.timeout_ms = timeout_ms
    return o


def capacitance_opts(offset=1.0, **kw) -> Opts:
    """Uniform start on the target grown by `offset`: capacitance weights on."""
    return opts(gauss_mode=GAUSS_OFFSET, gauss_param=offset, start_mode=START_UNIFORM, **kw)


def generate_layout(seed: int, n: int, domain: float, wmin: int = 5, wmax: int = 50, gap: float = 2.0):
    out = np.zeros((n, 4), dtype=np.float32)
    _check(lib().frw_generate_layout(seed, n, domain, wmin, wmax, gap, _ptr(out, _F)))
    return out


def parse_layout(path: str, layer: int = 0):
    """The product's layout reader on the host (Parser::parse + getLayerAt +
    getLayerSize): (rects (n, 4) float64 in file order, bounds[4], layers)."""
    n = C.c_int64()
    nl = C.c_int32()
    b = np.zeros(4)
    _check(lib().frw_parse_layout(path.encode(), layer, None, 0, C.byref(n), _ptr(b, _D), C.byref(nl)))
    out = np.zeros((n.value, 4))
    _check(lib().frw_parse_layout(path.encode(), layer, _ptr(out, _D), n.value, C.byref(n), None, None))
    return out, b, int(nl.value)


def write_layout(path: str, rects, name: str = "layer") -> None:
    r = np.ascontiguousarray(rects, dtype=np.float32)
    _check(lib().frw_write_layout(path.encode(), _ptr(r, _F), len(r), name.encode()))


@dataclass
class WalkResult:
    walks: int
    escaped: int
    aborted: int
    hops_total: int
    gauss: np.ndarray
    fraction_other: float
    kernel_ms: float
    conductor: np.ndarray
    hits: np.ndarray
    cap: np.ndarray
    cap_se: np.ndarray
    sum_w: np.ndarray
    sum_w2: np.ndarray
    extra: dict = field(default_factory=dict)

    def row(self, k: int):
        i = np.searchsorted(self.conductor, k)
        if i < len(self.conductor) and self.conductor[i] == k:
            return self.hits[i], self.cap[i], self.cap_se[i]
        return 0, 0.0, 0.0


class Layout:
    """A device-resident layout with its Morton quadtree."""

    def __init__(self, handle, n: int):
        self._h = handle
        self.n = n

    @classmethod
    def from_file(cls, path: str, layer: int = 0, device: int = 0) -> "Layout":
        h = _VP()
        _check(lib().frw_layout_from_file(path.encode(), layer, device, C.byref(h)))
        info = LayoutInfo()
        _check(lib().frw_layout_info_get(h, C.byref(info)))
        return cls(h, info.n_rects)

    @classmethod
    def from_rects(cls, rects, bounds=None, device: int = 0, stream: int = 0) -> "Layout":
        r = np.ascontiguousarray(rects, dtype=np.float32)
        if r.ndim != 2 or r.shape[1] != 4:
            raise ValueError("rects must be (n, 4)")
        b = None if bounds is None else np.ascontiguousarray(bounds, dtype=np.float64)
        h = _VP()
        _check(lib().frw_layout_create(_ptr(r, _F), len(r), _ptr(b, _D), device, stream or None, C.byref(h)))
        return cls(h, len(r))

    def close(self):
        if self._h:
            lib().frw_layout_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def info(self) -> LayoutInfo:
        info = LayoutInfo()
        _check(lib().frw_layout_info_get(self._h, C.byref(info)))
        return info

    @property
    def bounds(self) -> np.ndarray:
        return np.array(self.info.bounds[:])

    def rects(self) -> np.ndarray:
        out = np.zeros((self.n, 4))
        _check(lib().frw_layout_rects(self._h, _ptr(out, _D)))
        return out

    # ---- cell lists
    def set_cells(self, cells_per_rect: float, max_per_cell: int = 32):
        """Rebuild the cell lists (0 removes them: queries use the tree alone)."""
        _check(lib().frw_layout_set_cells(self._h, float(cells_per_rect), int(max_per_cell), None))

    @property
    def cells(self) -> CellsInfo:
        i = CellsInfo()
        _check(lib().frw_layout_cells_info(self._h, C.byref(i)))
        return i

    # ---- queries
    def query(self, pts):
        """drawBiggestSquareAtPoint + checkCollisons(point) for (n,2) points."""
        p = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 2)
        sq = np.zeros((len(p), 4))
        hit = np.zeros(len(p), dtype=np.int64)
        _check(lib().frw_query_batch(self._h, _ptr(p), len(p), _ptr(sq), _ptr(hit), MEM_HOST, None))
        return sq, hit

    def query_device(self, pts_t, sq_t, hit_t, stream: int = 0):
        """Device-resident variant on torch CUDA tensors (no host copies)."""
        _check(lib().frw_query_batch(self._h, C.c_void_p(pts_t.data_ptr()), pts_t.shape[0],
                                     C.c_void_p(sq_t.data_ptr()), C.c_void_p(hit_t.data_ptr()), MEM_DEVICE,
                                     stream or None))

    def draw_biggest_square(self, pts):
        return self.query(pts)[0]

    def check_collisions_point(self, pts):
        return self.query(pts)[1]

    def check_collisions(self, boxes, ignore=None):
        b = np.ascontiguousarray(boxes, dtype=np.float64).reshape(-1, 4)
        ig = None if ignore is None else np.ascontiguousarray(ignore, dtype=np.float64)
        out = np.zeros(len(b), dtype=np.uint8)
        _check(lib().frw_box_collides_batch(self._h, _ptr(b), len(b), _ptr(ig, _D), _ptr(out), MEM_HOST, None))
        return out.astype(bool)

    def gauss_surface(self, target: int, o: Opts | None = None):
        out = np.zeros(4)
        _check(lib().frw_gauss_surface(self._h, target, C.byref(o) if o else None, _ptr(out, _D), None))
        return out

    # ---- walks
    def walk(self, target: int, walks: int, seed: int, o: Opts | None = None, capacity: int | None = None,
             stream: int = 0) -> WalkResult:
        cap = self.n if capacity is None else capacity
        cond = np.zeros(cap, dtype=np.int64)
        hits = np.zeros(cap, dtype=np.uint64)
        c = np.zeros(cap)
        se = np.zeros(cap)
        s1 = np.zeros(cap)
        s2 = np.zeros(cap)
        r = Result()
        r.capacity = cap
        r.conductor = _ptr(cond, _I64)
        r.hits = _ptr(hits, C.POINTER(C.c_uint64))
        r.cap = _ptr(c, _D)
        r.cap_se = _ptr(se, _D)
        r.sum_w = _ptr(s1, _D)
        r.sum_w2 = _ptr(s2, _D)
        _check(lib().frw_walk(self._h, target, walks, seed, C.byref(o) if o else None, C.byref(r), stream or None))
        m = min(r.n_entries, cap)
        return WalkResult(r.walks, r.escaped, r.aborted, r.hops_total, np.array(r.gauss[:]), r.fraction_other,
                          r.kernel_ms, cond[:m], hits[:m], c[:m], se[:m], s1[:m], s2[:m],
                          extra={"n_entries": int(r.n_entries)})

    def walk_device(self, target: int, walks: int, seed: int, o: Opts | None, hits, sum_w, sum_w2, stats, status,
                    stream: int = 0):
        """frw_walk_device on torch CUDA tensors (uint64/float64 rows of n
        entries, uint64 stats[4], int32 status[1]); stream-ordered, no sync."""
        _check(lib().frw_walk_device(self._h, target, walks, seed, C.byref(o) if o else None,
                                     C.c_void_p(hits.data_ptr()), C.c_void_p(sum_w.data_ptr()),
                                     C.c_void_p(sum_w2.data_ptr()), C.c_void_p(stats.data_ptr()),
                                     C.c_void_p(status.data_ptr()), stream or None))

    def rows_compact(self, hits, sum_w, sum_w2, idx, out_hits, out_sum_w, out_sum_w2, count, stream: int = 0):
        """frw_rows_compact on torch CUDA tensors: the nonzero rows of
        frw_walk_device's arrays, at most len(idx) of them, count (uint64[1])
        = how many there are.  Stream-ordered, no sync."""
        _check(lib().frw_rows_compact(self._h, C.c_void_p(hits.data_ptr()), C.c_void_p(sum_w.data_ptr()),
                                      C.c_void_p(sum_w2.data_ptr()), idx.shape[0], C.c_void_p(idx.data_ptr()),
                                      C.c_void_p(out_hits.data_ptr()), C.c_void_p(out_sum_w.data_ptr()),
                                      C.c_void_p(out_sum_w2.data_ptr()), C.c_void_p(count.data_ptr()),
                                      stream or None))

    def cv_features(self, target: int, rec4) -> np.ndarray:
        q = np.ascontiguousarray(rec4, dtype=np.float64).reshape(-1, 4)
        out = np.zeros((len(q), 16), dtype=np.float32)
        _check(lib().frw_cv_features(self._h, target, _ptr(q, _D), len(q), _ptr(out, _F)))
        return out

    def walk_trace(self, target: int, first: int, walks: int, seed: int, o: Opts | None = None):
        end = np.zeros(walks, dtype=np.int64)
        hops = np.zeros(walks, dtype=np.int32)
        b1 = np.zeros(walks, dtype=np.int32)
        w = np.zeros(walks)
        _check(lib().frw_walk_trace(self._h, target, first, walks, seed, C.byref(o) if o else None, _ptr(end),
                                    _ptr(hops), _ptr(b1), _ptr(w), MEM_HOST, None))
        return end, hops, b1, w


class Batch:
    """frw_batch: many (layout, target, walks) jobs in one persistent graph-captured launch."""

    def __init__(self, layouts, targets, walks, o: Opts | None = None):
        self._layouts = list(layouts)  # keep alive
        n = len(self._layouts)
        arr = (_VP * n)(*[L._h for L in self._layouts])
        t = np.ascontiguousarray(targets, dtype=np.int64)
        w = np.ascontiguousarray(walks, dtype=np.uint64)
        self.walks = w
        h = _VP()
        _check(lib().frw_batch_create(arr, _ptr(t, _I64), _ptr(w, C.POINTER(C.c_uint64)), n,
                                      C.byref(o) if o else None, C.byref(h)))
        self._h = h

    def tune(self, trial_walks: int) -> Tuning:
        t = Tuning()
        _check(lib().frw_batch_tune(self._h, trial_walks, C.byref(t)))
        return t

    def set_tuning(self, blocks_per_sm: int, refill_min: int, chunk: int):
        t = Tuning(C.sizeof(Tuning), blocks_per_sm, refill_min, chunk, 0.0)
        _check(lib().frw_batch_set_tuning(self._h, C.byref(t)))

    @property
    def tuning(self) -> Tuning:
        t = Tuning()
        _check(lib().frw_batch_get_tuning(self._h, C.byref(t)))
        return t

    def run(self, seed: int, capacity: int = 64):
        n = len(self._layouts)
        res = (Result * n)()
        keep = []
        for j in range(n):
            cond = np.zeros(capacity, dtype=np.int64)
            hits = np.zeros(capacity, dtype=np.uint64)
            c = np.zeros(capacity)
            se = np.zeros(capacity)
            s1 = np.zeros(capacity)
            s2 = np.zeros(capacity)
            keep.append((cond, hits, c, se, s1, s2))
            r = res[j]
            r.capacity = capacity
            r.conductor = _ptr(cond, _I64)
            r.hits = _ptr(hits, C.POINTER(C.c_uint64))
            r.cap = _ptr(c, _D)
            r.cap_se = _ptr(se, _D)
            r.sum_w = _ptr(s1, _D)
            r.sum_w2 = _ptr(s2, _D)
        _check(lib().frw_batch_run(self._h, seed, res, None))
        out = []
        for j in range(n):
            r = res[j]
            m = min(r.n_entries, capacity)
            cond, hits, c, se, s1, s2 = keep[j]
            out.append(WalkResult(r.walks, r.escaped, r.aborted, r.hops_total, np.array(r.gauss[:]), r.fraction_other,
                                  r.kernel_ms, cond[:m], hits[:m], c[:m], se[:m], s1[:m], s2[:m]))
        return out

    def close(self):
        if self._h:
            lib().frw_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cv_opts(train_walks=1_000_000, train_seed=0x7E57C0DE, epochs=4, batch=32768, lr=6e-3) -> CvOpts:
    o = CvOpts()
    lib().frw_cv_opts_default(C.byref(o))
    o.train_walks, o.train_seed, o.epochs, o.batch, o.lr = train_walks, train_seed, epochs, batch, lr
    return o


class ControlVariate:
    """frw_cv: a trained control variate for C_tt of one layout and target."""

    def __init__(self, layout: "Layout", target: int, walk_opts: Opts, opts: CvOpts | None = None):
        self._layout = layout  # keeps the layout alive
        self._o = walk_opts
        h = _VP()
        _check(lib().frw_cv_train(layout._h, target, C.byref(walk_opts), C.byref(opts) if opts else None,
                                  C.byref(h), None))
        self._h = h

    @property
    def info(self) -> CvInfo:
        i = CvInfo()
        _check(lib().frw_cv_info_get(self._h, C.byref(i)))
        return i

    def walk(self, walks: int, seed: int) -> CvResult:
        r = CvResult()
        _check(lib().frw_cv_walk(self._h, walks, seed, C.byref(r), None))
        return r

    def params(self) -> np.ndarray:
        out = np.zeros(CV_PARAMS, dtype=np.float32)
        _check(lib().frw_cv_params(self._h, _ptr(out, _F)))
        return out

    def close(self):
        if self._h:
            lib().frw_cv_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mlp_forward(params, x, device: int = 0) -> np.ndarray:
    p = np.ascontiguousarray(params, dtype=np.float32)
    xx = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 16)
    out = np.zeros(len(xx), dtype=np.float32)
    _check(lib().frw_mlp_forward(_ptr(p, _F), _ptr(xx, _F), len(xx), _ptr(out, _F), device))
    return out


def mlp_grad(params, x, y, wt, inv_wsum: float, device: int = 0):
    p = np.ascontiguousarray(params, dtype=np.float32)
    xx = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 16)
    yy = np.ascontiguousarray(y, dtype=np.float32)
    ww = np.ascontiguousarray(wt, dtype=np.float32)
    g = np.zeros(CV_PARAMS, dtype=np.float32)
    loss = C.c_double()
    _check(lib().frw_mlp_grad(_ptr(p, _F), _ptr(xx, _F), _ptr(yy, _F), _ptr(ww, _F), len(xx), inv_wsum, _ptr(g, _F),
                              C.byref(loss), device))
    return loss.value, g


def get_avg_path_len_cuda(path: str, iter_num: int, rect_id: int, layer: int = 0, seed: int = 0, device: int = 0,
                          hist_path: str | None = None) -> float:
    """getAvgPathLenCUDA: fraction of walks that did not end on rect_id."""
    out = C.c_double()
    _check(lib().frw_avg_path_len(path.encode(), iter_num, rect_id, layer, seed, device,
                                  hist_path.encode() if hist_path else None, C.byref(out)))
    return out.value


def header_symbols(headers=(HEADER, HEADER3)):
    """Function names declared in include/frw.h and include/frw3d.h."""
    import re

    if isinstance(headers, str):
        headers = (headers,)
    names = set()
    for h in headers:
        txt = open(h).read()
        names |= set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(frw3?_[a-z_0-9]+)\s*\(", txt, re.M))
    return sorted(names)


# ---- 3-D path (include/frw3d.h) ------------------------------------------------
NSAMPLE3 = 50


def cube_green_table(n: int = NSAMPLE3):
    """precompute_unit_cube_green(g, dgdx, dgdy, dgdz, intg, n) (host, FP64)."""
    nb = 6 * n * n
    out = [np.zeros(nb) for _ in range(4)] + [np.zeros(nb + 1)]
    _check(lib().frw3_cube_green_table(n, *[_ptr(a, _D) for a in out]))
    return tuple(out)


def green_cube(a: float, eta: float, dzeta: float) -> float:
    g = C.c_double()
    _check(lib().frw3_green_cube(a, eta, dzeta, C.byref(g)))
    return g.value


def deriv_green_cube(a: float, eta: float, dzeta: float) -> np.ndarray:
    dg = np.zeros(3)
    _check(lib().frw3_deriv_green_cube(a, eta, dzeta, _ptr(dg, _D)))
    return dg


def opts3(gauss_offset=1.0, shell=0.0, hop_cap=100000, permittivity=PERMITTIVITY, stream_id=0, nsample=NSAMPLE3,
          first_walk=0, blocks_per_sm=0, refill_min=4, start_strata=0) -> Opts3:
    o = Opts3()
    lib().frw3_opts_default(C.byref(o))
    o.gauss_offset = gauss_offset
    o.shell = shell
    o.hop_cap = hop_cap
    o.permittivity = permittivity
    o.stream_id = stream_id
    o.nsample = nsample
    o.first_walk = first_walk
    o.blocks_per_sm = blocks_per_sm
    o.refill_min = refill_min
    o.start_strata = start_strata
    return o


def generate_layout3(seed: int, n: int, domain: float, zdomain: float, wmin: int = 5, wmax: int = 50,
                     zmin: int = 5, zmax: int = 50, gap: int = 2) -> np.ndarray:
    out = np.zeros((n, 6), dtype=np.float32)
    _check(lib().frw3_generate_layout(seed, n, domain, zdomain, wmin, wmax, zmin, zmax, gap, _ptr(out, _F)))
    return out


class Layout3:
    """A device-resident 3-D layout (boxes) with its cell grid."""

    def __init__(self, handle, n: int):
        self._h = handle
        self.n = n

    @classmethod
    def from_boxes(cls, boxes, bounds=None, cells_per_box: float = 0.0, device: int = 0) -> "Layout3":
        b = np.ascontiguousarray(boxes, dtype=np.float32)
        if b.ndim != 2 or b.shape[1] != 6:
            raise ValueError("boxes must be (n, 6)")
        bd = None if bounds is None else np.ascontiguousarray(bounds, dtype=np.float64)
        h = _VP()
        _check(lib().frw3_layout_create(_ptr(b, _F), len(b), _ptr(bd, _D), cells_per_box, device, C.byref(h)))
        return cls(h, len(b))

    @classmethod
    def from_file(cls, path: str, z0, z1, bounds=None, cells_per_box: float = 0.0, device: int = 0) -> "Layout3":
        a = np.ascontiguousarray(z0, dtype=np.float64)
        b = np.ascontiguousarray(z1, dtype=np.float64)
        bd = None if bounds is None else np.ascontiguousarray(bounds, dtype=np.float64)
        h = _VP()
        _check(lib().frw3_layout_from_file(path.encode(), _ptr(a, _D), _ptr(b, _D), len(a), _ptr(bd, _D),
                                           cells_per_box, device, C.byref(h)))
        info = Layout3Info()
        _check(lib().frw3_layout_info_get(h, C.byref(info)))
        return cls(h, info.n)

    def close(self):
        if self._h:
            lib().frw3_layout_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def info(self) -> Layout3Info:
        i = Layout3Info()
        _check(lib().frw3_layout_info_get(self._h, C.byref(i)))
        return i

    @property
    def bounds(self) -> np.ndarray:
        return np.array(self.info.bounds[:])

    def boxes(self) -> np.ndarray:
        out = np.zeros((self.n, 6), dtype=np.float32)
        _check(lib().frw3_layout_boxes(self._h, _ptr(out, _F)))
        return out

    def query(self, pts):
        """Clearance (L-infinity distance to the nearest box) and that box for (n,3) points."""
        p = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        d = np.zeros(len(p))
        k = np.zeros(len(p), dtype=np.int64)
        _check(lib().frw3_query_batch(self._h, _ptr(p), len(p), _ptr(d), _ptr(k), MEM_HOST, None))
        return d, k

    def query_device(self, pts_t, clear_t, nearest_t, stream: int = 0):
        _check(lib().frw3_query_batch(self._h, C.c_void_p(pts_t.data_ptr()), pts_t.shape[0],
                                      C.c_void_p(clear_t.data_ptr()), C.c_void_p(nearest_t.data_ptr()), MEM_DEVICE,
                                      stream or None))

    def walk(self, target: int, walks: int, seed: int, o: Opts3 | None = None, capacity: int | None = None,
             stream: int = 0) -> WalkResult:
        o = o or opts3()
        cap = self.n if capacity is None else capacity
        cond = np.zeros(cap, dtype=np.int64)
        hits = np.zeros(cap, dtype=np.uint64)
        c = np.zeros(cap)
        se = np.zeros(cap)
        s1 = np.zeros(cap)
        s2 = np.zeros(cap)
        r = Result3()
        r.capacity = cap
        r.conductor = _ptr(cond, _I64)
        r.hits = _ptr(hits, C.POINTER(C.c_uint64))
        r.cap = _ptr(c, _D)
        r.cap_se = _ptr(se, _D)
        r.sum_w = _ptr(s1, _D)
        r.sum_w2 = _ptr(s2, _D)
        _check(lib().frw3_walk(self._h, target, walks, seed, C.byref(o), C.byref(r), stream or None))
        m = min(r.n_entries, cap)
        return WalkResult(r.walks, r.escaped, r.aborted, r.hops_total, np.array(r.gauss[:]), r.fraction_other,
                          r.kernel_ms, cond[:m], hits[:m], c[:m], se[:m], s1[:m], s2[:m], {"shell": r.shell})

    def walk_batch(self, targets, walks_per_target: int, seed: int, o: Opts3 | None = None,
                   capacity: int | None = None, stream: int = 0):
        """frw3_walk_batch: one WalkResult per target, from one launch."""
        t = np.ascontiguousarray(targets, dtype=np.int64)
        cap = self.n if capacity is None else capacity
        T = len(t)
        arrs = [(np.zeros(cap, np.int64), np.zeros(cap, np.uint64), np.zeros(cap), np.zeros(cap), np.zeros(cap),
                 np.zeros(cap)) for _ in range(T)]
        rs = (Result3 * T)()
        for r, (cond, hits, c, se, s1, s2) in zip(rs, arrs):
            r.capacity = cap
            r.conductor = _ptr(cond, _I64)
            r.hits = _ptr(hits, C.POINTER(C.c_uint64))
            r.cap = _ptr(c, _D)
            r.cap_se = _ptr(se, _D)
            r.sum_w = _ptr(s1, _D)
            r.sum_w2 = _ptr(s2, _D)
        _check(lib().frw3_walk_batch(self._h, _ptr(t, _I64), T, walks_per_target, seed, C.byref(o) if o else None,
                                     rs, stream or None))
        out = []
        for r, (cond, hits, c, se, s1, s2) in zip(rs, arrs):
            m = min(r.n_entries, cap)
            out.append(WalkResult(r.walks, r.escaped, r.aborted, r.hops_total, np.array(r.gauss[:]),
                                  r.fraction_other, r.kernel_ms, cond[:m], hits[:m], c[:m], se[:m], s1[:m], s2[:m],
                                  {"shell": r.shell}))
        return out

    def walk_device(self, target: int, walks: int, seed: int, o: Opts3 | None, hits, sum_w, sum_w2, stats, status,
                    stream: int = 0):
        """frw3_walk_device on torch CUDA tensors (uint64/float64 rows of n
        entries, uint64 stats[4], int32 status[1]); stream-ordered, no sync."""
        _check(lib().frw3_walk_device(self._h, target, walks, seed, C.byref(o) if o else None,
                                      C.c_void_p(hits.data_ptr()), C.c_void_p(sum_w.data_ptr()),
                                      C.c_void_p(sum_w2.data_ptr()), C.c_void_p(stats.data_ptr()),
                                      C.c_void_p(status.data_ptr()), stream or None))

    def walk_trace(self, target: int, first: int, walks: int, seed: int, o: Opts3 | None = None):
        o = o or opts3()
        end = np.zeros(walks, dtype=np.int64)
        hops = np.zeros(walks, dtype=np.int32)
        b1 = np.zeros(walks, dtype=np.int32)
        w = np.zeros(walks)
        _check(lib().frw3_walk_trace(self._h, target, first, walks, seed, C.byref(o), _ptr(end), _ptr(hops),
                                     _ptr(b1), _ptr(w), MEM_HOST, None))
        return end, hops, b1, w
