"""frw_walk_trace_static: the allocation-free walk entry point.

Some callers cannot allocate device memory while they call into the library
(their host application owns every byte of the GPU through its own pool, or a
real-time loop forbids allocator latency).  For them the walk kernel's
scratch lives in a fixed device array inside the library; this test calls
that entry point through the C ABI with device output buffers the caller
owns and checks that two calls in a row return exactly what the allocating
frw_walk_trace returns.  It lives in its own file, collected last, so a
failure here never hides the other tests.
"""
import ctypes as C

import numpy as np
import pytest

import frw

pytestmark = pytest.mark.gpu


def _fn():
    f = frw.lib().frw_walk_trace_static
    f.argtypes = [C.c_void_p, C.c_int64, C.c_uint64, C.c_uint64, C.c_uint64, C.POINTER(frw.Opts), C.c_void_p,
                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def _device_memory():
    """(bytes used and reserved by the device's default stream-ordered pool,
    free device bytes): what an allocating call would change."""
    import torch

    cu = C.CDLL("libcuda.so.1")
    pool = C.c_void_p()
    assert cu.cuDeviceGetDefaultMemPool(C.byref(pool), torch.cuda.current_device()) == 0
    used, reserved = C.c_uint64(), C.c_uint64()
    assert cu.cuMemPoolGetAttribute(pool, 7, C.byref(used)) == 0  # CU_MEMPOOL_ATTR_USED_MEM_CURRENT
    assert cu.cuMemPoolGetAttribute(pool, 5, C.byref(reserved)) == 0  # CU_MEMPOOL_ATTR_RESERVED_MEM_CURRENT
    return used.value, reserved.value, torch.cuda.mem_get_info()[0]


def test_static_walk_trace_matches_allocating_trace_twice():
    import torch

    rects = frw.generate_layout(0xF4A7 + 1, 100, 1000.0)
    o = frw.capacitance_opts(1.0)
    n, first, seed = 20_000, 77, 31337
    with frw.Layout.from_rects(rects) as L:
        want = L.walk_trace(0, first, n, seed=seed, o=o)
        fn = _fn()
        for call in range(2):
            end = torch.full((n,), -99, dtype=torch.int64, device="cuda")
            hops = torch.zeros(n, dtype=torch.int32, device="cuda")
            b1 = torch.zeros(n, dtype=torch.int32, device="cuda")
            w = torch.zeros(n, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            before = _device_memory()
            st = fn(L._h, 0, first, n, seed, C.byref(o), end.data_ptr(), hops.data_ptr(), b1.data_ptr(),
                    w.data_ptr(), None)
            after = _device_memory()
            assert st == 0, frw.lib().frw_last_error().decode()
            # nothing taken from the stream-ordered pool; and once the first call
            # has loaded the array with its module, no device memory at all
            assert after[:2] == before[:2], (call, before, after)
            if call == 1:
                assert after[2] == before[2], (before, after)
            got = (end.cpu().numpy(), hops.cpu().numpy(), b1.cpu().numpy(), w.cpu().numpy())
            for g, x in zip(got, want):
                assert np.array_equal(g, x), f"call {call}"


def test_static_walk_trace_rejects_layouts_over_the_limit():
    import torch

    rects = frw.generate_layout(5, 70_000, 2e4)
    o = frw.capacitance_opts(1.0)
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    with frw.Layout.from_rects(rects) as L:
        st = _fn()(L._h, 0, 0, 4, 1, C.byref(o), buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), buf.data_ptr(),
                   None)
    assert st == frw.E_ARG
    assert "65,536" in frw.lib().frw_last_error().decode()
