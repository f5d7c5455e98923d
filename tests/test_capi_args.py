"""Argument checks of the device-buffer search entry points, made on the host before any device
call: a NULL buffer, a result row narrower than k, or the learned stop on the entry point that
allocates nothing come back as VDX_ERR_INVALID_ARGUMENT with no launch (no GPU needed)."""

import ctypes
from pathlib import Path

import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
P, U64, U32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32
FAKE = 0x1000  # never dereferenced: every call below is rejected before it reaches the device


def bind(lib):
    noalloc = lib.vdx_search_batch_device_noalloc
    noalloc.restype = ctypes.c_int
    noalloc.argtypes = [P, P, U64, U64, P, P, U32, U32, U32, P, P, P, P, P]
    device = lib.vdx_search_batch_device
    device.restype = ctypes.c_int
    device.argtypes = [P, P, U64, U64, P, P, U32, U32, U32, P, P, P, P, P, P]
    return noalloc, device


@pytest.mark.parametrize("missing", ["d_queries", "d_ids", "d_dists", "d_counts"])
def test_null_buffers_are_rejected(vdx, missing):
    lib = vdx.lib()
    noalloc, device = bind(lib)
    ix = vdx.HnswIndex.load(GOLDEN / "kat_m8.vdx")
    bufs = {n: (None if n == missing else FAKE) for n in ("d_queries", "d_ids", "d_dists", "d_counts")}
    opts = vdx.SearchOptions(0, 0, 0, 0.5, 0)
    st = noalloc(ix.handle, bufs["d_queries"], 4, 16, None, None, 10, 40, 10, bufs["d_ids"],
                 bufs["d_dists"], bufs["d_counts"], ctypes.byref(opts), None)
    assert st == 1 and f"{missing} is NULL" in lib.vdx_last_error().decode()
    st = device(ix.handle, bufs["d_queries"], 4, 16, None, None, 10, 40, 10, bufs["d_ids"],
                bufs["d_dists"], bufs["d_counts"], FAKE, ctypes.byref(opts), None)
    assert st == 1 and f"{missing} is NULL" in lib.vdx_last_error().decode()


def test_narrow_rows_and_learned_stop_are_rejected(vdx):
    lib = vdx.lib()
    noalloc, device = bind(lib)
    ix = vdx.HnswIndex.load(GOLDEN / "kat_m8.vdx")
    opts = vdx.SearchOptions(0, 0, 0, 0.5, 0)
    st = noalloc(ix.handle, FAKE, 4, 16, None, None, 10, 40, 8, FAKE, FAKE, FAKE,
                 ctypes.byref(opts), None)
    assert st == 1 and "out_stride is smaller than k" in lib.vdx_last_error().decode()
    st = device(ix.handle, FAKE, 4, 16, None, None, 10, 40, 8, FAKE, FAKE, FAKE, FAKE,
                ctypes.byref(opts), None)
    assert st == 1 and "out_stride is smaller than k" in lib.vdx_last_error().decode()
    learned = vdx.SearchOptions(1, 0, 1, 0.5, 0)
    st = noalloc(ix.handle, FAKE, 4, 16, None, None, 10, 40, 10, FAKE, FAKE, FAKE,
                 ctypes.byref(learned), None)
    assert st == 1 and "learned stop" in lib.vdx_last_error().decode()
