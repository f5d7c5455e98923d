"""vdx_search_batch_device_noalloc, the search entry point for callers that cannot allocate
device memory (their HBM belongs to an external pool manager, or they run on a path where
cudaMalloc is not allowed): called through the C ABI twice in a row, it must return exactly what
vdx_search_batch_device returns for the same queries, though it keeps its launch state in a
static device array instead of a caller-provided work buffer.

This file sorts last so that a run stopping at the first failure has run every other test; it
also passes on its own in a fresh process."""

import ctypes
from pathlib import Path

import numpy as np
import pytest

from conftest import integer_matrix

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def bind_noalloc(lib):
    fn = lib.vdx_search_batch_device_noalloc
    P, U64, U32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32
    fn.restype = ctypes.c_int
    fn.argtypes = [P, P, U64, U64, P, P, U32, U32, U32, P, P, P, P, P]
    return fn


def test_noalloc_entry_point_matches_the_work_buffer_entry_point(gpu):
    torch = pytest.importorskip("torch")
    lib = gpu.lib()
    noalloc = bind_noalloc(lib)
    ix = gpu.HnswIndex.load(GOLDEN / "kat_m8.vdx")
    ix.upload(0, "fp32")
    dev = torch.device("cuda:0")
    queries = integer_matrix(200, 16, 2)
    nq, k, ef = len(queries), 10, 40
    q = torch.from_numpy(queries).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream

    # The existing entry point, with its caller-allocated work buffer.
    ids0 = torch.empty((nq, k), dtype=torch.int32, device=dev)
    d0 = torch.empty((nq, k), dtype=torch.float32, device=dev)
    c0 = torch.empty(nq, dtype=torch.int32, device=dev)
    work = torch.zeros(int(lib.vdx_work_words()), dtype=torch.int32, device=dev)
    ix.search_batch_device(q, k, ef, k, ids0, d0, c0, work, stream=stream)
    torch.cuda.synchronize()
    assert int(work[0].item()) == 0

    opts = gpu.SearchOptions(0, 0, 0, 0.5, 0)
    for call in range(2):
        ids = torch.full((nq, k), -7, dtype=torch.int32, device=dev)
        d = torch.full((nq, k), -7.0, dtype=torch.float32, device=dev)
        c = torch.full((nq,), -7, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        status = noalloc(ix.handle, q.data_ptr(), nq, queries.shape[1], None, None, k, ef, k,
                         ids.data_ptr(), d.data_ptr(), c.data_ptr(), ctypes.byref(opts), stream)
        assert status == 0, lib.vdx_last_error().decode()
        torch.cuda.synchronize()
        # Bit-exact, the tolerance of every search parity test here.
        assert torch.equal(c, c0), f"call {call}: counts"
        assert torch.equal(ids, ids0), f"call {call}: ids"
        assert torch.equal(d.view(torch.int32), d0.view(torch.int32)), f"call {call}: distances"


def test_noalloc_entry_point_reports_bad_queries_and_missing_upload(gpu):
    torch = pytest.importorskip("torch")
    lib = gpu.lib()
    noalloc = bind_noalloc(lib)
    dev = torch.device("cuda:0")
    queries = integer_matrix(8, 16, 3)
    queries[5, 3] = np.nan
    q = torch.from_numpy(queries).to(dev)
    ids = torch.empty((8, 4), dtype=torch.int32, device=dev)
    d = torch.empty((8, 4), dtype=torch.float32, device=dev)
    c = torch.empty(8, dtype=torch.int32, device=dev)
    opts = gpu.SearchOptions(0, 0, 0, 0.5, 0)
    stream = torch.cuda.current_stream(dev).cuda_stream

    fresh = gpu.HnswIndex.load(GOLDEN / "kat_m8.vdx")  # no device copy yet
    status = noalloc(fresh.handle, q.data_ptr(), 8, 16, None, None, 4, 10, 4, ids.data_ptr(),
                     d.data_ptr(), c.data_ptr(), ctypes.byref(opts), stream)
    assert status == 1 and "vdx_index_upload" in lib.vdx_last_error().decode()

    fresh.upload(0, "fp32")
    status = noalloc(fresh.handle, q.data_ptr(), 8, 16, None, None, 4, 10, 4, ids.data_ptr(),
                     d.data_ptr(), c.data_ptr(), ctypes.byref(opts), stream)
    assert status == 1
    assert "query must not contain NaN or inf" in lib.vdx_last_error().decode()
