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


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
@pytest.mark.parametrize("per_query", [False, True])
@pytest.mark.parametrize("ef", [40, 200])
def test_noalloc_entry_point_matches_the_work_buffer_entry_point(gpu, precision, per_query, ef):
    """Both entry points on the same queries: uniform or per-query k / ef, FP32 or BF16 rows
    (with the default FP32 re-rank), a register result list (ef 40) or a shared-memory one
    (ef 200). Bit-exact, the tolerance of every search parity test here."""
    torch = pytest.importorskip("torch")
    lib = gpu.lib()
    noalloc = bind_noalloc(lib)
    ix = gpu.HnswIndex.load(GOLDEN / "kat_m8.vdx")
    ix.upload(0, precision)
    dev = torch.device("cuda:0")
    queries = integer_matrix(200, 16, 2)
    nq, k = len(queries), 10
    q = torch.from_numpy(queries).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    code = {"fp32": 0, "bf16": 1}[precision]
    k_t = ef_t = None
    if per_query:
        rng = np.random.default_rng(ef)
        ks = rng.integers(1, k + 1, size=nq).astype(np.int32)
        efs = (ks + rng.integers(0, ef - k + 1, size=nq)).astype(np.int32)
        k_t = torch.from_numpy(ks).to(dev)
        ef_t = torch.from_numpy(efs).to(dev)

    # The existing entry point, with its caller-allocated work buffer.
    ids0 = torch.empty((nq, k), dtype=torch.int32, device=dev)
    d0 = torch.empty((nq, k), dtype=torch.float32, device=dev)
    c0 = torch.empty(nq, dtype=torch.int32, device=dev)
    work = torch.zeros(int(lib.vdx_work_words()), dtype=torch.int32, device=dev)
    ix.search_batch_device(q, k, ef, k, ids0, d0, c0, work, k_per_query=k_t, ef_per_query=ef_t,
                           stream=stream, precision=precision)
    torch.cuda.synchronize()
    assert int(work[0].item()) == 0

    opts = gpu.SearchOptions(code, 0, 0, 0.5, 0)
    kp = None if k_t is None else k_t.data_ptr()
    ep = None if ef_t is None else ef_t.data_ptr()
    for call in range(2):
        ids = torch.full((nq, k), -7, dtype=torch.int32, device=dev)
        d = torch.full((nq, k), -7.0, dtype=torch.float32, device=dev)
        c = torch.full((nq,), -7, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        status = noalloc(ix.handle, q.data_ptr(), nq, queries.shape[1], kp, ep, k, ef, k,
                         ids.data_ptr(), d.data_ptr(), c.data_ptr(), ctypes.byref(opts), stream)
        assert status == 0, lib.vdx_last_error().decode()
        torch.cuda.synchronize()
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


def test_noalloc_entry_point_empty_batch_and_ef_above_capacity(gpu):
    """nq = 0 succeeds and touches no result buffer; a per-query ef beyond the result capacity
    the uniform ef sets (next power of two >= max(ef, 32)) fails that row with the capacity
    error, as vdx_search_batch_device reports it, and the next call succeeds."""
    torch = pytest.importorskip("torch")
    lib = gpu.lib()
    noalloc = bind_noalloc(lib)
    ix = gpu.HnswIndex.load(GOLDEN / "kat_m8.vdx")
    ix.upload(0, "fp32")
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev).cuda_stream
    opts = gpu.SearchOptions(0, 0, 0, 0.5, 0)
    queries = integer_matrix(16, 16, 4)
    q = torch.from_numpy(queries).to(dev)
    ids = torch.full((16, 10), -7, dtype=torch.int32, device=dev)
    d = torch.full((16, 10), -7.0, dtype=torch.float32, device=dev)
    c = torch.full((16,), -7, dtype=torch.int32, device=dev)

    status = noalloc(ix.handle, q.data_ptr(), 0, 16, None, None, 10, 40, 10, ids.data_ptr(),
                     d.data_ptr(), c.data_ptr(), ctypes.byref(opts), stream)
    assert status == 0, lib.vdx_last_error().decode()
    torch.cuda.synchronize()
    assert int((c == -7).sum().item()) == 16 and int((ids == -7).sum().item()) == 160

    efs = torch.full((16,), 40, dtype=torch.int32, device=dev)
    efs[9] = 65  # the uniform ef 40 sets a capacity of 64
    ks = torch.full((16,), 10, dtype=torch.int32, device=dev)
    status = noalloc(ix.handle, q.data_ptr(), 16, 16, ks.data_ptr(), efs.data_ptr(), 10, 40, 10,
                     ids.data_ptr(), d.data_ptr(), c.data_ptr(), ctypes.byref(opts), stream)
    assert status == 1
    assert "ef exceeds the GPU search capacity" in lib.vdx_last_error().decode()
    torch.cuda.synchronize()
    assert int(c[9].item()) == 0

    status = noalloc(ix.handle, q.data_ptr(), 16, 16, None, None, 10, 40, 10, ids.data_ptr(),
                     d.data_ptr(), c.data_ptr(), ctypes.byref(opts), stream)
    assert status == 0, lib.vdx_last_error().decode()
    torch.cuda.synchronize()
    assert int(c.min().item()) == 10
