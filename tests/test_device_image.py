"""The device-image sidecar (HnswIndex.save_device_image / load_device_image): the FP32 device
mirror written in its device layout, every section 4096-byte aligned, named by an XXH64 of the
graph. The host side (layout, contents, the checks that run before any device call) is tested
against a parse of the v1 index file (docs/FORMAT.md of the reference); the GPU side checks that
a mirror installed from the sidecar searches exactly as the uploaded one."""

import struct

import numpy as np
import pytest

from conftest import integer_matrix

NO_ID = 0xFFFFFFFF


def parse_v1(path):
    """The v1 file as arrays: header fields, levels, layer-0 blocks [n, 1 + 2M], upper blocks
    [sum(levels), 1 + M] and vectors [n, dim] (docs/FORMAT.md "Layout" of the reference)."""
    b = path.read_bytes()
    _, metric, dim, M, _, _, n, max_level, entry, blocks = struct.unpack_from("<II8Q", b, 8)
    at = 80
    levels = np.frombuffer(b, np.uint8, n, at)
    at += n
    layer0 = np.frombuffer(b, np.uint32, n * (1 + 2 * M), at).reshape(n, 1 + 2 * M)
    at += layer0.nbytes
    upper = np.frombuffer(b, np.uint32, blocks * (1 + M), at).reshape(blocks, 1 + M)
    at += upper.nbytes
    vectors = np.frombuffer(b, np.float32, n * dim, at).reshape(n, dim)
    return dict(metric=metric, dim=dim, M=M, n=n, max_level=max_level, entry=entry, blocks=blocks,
                levels=levels, layer0=layer0, upper=upper, vectors=vectors)


def padded_blocks(raw, stride):
    """[count, ids...] blocks as the device holds them: the ids, then 0xFFFFFFFF to `stride`."""
    out = np.full((raw.shape[0], stride), NO_ID, np.uint32)
    for i, blk in enumerate(raw):
        out[i, :blk[0]] = blk[1:1 + blk[0]]
    return out


def built_index(vdx, metric, n, dim, M, seed):
    ix = vdx.HnswIndex(dim, metric, M=M, ef_construction=40, seed=seed)
    ix.add(integer_matrix(n, dim, seed) if metric == "l2" else
           np.random.default_rng(seed).standard_normal((n, dim)).astype(np.float32), num_threads=1)
    return ix


@pytest.mark.parametrize("metric,dim,M", [("l2", 13, 6), ("cosine", 16, 8), ("ip", 5, 3)])
def test_sidecar_holds_the_device_layout_of_the_graph(vdx, tmp_path, metric, dim, M):
    ix = built_index(vdx, metric, 700, dim, M, seed=5)
    ix.save(tmp_path / "g.vdx")
    ix.save_device_image(tmp_path / "g.vdxdev")
    g = parse_v1(tmp_path / "g.vdx")
    b = (tmp_path / "g.vdxdev").read_bytes()
    assert b[:8] == b"VDXDEV01"
    version, metric_code, n, dim_, row32, M_, stride0, stride_up, max_level, entry, _, blocks, digest = \
        struct.unpack_from("<IIQIIIIIIIIQQ", b, 8)
    assert (version, metric_code, n, dim_, M_, max_level, entry, blocks) == \
        (1, g["metric"], g["n"], g["dim"], g["M"], g["max_level"], g["entry"], g["blocks"])
    assert (row32, stride0, stride_up) == (-(-dim // 4) * 4, -(-2 * M // 4) * 4, -(-M // 4) * 4)
    assert digest == vdx.xxh64(g["vectors"].tobytes() + g["levels"].tobytes() + g["layer0"].tobytes()
                               + g["upper"].tobytes())
    sections = [struct.unpack_from("<QQ", b, 72 + 16 * i) for i in range(4)]
    assert all(off % 4096 == 0 for off, _ in sections)
    assert sections[0][0] == 4096
    for (off, size), (nxt, _) in zip(sections, sections[1:]):
        assert off + size <= nxt < off + size + 4096
    assert len(b) == sections[3][0] + sections[3][1]

    def section(i, dtype, cols):
        off, size = sections[i]
        return np.frombuffer(b, dtype, size // np.dtype(dtype).itemsize, off).reshape(-1, cols)

    rows = np.zeros((n, row32), np.float32)
    rows[:, :dim] = g["vectors"]
    np.testing.assert_array_equal(section(0, np.float32, row32).view(np.uint32), rows.view(np.uint32))
    np.testing.assert_array_equal(section(1, np.uint32, stride0), padded_blocks(g["layer0"], stride0))
    first = np.concatenate([[0], np.cumsum(g["levels"].astype(np.uint64))[:-1]]).astype(np.uint32)
    np.testing.assert_array_equal(section(2, np.uint32, 1).ravel(), first)
    np.testing.assert_array_equal(section(3, np.uint32, stride_up), padded_blocks(g["upper"], stride_up))
    assert ix.graph_hash() == digest


def test_sidecar_of_another_graph_or_file_is_refused_before_any_device_call(vdx, tmp_path):
    a = built_index(vdx, "l2", 400, 8, 4, seed=1)
    b = built_index(vdx, "l2", 400, 8, 4, seed=2)
    a.save_device_image(tmp_path / "a.vdxdev")
    with pytest.raises(OSError, match="belongs to another graph"):
        b.load_device_image(tmp_path / "a.vdxdev")
    # Same shape and same graph except one link: the hash tells them apart.
    a.save(tmp_path / "a.vdx")
    raw = bytearray((tmp_path / "a.vdxdev").read_bytes())
    raw[64:72] = struct.pack("<Q", struct.unpack_from("<Q", raw, 64)[0] ^ 1)
    (tmp_path / "bad.vdxdev").write_bytes(bytes(raw))
    with pytest.raises(OSError, match="belongs to another graph"):
        vdx.HnswIndex.load(tmp_path / "a.vdx").load_device_image(tmp_path / "bad.vdxdev")
    raw = bytearray((tmp_path / "a.vdxdev").read_bytes())
    raw[8:12] = struct.pack("<I", 2)
    (tmp_path / "v2.vdxdev").write_bytes(bytes(raw))
    with pytest.raises(OSError, match="version 2 is not supported"):
        a.load_device_image(tmp_path / "v2.vdxdev")
    (tmp_path / "other").write_bytes(b"\0" * 5000)
    with pytest.raises(OSError, match="not a vdx device image"):
        a.load_device_image(tmp_path / "other")
    with pytest.raises(OSError, match="cannot open"):
        a.load_device_image(tmp_path / "missing")
    # An index grown after the sidecar was written no longer matches it.
    a.add(integer_matrix(3, 8, 9))
    with pytest.raises(OSError, match="belongs to another graph"):
        a.load_device_image(tmp_path / "a.vdxdev")


@pytest.mark.gpu
@pytest.mark.parametrize("metric", ["l2", "cosine"])
def test_mirror_from_the_sidecar_searches_as_the_uploaded_one(gpu, tmp_path, metric):
    ix = built_index(gpu, metric, 3000, 20, 8, seed=7)
    queries = integer_matrix(200, 20, 8) if metric == "l2" else \
        np.random.default_rng(8).standard_normal((200, 20)).astype(np.float32)
    ix.save(tmp_path / "g.vdx")
    ix.save_device_image(tmp_path / "g.vdxdev")
    want = ix.search_batch(queries, 10, 48)
    cold = gpu.HnswIndex.load(tmp_path / "g.vdx")
    cold.load_device_image(tmp_path / "g.vdxdev", 0)
    got = cold.search_batch(queries, 10, 48)
    for x, y in zip(got, want):
        np.testing.assert_array_equal(np.asarray(x).view(np.uint32), np.asarray(y).view(np.uint32))
    # A truncated sidecar is refused and leaves the index searchable (uploaded the usual way).
    data = (tmp_path / "g.vdxdev").read_bytes()
    (tmp_path / "cut.vdxdev").write_bytes(data[:len(data) - 100])
    fresh = gpu.HnswIndex.load(tmp_path / "g.vdx")
    with pytest.raises(OSError, match="truncated"):
        fresh.load_device_image(tmp_path / "cut.vdxdev", 0)
    for x, y in zip(fresh.search_batch(queries, 10, 48), want):
        np.testing.assert_array_equal(np.asarray(x).view(np.uint32), np.asarray(y).view(np.uint32))
