"""The product's host side on the CPU: the C ABI loads and exports what include/vdx_b200.h
declares; graph construction equals the reference's byte for byte; the file reader accepts every
file the reference writes and rejects what it rejects, with its messages; host distance kernels
and the checksum match the reference. No GPU is used here."""

import re
import struct
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, integer_matrix, uniform_matrix

GOLDEN = Path(__file__).resolve().parent / "golden"
HEADER = ROOT / "include" / "vdx_b200.h"

# Header field offsets (docs/FORMAT.md "Header" of the reference).
VERSION_AT, METRIC_AT, DIM_AT, M_AT, EFC_AT, SEED_AT = 8, 12, 16, 24, 32, 40
NODES_AT, MAXLEVEL_AT, ENTRY_AT, UPPER_AT = 48, 56, 64, 72


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"VDX_API\s+[\w\s\*]+?\b(vdx_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(vdx):
    names = declared_symbols()
    assert len(names) >= 20
    lib = vdx.lib()
    for name in names:
        assert hasattr(lib, name), name


def test_xxh64_reference_vectors(vdx):
    """XSUM_XXH64_testdata of xxHash v0.8.3, as tests/xxhash64_test.cpp:34-101 uses them."""
    prime32, prime64 = 2654435761, 11400714785074694797
    buf = bytearray()
    gen = prime32
    for _ in range(222):
        buf.append(gen >> 56)
        gen = (gen * prime64) & 0xFFFFFFFFFFFFFFFF
    cases = [(0, 0, 0xEF46DB3751D8E999), (0, prime32, 0xAC75FDA2929B17EF),
             (1, 0, 0xE934A84ADB052768), (1, prime32, 0x5014607643A9B4C3),
             (4, 0, 0x9136A0DCA57457EE), (14, 0, 0x8282DCC4994E35C8),
             (14, prime32, 0xC3BD6BF63DEB6DF0), (222, 0, 0xB641AE8CB691C174),
             (222, prime32, 0x20CB8AB7AE10C14A)]
    for length, seed, want in cases:
        assert vdx.xxh64(bytes(buf[:length]), seed) == want


def test_host_distances_are_bitwise_the_references(vdx):
    g = np.load(GOLDEN / "kat_results.npz")
    for a, b, dim, l2, ip in zip(g["pair_a"], g["pair_b"], g["pair_dim"], g["pair_l2"], g["pair_ip"]):
        assert np.float32(vdx.host_l2(a[:dim], b[:dim])) == l2, dim
        assert np.float32(vdx.host_ip(a[:dim], b[:dim])) == ip, dim


def test_loads_the_reference_graph(vdx):
    ix = vdx.HnswIndex.load(GOLDEN / "kat_m8.vdx")
    info = ix.info()
    assert (info["size"], info["dim"], info["M"], info["ef_construction"], info["seed"]) == (1000, 16, 8, 64, 42)
    rep = ix.inspect()
    assert rep["violations"] == 0 and rep["max_level"] == 3
    assert round(rep["mean_degree0"] * 1000) == 11157


def test_serial_build_is_byte_identical_to_the_references(vdx, tmp_path):
    base = integer_matrix(1000, 16, 1)
    ix = vdx.HnswIndex(16, "l2", M=8, ef_construction=64, seed=42)
    ix.add(base, num_threads=1)
    ix.save(tmp_path / "mine.vdx")
    assert (tmp_path / "mine.vdx").read_bytes() == (GOLDEN / "kat_m8.vdx").read_bytes()
    one = vdx.HnswIndex(16, "l2", M=8, ef_construction=64, seed=42)
    for row in base:
        one.add_one(row)
    one.save(tmp_path / "one.vdx")
    assert (tmp_path / "one.vdx").read_bytes() == (GOLDEN / "kat_m8.vdx").read_bytes()


@pytest.mark.parametrize("metric", [0, 1, 2])
def test_serial_build_matches_reference_on_real_valued_data(vdx, orc, tmp_path, metric):
    base = uniform_matrix(800, 13, 5)
    ref = orc.RefHnsw(13, metric, 6, 30, 7)
    ref.add(base, threads=1)
    ref.save(tmp_path / "ref.vdx")
    mine = vdx.HnswIndex(13, metric, M=6, ef_construction=30, seed=7)
    mine.add(base, num_threads=1)
    mine.save(tmp_path / "mine.vdx")
    assert (tmp_path / "mine.vdx").read_bytes() == (tmp_path / "ref.vdx").read_bytes()
    # memory_bytes (src/hnsw.cpp:207-214 of the reference) on the built and on a loaded graph.
    assert mine.info()["memory_bytes"] == ref.info()["memory_bytes"]
    assert vdx.HnswIndex.load(tmp_path / "ref.vdx").info()["memory_bytes"] == ref.info()["memory_bytes"]


@pytest.mark.parametrize("metric", [0, 1, 2])
def test_serial_build_matches_reference_under_heavy_ties(vdx, orc, tmp_path, metric):
    """Values in {1, 2, 3} over 6 dims: most distances tie, so every choice the build makes
    between equal distances (beam order, eviction, the heuristic's strict test, the greedy walk's
    first strict minimum) shows in the saved file."""
    base = np.random.default_rng(11).integers(1, 4, size=(1500, 6)).astype(np.float32)
    ref = orc.RefHnsw(6, metric, 4, 20, 3)
    ref.add(base, threads=1)
    ref.save(tmp_path / "ref.vdx")
    mine = vdx.HnswIndex(6, metric, M=4, ef_construction=20, seed=3)
    mine.add(base, num_threads=1)
    mine.save(tmp_path / "mine.vdx")
    assert (tmp_path / "mine.vdx").read_bytes() == (tmp_path / "ref.vdx").read_bytes()


def test_files_round_trip_both_ways(vdx, orc, tmp_path):
    mine = vdx.HnswIndex.load(GOLDEN / "kat_m8.vdx")
    mine.save(tmp_path / "again.vdx")
    assert (tmp_path / "again.vdx").read_bytes() == (GOLDEN / "kat_m8.vdx").read_bytes()
    back = orc.RefHnsw.load(tmp_path / "again.vdx")
    assert back.inspect()["violations"] == 0


def test_add_after_load_builds_the_same_graph(vdx, tmp_path):
    first, second = uniform_matrix(300, 8, 1), uniform_matrix(200, 8, 2)
    direct = vdx.HnswIndex(8, "l2", M=8, ef_construction=40)
    direct.add(first)
    direct.save(tmp_path / "half.vdx")
    direct.add(second)
    resumed = vdx.HnswIndex.load(tmp_path / "half.vdx")
    resumed.add(second)
    direct.save(tmp_path / "d.vdx")
    resumed.save(tmp_path / "r.vdx")
    assert (tmp_path / "d.vdx").read_bytes() == (tmp_path / "r.vdx").read_bytes()


def test_parallel_build_is_healthy(vdx):
    base = integer_matrix(3000, 16, 1)
    serial = vdx.HnswIndex(16, "l2", M=16, ef_construction=64)
    serial.add(base, num_threads=1)
    for threads in (2, 4, 8):
        ix = vdx.HnswIndex(16, "l2", M=16, ef_construction=64)
        ix.add(base, num_threads=threads)
        rep = ix.inspect()
        assert rep["violations"] == 0, rep["first_violation"]
        assert rep["reachable"] >= 3000 - 3
        assert rep["max_level"] == serial.inspect()["max_level"]


def test_empty_index_round_trips(vdx, tmp_path):
    ix = vdx.HnswIndex(5, "cosine", M=6, ef_construction=30)
    ix.save(tmp_path / "e.vdx")
    back = vdx.HnswIndex.load(tmp_path / "e.vdx")
    info = back.info()
    assert (info["size"], info["dim"], info["metric"], info["M"]) == (0, 5, 2, 6)


def test_bad_parameters_and_vectors_are_rejected(vdx):
    with pytest.raises(ValueError, match="M must be at least 2"):
        vdx.HnswIndex(4, M=1)
    with pytest.raises(ValueError, match="at most 10000"):
        vdx.HnswIndex(4, M=10001)
    with pytest.raises(ValueError, match="ef_construction must be positive"):
        vdx.HnswIndex(4, ef_construction=0)
    with pytest.raises(ValueError, match="dim must be positive"):
        vdx.HnswIndex(0)
    ix = vdx.HnswIndex(2)
    ix.add_one([1.0, 2.0])
    with pytest.raises(ValueError, match="HnswIndex::add: got dimension 3, index has 2"):
        ix.add_one([1.0, 2.0, 3.0])
    with pytest.raises(ValueError, match="must not contain NaN or inf"):
        ix.add(np.array([[0.0, 1.0], [np.nan, 0.0]], np.float32))
    assert len(ix) == 1
    cos = vdx.HnswIndex(2, "cosine")
    with pytest.raises(ValueError, match="zero length"):
        cos.add_one([0.0, 0.0])


# --- the reader against hostile files (tests/hnsw_io_test.cpp:422-647 of the reference) --------

def tiny_bytes():
    return bytearray((GOLDEN / "tiny.vdx").read_bytes())


def reseal(vdx, b: bytearray) -> bytearray:
    b[-8:] = struct.pack("<Q", vdx.xxh64(bytes(b[:-8])))
    return b


def rejected(vdx, path: Path, data: bytes, reason: str) -> None:
    path.write_bytes(bytes(data))
    with pytest.raises(OSError) as e:
        vdx.HnswIndex.load(path)
    msg = str(e.value)
    assert str(path) in msg, msg
    assert reason in msg, msg


def test_tiny_header_is_the_documented_example():
    """docs/FORMAT.md "Example": dim 2, M 2, ef_construction 8, seed 42, n 12, max level 3,
    entry point 4, U 10, 556 bytes."""
    b = tiny_bytes()
    assert len(b) == 556
    assert b[:8] == b"\x89VDXHNSW"
    assert struct.unpack("<II8Q", bytes(b[8:80])) == (1, 0, 2, 2, 8, 42, 12, 3, 4, 10)


def test_every_truncation_is_rejected(vdx, tmp_path):
    b = tiny_bytes()
    for length in range(len(b)):
        reason = "too small" if length < 88 else "truncated or corrupted"
        rejected(vdx, tmp_path / "cut.vdx", b[:length], reason)


def test_every_flipped_bit_is_rejected(vdx, tmp_path):
    b = tiny_bytes()
    p = tmp_path / "flip.vdx"
    for off in range(len(b)):
        for bit in range(8):
            f = bytearray(b)
            f[off] ^= 1 << bit
            rejected(vdx, p, f, "")


def put(b: bytearray, off: int, fmt: str, v) -> None:
    b[off:off + struct.calcsize(fmt)] = struct.pack(fmt, v)


def test_hostile_header_fields_are_rejected(vdx, tmp_path):
    nodes = 12
    cases = [(VERSION_AT, "<I", 0, "format version 0 is not supported"),
             (VERSION_AT, "<I", 2, "format version 2 is not supported"),
             (METRIC_AT, "<I", 3, "unknown metric code 3"),
             (DIM_AT, "<Q", 0, "dimension is 0"),
             (M_AT, "<Q", 1, "below the minimum of 2"),
             (M_AT, "<Q", 10001, "above the maximum of 10000"),
             (M_AT, "<Q", 1 << 40, "above the maximum of 10000"),
             (EFC_AT, "<Q", 0, "ef_construction is 0"),
             (NODES_AT, "<Q", 1 << 32, "more than 32-bit ids can address"),
             (NODES_AT, "<Q", nodes + 1, "truncated or corrupted"),
             (NODES_AT, "<Q", nodes - 1, "truncated or corrupted"),
             (MAXLEVEL_AT, "<Q", 256, "above 255"),
             (ENTRY_AT, "<Q", nodes, "is not one of the"),
             (UPPER_AT, "<Q", 0, "truncated or corrupted"),
             (DIM_AT, "<Q", 1 << 62, "overflow 64 bits"),
             (UPPER_AT, "<Q", 1 << 62, "overflow 64 bits")]
    for off, fmt, value, reason in cases:
        b = tiny_bytes()
        put(b, off, fmt, value)
        rejected(vdx, tmp_path / "bad.vdx", reseal(vdx, b), reason)


def test_hostile_graphs_are_rejected(vdx, tmp_path):
    b0 = tiny_bytes()
    n, M = 12, 2
    levels = list(b0[80:80 + n])
    layer0_at = 80 + n
    upper_at = layer0_at + n * (1 + 2 * M) * 4
    vectors_at = upper_at + sum(levels) * (1 + M) * 4

    def block(node):
        return layer0_at + node * (1 + 2 * M) * 4

    def upper_block(node, layer):
        return upper_at + (sum(levels[:node]) + layer - 1) * (1 + M) * 4

    linked = next(i for i in range(n) if struct.unpack_from("<I", b0, block(i))[0] >= 2)
    ground = next(i for i in range(n) if levels[i] == 0)
    low = next(i for i in range(n) if levels[i] < 3)
    up = next(i for i in range(n) if levels[i] >= 1 and struct.unpack_from("<I", b0, upper_block(i, 1))[0] > 0)
    blk = block(linked)
    first_id = struct.unpack_from("<I", b0, blk + 4)[0]
    cases = [
        (lambda b: put(b, 80 + ground, "<B", 255), "above the max level"),
        (lambda b: put(b, 80 + ground, "<B", 1), "the levels add up to"),
        (lambda b: put(b, ENTRY_AT, "<Q", low), "not the max level"),
        (lambda b: put(b, blk, "<I", 2 * M + 1), "links on layer 0 (max"),
        (lambda b: put(b, blk + 4, "<I", n), "but there are only"),
        (lambda b: put(b, blk + 4, "<I", linked), "links to itself"),
        (lambda b: put(b, blk + 8, "<I", first_id), "twice"),
        (lambda b: put(b, upper_block(up, 1) + 4, "<I", ground), "above its level"),
        (lambda b: put(b, vectors_at + 3 * 2 * 4, "<f", float("nan")), "NaN or infinity"),
        (lambda b: put(b, vectors_at + 5 * 2 * 4 + 4, "<f", float("inf")), "NaN or infinity"),
    ]
    for corrupt, reason in cases:
        b = tiny_bytes()
        corrupt(b)
        rejected(vdx, tmp_path / "bad.vdx", reseal(vdx, b), reason)


def test_other_files_are_rejected(vdx, tmp_path):
    b = tiny_bytes()
    b[0] = ord("v")
    rejected(vdx, tmp_path / "bad.vdx", reseal(vdx, b), "wrong magic")
    rejected(vdx, tmp_path / "text.vdx", b"Not an index, but longer than a header.\n" * 10, "wrong magic")
    rejected(vdx, tmp_path / "zeros.vdx", bytes(1000), "wrong magic")
    rejected(vdx, tmp_path / "empty.vdx", b"", "too small")
    with pytest.raises(OSError, match="no_such_file"):
        vdx.HnswIndex.load(tmp_path / "no_such_file.vdx")


def test_save_replaces_atomically_and_cleans_up(vdx, tmp_path):
    ix = vdx.HnswIndex(4, M=4, ef_construction=20)
    ix.add(uniform_matrix(20, 4, 1))
    ix.save(tmp_path / "index.vdx")
    ix.add(uniform_matrix(10, 4, 2))
    ix.save(tmp_path / "index.vdx")
    assert len(vdx.HnswIndex.load(tmp_path / "index.vdx")) == 30
    assert sorted(p.name for p in tmp_path.iterdir()) == ["index.vdx"]
    with pytest.raises(OSError, match="no_such_dir"):
        ix.save(tmp_path / "no_such_dir" / "index.vdx")
    (tmp_path / "target").mkdir()
    with pytest.raises(OSError):
        ix.save(tmp_path / "target")
    assert sorted(p.name for p in tmp_path.iterdir()) == ["index.vdx", "target"]
