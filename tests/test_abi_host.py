"""CPU-only checks of the C ABI library: it loads, exports every symbol that
include/gcgpu.h declares, and its host-side logic (edge-list parser, argument
validation, generators) behaves like the reference's. No kernel is launched."""
import os
import re

import numpy as np
import pytest

import gcgpu
from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "gcgpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gcg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 15
    lib = gcgpu._lib
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(gcgpu.EXPORTED)


def test_version_and_error_string():
    assert "sm_100a" in gcgpu.version()
    assert isinstance(gcgpu.last_error(), str)


def test_null_arguments_are_rejected_without_abort():
    import ctypes as C
    st = gcgpu._graph_from_edges(None, None, 0, 0, 0, 1, None)
    assert st == -1 and "null" in gcgpu.last_error()
    st = gcgpu._pagerank(None, None, None, None)
    assert st == -1
    st = gcgpu._graph_free(None)
    assert st == 0
    m = C.c_uint64(0)
    assert gcgpu._parse_file(None, None, None, 0, C.byref(m)) == -1


def write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_parser_matches_convert_edgelist(tmp_path):
    """conversions.hpp:210-288: '#'/'%' comments, delimiters tab/comma/space,
    a third token (edge value) ignored, atoi semantics; self-loops are kept by
    the parser and dropped by the sharder."""
    p = write(tmp_path, "g.txt",
              "# comment\n%another\n1\t2\n3,4\n5 6 0.5\n  7   8\n9\t9\n10,11,2.0\n12\t13\r\n+14 -1\n")
    s, d = gcgpu.parse_edgelist_file(p)
    assert s.tolist() == [1, 3, 5, 7, 9, 10, 12, 14]
    assert d.tolist() == [2, 4, 6, 8, 9, 11, 13, 0xFFFFFFFF]


def test_parser_rejects_short_line_with_line_number(tmp_path):
    p = write(tmp_path, "bad.txt", "1 2\n3\n4 5\n")
    with pytest.raises(gcgpu.GcgError) as e:
        gcgpu.parse_edgelist_file(p)
    assert e.value.status == -5 and "line 2" in str(e.value)


def test_parser_missing_file(tmp_path):
    with pytest.raises(gcgpu.GcgError) as e:
        gcgpu.parse_edgelist_file(str(tmp_path / "nope.txt"))
    assert e.value.status == -4


def test_parser_large_file_is_split_across_threads_in_order(tmp_path):
    rng = np.random.default_rng(3)
    s = rng.integers(0, 1 << 30, 300_000, dtype=np.uint64)
    d = rng.integers(0, 1 << 30, 300_000, dtype=np.uint64)
    p = tmp_path / "big.txt"
    with open(p, "w") as f:
        f.write("# header\n")
        np.savetxt(f, np.stack([s, d], 1), fmt="%d", delimiter=" ")
    ps, pd = gcgpu.parse_edgelist_file(str(p))
    assert np.array_equal(ps, s.astype(np.uint32)) and np.array_equal(pd, d.astype(np.uint32))


def test_generator_argument_checks():
    with pytest.raises(gcgpu.GcgError):
        gcgpu.generate_rmat(0, 10)
    with pytest.raises(gcgpu.GcgError):
        gcgpu.generate_rmat(10, 10, a=0.9, b=0.2, c=0.1)
    with pytest.raises(gcgpu.GcgError):
        gcgpu.generate_er(0, 10)


def test_write_vout_layout(tmp_path):
    """<base>.<sizeof>B.vout is a raw little-endian array (chifilenames.hpp:65-71)."""
    base = str(tmp_path / "g")
    v = np.arange(10, dtype=np.float32) * 0.5
    gcgpu.write_vout(base, v)
    assert np.array_equal(np.fromfile(base + ".4B.vout", dtype=np.float32), v)


def test_block_cache_is_empty_without_allocations():
    # nothing was allocated on a machine without a GPU: the cache holds nothing
    # and releasing it is a no-op
    assert gcgpu.cached_memory() == (0, 0)
    assert gcgpu.release_cached_memory() == 0


def test_vertex_count_beyond_the_limit_is_rejected_before_any_device_work():
    # at most 2^32 - 2^26 vertices: 32-bit grid-stride counters cannot wrap
    s = np.array([0, 1], np.uint32)
    d = np.array([1, 2], np.uint32)
    with pytest.raises(gcgpu.GcgError) as e:
        gcgpu.Graph.from_edges(s, d, num_vertices=(1 << 32) - (1 << 26) + 1)
    assert e.value.status == -6
