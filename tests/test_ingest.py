"""Fast ingest (CPU only): the parallel edge-list reader keeps the reference
reader's line rules (bc2d.c:214-247: '#' lines are comments, "Nodes:" echo,
"%lu %lu" fields, abort on an id >= N naming the line), and the binary CSR
cache round-trips and rejects corrupt files."""
import os

import numpy as np
import pytest

import bcg


def _ref_pairs(text, n):
    """Independent restatement of the line rules for the expected graph."""
    pairs = []
    for line in text.split("\n"):
        if "#" in line:
            continue
        f = line.split()
        try:
            u, v = int(f[0]), int(f[1])
        except (IndexError, ValueError):
            continue
        pairs.append((u, v))
    return pairs


def test_reader_matches_line_rules(tmp_path):
    text = ("# comment\n# Nodes: 9 Edges: 7\n0 1\n  1\t2  extra\n\n2 3\r\n#3 4\n"
            "x y\n4 5 # trailing comment makes the line a comment\n5 6\n+6 7\n007 8\n")
    p = tmp_path / "g.txt"
    p.write_text(text)
    offs, adj = bcg.read_edgelist(str(p), 9)
    eo, ea = bcg.from_pairs(_ref_pairs(text, 9), 9)
    assert np.array_equal(offs, eo) and np.array_equal(adj, ea)


def test_reader_error_names_the_line(tmp_path):
    p = tmp_path / "bad.txt"
    p.write_text("# header\n0 1\n\n1 2\n2 9\n3 4\n")
    with pytest.raises(bcg.BcgError) as ei:
        bcg.read_edgelist(str(p), 5)
    # non-comment lines are counted (the blank one too): "2 9" is line 4
    assert ei.value.code == bcg.ERR_IO and "line 4" in str(ei.value) and "(2, 9)" in str(ei.value)


def test_reader_large_parallel_equals_generator(tmp_path):
    offs, adj = bcg.generate("rmat:scale=14,ef=16,seed=3")
    p = tmp_path / "big.txt"
    bcg.write_edgelist(str(p), offs, adj)
    o2, a2 = bcg.read_edgelist(str(p), len(offs) - 1)
    assert np.array_equal(offs, o2) and np.array_equal(adj, a2)


def test_binary_cache_roundtrip_and_corruption(tmp_path):
    offs, adj = bcg.generate("rmat:scale=10,ef=8,seed=5,pendant_frac=0.1,pendant_mean=4")
    p = tmp_path / "g.bcsr"
    bcg.write_binary(str(p), offs, adj)
    o2, a2 = bcg.read_binary(str(p))
    assert np.array_equal(offs, o2) and np.array_equal(adj, a2)
    raw = bytearray(p.read_bytes())
    raw[-5] ^= 0x40  # flip a bit in the adjacency
    bad = tmp_path / "bad.bcsr"
    bad.write_bytes(bytes(raw))
    with pytest.raises(bcg.BcgError) as ei:
        bcg.read_binary(str(bad))
    assert ei.value.code == bcg.ERR_IO
    short = tmp_path / "short.bcsr"
    short.write_bytes(bytes(raw[:-8]))
    with pytest.raises(bcg.BcgError):
        bcg.read_binary(str(short))
    with pytest.raises(bcg.BcgError):
        bcg.read_binary(str(tmp_path / "missing.bcsr"))
