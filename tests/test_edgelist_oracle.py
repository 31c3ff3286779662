"""The CPU restatement of read_edgelist (oracle/edgelist_oracle.py) pinned to
the reference: its unit tests (src/algorithms/io/edgelist.rs:106-130) and the
karate fixture its tests read (fixtures/karate.edges, 34 vertices, 78 edges)."""
import json
import os

import pytest

import edgelist_oracle as E
from conftest import GOLDEN


def test_reference_unit_cases():
    assert E.read_edgelist(b"") == (0, [])                                   # :107-111
    n, edges = E.read_edgelist(b"# hi\n\n0 1\n   2 3   \n")                  # :114-119
    assert (n, len(edges)) == (4, 2)
    with pytest.raises(E.ParseErr) as ei:                                    # :122-129
        E.read_edgelist(b"0 1\nbroken\n")
    assert ei.value.line == 2


def test_round_trip_of_write_edgelist_format():
    # write_edgelist (edgelist.rs:93-100) writes "u v\n" per edge
    edges = [(0, 1), (2, 3), (1, 3)]
    text = "".join(f"{u} {v}\n" for u, v in edges).encode()
    assert E.read_edgelist(text) == (4, edges)


def test_karate_fixture():
    fx = json.load(open(os.path.join(GOLDEN, "reference_fixtures.json")))["edgelists"][0]
    n, edges = E.read_edgelist(fx["text"].encode())
    assert (n, len(edges)) == (fx["vcount"], fx["ecount"])


def test_rust_integer_and_whitespace_rules():
    assert E.read_edgelist(b"0 +5\n") == (6, [(0, 5)])
    assert E.read_edgelist(b"00 0007\r\n") == (8, [(0, 7)])
    for text, line, msg in [
        (b"0 -5\n", 1, "invalid vertex id `-5`: invalid digit found in string"),
        (b"+ 1\n", 1, "invalid vertex id `+`: invalid digit found in string"),
        (b"1 4294967296\n", 1, "invalid vertex id `4294967296`: number too large to fit in target type"),
        (b"1 99999999999x\n", 1, "invalid vertex id `99999999999x`: number too large to fit in target type"),
        (b"0 1\n7\n", 2, "missing vertex id"),
        (b"\n\n1 2 3\n", 3, "expected exactly two vertex ids"),
        (b"1\x1c2 3\n", 1, "invalid vertex id `1\x1c2`: invalid digit found in string"),
    ]:
        with pytest.raises(E.ParseErr) as ei:
            E.read_edgelist(text)
        assert (ei.value.line, ei.value.message) == (line, msg), text
    # Unicode White_Space separates tokens (U+00A0, U+3000)
    assert E.read_edgelist("1 2\n　3 4　\n".encode()) == (5, [(1, 2), (3, 4)])
    with pytest.raises(E.IoErr):
        E.read_edgelist(b"0 1\n# \xff\n")
    with pytest.raises(E.InternalErr):
        E.read_edgelist(b"0 4294967295\n")
