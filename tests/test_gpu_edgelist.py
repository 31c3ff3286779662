"""The GPU edge-list reader (prg_parse_edgelist / prg_read_edgelist) against
the CPU restatement of read_edgelist (src/algorithms/io/edgelist.rs:25-72):
identical edges in file order and n, or the identical first failing line and
message, on the reference's fixture, on crafted edge cases and on seeded
random texts; at scale (millions of lines) through size-independent
checks against the arrays a regular text was written from."""
import json
import os

import numpy as np
import pytest

import edgelist_oracle as E
import igraph_b200 as ig
import oracle as O
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def expect(text: bytes):
    """('ok', n, from, to) | ('parse', line, message) | ('io',) | ('internal', message)"""
    try:
        n, edges = E.read_edgelist(text)
    except E.ParseErr as e:
        return ("parse", e.line, e.message)
    except E.IoErr:
        return ("io",)
    except E.InternalErr as e:
        return ("internal", str(e))
    f = np.array([u for u, _ in edges], np.uint32)
    t = np.array([v for _, v in edges], np.uint32)
    return ("ok", n, f, t)


def got(text: bytes):
    try:
        n, f, t = ig.parse_edgelist(text)
    except ig.ParseError as e:
        return ("parse", e.line, e.message)
    except ig.IoError:
        return ("io",)
    except ig.Internal as e:
        return ("internal", str(e))
    return ("ok", n, f, t)


def same(a, b):
    if a[0] != b[0]:
        return False
    if a[0] == "ok":
        return a[1] == b[1] and np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])
    return a == b


CASES = [
    b"",
    b"\n\n\n",
    b"# only a comment",
    b"0 1",
    b"0 1\n",
    b"# hi\n\n0 1\n   2 3   \n",                       # edgelist.rs:114-119
    b"0 1\nbroken\n",                                   # edgelist.rs:122-129
    b"0 1\r\n2 3\r\n",
    b"\t0\t1\t\n\x0b2\x0c3\r\n",
    b"  # indented comment\n5 6\n",
    b"0 +5\n00 0007\n",
    b"0 -5\n",
    b"+ 1\n",
    b"1 4294967295\n",
    b"1 4294967294\n",
    b"1 4294967296\n",
    b"1 99999999999x\n",
    b"3\n",
    b"1 2 3\n",
    b"1 2\n3 4 # trailing comment is a token\n",
    b"1\x1c2 3\n",
    b"1\x002 3\n",
    "1\u00a02\n3\u20034\n\u30005 6\u3000\n".encode(),  # Unicode White_Space (U+00A0, U+2003, U+3000)
    "# caf\u00e9 comment\n1 2\n".encode(),
    b"0 1\n# \xff\n2 3\n",                               # invalid UTF-8 -> I/O error
    b"0 1\nbad\n# \xff\n",                              # the parse error comes first
    b"0 1\n\xc0\xaf 2\n",                                # overlong encoding
    "1 2\n\u00e9 3\n".encode(),                      # non-ASCII token
    b"7 7\n7 7\n",
]


@pytest.mark.parametrize("idx", range(len(CASES)))
def test_crafted_cases_match_the_restatement(cuda_ok, idx):
    text = CASES[idx]
    a, b = expect(text), got(text)
    assert same(a, b), (text, a, b)


def test_reference_fixture_and_drop_in_pagerank(cuda_ok, golden_cases):
    fx = json.load(open(os.path.join(GOLDEN, "reference_fixtures.json")))["edgelists"][0]
    text = fx["text"].encode()
    n, f, t = ig.parse_edgelist(text)
    assert (n, len(f)) == (fx["vcount"], fx["ecount"])
    assert same(expect(text), ("ok", n, f, t))
    g = ig.read_edgelist(text)
    assert (g.vcount(), g.ecount(), g.is_directed()) == (34, 78, False)
    # file -> GPU parse -> resident CSR -> PageRank, without the edges leaving the GPU
    with ig.DeviceGraph.from_edgelist(text) as dg:
        x, _ = dg.solve()
    ref = O.pagerank(34, f, t, False)
    assert np.max(np.abs(x - ref)) <= 1e-10
    assert ig.DeviceGraph.from_edgelist(b"# nothing\n") is None


def _random_text(rng, lines):
    out = []
    ws = [b" ", b"\t", b"  ", b"\x0b", b"\x0c", b" \t "]
    for _ in range(lines):
        r = rng.random()
        if r < 0.05:
            out.append(b"# " + bytes(rng.integers(32, 127, rng.integers(0, 30)).astype(np.uint8)))
        elif r < 0.08:
            out.append(rng.choice(ws))
        else:
            u, v = (int(x) for x in rng.integers(0, 100_000, 2))
            su = (b"+" if rng.random() < 0.02 else b"") + (b"0" if rng.random() < 0.02 else b"") + str(u).encode()
            line = rng.choice(ws) * int(rng.integers(0, 2)) + su + rng.choice(ws) + str(v).encode()
            line += rng.choice(ws) * int(rng.integers(0, 2))
            out.append(line)
    ending = [b"\n", b"\r\n"][int(rng.integers(0, 2))]
    return ending.join(out) + (ending if rng.random() < 0.5 else b"")


@pytest.mark.parametrize("seed", range(6))
def test_seeded_random_texts(cuda_ok, seed):
    rng = np.random.default_rng(seed)
    text = _random_text(rng, int(rng.integers(1, 20_000)))
    if seed % 2:  # plant one failing line
        lines = text.split(b"\n")
        k = int(rng.integers(0, len(lines)))
        lines[k] = [b"1 2 3", b"x 1", b"4", b"1 99999999999"][seed % 4]
        text = b"\n".join(lines)
    a, b = expect(text), got(text)
    assert same(a, b), (seed, a[:2], b[:2])


def test_large_text_properties(cuda_ok):
    # 8 M lines, ~110 MB of text: many 512-byte chunks and scan tiles;
    # checked against the generating arrays
    rng = np.random.default_rng(11)
    m = 8_000_000
    u = rng.integers(0, 1 << 24, m, dtype=np.uint32)
    v = rng.integers(0, 1 << 24, m, dtype=np.uint32)
    text = ("\n".join(f"{a} {b}" for a, b in zip(u.tolist(), v.tolist())) + "\n").encode()
    n, f, t = ig.parse_edgelist(text)
    assert n == int(max(u.max(), v.max())) + 1
    assert np.array_equal(f, u) and np.array_equal(t, v)
    # a failing line at the very end is found with its line number
    with pytest.raises(ig.ParseError) as ei:
        ig.parse_edgelist(text + b"12 x\n")
    assert ei.value.line == m + 1 and ei.value.message == "invalid vertex id `x`: invalid digit found in string"
