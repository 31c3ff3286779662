"""CPU restatement of rust-igraph's read_edgelist (src/algorithms/io/edgelist.rs:25-72).

TEST INFRASTRUCTURE ONLY: the tests compare the GPU reader against it.

Rust semantics restated here:
  * `BufRead::lines()` splits on b"\\n", drops one "\\r" before it, and fails
    with an I/O error ("stream did not contain valid UTF-8") on the first line
    that is not valid UTF-8;
  * `str::trim` / `split_whitespace` use char::is_whitespace, the Unicode
    White_Space property (note: U+001C..U+001F are NOT whitespace in Rust,
    unlike Python's str.split());
  * `u32::from_str` accepts an optional '+', then ASCII digits; scanning left
    to right, a non-digit gives "invalid digit found in string" and an
    overflow "number too large to fit in target type"; a lone sign is an
    invalid digit;
  * the first failing line (1-based) is reported as
    `IgraphError::Parse { line, message }`.
"""
from __future__ import annotations

WHITE_SPACE = frozenset([*range(0x09, 0x0E), 0x20, 0x85, 0xA0, 0x1680, *range(0x2000, 0x200B), 0x2028, 0x2029,
                         0x202F, 0x205F, 0x3000])


class ParseErr(Exception):
    def __init__(self, line, message):
        super().__init__(f"parse error at line {line}: {message}")
        self.line = line
        self.message = message


class IoErr(Exception):
    pass


class InternalErr(Exception):
    pass


def _is_ws(ch: str) -> bool:
    return ord(ch) in WHITE_SPACE


def _trim(s: str) -> str:
    b, e = 0, len(s)
    while b < e and _is_ws(s[b]):
        b += 1
    while e > b and _is_ws(s[e - 1]):
        e -= 1
    return s[b:e]


def _split_ws(s: str):
    toks, cur = [], []
    for ch in s:
        if _is_ws(ch):
            if cur:
                toks.append("".join(cur))
                cur = []
        else:
            cur.append(ch)
    if cur:
        toks.append("".join(cur))
    return toks


def _parse_u32(tok: str):
    """Returns (value, None) or (None, ParseIntError text)."""
    if tok == "":
        return None, "cannot parse integer from empty string"
    s = tok
    if s[0] in "+-" and len(s) == 1:
        return None, "invalid digit found in string"
    if s[0] == "+":
        s = s[1:]
    acc = 0
    for ch in s:
        if not ("0" <= ch <= "9"):  # ASCII digits only
            return None, "invalid digit found in string"
        acc = acc * 10 + (ord(ch) - 48)
        if acc > 0xFFFFFFFF:
            return None, "number too large to fit in target type"
    return acc, None


def _parse_id(tok, line):
    if tok is None:
        raise ParseErr(line, "missing vertex id")
    v, err = _parse_u32(tok)
    if err is not None:
        raise ParseErr(line, f"invalid vertex id `{tok}`: {err}")
    return v


def _lines(data: bytes):
    pos = 0
    n = len(data)
    while pos < n:
        nl = data.find(b"\n", pos)
        if nl < 0:
            raw, pos = data[pos:], n
        else:
            raw, pos = data[pos:nl], nl + 1
            if raw.endswith(b"\r"):
                raw = raw[:-1]
        try:
            yield raw.decode("utf-8", errors="strict")
        except UnicodeDecodeError:
            raise IoErr("stream did not contain valid UTF-8")


def read_edgelist(data: bytes):
    """(n, [(u, v), ...]) in file order, or raises ParseErr / IoErr."""
    edges = []
    max_id = 0
    had_any = False
    for line_no, line in enumerate(_lines(bytes(data)), start=1):
        t = _trim(line)
        if t == "" or t.startswith("#"):
            continue
        parts = _split_ws(t)
        u = _parse_id(parts[0] if len(parts) > 0 else None, line_no)
        v = _parse_id(parts[1] if len(parts) > 1 else None, line_no)
        if len(parts) > 2:
            raise ParseErr(line_no, "expected exactly two vertex ids")
        max_id = max(max_id, u, v)
        edges.append((u, v))
        had_any = True
    if had_any and max_id == 0xFFFFFFFF:
        raise InternalErr("vertex id u32::MAX cannot be sized into n")  # edgelist.rs:50-55
    return (max_id + 1 if had_any else 0), edges
