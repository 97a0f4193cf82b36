"""Pure-Python restatement of the reference's ESRI ASCII grid reader.

TEST INFRASTRUCTURE ONLY: the checker for hydroflux_b200's C++ reader
(hf_read_ascii_grid); never part of the product path.

Follows solver-2d/src/ascii_grid.rs:
- parse_ascii_grid (ascii_grid.rs:115-156): `str::lines`, six header lines
  in a fixed order, then the remaining lines joined and split on Unicode
  White_Space (`split_whitespace`), each token parsed as f64, and exactly
  ncols * nrows values;
- header_value (ascii_grid.rs:158-180): first token is the key
  (ASCII-case-insensitive), second the value, further tokens ignored;
- read_ascii_grid (ascii_grid.rs:101-113): gzip when the path's extension is
  "gz" (GzDecoder: the first gzip member), and the text must be UTF-8
  (`read_to_string`);
- esa_worldcover_to_manning (io.rs:192-207) as a table.
Errors are returned as the variant name of AsciiGridError.
"""
from __future__ import annotations

import re
import zlib

# Unicode White_Space, the separator set of str::split_whitespace.
WHITE_SPACE = frozenset(
    [chr(c) for c in range(0x09, 0x0E)] + [chr(c) for c in range(0x2000, 0x200B)]
    + [chr(c) for c in (0x20, 0x85, 0xA0, 0x1680, 0x2028, 0x2029, 0x202F, 0x205F, 0x3000)])

# f64::from_str: optional sign, then inf / infinity / nan (any case) or a
# decimal with optional fraction and exponent.
_F64 = re.compile(r"[+-]?(?:(?:[0-9]+\.?[0-9]*|\.[0-9]+)(?:[eE][+-]?[0-9]+)?|[iI][nN][fF]"
                  r"|[iI][nN][fF][iI][nN][iI][tT][yY]|[nN][aA][nN])\Z")

ESA_WORLDCOVER_MANNING = {10: 0.100, 20: 0.060, 30: 0.040, 40: 0.035, 50: 0.015, 60: 0.025,
                          70: 0.030, 80: 0.030, 90: 0.050, 95: 0.100, 100: 0.045}


def esa_worldcover_to_manning(code: int) -> float:
    return ESA_WORLDCOVER_MANNING.get(code, 0.040)


class GridError(Exception):
    def __init__(self, kind: str, detail: str = ""):
        super().__init__(f"{kind}: {detail}")
        self.kind = kind


def rust_lines(text: str):
    """str::lines: split at '\\n', drop one '\\r' before it, no final empty line."""
    if not text:
        return []
    parts = text.split("\n")
    if parts[-1] == "":
        parts.pop()
    return [p[:-1] if p.endswith("\r") else p for p in parts]


def split_whitespace(s: str):
    out, cur = [], []
    for ch in s:
        if ch in WHITE_SPACE:
            if cur:
                out.append("".join(cur))
                cur = []
        else:
            cur.append(ch)
    if cur:
        out.append("".join(cur))
    return out


def parse_f64(tok: str) -> float:
    if not _F64.match(tok):
        raise GridError("Parse", tok)
    return float(tok)


def as_usize(v: float) -> int:
    if v != v or v <= 0.0:
        return 0
    if v == float("inf"):
        return 2 ** 64 - 1
    return int(v)


def _header_value(lines, i: int, key: str) -> float:
    if i >= len(lines):
        raise GridError("Header", f"missing {key}")
    parts = split_whitespace(lines[i])
    if not parts:
        raise GridError("Header", f"empty line, expected {key}")
    if parts[0].lower() != key.lower() or not parts[0].isascii():
        raise GridError("Header", f"expected key {key}, got {parts[0]}")
    if len(parts) < 2:
        raise GridError("Header", f"missing value for {key}")
    return parse_f64(parts[1])


def parse_ascii_grid(text: str):
    """(values as a flat list, header dict) or GridError."""
    lines = rust_lines(text)
    keys = ["ncols", "nrows", "xllcorner", "yllcorner", "cellsize", "NODATA_value"]
    vals = [_header_value(lines, i, k) for i, k in enumerate(keys)]
    ncols, nrows = as_usize(vals[0]), as_usize(vals[1])
    data = [parse_f64(tok) for tok in split_whitespace(" ".join(lines[6:]))]
    if len(data) != ncols * nrows:
        raise GridError("ValueCount", f"expected {ncols * nrows}, found {len(data)}")
    header = dict(ncols=ncols, nrows=nrows, xllcorner=vals[2], yllcorner=vals[3],
                  cellsize=vals[4], nodata_value=vals[5])
    return data, header


def read_ascii_grid(path: str):
    raw = open(path, "rb").read()
    if str(path).endswith(".gz"):
        # flate2's GzDecoder: the first gzip member only.
        d = zlib.decompressobj(16 + zlib.MAX_WBITS)
        try:
            raw = d.decompress(raw) + d.flush()
        except zlib.error as e:
            raise GridError("Io", str(e))
        if not d.eof:
            raise GridError("Io", "truncated gzip stream")
    try:
        text = raw.decode("utf-8")
    except UnicodeDecodeError as e:
        raise GridError("Io", str(e))
    return parse_ascii_grid(text)
