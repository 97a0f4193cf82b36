"""ESRI ASCII grid I/O through the C ABI (hf_read_ascii_grid and friends),
checked against the reference's own unit tests (solver-2d/src/ascii_grid.rs
tests module, re-encoded), against the pure-Python restatement in
oracle/ascii_grid.py on edge and randomised inputs, and on the reference's
own data files when they are present. Host code only: runs without a GPU."""
import gzip
import math
import os
import struct

import numpy as np
import pytest

from oracle import ascii_grid as O

SAMPLE = ("ncols         4\n"
          "nrows         3\n"
          "xllcorner     0.0\n"
          "yllcorner     0.0\n"
          "cellsize      10\n"
          "NODATA_value  -9999\n"
          "1 2 3 4\n"
          "5 6 7 8\n"
          "9 10 11 12\n")

# A checkout of the reference, when one is named, adds its Huasco result grid;
# the Test 8A grids are committed fixtures (tests/golden/uk_ea).
REF_DATA = os.environ.get("HYDROFLUX_REFERENCE_DIR")
UK_EA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "uk_ea")


@pytest.fixture(scope="module")
def R():
    from hydroflux_b200 import build
    build.build()
    from hydroflux_b200 import raster
    return raster


def write(tmp_path, text, name="g.asc", raw=None):
    p = tmp_path / name
    data = raw if raw is not None else text.encode("utf-8")
    if name.endswith(".gz") and raw is None:
        data = gzip.compress(data)
    p.write_bytes(data)
    return str(p)


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def check_against_oracle(R, path):
    """C reader and the restatement agree: same error variant, or the same
    header and bit-identical values."""
    try:
        ref = O.read_ascii_grid(path)
        ref_err = None
    except O.GridError as e:
        ref, ref_err = None, e.kind
    kinds = {"Io": R.AsciiGridIoError, "Header": R.AsciiGridHeaderError,
             "ValueCount": R.AsciiGridValueCountError, "Parse": R.AsciiGridParseError}
    if ref_err is not None:
        with pytest.raises(kinds[ref_err]):
            R.read_ascii_grid(path)
        return None
    data, h = R.read_ascii_grid(path)
    vals, hd = ref
    assert (h.ncols, h.nrows) == (hd["ncols"], hd["nrows"])
    for k in ("xllcorner", "yllcorner", "cellsize", "nodata_value"):
        assert bits(getattr(h, k)) == bits(hd[k]), k
    assert data.shape == (hd["nrows"], hd["ncols"])
    assert np.array_equal(bits(data.ravel()), bits(np.array(vals, dtype=np.float64)))
    return data, h


# --- the reference's unit tests (ascii_grid.rs tests module) ----------------

def test_parses_header_fields(R, tmp_path):
    _, h = R.read_ascii_grid(write(tmp_path, SAMPLE))
    assert h.ncols == 4 and h.nrows == 3
    assert h.cellsize == 10.0 and h.nodata_value == -9999.0


def test_row_zero_is_the_first_data_row_after_header(R, tmp_path):
    data, _ = R.read_ascii_grid(write(tmp_path, SAMPLE))
    assert data[0].tolist() == [1.0, 2.0, 3.0, 4.0]
    assert data[2].tolist() == [9.0, 10.0, 11.0, 12.0]


def test_rejects_wrong_value_count(R, tmp_path):
    with pytest.raises(R.AsciiGridValueCountError):
        R.read_ascii_grid(write(tmp_path, SAMPLE.replace("9 10 11 12\n", "")))


def test_rejects_out_of_order_header(R, tmp_path):
    with pytest.raises(R.AsciiGridHeaderError):
        R.read_ascii_grid(write(tmp_path, SAMPLE.replace("ncols         4\n", "", 1)))


def test_cell_at_maps_south_west_corner_to_bottom_row(R, tmp_path):
    _, h = R.read_ascii_grid(write(tmp_path, SAMPLE))
    assert h.cell_at(5.0, 5.0) == (2, 0)
    assert h.cell_at(35.0, 25.0) == (0, 3)
    assert h.cell_at(-1.0, 5.0) is None
    assert h.cell_at(5.0, 1000.0) is None


def test_rows_overlapping_y_range_matches_expected_band(R, tmp_path):
    _, h = R.read_ascii_grid(write(tmp_path, SAMPLE))
    assert sorted(h.rows_overlapping_y_range(12.0, 22.0)) == [0, 1]


# --- header helpers at their edges --------------------------------------------

def test_header_helpers_edges(R):
    h = R.AsciiGridHeader(4, 3, 100.0, 200.0, 10.0, -9999.0)
    assert h.cell_at(100.0, 200.0) == (2, 0)          # the south-west corner itself
    assert h.cell_at(139.999, 229.999) == (0, 3)
    assert h.cell_at(140.0, 205.0) is None            # east edge is exclusive
    assert h.cell_at(105.0, 230.0) is None            # north edge is exclusive
    assert h.cell_at(math.nan, 205.0) == (2, 0)       # NaN casts to 0 like `as usize`
    assert h.cell_at(math.inf, 205.0) is None
    assert h.rows_overlapping_y_range(200.0, 210.0) == [2]
    assert h.rows_overlapping_y_range(200.0, 210.5) == [2, 1]
    assert h.rows_overlapping_y_range(150.0, 1e9) == [2, 1, 0]
    assert h.rows_overlapping_y_range(250.0, 260.0) == []
    assert h.rows_overlapping_y_range(210.0, 190.0) == []
    assert h.rows_overlapping_y_range(math.nan, math.inf) == [2, 1, 0]


# --- format edges, C reader vs the restatement --------------------------------

HEADER = "ncols 3\nnrows 2\nxllcorner 1.5\nyllcorner -2.25\ncellsize 0.5\nNODATA_value -9999\n"
EDGE_TEXTS = {
    "crlf": SAMPLE.replace("\n", "\r\n"),
    "wrapped": HEADER + "1 2\n3\n4 5\n6\n",
    "one_line_data": HEADER + "1 2 3 4 5 6",
    "no_final_newline": SAMPLE.rstrip("\n"),
    "case_keys": SAMPLE.replace("ncols", "NCOLS").replace("NODATA_value", "nodata_VALUE"),
    "tabs_and_extra_tokens": HEADER.replace("ncols 3", "\t ncols\t3  trailing words") + "1\t2 3\n4 5 6\n",
    "unicode_spaces": HEADER + "1\u00a02\u30003\n4\u20035\u00856\n",
    "unicode_space_in_header": HEADER.replace("nrows 2", "nrows\u20002") + "1 2 3 4 5 6\n",
    "blank_lines_in_data": HEADER + "\n1 2 3\n\n\n4 5 6\n\n",
    "fractional_ncols": HEADER.replace("ncols 3", "ncols 3.9") + "1 2 3 4 5 6\n",
    "exponent_ncols": HEADER.replace("ncols 3", "ncols 3e0") + "1 2 3 4 5 6\n",
    "negative_nrows_no_data": HEADER.replace("nrows 2", "nrows -2"),
    "negative_nrows_with_data": HEADER.replace("nrows 2", "nrows -2") + "1\n",
    "nan_nrows": HEADER.replace("nrows 2", "nrows NaN"),
    "zero_cells": HEADER.replace("ncols 3", "ncols 0"),
    "specials": HEADER + "inf -Infinity +nan NAN 1e400 -1e-400\n",
    "number_forms": HEADER + "1. .5 +7 -0 1E+3 0000.000100e-0002\n",
    "subnormal_and_long": HEADER + "4.9e-324 2.2250738585072011e-308 "
                          "0.1000000000000000055511151231257827021181583404541015625 "
                          "1.7976931348623157e308 123456789012345678901234567890 3\n",
    "hex_rejected": HEADER + "1 2 3 4 5 0x10\n",
    "bad_exponent": HEADER + "1 2 3 4 5 1e\n",
    "lone_point": HEADER + "1 2 3 4 5 .\n",
    "underscore": HEADER + "1 2 3 4 5 1_0\n",
    "double_sign": HEADER + "1 2 3 4 5 +-1\n",
    "comma_decimal": HEADER + "1 2 3 4 5 1,5\n",
    "inf_prefix": HEADER + "1 2 3 4 5 infin\n",
    "fullwidth_digit": HEADER + "1 2 3 4 5 \uff11\n",
    "bad_header_value": HEADER.replace("cellsize 0.5", "cellsize abc") + "1 2 3 4 5 6\n",
    "missing_value": HEADER.replace("cellsize 0.5", "cellsize") + "1 2 3 4 5 6\n",
    "empty_header_line": HEADER.replace("cellsize 0.5", "   ") + "1 2 3 4 5 6\n",
    "wrong_key": HEADER.replace("xllcorner", "xllcenter") + "1 2 3 4 5 6\n",
    "key_prefix": HEADER.replace("cellsize", "cellsizes") + "1 2 3 4 5 6\n",
    "short_file": "ncols 3\nnrows 2\n",
    "empty_file": "",
    "bom": "\ufeff" + SAMPLE,
    "too_many_values": SAMPLE + "13\n",
}


@pytest.mark.parametrize("name", sorted(EDGE_TEXTS))
def test_edges_match_restatement(R, tmp_path, name):
    check_against_oracle(R, write(tmp_path, EDGE_TEXTS[name]))


def test_edge_values(R, tmp_path):
    data, h = R.read_ascii_grid(write(tmp_path, EDGE_TEXTS["specials"]))
    v = data.ravel()
    assert v[0] == math.inf and v[1] == -math.inf and math.isnan(v[2]) and math.isnan(v[3])
    assert v[4] == math.inf and v[5] == 0.0 and math.copysign(1.0, v[5]) == -1.0
    _, h = R.read_ascii_grid(write(tmp_path, EDGE_TEXTS["fractional_ncols"].replace(
        "1 2 3 4 5 6", "1 2 3 4 5 6")))
    assert h.ncols == 3
    data, h = R.read_ascii_grid(write(tmp_path, EDGE_TEXTS["zero_cells"]))
    assert data.shape == (2, 0) and h.ncols == 0
    with pytest.raises(R.AsciiGridParseError):
        R.read_ascii_grid(write(tmp_path, EDGE_TEXTS["hex_rejected"]))
    with pytest.raises(R.AsciiGridHeaderError):
        R.read_ascii_grid(write(tmp_path, EDGE_TEXTS["bom"]))


def test_io_errors(R, tmp_path):
    with pytest.raises(R.AsciiGridIoError):
        R.read_ascii_grid(str(tmp_path / "missing.asc"))
    # invalid UTF-8 is an I/O error, as in read_to_string
    p = write(tmp_path, None, raw=SAMPLE.encode().replace(b"12", b"1\xff"))
    check_against_oracle(R, p)
    with pytest.raises(R.AsciiGridIoError):
        R.read_ascii_grid(p)
    # a .gz name with plain text inside, and a truncated gzip stream
    p = write(tmp_path, None, "plain.asc.gz", raw=SAMPLE.encode())
    check_against_oracle(R, p)
    with pytest.raises(R.AsciiGridIoError):
        R.read_ascii_grid(p)
    z = gzip.compress(SAMPLE.encode())
    for cut in (5, len(z) // 2, len(z) - 4):
        p = write(tmp_path, None, f"cut{cut}.asc.gz", raw=z[:cut])
        check_against_oracle(R, p)
        with pytest.raises(R.AsciiGridIoError):
            R.read_ascii_grid(p)
    # a corrupted checksum
    bad = z[:-8] + struct.pack("<I", (struct.unpack("<I", z[-8:-4])[0] ^ 1)) + z[-4:]
    p = write(tmp_path, None, "crc.asc.gz", raw=bad)
    check_against_oracle(R, p)
    with pytest.raises(R.AsciiGridIoError):
        R.read_ascii_grid(p)


def test_gzip_first_member_only(R, tmp_path):
    """Like flate2's GzDecoder, only the first gzip member is read."""
    two = gzip.compress(SAMPLE.encode()) + gzip.compress(b"13 14 15\n")
    p = write(tmp_path, None, "two.asc.gz", raw=two)
    data, _ = check_against_oracle(R, p)
    assert data.shape == (3, 4)


def test_plain_name_is_not_gunzipped(R, tmp_path):
    p = write(tmp_path, None, "zipped.asc", raw=gzip.compress(SAMPLE.encode()))
    check_against_oracle(R, p)
    with pytest.raises(R.AsciiGridIoError):
        R.read_ascii_grid(p)


def test_randomised_layouts_match_restatement(R, tmp_path):
    rng = np.random.default_rng(7)
    seps = [" ", "  ", "\t", "\n", "\r\n", " \n ", "\u00a0", "\u2028", "\u3000", "\x0b", "\x0c"]
    for k in range(40):
        nr, nc = int(rng.integers(0, 6)), int(rng.integers(0, 6))
        vals = rng.standard_normal(nr * nc) * 10.0 ** rng.integers(-300, 300, nr * nc)
        toks = [repr(float(v)) if rng.random() < 0.5 else f"{v:.6e}" for v in vals]
        body = ""
        for t in toks:
            body += t + seps[int(rng.integers(0, len(seps)))]
        keys = ["ncols", "nrows", "xllcorner", "yllcorner", "cellsize", "NODATA_value"]
        hv = [nc, nr, rng.uniform(-1e6, 1e6), rng.uniform(-1e6, 1e6), rng.uniform(0.1, 50), -9999]
        head = "".join(
            (k2.upper() if rng.random() < 0.3 else k2) + " " * int(rng.integers(1, 4))
            + str(v) + ("\r\n" if rng.random() < 0.3 else "\n") for k2, v in zip(keys, hv))
        if rng.random() < 0.2 and toks:     # damage: drop a value, add one, or break one
            body += rng.choice(["", "7", "x1"])
        name = f"r{k}.asc" + (".gz" if k % 3 == 0 else "")
        check_against_oracle(R, write(tmp_path, head + body, name))


# --- writer round trips -------------------------------------------------------

@pytest.mark.parametrize("name", ["w.asc", "w.asc.gz"])
def test_write_read_bit_exact(R, tmp_path, name):
    rng = np.random.default_rng(3)
    a = rng.standard_normal((17, 23)) * 10.0 ** rng.integers(-308, 308, (17, 23))
    a.ravel()[:8] = [0.0, -0.0, 5e-324, -2.2250738585072014e-308, math.inf, -math.inf,
                     math.nan, 1.7976931348623157e308]
    h = R.AsciiGridHeader(23, 17, 263977.0, 664409.0, 2.0, -9999.0)
    p = str(tmp_path / name)
    R.write_ascii_grid(p, a, h)
    b, h2 = check_against_oracle(R, p)
    assert h2 == h
    assert np.array_equal(bits(b), bits(a))
    if name.endswith(".gz"):
        assert open(p, "rb").read(2) == b"\x1f\x8b"


def test_write_checks_shape(R, tmp_path):
    with pytest.raises(ValueError):
        R.write_ascii_grid(str(tmp_path / "x.asc"), np.zeros((2, 3)),
                           R.AsciiGridHeader(2, 3, 0.0, 0.0, 1.0, -9999.0))
    with pytest.raises(R.AsciiGridIoError):
        R.write_ascii_grid(str(tmp_path / "no_such_dir" / "x.asc"), np.zeros((3, 2)),
                           R.AsciiGridHeader(2, 3, 0.0, 0.0, 1.0, -9999.0))


# --- depth raster, land-cover table, mesh builders -----------------------------

def test_depth_raster_from_states(R):
    h = np.array([[0.0, 1e-6, 1.0000000000000002e-6, -1.0], [0.5, math.nan, math.inf, 2e-7]])
    assert np.array_equal(bits(R.depth_raster_from_states(h)), bits(h))
    d = R.depth_raster_from_states(h, nodata=-9999.0)
    want = np.where(h <= R.H_DRY, -9999.0, h)   # NaN <= H_DRY is false: NaN is kept
    assert np.array_equal(bits(d), bits(want))
    assert d[0, 1] == -9999.0 and d[0, 2] == h[0, 2]


def test_esa_worldcover_table(R):
    for code in range(256):
        assert R.esa_worldcover_to_manning(code) == O.esa_worldcover_to_manning(code), code
    with pytest.raises(ValueError):
        R.esa_worldcover_to_manning(256)


def test_mesh_builders(R, tmp_path):
    hd = R.AsciiGridHeader(4, 3, 0.0, 0.0, 2.0, -9999.0)
    bed = np.arange(12, dtype=np.float64).reshape(3, 4)
    R.write_ascii_grid(str(tmp_path / "dem.asc"), bed, hd)
    mesh, h = R.mesh_from_ascii_grid(str(tmp_path / "dem.asc"), 0.03)
    assert h == hd and mesh.dx == 2.0 and mesh.dy == 2.0
    assert np.array_equal(mesh.bed, bed) and np.all(mesh.manning == 0.03)
    n = np.where(bed > 5, 0.05, 0.02)
    R.write_ascii_grid(str(tmp_path / "n.asc.gz"), n, hd)
    mesh, _ = R.mesh_from_ascii_grid(str(tmp_path / "dem.asc"), str(tmp_path / "n.asc.gz"))
    assert np.array_equal(mesh.manning, n)
    lc = np.array([[10, 20, 30, 40], [50, 60, 70, 80], [90, 95, 100, 7]], dtype=np.float64)
    R.write_ascii_grid(str(tmp_path / "lc.asc"), lc, hd)
    mesh, _ = R.mesh_from_ascii_grid_with_landcover(str(tmp_path / "dem.asc"),
                                                    str(tmp_path / "lc.asc"))
    assert mesh.manning.tolist() == [[O.esa_worldcover_to_manning(int(c)) for c in r]
                                     for r in lc.tolist()]
    R.write_ascii_grid(str(tmp_path / "lc_bad.asc"), lc + 0.5, hd)
    with pytest.raises(ValueError):
        R.mesh_from_ascii_grid_with_landcover(str(tmp_path / "dem.asc"),
                                              str(tmp_path / "lc_bad.asc"))
    R.write_ascii_grid(str(tmp_path / "lc_small.asc"), lc[:2],
                       R.AsciiGridHeader(4, 2, 0.0, 0.0, 2.0, -9999.0))
    with pytest.raises(R.RasterShapeMismatch):
        R.mesh_from_ascii_grid_with_landcover(str(tmp_path / "dem.asc"),
                                              str(tmp_path / "lc_small.asc"))
    R.write_ascii_grid(str(tmp_path / "flat.asc"), bed,
                       R.AsciiGridHeader(4, 3, 0.0, 0.0, 0.0, -9999.0))
    with pytest.raises(R.InvalidPixelSize):
        R.mesh_from_ascii_grid(str(tmp_path / "flat.asc"), 0.03)
    R.write_ascii_grid(str(tmp_path / "empty.asc"), np.zeros((0, 4)),
                       R.AsciiGridHeader(4, 0, 0.0, 0.0, 1.0, -9999.0))
    with pytest.raises(R.EmptyRaster):
        R.mesh_from_ascii_grid(str(tmp_path / "empty.asc"), 0.03)


# --- the reference's own data files ------------------------------------------

REF_GRIDS = [
    ("reference", "examples/huasco_2d_phase2/data/synxflow_noflow_h_86400.asc.gz"),
    ("fixture", "test8a_glasgow/ea8-2m.dem.gz"),
    ("fixture", "test8a_glasgow/ea8-2m.n.gz"),
]


@pytest.mark.parametrize("where,rel", REF_GRIDS)
def test_reference_data_files(R, where, rel):
    if where == "reference":
        if not REF_DATA or not os.path.exists(os.path.join(REF_DATA, rel)):
            pytest.skip("HYDROFLUX_REFERENCE_DIR does not name a reference checkout")
        path = os.path.join(REF_DATA, rel)
    else:
        path = os.path.join(UK_EA, rel)
    data, h = check_against_oracle(R, path)
    assert data.shape == (h.nrows, h.ncols) and np.all(np.isfinite(data))


def test_reference_urban_grids(R):
    """The urban rain/point-inflow case (solver-2d/examples/
    uk_ea_test8a_official.rs): a 481 x 199 DEM at 2 m without NODATA, a
    Manning grid of the same geometry with two values, and every control
    point and the inflow point inside the grid."""
    d = os.path.join(UK_EA, "test8a_glasgow")
    mesh, h = R.mesh_from_ascii_grid(os.path.join(d, "ea8-2m.dem.gz"),
                                     os.path.join(d, "ea8-2m.n.gz"))
    assert (h.nrows, h.ncols, h.cellsize) == (199, 481, 2.0)
    assert 21.0 < mesh.bed.min() < mesh.bed.max() < 37.5
    assert sorted(np.unique(mesh.manning).tolist()) == [0.02, 0.05]
    pts = []
    for line in open(os.path.join(d, "ea8-2m.stage")).read().split("\n")[1:]:
        if line.strip():
            x, y = map(float, line.split())
            pts.append((x, y))
    assert len(pts) == 9
    assert all(h.cell_at(x, y) is not None for x, y in pts)
