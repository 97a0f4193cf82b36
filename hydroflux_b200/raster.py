"""Rasters on the host: ESRI ASCII grids and the helpers around them.

Mirrors hydroflux-solver-2d's `ascii_grid` module (solver-2d/src/ascii_grid.rs)
and the format-independent parts of its `io` module (solver-2d/src/io.rs):
the reader, the header's geographic lookups, the depth raster, the ESA
WorldCover roughness table and the mesh builders. The reader and writer are
C++ in libhydroflux_gpu.so (hf_read_ascii_grid / hf_write_ascii_grid); the
GeoTIFF side of io.rs is not provided (it needs a GeoTIFF library), so the
mesh builders take ASCII grids.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass
from typing import Callable, List, Optional, Tuple

import numpy as np

from . import abi
from ._lib import last_error, lib
from .sim import H_DRY, Mesh2D


class AsciiGridError(Exception):
    """AsciiGridError (ascii_grid.rs:78-98)."""


class AsciiGridIoError(AsciiGridError):
    """AsciiGridError::Io: the file cannot be read, is not gzip when named
    .gz, or is not UTF-8 text."""


class AsciiGridHeaderError(AsciiGridError):
    """AsciiGridError::Header: a header line missing, out of order or empty."""


class AsciiGridValueCountError(AsciiGridError):
    """AsciiGridError::ValueCount: not exactly ncols * nrows data values."""


class AsciiGridParseError(AsciiGridError):
    """AsciiGridError::Parse: a token that is not an f64."""


class IoError(Exception):
    """IoError (io.rs:45-73): properties of the user's input files."""


class InvalidPixelSize(IoError):
    pass


class EmptyRaster(IoError):
    pass


class RasterShapeMismatch(IoError):
    pass


def _as_usize(v: float) -> int:
    """Rust's saturating `f64 as usize`: truncation, NaN and negatives to 0."""
    if v != v or v <= 0.0:
        return 0
    if v == math.inf:
        return 2 ** 64 - 1
    return int(v)


def _floor(v: float) -> float:
    """f64::floor, which keeps infinities and NaN."""
    return float(math.floor(v)) if math.isfinite(v) else v


@dataclass(frozen=True)
class AsciiGridHeader:
    """AsciiGridHeader (ascii_grid.rs:26-41)."""
    ncols: int
    nrows: int
    xllcorner: float
    yllcorner: float
    cellsize: float
    nodata_value: float

    def cell_at(self, x: float, y: float) -> Optional[Tuple[int, int]]:
        """(row, col) of the cell holding (x, y), row 0 = north, or None
        outside the grid (ascii_grid.rs:48-60)."""
        col = (x - self.xllcorner) / self.cellsize
        row_from_south = (y - self.yllcorner) / self.cellsize
        if col < 0.0 or row_from_south < 0.0:
            return None
        col = _as_usize(_floor(col))
        row_from_south = _as_usize(_floor(row_from_south))
        if col >= self.ncols or row_from_south >= self.nrows:
            return None
        return self.nrows - 1 - row_from_south, col

    def rows_overlapping_y_range(self, y_min: float, y_max: float) -> List[int]:
        """Rows (row 0 = north) whose extent overlaps [y_min, y_max)
        (ascii_grid.rs:66-75)."""
        lo_f = _floor((y_min - self.yllcorner) / self.cellsize)
        lo = _as_usize(max(lo_f, 0.0) if lo_f == lo_f else 0.0)  # f64::max ignores NaN
        hi_f = (y_max - self.yllcorner) / self.cellsize
        hi = min(_as_usize(math.ceil(hi_f) if math.isfinite(hi_f) else hi_f), self.nrows)
        return [self.nrows - 1 - r for r in range(lo, hi)]

    def _c(self) -> abi.hf_ascii_grid_header:
        return abi.hf_ascii_grid_header(int(self.ncols), int(self.nrows), float(self.xllcorner),
                                        float(self.yllcorner), float(self.cellsize),
                                        float(self.nodata_value))


def _raise_grid_error(rc: int):
    msg = last_error()
    if rc == abi.HF_ERR_SHAPE_MISMATCH:
        raise AsciiGridValueCountError(msg)
    if rc == abi.HF_ERR_OUT_OF_MEMORY:
        raise MemoryError(msg)
    if msg.startswith("malformed ASCII grid header"):
        raise AsciiGridHeaderError(msg)
    if msg.startswith("value ") and msg.endswith("is not a valid number"):
        raise AsciiGridParseError(msg)
    raise AsciiGridIoError(msg)


def read_ascii_grid(path) -> Tuple[np.ndarray, AsciiGridHeader]:
    """read_ascii_grid (ascii_grid.rs:101-160): the (nrows, ncols) values,
    row 0 = the first data row (north), and the header. A path ending in
    .gz is gunzipped."""
    h = abi.hf_ascii_grid_header()
    buf = C.POINTER(C.c_double)()
    rc = lib().hf_read_ascii_grid(os.fsencode(path), C.byref(h), C.byref(buf))
    if rc != 0:
        _raise_grid_error(rc)
    try:
        n = h.ncols * h.nrows
        data = np.ctypeslib.as_array(buf, shape=(max(n, 1),))[:n].copy() if n else \
            np.empty(0, dtype=np.float64)
    finally:
        lib().hf_free_buffer(C.cast(buf, C.c_void_p))
    header = AsciiGridHeader(h.ncols, h.nrows, h.xllcorner, h.yllcorner, h.cellsize,
                             h.nodata_value)
    return data.reshape(h.nrows, h.ncols), header


def write_ascii_grid(path, data, header: AsciiGridHeader) -> None:
    """Write `data` ((nrows, ncols), row 0 = north) as an ESRI ASCII grid that
    read_ascii_grid returns bit for bit; gzip when the path ends in .gz."""
    a = np.ascontiguousarray(data, dtype=np.float64)
    if a.shape != (header.nrows, header.ncols):
        raise ValueError(f"data shape {a.shape} does not match the header "
                         f"({header.nrows}, {header.ncols})")
    h = header._c()
    rc = lib().hf_write_ascii_grid(os.fsencode(path), C.byref(h),
                                   a.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise AsciiGridIoError(last_error())


def depth_raster_from_states(h, nodata: Optional[float] = None) -> np.ndarray:
    """depth_raster_from_states (io.rs:216-234) on a depth array: h, or
    `nodata` where h <= H_DRY when nodata is given."""
    a = np.ascontiguousarray(h, dtype=np.float64)
    out = np.empty_like(a)
    rc = lib().hf_depth_raster(a.size, a.ctypes.data_as(C.POINTER(C.c_double)),
                               0 if nodata is None else 1,
                               0.0 if nodata is None else float(nodata),
                               out.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise ValueError(last_error())
    return out


def write_depth_ascii_grid(path, h, header: AsciiGridHeader,
                           nodata: Optional[float] = None) -> None:
    """write_depth_geotiff (io.rs:241-254) with an ESRI ASCII grid for the
    file: the depth raster on the DEM's geometry, with `nodata` recorded as
    the grid's no-data value when given."""
    depth = depth_raster_from_states(h, nodata)
    hdr = header if nodata is None else AsciiGridHeader(
        header.ncols, header.nrows, header.xllcorner, header.yllcorner, header.cellsize,
        float(nodata))
    write_ascii_grid(path, depth, hdr)


def esa_worldcover_to_manning(code: int) -> float:
    """esa_worldcover_to_manning (io.rs:192-207)."""
    code = int(code)
    if not 0 <= code <= 255:
        raise ValueError(f"land-cover code {code} is not a u8")
    return float(lib().hf_worldcover_manning(code))


def _mesh_checks(bed: np.ndarray, header: AsciiGridHeader):
    cs = header.cellsize
    if not cs > 0.0:
        raise InvalidPixelSize(f"pixel size must be strictly positive, got dx = {cs}, dy = {cs}")
    if bed.size == 0:
        raise EmptyRaster("raster is empty")


def mesh_from_ascii_grid(path, manning) -> Tuple[Mesh2D, AsciiGridHeader]:
    """mesh_from_geotiff (io.rs:84-105) for an ASCII-grid DEM. `manning` is a
    uniform n, or the path of a Manning-n grid on the DEM's geometry
    (Mesh2D::with_manning_field, as the urban rain/point-inflow example
    solver-2d/examples/uk_ea_test8a_official.rs:141-160 builds its mesh)."""
    bed, header = read_ascii_grid(path)
    _mesh_checks(bed, header)
    if isinstance(manning, (str, bytes, os.PathLike)):
        n, nh = read_ascii_grid(manning)
        if (nh.nrows, nh.ncols) != (header.nrows, header.ncols):
            raise RasterShapeMismatch(
                f"DEM shape {(header.nrows, header.ncols)} does not match Manning grid shape "
                f"{(nh.nrows, nh.ncols)}")
        return Mesh2D.with_manning_field(bed, header.cellsize, header.cellsize, n), header
    return Mesh2D(bed, header.cellsize, header.cellsize, float(manning)), header


def mesh_from_ascii_grid_with_landcover(
        dem_path, landcover_path,
        landcover_to_manning: Callable[[int], float] = esa_worldcover_to_manning,
) -> Tuple[Mesh2D, AsciiGridHeader]:
    """mesh_from_geotiff_with_landcover (io.rs:132-165): the DEM's geometry,
    Manning n from the land-cover class (a u8) of each cell."""
    bed, header = read_ascii_grid(dem_path)
    lc, lh = read_ascii_grid(landcover_path)
    if (lh.nrows, lh.ncols) != (header.nrows, header.ncols):
        raise RasterShapeMismatch(
            f"DEM shape {(header.nrows, header.ncols)} does not match landcover shape "
            f"{(lh.nrows, lh.ncols)}")
    _mesh_checks(bed, header)
    if not (np.all(np.isfinite(lc)) and np.all(lc == np.floor(lc))
            and lc.min(initial=0) >= 0 and lc.max(initial=0) <= 255):
        raise ValueError("land-cover grid values must be integers in 0..=255")
    codes = lc.astype(np.int64)
    table = {int(c): float(landcover_to_manning(int(c))) for c in np.unique(codes)}
    manning = np.vectorize(table.__getitem__, otypes=[np.float64])(codes) if codes.size else \
        np.zeros(codes.shape)
    return Mesh2D.with_manning_field(bed, header.cellsize, header.cellsize, manning), header


__all__ = [
    "AsciiGridError", "AsciiGridIoError", "AsciiGridHeaderError", "AsciiGridValueCountError",
    "AsciiGridParseError", "IoError", "InvalidPixelSize", "EmptyRaster", "RasterShapeMismatch",
    "AsciiGridHeader", "read_ascii_grid", "write_ascii_grid", "depth_raster_from_states",
    "write_depth_ascii_grid", "esa_worldcover_to_manning", "mesh_from_ascii_grid",
    "mesh_from_ascii_grid_with_landcover", "H_DRY",
]
