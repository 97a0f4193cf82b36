// hf_io.cu -- ESRI ASCII grid rasters in and out (host code).
//
// The reference reads its benchmark DEMs from ESRI ASCII grids, optionally
// gzip-compressed (solver-2d/src/ascii_grid.rs:101-160), and writes depth
// rasters from the state (io.rs:216-240). This is the same format on the
// library's side of the C ABI: a strict reader (the six header lines in the
// reference's order, keys matched case-insensitively, then exactly
// ncols * nrows whitespace-separated values in any line layout; row 0 is the
// first data row, the northern one) and a writer whose output the reader
// returns bit for bit. Paths ending in ".gz" are gzip streams.
#include <strings.h>
#include <zlib.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/hydroflux_gpu.h"
#include "hf_internal.h"

namespace {

int io_fail(int code, const std::string& m) { return hf::record_error(code, m.c_str()); }

bool ends_with_gz(const char* path) {
  const size_t n = std::strlen(path);
  return n >= 3 && std::strcmp(path + n - 3, ".gz") == 0;
}

// Byte length of the Unicode White_Space code point at p (0 if there is
// none): the separators of str::split_whitespace, which the reference splits
// its header lines and data section on.
size_t ws_len(const char* p, const char* e) {
  const unsigned char c = (unsigned char)*p;
  if (c == ' ' || (c >= 0x09 && c <= 0x0D)) return 1;
  if (c < 0xC2 || e - p < 2) return 0;
  const unsigned char c1 = (unsigned char)p[1];
  if (c == 0xC2) return (c1 == 0x85 || c1 == 0xA0) ? 2 : 0;
  if (e - p < 3) return 0;
  const unsigned char c2 = (unsigned char)p[2];
  if (c == 0xE1) return (c1 == 0x9A && c2 == 0x80) ? 3 : 0;  // U+1680
  if (c == 0xE2 && c1 == 0x80)                               // U+2000-200A, 2028, 2029, 202F
    return (c2 <= 0x8A || c2 == 0xA8 || c2 == 0xA9 || c2 == 0xAF) ? 3 : 0;
  if (c == 0xE2 && c1 == 0x81) return c2 == 0x9F ? 3 : 0;    // U+205F
  if (c == 0xE3) return (c1 == 0x80 && c2 == 0x80) ? 3 : 0;  // U+3000
  return 0;
}

const char* skip_ws(const char* p, const char* e) {
  size_t n;
  while (p < e && (n = ws_len(p, e)) > 0) p += n;
  return p;
}

const char* skip_word(const char* p, const char* e) {
  while (p < e && ws_len(p, e) == 0) ++p;
  return p;
}

// The reference reads the file into a String, so bytes that are not UTF-8
// are an I/O error there too.
bool valid_utf8(const std::string& s) {
  const unsigned char* p = (const unsigned char*)s.data();
  const unsigned char* e = p + s.size();
  while (p < e) {
    const unsigned c = *p;
    if (c < 0x80) { ++p; continue; }
    int n;
    unsigned lo = 0x80, hi = 0xBF;
    if (c >= 0xC2 && c <= 0xDF) n = 1;
    else if (c >= 0xE0 && c <= 0xEF) {
      n = 2;
      if (c == 0xE0) lo = 0xA0;  // no overlong forms
      if (c == 0xED) hi = 0x9F;  // no surrogates
    } else if (c >= 0xF0 && c <= 0xF4) {
      n = 3;
      if (c == 0xF0) lo = 0x90;
      if (c == 0xF4) hi = 0x8F;  // nothing above U+10FFFF
    } else {
      return false;
    }
    if (e - p <= n) return false;
    if (p[1] < lo || p[1] > hi) return false;
    for (int k = 2; k <= n; ++k)
      if (p[k] < 0x80 || p[k] > 0xBF) return false;
    p += n + 1;
  }
  return true;
}

// First gzip member of `raw` (flate2's GzDecoder, which the reference reads
// .gz files with, stops there too); a bad header, a corrupt or truncated
// stream or a checksum mismatch is an error.
int gunzip_first_member(const std::string& raw, const char* path, std::string& out) {
  z_stream zs;
  std::memset(&zs, 0, sizeof zs);
  if (inflateInit2(&zs, 16 + MAX_WBITS) != Z_OK)
    return io_fail(HF_ERR_INVALID_ARG, "zlib initialisation failed");
  zs.next_in = (Bytef*)raw.data();
  std::vector<char> buf(1 << 20);
  size_t left = raw.size();
  int zr = Z_OK;
  while (zr != Z_STREAM_END) {
    if (zs.avail_in == 0 && left > 0) {
      const uInt chunk = (uInt)std::min<size_t>(left, 1u << 30);
      zs.avail_in = chunk;
      left -= chunk;
    }
    zs.next_out = (Bytef*)buf.data();
    zs.avail_out = (uInt)buf.size();
    zr = inflate(&zs, Z_NO_FLUSH);
    if (zr != Z_OK && zr != Z_STREAM_END) break;
    out.append(buf.data(), buf.size() - zs.avail_out);
    if (zr == Z_OK && zs.avail_in == 0 && left == 0 && zs.avail_out != 0) {
      zr = Z_BUF_ERROR;  // input ended inside the member
      break;
    }
  }
  const std::string msg = zs.msg ? zs.msg : "truncated gzip stream";
  inflateEnd(&zs);
  if (zr != Z_STREAM_END)
    return io_fail(HF_ERR_INVALID_ARG, std::string("gzip error in ") + path + ": " + msg);
  return HF_OK;
}

// Whole file; a path ending in ".gz" must hold a gzip stream (the reference
// picks its decoder by the extension alone) and the text must be UTF-8.
int slurp(const char* path, std::string& out) {
  out.clear();
  std::string raw;
  FILE* f = std::fopen(path, "rb");
  if (!f) return io_fail(HF_ERR_INVALID_ARG, std::string("cannot open ") + path);
  char buf[1 << 16];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) raw.append(buf, n);
  const bool err = std::ferror(f) != 0;
  std::fclose(f);
  if (err) return io_fail(HF_ERR_INVALID_ARG, std::string("read error in ") + path);
  if (ends_with_gz(path)) {
    const int rc = gunzip_first_member(raw, path, out);
    if (rc) return rc;
  } else {
    out.swap(raw);
  }
  if (!valid_utf8(out))
    return io_fail(HF_ERR_INVALID_ARG, std::string("stream did not contain valid UTF-8: ") + path);
  return HF_OK;
}

// A decimal number token as the reference's f64 parser takes it: optional
// sign, digits with an optional point, optional exponent, or inf / infinity
// / nan in any case. The value is strtod's (correctly rounded).
// [b, e) is checked in place; strtod parses a copy of it.
bool parse_number(const char* b, const char* e, double* out) {
  const char* p = b;
  if (p < e && (*p == '+' || *p == '-')) ++p;
  bool ok;
  if (p < e && std::isalpha((unsigned char)*p)) {
    const size_t n = (size_t)(e - p);
    ok = (n == 3 && (strncasecmp(p, "inf", 3) == 0 || strncasecmp(p, "nan", 3) == 0)) ||
         (n == 8 && strncasecmp(p, "infinity", 8) == 0);
  } else {
    bool digits = false;
    while (p < e && std::isdigit((unsigned char)*p)) { ++p; digits = true; }
    if (p < e && *p == '.') {
      ++p;
      while (p < e && std::isdigit((unsigned char)*p)) { ++p; digits = true; }
    }
    if (digits && p < e && (*p == 'e' || *p == 'E')) {
      ++p;
      if (p < e && (*p == '+' || *p == '-')) ++p;
      bool ed = false;
      while (p < e && std::isdigit((unsigned char)*p)) { ++p; ed = true; }
      if (!ed) digits = false;
    }
    ok = digits && p == e;
  }
  if (!ok) return false;
  char small[64];
  std::string big;
  const size_t n = (size_t)(e - b);
  const char* s;
  if (n < sizeof small) {
    std::memcpy(small, b, n);
    small[n] = '\0';
    s = small;
  } else {
    big.assign(b, e);
    s = big.c_str();
  }
  char* end = nullptr;
  const double v = std::strtod(s, &end);
  if (end != s + n) return false;
  *out = v;  // overflow gives +-inf like the reference's parser
  return true;
}

// Next line of text (without the line break and a trailing '\r').
bool next_line(const std::string& text, size_t& pos, const char*& b, const char*& e) {
  if (pos >= text.size()) return false;
  size_t nl = text.find('\n', pos);
  if (nl == std::string::npos) nl = text.size();
  b = text.data() + pos;
  e = text.data() + nl;
  if (e > b && e[-1] == '\r') --e;
  pos = nl + 1;
  return true;
}

int header_value(const std::string& text, size_t& pos, const char* key, double* v) {
  const char *b, *e;
  if (!next_line(text, pos, b, e))
    return io_fail(HF_ERR_INVALID_ARG, std::string("malformed ASCII grid header: missing ") + key);
  const char* k0 = skip_ws(b, e);
  const char* k1 = skip_word(k0, e);
  if (k0 == k1)
    return io_fail(HF_ERR_INVALID_ARG,
                   std::string("malformed ASCII grid header: empty line, expected ") + key);
  if ((size_t)(k1 - k0) != std::strlen(key) || strncasecmp(k0, key, k1 - k0) != 0)
    return io_fail(HF_ERR_INVALID_ARG, std::string("malformed ASCII grid header: expected key ") +
                                           key + ", got " + std::string(k0, k1));
  const char* v0 = skip_ws(k1, e);
  const char* v1 = skip_word(v0, e);
  if (v0 == v1)
    return io_fail(HF_ERR_INVALID_ARG,
                   std::string("malformed ASCII grid header: missing value for ") + key);
  if (!parse_number(v0, v1, v))
    return io_fail(HF_ERR_INVALID_ARG, "value " + std::string(v0, v1) + " is not a valid number");
  return HF_OK;
}

// `as usize` of a parsed f64: truncation toward zero, negatives and NaN to 0.
int64_t as_count(double v) {
  if (!(v > 0.0)) return 0;
  if (v >= 9.0e18) return INT64_MAX;
  return (int64_t)v;
}

}  // namespace

extern "C" {

int hf_read_ascii_grid(const char* path, hf_ascii_grid_header* header, double** data) {
  if (!path || !header || !data) return io_fail(HF_ERR_INVALID_ARG, "null argument");
  *data = nullptr;
  std::string text;
  int rc = slurp(path, text);
  if (rc) return rc;
  size_t pos = 0;
  double ncols, nrows, xll, yll, cs, nodata;
  if ((rc = header_value(text, pos, "ncols", &ncols)) ||
      (rc = header_value(text, pos, "nrows", &nrows)) ||
      (rc = header_value(text, pos, "xllcorner", &xll)) ||
      (rc = header_value(text, pos, "yllcorner", &yll)) ||
      (rc = header_value(text, pos, "cellsize", &cs)) ||
      (rc = header_value(text, pos, "NODATA_value", &nodata)))
    return rc;
  const int64_t nc = as_count(ncols), nr = as_count(nrows);
  if (nc > 0 && nr > INT64_MAX / nc)
    return io_fail(HF_ERR_INVALID_ARG, "ASCII grid too large");
  const int64_t expected = nc * nr;
  std::vector<double> vals;
  vals.reserve((size_t)std::min<int64_t>(expected, (int64_t)1 << 28));
  const char* p = text.data() + std::min(pos, text.size());
  const char* end = text.data() + text.size();
  while (true) {
    p = skip_ws(p, end);
    if (p >= end) break;
    const char* q = skip_word(p, end);
    double v;
    if (!parse_number(p, q, &v))
      return io_fail(HF_ERR_INVALID_ARG, "value " + std::string(p, q) + " is not a valid number");
    vals.push_back(v);
    p = q;
  }
  if ((int64_t)vals.size() != expected)
    return io_fail(HF_ERR_SHAPE_MISMATCH, "expected " + std::to_string(expected) +
                                              " data values (ncols * nrows), found " +
                                              std::to_string(vals.size()));
  double* out = (double*)std::malloc(std::max<size_t>(1, vals.size()) * sizeof(double));
  if (!out) return io_fail(HF_ERR_OUT_OF_MEMORY, "out of host memory");
  if (!vals.empty()) std::memcpy(out, vals.data(), vals.size() * sizeof(double));
  header->ncols = nc;
  header->nrows = nr;
  header->xllcorner = xll;
  header->yllcorner = yll;
  header->cellsize = cs;
  header->nodata_value = nodata;
  *data = out;
  return HF_OK;
}

void hf_free_buffer(void* p) { std::free(p); }

int hf_write_ascii_grid(const char* path, const hf_ascii_grid_header* h, const double* data) {
  if (!path || !h || (!data && h->ncols * h->nrows > 0))
    return io_fail(HF_ERR_INVALID_ARG, "null argument");
  if (h->ncols < 0 || h->nrows < 0) return io_fail(HF_ERR_INVALID_ARG, "negative grid size");
  // %.17g round-trips every double; the reader parses the text back exactly.
  std::string out;
  char buf[64];
  auto num = [&](double v) {
    if (std::isnan(v)) return std::string("NaN");
    if (std::isinf(v)) return std::string(v > 0 ? "inf" : "-inf");
    std::snprintf(buf, sizeof buf, "%.17g", v);
    return std::string(buf);
  };
  out += "ncols " + std::to_string(h->ncols) + "\n";
  out += "nrows " + std::to_string(h->nrows) + "\n";
  out += "xllcorner " + num(h->xllcorner) + "\n";
  out += "yllcorner " + num(h->yllcorner) + "\n";
  out += "cellsize " + num(h->cellsize) + "\n";
  out += "NODATA_value " + num(h->nodata_value) + "\n";
  for (int64_t i = 0; i < h->nrows; ++i) {
    for (int64_t j = 0; j < h->ncols; ++j) {
      if (j) out += ' ';
      out += num(data[i * h->ncols + j]);
    }
    out += '\n';
  }
  if (ends_with_gz(path)) {
    gzFile f = gzopen(path, "wb");
    if (!f) return io_fail(HF_ERR_INVALID_ARG, std::string("cannot create ") + path);
    size_t off = 0;
    while (off < out.size()) {
      const unsigned chunk = (unsigned)std::min<size_t>(out.size() - off, 1u << 30);
      if (gzwrite(f, out.data() + off, chunk) != (int)chunk) {
        gzclose(f);
        return io_fail(HF_ERR_INVALID_ARG, std::string("write error in ") + path);
      }
      off += chunk;
    }
    if (gzclose(f) != Z_OK) return io_fail(HF_ERR_INVALID_ARG, std::string("write error in ") + path);
  } else {
    FILE* f = std::fopen(path, "wb");
    if (!f) return io_fail(HF_ERR_INVALID_ARG, std::string("cannot create ") + path);
    const size_t n = std::fwrite(out.data(), 1, out.size(), f);
    if (std::fclose(f) != 0 || n != out.size())
      return io_fail(HF_ERR_INVALID_ARG, std::string("write error in ") + path);
  }
  return HF_OK;
}

// depth_raster_from_states (io.rs:216-234): h, with `nodata` for cells with
// h <= H_DRY when use_nodata is set.
int hf_depth_raster(int64_t ncell, const double* h, int use_nodata, double nodata, double* out) {
  if (ncell < 0 || (ncell > 0 && (!h || !out))) return io_fail(HF_ERR_INVALID_ARG, "bad arguments");
  for (int64_t k = 0; k < ncell; ++k) out[k] = (use_nodata && h[k] <= 1.0e-6) ? nodata : h[k];
  return HF_OK;
}

// esa_worldcover_to_manning (io.rs:192-207).
double hf_worldcover_manning(int code) {
  switch (code) {
    case 10: return 0.100;
    case 20: return 0.060;
    case 30: return 0.040;
    case 40: return 0.035;
    case 50: return 0.015;
    case 60: return 0.025;
    case 70: return 0.030;
    case 80: return 0.030;
    case 90: return 0.050;
    case 95: return 0.100;
    case 100: return 0.045;
    default: return 0.040;
  }
}

}  // extern "C"
