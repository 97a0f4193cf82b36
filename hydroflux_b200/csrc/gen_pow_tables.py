#!/usr/bin/env python
"""Writes hf_pow_tables.h: the two 128-entry tables of the libm-rounded pow
(hf_pow.h), computed exactly from their defining rules.

log table, entry i (x = 2^k z, z in [0x1.69555p-1, 0x1.69555p0) split into
128 subintervals by the 7 bits below the exponent of z's pattern, counted
from 0x3fe6955500000000):
    center = midpoint of subinterval i
    1/c    = round(128/center)/128 if center < 1 else round(256/center)/256
    logc   = round(2^43 log c) / 2^43        (k*ln2hi + logc is then exact)
    ctail  = RN(log c - logc)
exp table, entry j: H = RN(2^(j/128)) and T = RN(2^(j/128)/H - 1), so that
2^(j/128) = H (1 + T) to ~2^-106.

These are the definitions published with the table-driven pow of Szabolcs
Nagy (ARM optimized-routines, 2018), which glibc has used since 2.28; the
values follow from them with 80-digit decimal arithmetic and exact rationals.

    python hydroflux_b200/csrc/gen_pow_tables.py [--check]
"""
from __future__ import annotations

import os
import struct
import sys
from decimal import Decimal, getcontext
from fractions import Fraction

getcontext().prec = 80
N = 128
LOG_OFF = 0x3fe6955500000000
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hf_pow_tables.h")


def rn(x) -> float:
    """Nearest double (ties to even) of an exact Decimal or Fraction."""
    return float(Fraction(x))


def from_bits(b: int) -> float:
    return struct.unpack("<d", struct.pack("<Q", b))[0]


def log_table():
    rows = []
    for i in range(N):
        lo = Fraction(from_bits(LOG_OFF + (i << 45)))
        hi = Fraction(from_bits(LOG_OFF + ((i + 1) << 45)))
        center = (lo + hi) / 2
        invc = Fraction(round(N / center), N) if center < 1 else Fraction(round(2 * N / center),
                                                                          2 * N)
        log_c = -(Decimal(invc.numerator) / Decimal(invc.denominator)).ln()
        scale = Decimal(2) ** 43
        logc = Decimal(round(log_c * scale)) / scale
        rows.append((float(invc), float(logc), rn(log_c - logc)))
    return rows


def exp_table():
    ln2 = Decimal(2).ln()
    rows = []
    for j in range(N):
        v = (ln2 * j / N).exp()
        h = rn(v)
        rows.append((h, rn(v / Decimal(h) - 1)))
    return rows


def render() -> str:
    out = ["// Generated by gen_pow_tables.py from the tables' defining rules; do not edit.",
           "#pragma once", "",
           "// {1/c, logc, ctail} for the 128 subintervals of the log reduction.",
           "#define HF_POW_LOG_TABLE { \\"]
    out += [f"  {{{a.hex()}, {b.hex()}, {c.hex()}}}, \\" for a, b, c in log_table()]
    out += ["}", "", "// {H, T} with 2^(j/128) = H (1 + T), j = 0..127.",
            "#define HF_POW_EXP_TABLE { \\"]
    out += [f"  {{{h.hex()}, {t.hex()}}}, \\" for h, t in exp_table()]
    out += ["}", ""]
    return "\n".join(out)


if __name__ == "__main__":
    text = render()
    if "--check" in sys.argv:
        sys.exit(0 if open(OUT).read() == text else "hf_pow_tables.h is out of date")
    with open(OUT, "w") as f:
        f.write(text)
    print(OUT)
