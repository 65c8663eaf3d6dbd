"""Generate libm_tables.cuh: the tables of the elementary functions in
elementary.cuh, computed from their definitions with 300-bit arithmetic.

* DCLAW_EXP_TABLE_DATA, 128 pairs (bits(T), bits(H) - k 2^52/128) for
  k = 0 .. 127: H is 2^(k/128) rounded to the nearest double and
  T = 2^(k/128)/H - 1 rounded to the nearest double, so that 2^(k/128) =
  H (1 + T) to about 2^-106. This is the table of the published exp of ARM's
  optimized-routines (math/exp.c, math/exp_data.c), which glibc 2.28 and
  later use as sysdeps/ieee754/dbl-64/e_exp.c.
* DCLAW_ATAN_TABLE_DATA, 65 pairs (hi, lo) with hi + lo = atan(k/64) to
  about 2^-106 (hi the nearest double, lo the nearest double to the rest),
  k = 0 .. 64.
* DCLAW_TAN_TABLE_DATA, 52 pairs (hi, lo) with hi + lo = tan(k/64),
  k = 0 .. 51.
* DCLAW_POW_LOG_TABLE_DATA, 128 triples (invc, logc, logctail) of the
  logarithm inside the published pow of ARM's optimized-routines
  (math/pow.c, math/pow_log_data.c; glibc's sysdeps/ieee754/dbl-64/e_pow.c):
  z in [0x1.69555p-1, 0x1.69555p0) is split by the top 7 bits of
  bits(z) - 0x3fe6955500000000 into 128 subintervals; for the centre of
  subinterval i, 1/c = round(128/centre)/128 when the centre is below 1,
  round(256/centre)/256 otherwise (a few bits, so z/c - 1 is exact);
  logc = log(c) rounded to a multiple of 2^-43 and logctail = log(c) -
  logc rounded to the nearest double.

Run: python dclaw_b200/csrc/gen_libm_tables.py  (needs mpmath)
"""
import struct
from pathlib import Path

import mpmath


def bits(d: float) -> int:
    return struct.unpack("<Q", struct.pack("<d", d))[0]


def exp_table():
    n = 128
    out = []
    for k in range(n):
        v = mpmath.mpf(2) ** (mpmath.mpf(k) / n)
        h = float(v)  # nearest double
        t = float((v - h) / h)
        out.append(f"0x{bits(t):016x}ull, 0x{(bits(h) - (k << 52) // n) & (2**64 - 1):016x}ull")
    return out


def dd_table(fn, count):
    out = []
    for k in range(count):
        v = fn(mpmath.mpf(k) / 64)
        hi = float(v)
        lo = float(v - hi)
        out.append(f"{hi.hex()}, {lo.hex()}")
    return out


def pow_log_table():
    n, off = 128, 0x3fe6955500000000

    def asd(u):
        return struct.unpack("<d", struct.pack("<Q", u))[0]

    out = []
    for i in range(n):
        zlo, zhi = asd(off + i * (1 << 45)), asd(off + (i + 1) * (1 << 45))
        centre = (mpmath.mpf(zlo) + mpmath.mpf(zhi)) / 2
        invc = mpmath.nint(n / centre) / n if centre < 1 else mpmath.nint(2 * n / centre) / n / 2
        lc = mpmath.log(1 / invc)
        logc = mpmath.nint(lc * 2**43) / 2**43
        out.append(f"{float(invc).hex()}, {float(logc).hex()}, {float(lc - logc).hex()}")
    return out


def macro(name, rows):
    return f"#define {name} \\\n" + " \\\n".join("    " + r + ("," if i + 1 < len(rows) else "")
                                              for i, r in enumerate(rows)) + "\n"


def main():
    mpmath.mp.prec = 300
    text = (
        "// libm_tables.cuh -- generated by gen_libm_tables.py; do not edit.\n"
        "#pragma once\n"
        "// 2^(k/128) = H (1 + T), k = 0..127: pairs (bits(T), bits(H) - k 2^52/128)\n"
        + macro("DCLAW_EXP_TABLE_DATA", exp_table())
        + "// atan(k/64) = hi + lo, k = 0..64\n"
        + macro("DCLAW_ATAN_TABLE_DATA", dd_table(mpmath.atan, 65))
        + "// tan(k/64) = hi + lo, k = 0..51\n"
        + macro("DCLAW_TAN_TABLE_DATA", dd_table(mpmath.tan, 52))
        + "// pow's logarithm: (1/c, log(c) to a multiple of 2^-43, the rest), i = 0..127\n"
        + macro("DCLAW_POW_LOG_TABLE_DATA", pow_log_table())
    )
    Path(__file__).with_name("libm_tables.cuh").write_text(text)


if __name__ == "__main__":
    main()
