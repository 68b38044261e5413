"""Writes sidr_pow_table.h: the 128-entry logarithm table of the power
function in sidr_libm.cuh (glibc 2.28+'s pow, from ARM optimized-routines).

For x = 2^k z with z in [0x1.69555p-1, 0x1.69555p0), the z range is cut into
128 subintervals by bits 45..51 of (bits(x) - 0x3fe6955500000000).  For the
subinterval of index i, c is a point near its centre whose reciprocal has few
bits, so that z/c - 1 is exact:

    1/c = round(128/centre)/128        when centre < 1,
          round(256/centre)/256        otherwise,

and the table holds {1/c, logc, logctail} with logc = log(c) rounded to a
multiple of 2^-43 (so k*ln2hi + logc is exact) and logctail = log(c) - logc
rounded to a double.  This is the construction that library documents for
its table; the values are computed here with 300-bit arithmetic.

    python gen_pow_table.py      (needs mpmath; output is committed)
"""
import os
import struct

import mpmath

mpmath.mp.prec = 300
N = 128
OFF = 0x3fe6955500000000


def value(bits: int) -> mpmath.mpf:
    return mpmath.mpf(struct.unpack("<d", struct.pack("<Q", bits))[0])


def main() -> None:
    lines = []
    for i in range(N):
        lo, hi = value(OFF + i * (1 << 45)), value(OFF + (i + 1) * (1 << 45))
        centre = (lo + hi) / 2
        if centre < 1:
            invc = mpmath.nint(N / centre) / N
        else:
            invc = mpmath.nint(2 * N / centre) / (2 * N)
        logc_exact = -mpmath.log(invc)
        logc = mpmath.nint(logc_exact * mpmath.mpf(2) ** 43) / mpmath.mpf(2) ** 43
        tail = float(logc_exact - logc)
        lines.append(f"    {float(invc).hex()}, {float(logc).hex()}, {tail.hex()},")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sidr_pow_table.h")
    with open(out, "w") as f:
        f.write("// Generated by gen_pow_table.py: {1/c, logc, logctail} for the 128\n"
                "// subintervals of the power function's logarithm.\n")
        f.write("#pragma once\n\n")
        f.write("#define SIDR_POW_LOG_TABLE_ENTRIES \\\n")
        f.write(" \\\n".join(lines) + "\n")
    print("wrote", out)


if __name__ == "__main__":
    main()
