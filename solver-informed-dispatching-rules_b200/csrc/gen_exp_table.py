"""Writes sidr_exp_table.h: the 2^(k/128) table of the exponential in
sidr_libm.cuh (k = 0..127).  Each entry splits 2^(k/128) into the double S_k
nearest to it and the relative remainder tail_k = (2^(k/128) - S_k) / S_k
rounded to a double, so that 2^(k/128) = S_k * (1 + tail_k) to about 2^-106;
S_k is stored with k << 45 subtracted from its bit pattern, which the
exponential adds back together with the power of two of the reduced argument.

    python gen_exp_table.py      (needs mpmath; output is committed)
"""
import os
import struct

import mpmath

mpmath.mp.prec = 300


def bits(x: float) -> int:
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def main() -> None:
    lines = []
    for k in range(128):
        v = mpmath.power(2, mpmath.mpf(k) / 128)
        s = float(v)  # round to nearest
        tail = float((v - mpmath.mpf(s)) / mpmath.mpf(s))
        lines.append(f"    0x{bits(tail):016x}ull, 0x{(bits(s) - (k << 45)) & (2**64 - 1):016x}ull,")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sidr_exp_table.h")
    with open(out, "w") as f:
        f.write("// Generated by gen_exp_table.py: {tail_k, S_k - (k << 45)} bit patterns of\n"
                "// 2^(k/128) = S_k * (1 + tail_k), k = 0..127.\n")
        f.write("#pragma once\n#include <stdint.h>\n\n")
        f.write("#define SIDR_EXP_TABLE_ENTRIES \\\n")
        f.write(" \\\n".join(lines) + "\n")
    print("wrote", out)


if __name__ == "__main__":
    main()
