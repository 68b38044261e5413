"""Writes sidr_sample_consts.h: the double-double constants of the on-device
scenario sampler (sidr_sample.cuh) -- ln 2, pi/2 in three parts, 1/n! for
n = 0..33 and 1/(2k+1) for k = 0..27 -- each the double nearest the value and
the double nearest the remainder (pi/2: a third part).

    python gen_sample_consts.py      (needs mpmath; output is committed)
"""
import os

import mpmath

mpmath.mp.prec = 400


def parts(x, n=2):
    out, r = [], mpmath.mpf(x)
    for _ in range(n):
        h = float(r)  # round to nearest
        out.append(h)
        r -= mpmath.mpf(h)
    return out


def dd(x):
    h, l = parts(x)
    return f"{{{h.hex()}, {l.hex()}}}"


def main() -> None:
    lines = ["// Generated by gen_sample_consts.py: double-double constants (hi, lo) of the", "// on-device scenario sampler.  Do not edit.", "#pragma once", ""]
    lines.append(f"#define SIDR_LN2_HI {parts(mpmath.log(2))[0].hex()}")
    lines.append(f"#define SIDR_LN2_LO {parts(mpmath.log(2))[1].hex()}")
    p = parts(mpmath.pi / 2, 3)
    for i, v in enumerate(p, 1):
        lines.append(f"#define SIDR_PIO2_{i} {v.hex()}")
    lines.append(f"#define SIDR_TWO_OVER_PI {float(2 / mpmath.pi).hex()}")
    lines.append("")
    lines.append("// 1/n!, n = 0..33")
    lines.append("#define SIDR_INV_FACT_TABLE \\")
    for n in range(34):
        lines.append(f"    {dd(1 / mpmath.factorial(n))}, \\")
    lines.append("")
    lines.append("")
    lines.append("// 1/(2k+1), k = 0..27")
    lines.append("#define SIDR_INV_ODD_TABLE \\")
    for k in range(28):
        lines.append(f"    {dd(mpmath.mpf(1) / (2 * k + 1))}, \\")
    lines.append("")
    lines.append("")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sidr_sample_consts.h")
    with open(out, "w") as f:
        f.write("\n".join(lines))


if __name__ == "__main__":
    main()
