"""Writes fft_trig.h: cos(2 pi k / R) and sin(2 pi k / R), k = 0 .. (R-1)/2, for
the odd radices of the DFT engine (the primes, and 9 for the direct radix-9
butterfly of the 126-point Rader convolution), as correctly rounded FP64
literals.

The values come from 60-digit Taylor series in Python's decimal module (no
floating-point library is involved); float(Decimal) rounds to nearest.  Run
it from this directory after changing RADICES:  python gen_fft_trig.py
"""
from decimal import Decimal, getcontext

RADICES = (3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 9)

getcontext().prec = 60


def pi():
    # Machin: pi = 16 atan(1/5) - 4 atan(1/239)
    def atan_inv(x):
        x = Decimal(x)
        term = 1 / x
        s, k, sign = term, 1, 1
        while True:
            term /= x * x
            k += 2
            sign = -sign
            t = term / k
            if t < Decimal(10) ** -70:
                return s
            s += sign * t
    return 16 * atan_inv(5) - 4 * atan_inv(239)


def cos_sin(a):
    c, s = Decimal(0), Decimal(0)
    term = Decimal(1)
    n = 0
    while abs(term) > Decimal(10) ** -70 or n < 4:
        if n % 4 == 0:
            c += term
        elif n % 4 == 1:
            s += term
        elif n % 4 == 2:
            c -= term
        else:
            s -= term
        n += 1
        term = term * a / n
    return c, s


def render():
    """The text of fft_trig.h."""
    P = pi()
    lines = [
        "// Generated by gen_fft_trig.py: cos / sin (2 pi k / R), k = 0 .. (R-1)/2, for the odd",
        "// radices of the DFT engine, at kTrigCos[TrigOff<R>::v + k].  Do not edit by hand.",
        "// Indexed with compile-time offsets, the values are constant-bank operands.",
        "#pragma once",
        "",
        "namespace so3g {",
        "",
        "template <int R>",
        "struct TrigOff;",
    ]
    cs, sn, off = [], [], 0
    for R in RADICES:
        H = (R - 1) // 2
        lines.append(f"template <>\nstruct TrigOff<{R}> {{\n  static constexpr int v = {off};\n}};")
        for k in range(0, H + 1):
            c, s = cos_sin(2 * P * k / R)
            cs.append(float(c).hex())
            sn.append(float(s).hex())
        off += H + 1

    def table(name, vals):
        out = [f"static __constant__ double {name}[{len(vals)}] = {{"]
        for i in range(0, len(vals), 4):
            out.append("    " + ", ".join(vals[i:i + 4]) + ",")
        out.append("};")
        return out

    lines += [""] + table("kTrigCos", cs) + table("kTrigSin", sn)
    lines += ["", "}  // namespace so3g", ""]
    return "\n".join(lines)


def main():
    open("fft_trig.h", "w").write(render())


if __name__ == "__main__":
    main()
