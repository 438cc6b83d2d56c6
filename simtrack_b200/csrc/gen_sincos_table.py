"""Writes stb_sincos_table.cuh: the constants of the table-driven fast path
of cr_sin / cr_cos / cr_sincos (stb_crmath.cuh).

  * pi/128 split into three parts: two of 36 significant bits (k * part is
    exact for |k| < 2^17) and the rounded remainder;
  * sin(i pi/128) and cos(i pi/128), i = 0..63, each as a double-double
    (the rounded value and the rounded remainder).

Every value is computed with mpmath at 200 bits and rounded once to double.
Run from the repository root: python simtrack_b200/csrc/gen_sincos_table.py
"""
from pathlib import Path

import mpmath

OUT = Path(__file__).resolve().parent / "stb_sincos_table.cuh"


def rnd(v) -> float:
    with mpmath.workprec(53):
        return float(+v)


def round_bits(v, bits: int) -> float:
    with mpmath.workprec(bits):
        return float(+v)  # exact in a double for bits <= 53


def split_dd(v):
    hi = rnd(v)
    lo = rnd(v - mpmath.mpf(hi))
    return hi, lo


def text() -> str:
    with mpmath.workprec(200):
        h = mpmath.pi / 128
        c1 = round_bits(h, 36)
        c2 = round_bits(h - mpmath.mpf(c1), 36)
        c3 = rnd(h - mpmath.mpf(c1) - mpmath.mpf(c2))
        rows = []
        for i in range(64):
            s = split_dd(mpmath.sin(i * h))
            c = split_dd(mpmath.cos(i * h))
            rows.append(f"    {s[0].hex()}, {s[1].hex()}, {c[0].hex()}, {c[1].hex()},  /* i = {i} */")
        inv = rnd(128 / mpmath.pi)
    lines = [
        "// Generated by gen_sincos_table.py (mpmath, 200-bit evaluation, one rounding",
        "// per value); do not edit.",
        "#pragma once",
        "",
        "namespace stb {",
        "",
        f"constexpr double kPi128Inv = {inv.hex()};  // RN(128/pi)",
        f"constexpr double kPi128A = {c1.hex()};  // pi/128, leading 36 bits",
        f"constexpr double kPi128B = {c2.hex()};  // next 36 bits",
        f"constexpr double kPi128C = {c3.hex()};  // rounded remainder",
        "",
        "// [sin(i pi/128) hi, lo, cos(i pi/128) hi, lo], i = 0..63",
        "#define STB_SINCOS_TABLE_INIT \\",
        "  { \\",
    ]
    lines += [r + " \\" for r in rows]
    lines += ["  }", "", "}  // namespace stb", ""]
    return "\n".join(lines)


if __name__ == "__main__":
    OUT.write_text(text())
    print(f"wrote {OUT}")
