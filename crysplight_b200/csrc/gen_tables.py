"""Generate cl_tables.h: constants for the device's Float32 elementary functions.

Every value is computed here from its mathematical definition with Python's
``decimal`` module at 60 significant digits and rounded once to IEEE double
(``float(Decimal)`` rounds correctly):

* pi/2 as a two-term double split (hi + lo) and 2/pi, for the Cody-Waite
  argument reduction of sin/cos;
* the Taylor coefficients (-1)^k / (2k+1)! and (-1)^k / (2k)! of sin and cos;
* ln 2 and, for F_j = 1 + j/64 (j = -19..27), the pairs (1/F_j, ln F_j) of a
  table-driven logarithm in the manner of P. T. P. Tang, "Table-driven
  implementation of the logarithm function in IEEE floating-point arithmetic",
  ACM TOMS 16(4), 1990;
* the Taylor coefficients (-1)^(k+1)/k of log1p.

Run: python gen_tables.py > cl_tables.h
"""
from decimal import Decimal, getcontext
import math

getcontext().prec = 60

LOG_JMIN, LOG_JMAX = -19, 27   # round(64*(m-1)) for m in [sqrt(1/2), sqrt(2))


def d_pi() -> Decimal:
    """pi by Machin's formula: 16 atan(1/5) - 4 atan(1/239)."""
    def atan_inv(n: int) -> Decimal:
        x = Decimal(1) / n
        x2 = x * x
        term, total, k = x, x, 1
        eps = Decimal(10) ** (-(getcontext().prec + 2))
        while abs(term) > eps:
            term *= -x2
            total += term / (2 * k + 1)
            k += 1
        return total
    return 16 * atan_inv(5) - 4 * atan_inv(239)


def d_sin_cos(x: Decimal) -> tuple:
    """sin and cos by their Taylor series at 60 digits (|x| <= 2 pi)."""
    eps = Decimal(10) ** (-(getcontext().prec + 2))
    s, c = Decimal(0), Decimal(0)
    term, n = Decimal(1), 0          # x^n / n!
    while True:
        if n % 4 == 0: c += term
        elif n % 4 == 1: s += term
        elif n % 4 == 2: c -= term
        else: s -= term
        n += 1
        term = term * x / n
        if abs(term) < eps and n > 4:
            break
    return s, c


def dbl(x: Decimal) -> float:
    return float(x)


def hexd(v: float) -> str:
    return float.hex(v)


def main() -> None:
    pi = d_pi()
    pio2 = pi / 2
    pio2_hi = dbl(pio2)
    pio2_lo = dbl(pio2 - Decimal(pio2_hi))
    two_over_pi = dbl(2 / pi)
    ln2 = dbl(Decimal(2).ln())

    out = []
    out.append("/* Generated by gen_tables.py from exact arithmetic (decimal, 60 digits). */")
    out.append("#pragma once")
    out.append("")
    out.append(f"#define CLM_PIO2_HI {hexd(pio2_hi)}  /* {pio2_hi!r} */")
    out.append(f"#define CLM_PIO2_LO {hexd(pio2_lo)}  /* {pio2_lo!r} */")
    out.append(f"#define CLM_2_OVER_PI {hexd(two_over_pi)}  /* {two_over_pi!r} */")
    out.append(f"#define CLM_LN2 {hexd(ln2)}  /* {ln2!r} */")
    out.append("")
    # sin: r + r^3 (S3 + r^2 (S5 + ... + r^2 S17)); cos: 1 + r^2 (C2 + ... + r^2 C16)
    for n in range(3, 18, 2):
        c = Decimal((-1) ** ((n - 1) // 2)) / Decimal(math.factorial(n))
        out.append(f"#define CLM_S{n} {hexd(dbl(c))}")
    for n in range(2, 17, 2):
        c = Decimal((-1) ** (n // 2)) / Decimal(math.factorial(n))
        out.append(f"#define CLM_C{n} {hexd(dbl(c))}")
    out.append("")
    # log1p(r) = r + r^2 (L2 + r (L3 + ... + r L8)), L_k = (-1)^(k+1)/k
    for k in range(2, 9):
        c = Decimal((-1) ** (k + 1)) / Decimal(k)
        out.append(f"#define CLM_L{k} {hexd(dbl(c))}")
    out.append("")
    out.append(f"#define CLM_LOG_JMIN ({LOG_JMIN})")
    out.append(f"#define CLM_LOG_NTAB {LOG_JMAX - LOG_JMIN + 1}")
    out.append("/* (1/F_j, ln F_j), F_j = 1 + j/64, j = CLM_LOG_JMIN .. */")
    out.append("#define CLM_LOG_TAB_INIT \\")
    for j in range(LOG_JMIN, LOG_JMAX + 1):
        F = Decimal(64 + j) / Decimal(64)
        inv = dbl(1 / F)
        lg = dbl(F.ln()) if j != 0 else 0.0
        out.append(f"    {hexd(inv)}, {hexd(lg)},  /* j = {j} */ \\")
    out.append("")
    # table-driven sincos: x = j*delta + r, delta = 2 pi / 256, |r| <= delta/2
    n_sc = 256
    delta = 2 * pi / n_sc
    d_hi = dbl(delta)
    d_lo = dbl(delta - Decimal(d_hi))
    out.append("")
    out.append(f"#define CLM_SC_N {n_sc}")
    out.append(f"#define CLM_SC_DELTA_HI {hexd(d_hi)}")
    out.append(f"#define CLM_SC_DELTA_LO {hexd(d_lo)}")
    out.append(f"#define CLM_SC_INV_DELTA {hexd(dbl(1 / delta))}")
    for n in (3, 5, 7):
        c = Decimal((-1) ** ((n - 1) // 2)) / Decimal(math.factorial(n))
        out.append(f"#define CLM_TS{n} {hexd(dbl(c))}")
    for n in (2, 4, 6, 8):
        c = Decimal((-1) ** (n // 2)) / Decimal(math.factorial(n))
        out.append(f"#define CLM_TC{n} {hexd(dbl(c))}")
    out.append("/* (sin, cos)(j * 2 pi / 256), j = 0..255; exact zeros where the value is 0 */")
    out.append("#define CLM_SC_TAB_INIT \\")
    for j in range(n_sc):
        if j % 64 == 0:
            sj, cj = (0.0, [1.0, 0.0, -1.0, 0.0][j // 64]) if j % 128 == 0 else (
                [0.0, 1.0, 0.0, -1.0][j // 64], 0.0)
        else:
            sd, cd = d_sin_cos(delta * j)
            sj, cj = dbl(sd), dbl(cd)
        out.append(f"    {hexd(sj)}, {hexd(cj)},  /* j = {j} */ \\")
    out.append("")
    print("\n".join(out))


if __name__ == "__main__":
    main()
