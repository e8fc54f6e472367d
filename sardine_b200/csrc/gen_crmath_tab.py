"""Generates crmath_tab.h: the constants of crmath.cuh, computed here in
decimal arithmetic at 80 significant digits (no libm involved).

    python sardine_b200/csrc/gen_crmath_tab.py > sardine_b200/csrc/crmath_tab.h

* pi/2 split into PIO2_1, PIO2_2 (33 significant bits each, so k * PIO2_i is
  exact for |k| < 2^20) and PIO2_3, PIO2_4 (53 bits each); ln 2 split the
  same way into LN2_1 (33 bits) and LN2_2;
* sin(j/256) and cos(j/256), j = 0..202, each as a double-double (hi, lo);
* 1/n!, n = 0..31, as double-doubles (the slow path's Taylor series) and
  1/(2n+1), n = 0..31, as doubles (the arctangent series).
"""
import math
from decimal import Decimal, getcontext

getcontext().prec = 80
TAB_N = 256
TAB_J = 203  # j/256 covers [0, pi/4 + 1/512]


def pi():
    # Machin: pi = 16 atan(1/5) - 4 atan(1/239)
    def atan_inv(n):
        x = Decimal(1) / n
        x2 = x * x
        s, t, k = Decimal(0), x, 1
        while True:
            term = t / k
            if abs(term) < Decimal(10) ** -85:
                return s + term
            s += term if (k // 2) % 2 == 0 else -term
            t *= x2
            k += 2
    return 16 * atan_inv(5) - 4 * atan_inv(239)


def sin_cos(x):
    s, c = Decimal(0), Decimal(0)
    t, n = Decimal(1), 0
    while True:
        if n % 4 == 0:
            c += t
        elif n % 4 == 1:
            s += t
        elif n % 4 == 2:
            c -= t
        else:
            s -= t
        n += 1
        t = t * x / n
        if abs(t) < Decimal(10) ** -85:
            return s, c


def dd(x):
    hi = float(x)  # float(Decimal) rounds to nearest
    lo = float(x - Decimal(hi))
    return hi, lo


def truncate_bits(x, bits):
    """x (a positive Decimal) rounded down to `bits` significant bits."""
    _, e = math.frexp(float(x))
    scale = Decimal(2) ** (bits - e)
    return float(int(x * scale) / scale)


def main():
    half_pi = pi() / 2
    p1 = truncate_bits(half_pi, 33)
    r = half_pi - Decimal(p1)
    p2 = truncate_bits(r, 33)
    r -= Decimal(p2)
    p3 = float(r)
    r -= Decimal(p3)
    p4 = float(r)
    print("// crmath_tab.h: generated by gen_crmath_tab.py (decimal arithmetic, 80 digits).")
    print("// Do not edit by hand.")
    print("#pragma once")
    print(f"#define CRM_TAB_N {TAB_N}")
    print(f"#define CRM_TAB_J {TAB_J}")
    print(f"#define CRM_TWO_OVER_PI {float(2 / pi()).hex()}")
    for i, p in enumerate((p1, p2, p3, p4), 1):
        print(f"#define CRM_PIO2_{i} {p.hex()}")
    ln2 = Decimal(2).ln()
    l1 = truncate_bits(ln2, 33)
    print(f"#define CRM_INV_LN2 {float(1 / ln2).hex()}")
    print(f"#define CRM_LN2_1 {l1.hex()}")
    print(f"#define CRM_LN2_2 {float(ln2 - Decimal(l1)).hex()}")
    print("// sin(j/256) hi, lo, cos(j/256) hi, lo")
    print("#define CRM_SINCOS_TABLE \\")
    for j in range(TAB_J):
        s, c = sin_cos(Decimal(j) / TAB_N)
        sh, sl = dd(s)
        ch, cl = dd(c)
        end = "," if j + 1 < TAB_J else ""
        print(f"  {sh.hex()}, {sl.hex()}, {ch.hex()}, {cl.hex()}{end} \\")
    print("")
    print("// 1/n! hi, lo (n = 0..31)")
    print("#define CRM_INVFACT_TABLE \\")
    f = Decimal(1)
    for n in range(32):
        if n:
            f *= n
        h, lo = dd(Decimal(1) / f)
        end = "," if n < 31 else ""
        print(f"  {h.hex()}, {lo.hex()}{end} \\")
    print("")
    print("// 1/(2n+1) (n = 0..31)")
    print("#define CRM_INVODD_TABLE \\")
    for n in range(32):
        end = "," if n < 31 else ""
        print(f"  {float(Decimal(1) / (2 * n + 1)).hex()}{end} \\")
    print("")


if __name__ == "__main__":
    main()
