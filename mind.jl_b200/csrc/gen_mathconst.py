"""Derive the constants of mind_math.h from first principles with exact decimal arithmetic.

Run:  python mind.jl_b200/csrc/gen_mathconst.py
It prints C99 hex-float literals; mind_math.h embeds its output verbatim.

* ln 2 comes from the series ln 2 = sum_{k>=1} 1/(k 2^k) evaluated to 60 digits.
* LN2_HI keeps the leading 32 significant bits of ln 2 so that k * LN2_HI is
  exact for every |k| < 2^21 (Cody and Waite's additive range reduction);
  LN2_LO is the double nearest to ln 2 - LN2_HI.
* The exp polynomial is the Taylor series of e^r, coefficients 1/n!.
* The log polynomial is the series of 2 atanh(s) = ln((1+s)/(1-s)),
  coefficients 2/(2k+1).
"""
from decimal import Decimal, getcontext
from fractions import Fraction
import math

getcontext().prec = 60


def ln2_decimal() -> Decimal:
    total = Decimal(0)
    for k in range(1, 220):
        total += Decimal(1) / (Decimal(k) * (Decimal(2) ** k))
    return total


def nearest_double(value: Fraction) -> float:
    """Round an exact rational to the nearest double (ties to even)."""
    # float(Fraction) is correctly rounded in CPython.
    return float(value)


def truncate_bits(value: float, bits: int) -> float:
    mantissa, exponent = math.frexp(value)
    scaled = math.floor(mantissa * (1 << bits))
    return math.ldexp(scaled, exponent - bits)


def main() -> None:
    ln2 = ln2_decimal()
    ln2_frac = Fraction(ln2)
    ln2_hi = truncate_bits(nearest_double(ln2_frac), 32)
    ln2_lo = nearest_double(ln2_frac - Fraction(ln2_hi))
    inv_ln2 = nearest_double(1 / ln2_frac)
    print(f"#define MIND_LN2_HI {ln2_hi.hex()}")
    print(f"#define MIND_LN2_LO {ln2_lo.hex()}")
    print(f"#define MIND_INV_LN2 {inv_ln2.hex()}")
    print(f"#define MIND_SQRT2 {nearest_double(Fraction(Decimal(2).sqrt())).hex()}")
    # Random123's open-interval uniform: (word + 1) * (1 / (2^32 + 1)).
    print(f"#define MIND_INV_2P32P1 {nearest_double(Fraction(1, 2**32 + 1)).hex()}")
    for n in range(2, 14):
        print(f"#define MIND_EXP_C{n} {nearest_double(Fraction(1, math.factorial(n))).hex()}")
    for k in range(1, 12):
        print(f"#define MIND_LOG_C{k} {nearest_double(Fraction(2, 2 * k + 1)).hex()}")


if __name__ == "__main__":
    main()
