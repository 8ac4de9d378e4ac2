"""Writes the tables of the dense3D decimal formatter (dense3d.cu).

pow10_table.inc: 128-bit truncated mantissas of the powers of ten, as the
entries of an initializer list {hi, lo, S}: for every k in [KMIN, KMAX],
10^k = (M_k + d) * 2^S_k with 2^127 <= M_k < 2^128 and 0 <= d < 1 (M_k is the
power rounded toward zero).

exp_thresholds.inc (with --thresholds): for the text with P significant
digits, the bit pattern of the smallest positive double (P = 18) or float
(P = 10) whose rounding to P digits (ties to even) is at least 10^E, i.e.
the first value at or above 10^E - 5 * 10^(E-P); a value's printed exponent is
the largest E whose threshold it reaches.

Run from this folder:
    python gen_pow10.py > pow10_table.inc
    python gen_pow10.py --thresholds > exp_thresholds.inc
"""
import struct
import sys
from fractions import Fraction
KMIN, KMAX = -300, 350


def entry(k):
    if k >= 0:
        v = 10 ** k
        s = v.bit_length() - 128
        m = v >> s if s >= 0 else v << -s
    else:
        d = 10 ** (-k)
        t = 127 + d.bit_length()
        m = (1 << t) // d
        s = -t
        if m >= 1 << 128:  # never for k < 0 (10^j is no power of two)
            m >>= 1
            s += 1
    assert (1 << 127) <= m < (1 << 128)
    return m >> 64, m & ((1 << 64) - 1), s


E64 = (-330, 310)
E32 = (-50, 40)


def smallest_at_least(q: Fraction, fmt: str):
    """Bit pattern of the smallest positive finite value of the format at or
    above q, or None when q exceeds the largest finite value."""
    if fmt == "d":
        lo, hi = 1, 0x7FEFFFFFFFFFFFFF
        unpack = lambda b: struct.unpack("<d", struct.pack("<Q", b))[0]
    else:
        lo, hi = 1, 0x7F7FFFFF
        unpack = lambda b: struct.unpack("<f", struct.pack("<I", b))[0]
    if Fraction(unpack(hi)) < q:
        return None
    if Fraction(unpack(lo)) >= q:
        return lo
    while hi - lo > 1:  # positive values are ordered like their bit patterns
        mid = (lo + hi) // 2
        if Fraction(unpack(mid)) >= q:
            hi = mid
        else:
            lo = mid
    return hi


def thresholds():
    print("// Generated by gen_pow10.py --thresholds: exponent thresholds of the dense3D text.")
    for name, fmt, p, (e0, e1), top in (("kExpThr64", "d", 18, E64, "0x7FF0000000000000ull"),
                                         ("kExpThr32", "f", 10, E32, "0x7F800000ull")):
        print("#define %s_MIN %d" % (name.upper(), e0))
        print("#define %s_LIST \\" % name.upper())
        for e in range(e0, e1 + 1):
            q = Fraction(10) ** e - 5 * Fraction(10) ** (e - p)
            b = smallest_at_least(q, fmt)
            print("    %s, /* 1e%d */ \\" % (("0x%xull" % b) if b is not None else top, e))
        print("")


def main():
    print("// Generated by gen_pow10.py: {hi, lo, binary exponent} of 10^k, k = %d .. %d." % (KMIN, KMAX))
    for k in range(KMIN, KMAX + 1):
        hi, lo, s = entry(k)
        print("{0x%016xull, 0x%016xull, %d},  // 1e%d" % (hi, lo, s, k))


if __name__ == "__main__":
    if "--thresholds" in sys.argv:
        thresholds()
    else:
        main()
