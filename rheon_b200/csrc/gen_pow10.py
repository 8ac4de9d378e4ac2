"""Writes pow10_table.inc: 128-bit truncated mantissas of the powers of ten
used by the dense3D decimal formatter (dense3d.cu), as the entries of an
initializer list {hi, lo, S} (dense3d.cu includes the list for the host and
for the device table).

For every k in [KMIN, KMAX], 10^k = (M_k + d) * 2^S_k with 2^127 <= M_k < 2^128
and 0 <= d < 1 (M_k is the power rounded toward zero). Run from this folder:
    python gen_pow10.py > pow10_table.inc
"""
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


def main():
    print("// Generated by gen_pow10.py: {hi, lo, binary exponent} of 10^k, k = %d .. %d." % (KMIN, KMAX))
    for k in range(KMIN, KMAX + 1):
        hi, lo, s = entry(k)
        print("{0x%016xull, 0x%016xull, %d},  // 1e%d" % (hi, lo, s, k))


if __name__ == "__main__":
    main()
