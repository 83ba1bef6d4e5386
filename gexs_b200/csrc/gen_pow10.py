"""Generate pow10_dd.h: 10^k as an unevaluated sum hi + lo of two doubles,
k = POW10_MIN..POW10_MAX, for the GPU decimal parser (gexs_ingest.cu).

hi is 10^k rounded to the nearest double and lo the nearest double to the
remainder 10^k - hi, both computed exactly with rational arithmetic, so
hi + lo carries ~106 bits of 10^k.  For k < SCALED_BELOW the pair holds
10^k * 2^SCALE_BITS (so both stay normal doubles); the parser multiplies its
result by 2^-SCALE_BITS, which is exact for normal results.

    python gen_pow10.py > pow10_dd.h
"""
from fractions import Fraction

POW10_MIN, POW10_MAX = -343, 308
SCALED_BELOW, SCALE_BITS = -280, 256


def main():
    print("/* generated by gen_pow10.py: 10^k = hi + lo, k = %d..%d */" % (POW10_MIN, POW10_MAX))
    print("#pragma once")
    print("#define GEXS_POW10_MIN (%d)" % POW10_MIN)
    print("#define GEXS_POW10_MAX (%d)" % POW10_MAX)
    print("#define GEXS_POW10_SCALED_BELOW (%d)" % SCALED_BELOW)
    print("#define GEXS_POW10_SCALE_BITS (%d)" % SCALE_BITS)
    print("static __device__ const double gexs_pow10_dd[%d][2] = {" % (POW10_MAX - POW10_MIN + 1))
    for k in range(POW10_MIN, POW10_MAX + 1):
        p = Fraction(10) ** k
        if k < SCALED_BELOW:
            p *= Fraction(2) ** SCALE_BITS
        hi = float(p)
        lo = float(p - Fraction(hi))
        print("    {%r, %r}," % (hi, lo))
    print("};")


if __name__ == "__main__":
    main()
