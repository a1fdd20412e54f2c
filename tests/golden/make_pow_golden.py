"""Golden vectors for the Manning power x^(4./3): correctly rounded values computed with
60-digit decimal arithmetic (ln then exp, then one rounding to double), and glibc's pow
for comparison.  Run: python tests/golden/make_pow_golden.py"""
import ctypes
import decimal
import os
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    decimal.getcontext().prec = 60
    p = Fraction(4.0 / 3)
    P = decimal.Decimal(p.numerator) / decimal.Decimal(p.denominator)
    rng = np.random.default_rng(42)
    x = np.concatenate([np.exp(rng.uniform(np.log(1e-6), np.log(1e3), 12000)),
                        1e-3 + rng.uniform(-2e-5, 2e-5, 3000),
                        np.array([1.0, 8.0, 27.0, 64.0, 0.125, 1e-3, 0.5e-3, 2.0, 3.0, 1e-200, 1e200])])
    cr = np.array([float((P * decimal.Decimal(float(v)).ln()).exp()) for v in x])
    libm = ctypes.CDLL("libm.so.6")
    libm.pow.restype = ctypes.c_double
    libm.pow.argtypes = [ctypes.c_double, ctypes.c_double]
    glibc = np.array([libm.pow(float(v), 4.0 / 3) for v in x])
    np.savez_compressed(os.path.join(HERE, "pow43_cr.npz"), x=x, cr=cr, glibc=glibc)
    print("written pow43_cr.npz:", len(x), "values;", int((cr != glibc).sum()), "where glibc is not CR")


if __name__ == "__main__":
    main()
