"""Coefficients of the portable sine, cosine and arctangent in pmath.hpp.

The candidate stage runs on the host and on the GPU and must give the same
bits on both, so it cannot call the platform's libm on one side and CUDA's on
the other.  pmath.hpp evaluates each function in double precision from a
polynomial fitted here (least squares on Chebyshev nodes against 50-digit
mpmath values), then rounds once to float; both compilers then perform the
same IEEE operations in the same order.

    python include/cctag_b200/portable/gen_pmath.py      # prints the coefficient tables
"""
import mpmath
import numpy as np

mpmath.mp.dps = 50


def lsq(f, lo, hi, powers, n=3000):
    k = np.arange(n)
    xs = [mpmath.mpf(lo + hi) / 2 + mpmath.mpf(hi - lo) / 2 * mpmath.cos(mpmath.pi * (kk + mpmath.mpf(0.5)) / n)
          for kk in k]
    A = mpmath.matrix([[x ** p for p in powers] for x in xs])
    y = mpmath.matrix([f(x) for x in xs])
    # normal equations in 50-digit arithmetic (well conditioned at these degrees)
    c = mpmath.lu_solve(A.T * A, A.T * y)
    return [float(v) for v in c], xs


def report(name, f, c, powers, xs):
    err = 0.0
    for x in xs[::7]:
        v = sum(mpmath.mpf(ci) * x ** p for ci, p in zip(c, powers))
        fx = f(x)
        if fx != 0:
            err = max(err, float(abs((v - fx) / fx)))
    print("// %s: max relative error %.2e" % (name, err))
    print("%s = [%s]" % (name, ", ".join(repr(v) for v in c)))


if __name__ == "__main__":
    q = mpmath.pi / 4
    # sin r = r + r^3 P(r^2), |r| <= pi/4: fit (sin r - r) / r^3 in r^2
    ps = list(range(0, 7))
    # the fit variable is u = r^2
    c, xs = lsq(lambda u: (mpmath.sin(mpmath.sqrt(u)) - mpmath.sqrt(u)) / mpmath.sqrt(u) ** 3, 1e-8,
                float(q) ** 2, ps)
    report("SinP", lambda u: (mpmath.sin(mpmath.sqrt(u)) - mpmath.sqrt(u)) / mpmath.sqrt(u) ** 3, c, ps, xs)
    # cos r = 1 - r^2/2 + r^4 Q(r^2)
    c, xs = lsq(lambda u: (mpmath.cos(mpmath.sqrt(u)) - 1 + u / 2) / u ** 2, 1e-8, float(q) ** 2, ps)
    report("CosQ", lambda u: (mpmath.cos(mpmath.sqrt(u)) - 1 + u / 2) / u ** 2, c, ps, xs)
    # atan u = u + u^3 R(u^2), |u| <= tan(pi/8)
    t8 = float(mpmath.tan(mpmath.pi / 8)) + 1e-9
    pa = list(range(0, 11))
    c, xs = lsq(lambda u: (mpmath.atan(mpmath.sqrt(u)) - mpmath.sqrt(u)) / mpmath.sqrt(u) ** 3, 1e-8, t8 ** 2,
                pa)
    report("AtanR", lambda u: (mpmath.atan(mpmath.sqrt(u)) - mpmath.sqrt(u)) / mpmath.sqrt(u) ** 3, c, pa, xs)
    # pi/2 split for the argument reduction: 33-bit head, 33-bit middle, tail
    h = mpmath.pi / 2
    c1 = float(mpmath.mpf(int(h * 2 ** 31)) / 2 ** 31)
    c2 = float(mpmath.mpf(int((h - c1) * 2 ** 64)) / 2 ** 64)
    c3 = float(h - c1 - c2)
    print("static constexpr double kPio2Hi = %r, kPio2Mid = %r, kPio2Lo = %r;" % (c1, c2, c3))
    print("static constexpr double kPi = %r, kPio2 = %r, kPio4 = %r, kTanPio8 = %r;" % (
        float(mpmath.pi), float(mpmath.pi / 2), float(mpmath.pi / 4), float(mpmath.tan(mpmath.pi / 8))))
