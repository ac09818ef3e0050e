"""The polynomial coefficients and constants of box_muller_math.h.

Near-minimax fits by Lawson's algorithm (iteratively reweighted least
squares on a Chebyshev basis, the weights multiplied by the error each
round), in double precision, then rounded to float:

  ln(1 + f) = f + f^2 Q(f),      f in [1/sqrt2 - 1, sqrt2 - 1], Q of degree 8,
                                 weighted to the relative error of ln(1 + f);
  sin r = r + r^3 S(r^2),        |r| <= pi/4 (0.1 % margin), S of degree 2;
  cos r = 1 - r^2/2 + r^4 C(r^2),                            C of degree 2;

and pi/2 split into three floats (each the float nearest to what the parts
before leave), ln2 into a 16-bit head and a float tail.

usage: python box_muller_fit.py   (prints the constants as C hex floats)
"""
from fractions import Fraction

import numpy as np
from numpy.polynomial import chebyshev as cheb
from numpy.polynomial import polynomial as poly


def lawson(x, target, weight, deg, iters=300):
    """Coefficients (monomials in x, ascending) of the near-minimax weighted
    fit, and its largest weighted error on the sample."""
    a, b = x.min(), x.max()
    t = (2.0 * x - (a + b)) / (b - a)
    v = cheb.chebvander(t, deg)
    w = np.full_like(x, 1.0 / len(x))
    for _ in range(iters):
        sw = np.sqrt(w)
        c, *_ = np.linalg.lstsq(v * (sw * weight)[:, None], target * weight * sw, rcond=None)
        e = np.abs(v @ c - target) * weight
        w = w * e
        w /= w.sum()
    pc = cheb.cheb2poly(c)
    lin = np.array([-(a + b) / (b - a), 2.0 / (b - a)])      # t as a polynomial in x
    mono = np.zeros(deg + 1)
    pt = np.array([1.0])
    for k in range(deg + 1):
        mono[:len(pt)] += pc[k] * pt
        pt = poly.polymul(pt, lin)
    return mono, float(e.max())


def f32hex(v):
    return float(np.float32(v)).hex().replace("0000000p", "p") + "f"


def main():
    lo, hi = 2.0 ** -0.5 - 1.0, 2.0 ** 0.5 - 1.0
    f = np.linspace(lo, hi, 20001)
    f = f[np.abs(f) > 1e-6]
    q, eq = lawson(f, (np.log1p(f) - f) / f ** 2, f ** 2 / np.abs(np.log1p(f)), 8)
    r = np.linspace(1e-3, np.pi / 4 * 1.001, 20001)
    s, es = lawson(r * r, (np.sin(r) - r) / r ** 3, r ** 3 / np.sin(r), 2)
    c, ec = lawson(r * r, (np.cos(r) - 1.0 + r * r / 2.0) / r ** 4, r ** 4 / np.cos(r), 2)
    print(f"// Q (ascending), fit error {eq:.2e}:", ", ".join(f32hex(v) for v in q))
    print(f"// S (ascending), fit error {es:.2e}:", ", ".join(f32hex(v) for v in s))
    print(f"// C (ascending), fit error {ec:.2e}:", ", ".join(f32hex(v) for v in c))
    pi = Fraction("3.14159265358979323846264338327950288419716939937510582097494459230781640628620899862803482534211706798")
    half = pi / 2
    p1 = Fraction(float(np.float32(float(half))))
    p2 = Fraction(float(np.float32(float(half - p1))))
    p3 = Fraction(float(np.float32(float(half - p1 - p2))))
    print("// pi/2 parts:", f32hex(float(p1)), f32hex(float(p2)), f32hex(float(p3)))
    print("// 2/pi:", f32hex(float(1 / half)))
    ln2 = Fraction("0.693147180559945309417232121458176568075500134360255254120680009493393621969694715605863326996418688")
    head = Fraction(0.693145751953125)                         # 0x1.62e4p-1: 16 significant bits
    print("// ln2 head, tail:", f32hex(float(head)), f32hex(float(ln2 - head)))


if __name__ == "__main__":
    main()
