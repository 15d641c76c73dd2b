"""Generate ipg_bessel_coeffs.h: polynomial coefficients for K0, K1.

The kernels evaluate the modified Bessel functions K0, K1 (and K2 by the
recurrence K2 = K0 + 2 K1 / x) without divisions in loops:

  x <= 2   ascending series (Abramowitz & Stegun 9.6.10-9.6.11) in y = x^2/4,
           with the exact coefficients
             I0 : 1 / (k!)^2                     K0 reg.: H_k / (k!)^2
             I1 : 1 / (k! (k+1)!)                K1 reg.: (H_k + H_{k+1} - 2 gamma) / (k! (k+1)!)
  x in (2, 8]  Chebyshev expansion of K_n(x) sqrt(x) e^x in s = (16/x - 5)/3
  x > 8        Chebyshev expansion of K_n(x) sqrt(x) e^x in s = 16/x - 1

The Chebyshev coefficients are computed here with mpmath (50 digits) at
Chebyshev nodes and truncated below 1e-18.

    python ipole_b200/csrc/gen_bessel_coeffs.py > ipole_b200/csrc/ipg_bessel_coeffs.h
"""
import mpmath as mp

mp.mp.dps = 50
NSERIES = 16


def series():
    i0, k0r, i1, k1r = [], [], [], []
    H = [mp.mpf(0)]
    for k in range(1, NSERIES + 2):
        H.append(H[-1] + mp.mpf(1) / k)
    for k in range(NSERIES):
        f = mp.factorial(k)
        f1 = mp.factorial(k + 1)
        i0.append(1 / f ** 2)
        k0r.append(H[k] / f ** 2)
        i1.append(1 / (f * f1))
        k1r.append((H[k] + H[k + 1] - 2 * mp.euler) / (f * f1))
    return i0, k0r, i1, k1r


def cheb(fn, n=60):
    nodes = [mp.cos(mp.pi * (j + mp.mpf(1) / 2) / n) for j in range(n)]
    vals = [fn(s) for s in nodes]
    c = []
    for k in range(n):
        ck = 2 * mp.fsum(vals[j] * mp.cos(mp.pi * k * (j + mp.mpf(1) / 2) / n) for j in range(n)) / n
        c.append(ck)
    c[0] /= 2
    while len(c) > 1 and abs(c[-1]) < mp.mpf("1e-18"):
        c.pop()
    return c


def scaled(nu, x):
    return mp.besselk(nu, x) * mp.sqrt(x) * mp.exp(x)


def emit(name, vals):
    body = ",\n  ".join(mp.nstr(v, 20, min_fixed=0, max_fixed=0) for v in vals)
    return f"static __constant__ const double {name}[{len(vals)}] = {{\n  {body}}};\n"


def main():
    i0, k0r, i1, k1r = series()
    mid = lambda nu: cheb(lambda s: scaled(nu, 16 / (3 * s + 5)))   # s = (16/x - 5)/3 -> x = 16/(3s+5)
    far = lambda nu: cheb(lambda s: scaled(nu, 16 / (s + 1)))       # s = 16/x - 1     -> x = 16/(s+1)
    out = ["/* Generated by gen_bessel_coeffs.py -- coefficients for K0/K1 (see there). */", "#pragma once", ""]
    out += [emit("kI0", i0), emit("kK0R", k0r), emit("kI1", i1), emit("kK1R", k1r)]
    out += [emit("kK0M", mid(0)), emit("kK1M", mid(1)), emit("kK0F", far(0)), emit("kK1F", far(1))]
    print("\n".join(out))


if __name__ == "__main__":
    main()
