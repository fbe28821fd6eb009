"""Writes erfcx_poly.h: a polynomial form of the scaled complementary error function
erfcx(x) = e^{x^2} erfc(x) on [0, inf), used by the assembly kernels' Ewald spectral terms.

The substitution t = P / (P + x) maps [0, inf) onto (0, 1]; erfcx(x) / t is smooth on [0, 1]
(it tends to P^{-1} pi^{-1/2} as t -> 0, since erfcx(x) ~ 1 / (x sqrt(pi))), so

    erfcx(x) = t * sum_{k=0}^{D} c_k s^k,      s = 2 t - 1,

with c_k the monomial coefficients of the degree-D Chebyshev interpolant of erfcx(x) / t in s at the
D + 1 Chebyshev points of the first kind (the standard near-minimax interpolant).  Everything is
computed with mpmath at 50 digits (erfcx through mpmath's erfc), converted to monomials in s there,
and rounded to double once.  P = 4, D = 22: the interpolant's own error is below 1e-16 relative; in
double, Horner evaluation adds a few units in the last place (coefficients are all below 0.3 in
magnitude).  tests/test_oracle_and_math.py checks the evaluation (host build of the same code)
against mpmath; the GPU parity tests check the assembly rows that use it against the reference.

  python bem3_emf_qd2_b200/csrc/gen_erfcx_poly.py   (rewrites the header beside it)
"""
import os

import mpmath as mp

P = 4
D = 22
mp.mp.dps = 50


def erfcx(x):
    return mp.exp(x * x) * mp.erfc(x)


def coefficients(p=P, d=D):
    n = d + 1
    nodes = [mp.cos(mp.pi * (j + mp.mpf(1) / 2) / n) for j in range(n)]  # s in (-1, 1)
    vals = []
    for s in nodes:
        t = (s + 1) / 2
        x = p * (1 - t) / t
        vals.append(erfcx(x) / t)
    # Chebyshev coefficients of the interpolant
    cheb = []
    for k in range(n):
        acc = mp.mpf(0)
        for j in range(n):
            acc += vals[j] * mp.cos(k * mp.pi * (j + mp.mpf(1) / 2) / n)
        cheb.append(acc * (1 if k == 0 else 2) / n)
    # Chebyshev -> monomial in s: T_0 = 1, T_1 = s, T_{k+1} = 2 s T_k - T_{k-1}
    Tm1, T = [mp.mpf(1)], [mp.mpf(0), mp.mpf(1)]
    mono = [mp.mpf(0)] * n
    mono[0] += cheb[0]
    if n > 1:
        mono[1] += cheb[1]
    for k in range(1, n - 1):
        Tn = [mp.mpf(0)] * (k + 2)
        for i, c in enumerate(T):
            Tn[i + 1] += 2 * c
        for i, c in enumerate(Tm1):
            Tn[i] -= c
        for i, c in enumerate(Tn):
            mono[i] += cheb[k + 1] * c
        Tm1, T = T, Tn
    return mono


def main():
    mono = coefficients()
    here = os.path.dirname(os.path.abspath(__file__))
    lines = [
        "// erfcx_poly.h -- generated by gen_erfcx_poly.py (do not edit): erfcx(x), x >= 0, as",
        f"// t * sum_k c_k s^k with t = {P} / ({P} + x), s = 2 t - 1, degree {D} (see the generator).",
        "#pragma once",
        f"#define ERFCX_P {P}.0",
        f"#define ERFCX_DEG {D}",
        "BEM_CONST double erfcx_c[ERFCX_DEG + 1] = {",
    ]
    for c in mono:
        lines.append("    %s," % mp.nstr(c, 17, min_fixed=-1, max_fixed=-1, strip_zeros=False).replace("e-0", "e-").replace("e+0", "e+"))
    lines.append("};")
    with open(os.path.join(here, "erfcx_poly.h"), "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
