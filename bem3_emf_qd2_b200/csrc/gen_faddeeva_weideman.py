"""Writes faddeeva_weideman.h: the coefficients of Weideman's rational approximation of the
Faddeeva function, used by the assembly kernels' w(z) for |z| < 8, Im z >= 0.

J. A. C. Weideman, "Computation of the complex error function", SIAM J. Numer. Anal. 31 (1994)
1497-1518: with L > 0 and Z = (L + iz) / (L - iz), which maps the upper half plane onto the unit
disk,

    w(z) = pi^{-1/2} / (L - iz) + 2 / (L - iz)^2 * sum_{n=0}^{N-1} a_{n+1} Z^n,

where a_n are the Fourier coefficients, in theta (t = L tan(theta / 2)), of
f(t) = e^{-t^2} (L^2 + t^2):  a_n = (1 / 2M) sum_{k=-M+1}^{M-1} f(t_k) cos(n theta_k),
theta_k = k pi / M.  L = (N / sqrt(2))^{1/2} is the paper's choice.  Here N = 40, M = 2N, and the
sums are done with mpmath at 40 digits, then rounded to double.  With these coefficients w(z)
agrees with the reference's Faddeeva_w to 4e-15 (relative to |w|) on the real-space lattice terms
and 2e-14 on the propagating spectral ones (tests/test_oracle_and_math.py).

  python bem3_emf_qd2_b200/csrc/gen_faddeeva_weideman.py   (rewrites the header beside it)
"""
import os

import mpmath as mp

N = 40
mp.mp.dps = 40


def coefficients(n_terms: int):
    M = 2 * n_terms
    L = mp.sqrt(mp.mpf(n_terms) / mp.sqrt(2))
    f = {}
    for k in range(-M + 1, M):
        th = k * mp.pi / M
        t = L * mp.tan(th / 2)
        f[k] = mp.exp(-t * t) * (L * L + t * t)
    a = []
    for n in range(1, n_terms + 1):
        s = mp.mpf(0)
        for k in range(-M + 1, M):
            s += f[k] * mp.cos(n * k * mp.pi / M)
        a.append(s / (2 * M))
    return L, a


def main():
    L, a = coefficients(N)
    here = os.path.dirname(os.path.abspath(__file__))
    lines = [
        "// faddeeva_weideman.h -- generated by gen_faddeeva_weideman.py (do not edit): the",
        "// coefficients of Weideman's rational approximation of w(z), N = %d, highest degree first" % N,
        "// (fad_wc[0] = a_N, ..., fad_wc[N - 1] = a_1), and its parameter L.",
        "#pragma once",
        "#define FAD_WN %d" % N,
        "#define FAD_WL %s" % mp.nstr(L, 20, min_fixed=-1, max_fixed=1),
        "BEM_CONST double fad_wc[FAD_WN] = {",
    ]
    vals = [mp.nstr(c, 17, strip_zeros=False) for c in reversed(a)]
    for i in range(0, N, 3):
        lines.append("    " + ", ".join(vals[i:i + 3]) + ("," if i + 3 < N else ""))
    lines.append("};")
    with open(os.path.join(here, "faddeeva_weideman.h"), "w") as fh:
        fh.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
