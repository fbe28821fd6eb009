"""Algorithmic FP64 operations of the regular periodic element pairs -- MEASUREMENT INFRASTRUCTURE.

The roofline numerator of the assembly's dominant kernel: FP64 operations per regular periodic pair,
counted by running the CPU restatement of the lattice sums (opcount.cpp: qpgf_oracle.c's terms, loop
nests and stop rules on a counting number type) at every Gauss point of a seeded sample of the
workload's pairs, with the method choice the assembly kernels use (the reference's rule plus the
cost rule for the Fourier-domain sum).  Special functions are charged at the counts of compact
published methods (opcount.cpp's header), each checked here against the C library first.

The per-point element work (geometry at the Gauss point, the four shape functions, the accumulation
of G, H, F and dF/dt, as in q0_bil_dcoef_v2_cc_GL, q0_bil_dcoef_v2_cc.c:129-204, once per point rather
than once per shape function) is counted from the same formulas, below (ELEMENT_OPS).

  python oracle/opcount.py [workload ...]      prints ops per pair / per point / per term

bench.py holds the figures this prints (frozen); tests/test_opcount.py recomputes them.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
SO = os.path.join(HERE, "_build", "libopcount.so")
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")

# the assembly kernels' cost rule for the Fourier-domain sum (QP_FD_ZFAC in csrc/qpgf.cuh)
ZFAC = 4.5

# Operations of one Gauss point's element work outside the Green's function (quads; triangles in
# parentheses), counted from the formulas: point map r = cr [1, z, e, z e] and normal W = cw [1, z, e]
# (3 x (6 + 4) = 30; triangles 3 x 4 = 12), R = r - r_t (3), |R| (5 + sqrt = 6), 1/|R| (1),
# R.W/|R|, R.v0/|R|, R.v1/|R| (3 x 6 = 18), W.v0, W.v1 (10), grad G . W (complex, 10), |W| (6; -),
# shape functions (bilinear 4 x 4 = 16; linear 3 x 2 = 6), weights G w |W|, H w (complex, 6),
# accumulation of G and H over the shape functions (4 x 8 = 32; 3 x 8 = 24), F and dF/dt (17).
ELEMENT_OPS = {4: 30 + 3 + 6 + 1 + 18 + 10 + 10 + 6 + 16 + 6 + 32 + 17,
               3: 12 + 3 + 6 + 1 + 18 + 10 + 10 + 0 + 6 + 6 + 24 + 17}


def weideman(N: int):
    """Coefficients (highest power first) and L of Weideman's rational approximation of w(z)
    (SIAM J. Numer. Anal. 31 (1994) 1497, its published FFT recipe)."""
    M = 2 * N
    k = np.arange(-M + 1, M)
    L = np.sqrt(N / np.sqrt(2.0))
    t = L * np.tan(k * np.pi / M / 2.0)
    f = np.concatenate([[0.0], np.exp(-t * t) * (L * L + t * t)])
    a = np.real(np.fft.fft(np.fft.fftshift(f))) / (2 * M)
    return np.ascontiguousarray(np.flipud(a[1:N + 1])), float(L)


def build() -> str:
    os.makedirs(os.path.dirname(SO), exist_ok=True)
    src = os.path.join(HERE, "opcount.cpp")
    if not os.path.exists(SO) or os.path.getmtime(SO) < os.path.getmtime(src):
        subprocess.run(["g++", "-O2", "-fPIC", "-shared", src, "-o", SO], check=True)
    return SO


class OpCount:
    def __init__(self):
        L = C.CDLL(build())
        self.lib = L
        L.oc_set_tables.argtypes = [_dp, C.c_double, _dp, C.c_double]
        L.oc_exp.argtypes = [C.c_double, _up]
        L.oc_exp.restype = C.c_double
        L.oc_erfc.argtypes = [C.c_double, _up]
        L.oc_erfc.restype = C.c_double
        L.oc_sincos.argtypes = [C.c_double, _dp, _up]
        L.oc_w.argtypes = [C.c_double, C.c_double, _dp, _up]
        L.oc_point.argtypes = [_dp, _dp, C.c_double, _dp, _up]
        L.oc_point.restype = C.c_int
        self.ax, Lx = weideman(36)
        self.aw, Lw = weideman(40)
        L.oc_set_tables(self.ax, Lx, self.aw, Lw)

    def check_special_functions(self):
        """Largest relative errors of the counted methods against the C library / scipy, and their
        operation counts."""
        from scipy.special import erfc, wofz
        ops = np.zeros(1, np.uint64)
        xs = np.linspace(-40.0, 5.0, 4001)
        e_exp = max(abs(self.lib.oc_exp(x, ops) - np.exp(x)) / np.exp(x) for x in xs)
        n_exp = int(ops[0])
        xs = np.linspace(-3.0, 25.0, 2801)
        e_erfc = max(abs(self.lib.oc_erfc(x, ops) - erfc(x)) / erfc(x) for x in xs)
        sc = np.zeros(2)
        e_sc = 0.0
        for x in np.linspace(-60.0, 60.0, 4001):
            self.lib.oc_sincos(x, sc, ops)
            e_sc = max(e_sc, abs(sc[0] - np.sin(x)), abs(sc[1] - np.cos(x)))
        n_sc = int(ops[0])
        rng = np.random.default_rng(5)
        w = np.zeros(2)
        e_w = 0.0
        for x, y in zip(rng.uniform(-8, 8, 3000), rng.uniform(0, 8, 3000)):
            self.lib.oc_w(x, y, w, ops)
            ref = wofz(x + 1j * y)
            e_w = max(e_w, abs(w[0] + 1j * w[1] - ref) / abs(ref))
        self.lib.oc_w(1.0, 1.0, w, ops)
        n_w = int(ops[0])
        self.lib.oc_erfc(1.0, ops)
        n_erfc = int(ops[0])
        return dict(exp=(e_exp, n_exp), erfc=(e_erfc, n_erfc), sincos=(e_sc, n_sc), w=(e_w, n_w))

    def point(self, p, r, zfac=ZFAC):
        out = np.zeros(8)
        info = np.zeros(3, np.uint64)
        ret = self.lib.oc_point(np.ascontiguousarray(p, np.float64), np.ascontiguousarray(r, np.float64), zfac,
                                out, info)
        return ret, out, int(info[0]), int(info[1]), int(info[2])


def _gauss_points(cr, nv, x, w):
    """Gauss points of one source element: the 12 x 12 rule (quads) or three 12 x 12 sub-quads
    (triangles), as the element rules lay them out."""
    s3 = np.sqrt(3.0)
    pts = []
    if nv == 4:
        for a in x:
            for b in x:
                pts.append(cr[:, 0] + cr[:, 1] * a + cr[:, 2] * b + cr[:, 3] * a * b)
    else:
        for part in range(3):
            for a in x:
                for b in x:
                    if part == 0:
                        z, e = 0.125 * (3 + 2 * a + 2 * b + a * b), 0.125 * s3 * (-a + b)
                    elif part == 1:
                        z, e = 0.0625 * (-3 + a - 5 * b - a * b), 0.0625 * s3 * (3 + 3 * a + b + a * b)
                    else:
                        z, e = 0.0625 * (-3 - 5 * a + b - a * b), 0.0625 * s3 * (-3 - a - 3 * b - a * b)
                    pts.append(cr[:, 0] + cr[:, 1] * z + cr[:, 2] * e)
    return np.array(pts)


def workload_ops(name: str, pairs: int = 24, seed: int = 2024, zfac: float = ZFAC):
    """Mean algorithmic operations per regular periodic pair of a named workload (seeded sample of
    pairs, every Gauss point of each), with the term count and the share of the operations that the
    lattice sums take.  Near-singular pairs (the 64 x 64 rule) are not in the sample: the kernel this
    figure is for recomputes none of them (they go to their own kernel)."""
    sys.path.insert(0, REPO)
    from bem3_emf_qd2_b200 import meshgen
    p, _ = meshgen.problem(name, tempfile.mkdtemp(prefix="bem3_oc_"))
    oc = OpCount()
    qpd = np.array([p.qpd["k"], *p.qpd["vk"], *p.qpd["vd1"], *p.qpd["vd2"]])
    x, _w = np.polynomial.legendre.leggauss(12)
    sid = p.sid[0]
    ne = len(sid)
    rng = np.random.default_rng(seed)
    tot_ops = tot_terms = tot_pts = tot_fd = 0
    for _ in range(pairs):
        t, s = rng.integers(0, ne, 2)
        while s == t:
            s = rng.integers(0, ne)
        td, sd = abs(int(sid[t])), abs(int(sid[s]))
        tn = int(rng.integers(0, p.nv[td]))
        rt = p.ren[td, tn]
        for q in _gauss_points(p.cr[sd], p.nv[sd], x, _w):
            ret, _, terms, ops, fd = oc.point(qpd, q - rt, zfac)
            if ret < 0:
                raise RuntimeError(f"lattice sum failed ({ret}) at {q - rt}")
            tot_ops += ops + ELEMENT_OPS[int(p.nv[sd])]
            tot_terms += terms
            tot_pts += 1
            tot_fd += fd
    return dict(workload=name, pairs=pairs, points=tot_pts, ops_per_pair=tot_ops / pairs,
                ops_per_point=tot_ops / tot_pts, terms_per_point=tot_terms / tot_pts,
                ops_per_term=tot_ops / tot_terms, fourier_share=tot_fd / tot_pts)


if __name__ == "__main__":
    oc = OpCount()
    for k, (err, n) in oc.check_special_functions().items():
        print(f"{k:7s} max rel err {err:.1e}  ops {n}")
    for name in (sys.argv[1:] or ["twolayer3072", "sphere384", "cone3360"]):
        r = workload_ops(name, pairs=96)
        print({k: (round(v, 2) if isinstance(v, float) else v) for k, v in r.items()}, flush=True)
        ref = workload_ops(name, pairs=96, zfac=0.0)
        print("  with the reference's method choice:", {k: round(ref[k], 2) for k in
                                                         ("ops_per_pair", "terms_per_point", "ops_per_term",
                                                          "fourier_share")}, flush=True)
