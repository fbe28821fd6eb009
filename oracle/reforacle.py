"""ctypes access to the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Two libraries live here, both built by ``oracle/Makefile``:

* ``_ref/libbem3ref.so``: the reference (akohta/bem3_emf_qd2) compiled from its own sources
  plus ``ref_probe.c``/``ref_shims.c``.  Available wherever the reference checkout was
  present at build time (the built file travels with the repository snapshot).
* ``_build/libqpgf_oracle.so``: the C restatement in ``qpgf_oracle.c`` (Faddeeva, QPGF and the
  regular element-pair rules), pinned against the reference by the tests.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this
module.  The product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libbem3ref.so")
PORT_SO = os.path.join(HERE, "_build", "libqpgf_oracle.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_cp = np.ctypeslib.ndpointer(dtype=np.complex128, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build(ref_dir, quiet: bool = True) -> None:
    """Build the oracle libraries.  ref_dir: a checkout of the reference, or None; the reference
    part is built only when its sources are there, the C restatement always."""
    targets = ["port"]
    args = []
    if ref_dir and os.path.isdir(os.path.join(ref_dir, "d3qd2_src")):
        targets.insert(0, "ref")
        args.append(f"REF={ref_dir}")
    out = subprocess.run(["make", "-C", HERE, *args, "-j8", *targets],
                         capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout[-4000:] + out.stderr[-4000:])


def have_ref() -> bool:
    return os.path.exists(REF_SO)


def have_port() -> bool:
    return os.path.exists(PORT_SO)


class RefOracle:
    """The compiled reference.  One problem is held at a time (a static in ref_probe.c)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        lib = C.CDLL(path)
        self.lib = lib
        lib.rp_load.argtypes = [C.c_char_p] * 4
        lib.rp_load_dat.argtypes = [C.c_char_p]
        lib.rp_write_dat.argtypes = [C.c_char_p]
        lib.rp_info.argtypes = [_ip]
        lib.rp_info.restype = C.c_int
        lib.rp_get_elems.argtypes = [_dp, _dp, _dp, _dp, _ip, _ip, _ip, _ip]
        lib.rp_get_nodes.argtypes = [_dp]
        lib.rp_get_sid.argtypes = [C.c_int, _ip]
        lib.rp_get_qpd.argtypes = [_dp]
        lib.rp_get_media.argtypes = [_dp, _dp]
        lib.rp_get_pw.argtypes = [_dp]
        lib.rp_get_quad.argtypes = [_dp, _dp, _dp, _dp]
        lib.rp_get_incident.argtypes = [_cp, _cp]
        lib.rp_pair.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _cp]
        lib.rp_pairs.argtypes = [C.c_int, _ip, _cp, C.c_int]
        lib.rp_assemble_rows.argtypes = [C.c_int, C.c_int, C.c_int, _cp, _cp, _cp, _cp, _dp, C.c_int]
        lib.rp_assemble_rows_list.argtypes = [C.c_int, C.c_int, _ip, _cp, _cp, _cp, _cp, _dp, C.c_int]
        lib.rp_assemble_rows_zshift.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _cp, _cp, _cp, _cp, _dp, C.c_int]
        for f in (lib.rp_qpgf_v1, lib.rp_qpgf_qG, lib.rp_qpgf_dqG):
            f.argtypes = [C.c_int, _dp, _dp, C.c_double, _cp, _ip]
        lib.rp_dcoef_rt_grad.argtypes = [C.c_int, _dp, C.c_int, C.c_int, _cp, _cp]
        lib.rp_qpgf_v2.argtypes = [C.c_int, _dp, _dp, C.c_double, _cp, _ip]
        lib.rp_faddeeva.argtypes = [C.c_int, _cp, C.c_double, _cp]
        lib.rp_coef_rt.argtypes = [C.c_int, _dp, C.c_int, C.c_int, _cp]
        lib.rp_get_bv.argtypes = [C.c_int, _cp, _cp, _cp, _cp, _cp, _cp]
        lib.rp_set_bv.argtypes = [C.c_int, _cp, _cp, _cp, _cp, _cp, _cp]
        lib.rp_EH.argtypes = [C.c_int, _dp, C.c_int, C.c_int, _cp, _cp, _ip]
        lib.rp_mEMP.argtypes = [C.c_int, _dp, C.c_int, C.c_int, _cp, _ip]
        lib.rp_EH_mEMP.argtypes = [C.c_int, _dp, C.c_int, C.c_int, _cp, _cp, _ip]
        lib.rp_force.argtypes = [_dp, _dp, _dp, C.c_int]
        lib.rp_force.restype = C.c_int
        lib.rp_domain_id.argtypes = [_dp]
        lib.rp_domain_id.restype = C.c_int

    # ---- problem loading -------------------------------------------------------------
    def load(self, ipw: str, ped: str, med: str, msh: str) -> "RefOracle":
        self.lib.rp_load(ipw.encode(), ped.encode(), med.encode(), msh.encode())
        return self

    def load_dat(self, dat: str) -> "RefOracle":
        self.lib.rp_load_dat(dat.encode())
        return self

    def write_dat(self, dat: str) -> None:
        self.lib.rp_write_dat(dat.encode())

    def info(self) -> dict:
        buf = np.zeros(64, np.int32)
        self.lib.rp_info(buf)
        mn = int(buf[0])
        return dict(MN=mn, Ne=int(buf[1]), Nn=int(buf[2]), NN=int(buf[3]), ps=int(buf[4]),
                    Ne_d=[int(x) for x in buf[5:5 + mn + 1]])

    def geometry(self) -> dict:
        inf = self.info()
        ne = inf["Ne"]
        cr = np.zeros((ne + 1, 3, 4)); cw = np.zeros((ne + 1, 3, 3))
        ren = np.zeros((ne + 1, 4, 3)); wen = np.zeros((ne + 1, 4, 3))
        ed = np.zeros((ne + 1, 4), np.int32); eni = np.zeros((ne + 1, 4), np.int32)
        md = np.zeros(ne + 1, np.int32); sd = np.zeros(ne + 1, np.int32)
        self.lib.rp_get_elems(cr, cw, ren, wen, ed, eni, md, sd)
        rn = np.zeros((inf["Nn"] + 1, 3))
        self.lib.rp_get_nodes(rn)
        sids = []
        for d in range(inf["MN"] + 1):
            s = np.zeros(inf["Ne_d"][d] + 1, np.int32)
            self.lib.rp_get_sid(d, s)
            sids.append(s)
        qpd = np.zeros(8)
        self.lib.rp_get_qpd(qpd)
        kn = np.zeros(2 * (inf["MN"] + 1)); n = np.zeros(2 * (inf["MN"] + 1))
        self.lib.rp_get_media(kn, n)
        pw = np.zeros(3)
        self.lib.rp_get_pw(pw)
        xli = np.zeros(12); wli = np.zeros(12); xhi = np.zeros(64); whi = np.zeros(64)
        self.lib.rp_get_quad(xli, wli, xhi, whi)
        Ui = np.zeros((ne + 1, 4, 4), np.complex128); dUi = np.zeros((ne + 1, 4, 4), np.complex128)
        self.lib.rp_get_incident(Ui, dUi)
        return dict(info=inf, cr=cr, cw=cw, ren=ren, wen=wen, ed=ed, eni=eni, md=md, sd=sd, rn=rn,
                    sid=sids, qpd=qpd, kn=kn[0::2] + 1j * kn[1::2], n=n[0::2] + 1j * n[1::2],
                    lambda0=pw[0], n0=pw[1], xli=xli, wli=wli, xhi=xhi, whi=whi, Ui=Ui, dUi=dUi)

    # ---- element pairs ---------------------------------------------------------------
    def pair(self, did: int, t: int, tn: int, s: int) -> np.ndarray:
        out = np.zeros(27, np.complex128)
        self.lib.rp_pair(did, t, tn, s, out)
        return out

    def pairs(self, quads: np.ndarray, nthreads: int = 0) -> np.ndarray:
        q = np.ascontiguousarray(quads, dtype=np.int32).reshape(-1, 4)
        out = np.zeros((len(q), 27), np.complex128)
        self.lib.rp_pairs(len(q), q, out, nthreads)
        return out

    def assemble_rows(self, did: int, t0: int, t1: int, nthreads: int = 0):
        """Rows of create_cmatrix_domain for elements t0..t1 (1-based, inclusive)."""
        ne = self.info()["Ne_d"][did]
        n = 4 * ne
        nr = 4 * (t1 - t0 + 1)
        G = np.zeros((nr, n), np.complex128); H = np.zeros((nr, n), np.complex128)
        dG = np.zeros((nr * 2, n), np.complex128); dH = np.zeros((nr * 2, n), np.complex128)
        dF = np.zeros((nr, 3))
        self.lib.rp_assemble_rows(did, t0, t1, G, H, dG, dH, dF, nthreads)
        return G, H, dG, dH, dF

    def assemble_rows_list(self, did: int, ts, nthreads: int = 0):
        """assemble_rows for the elements ts (1-based), parallel over every (element, node, source):
        rows 4 i + tn for element ts[i]."""
        ts = np.ascontiguousarray(ts, dtype=np.int32)
        n = 4 * self.info()["Ne_d"][did]
        nr = 4 * len(ts)
        G = np.zeros((nr, n), np.complex128); H = np.zeros((nr, n), np.complex128)
        dG = np.zeros((nr * 2, n), np.complex128); dH = np.zeros((nr * 2, n), np.complex128)
        dF = np.zeros((nr, 3))
        self.lib.rp_assemble_rows_list(did, len(ts), ts, G, H, dG, dH, dF, nthreads)
        return G, H, dG, dH, dF

    def assemble_rows_zshift(self, did: int, t0: int, t1: int, ulps: int, nthreads: int = 0):
        """assemble_rows with the rows' collocation nodes moved by `ulps` units in the last place in z."""
        ne = self.info()["Ne_d"][did]
        n = 4 * ne
        nr = 4 * (t1 - t0 + 1)
        G = np.zeros((nr, n), np.complex128); H = np.zeros((nr, n), np.complex128)
        dG = np.zeros((nr * 2, n), np.complex128); dH = np.zeros((nr * 2, n), np.complex128)
        dF = np.zeros((nr, 3))
        self.lib.rp_assemble_rows_zshift(did, t0, t1, ulps, G, H, dG, dH, dF, nthreads)
        return G, H, dG, dH, dF

    # ---- Green's function ------------------------------------------------------------
    def qpgf(self, r: np.ndarray, qpd: np.ndarray, kind: str = "v1", eps: float = 1e-15):
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 3)
        n = len(r)
        ret = np.zeros(n, np.int32)
        qpd = np.ascontiguousarray(qpd, dtype=np.float64)
        if kind == "v1":
            out = np.zeros((n, 4), np.complex128)
            self.lib.rp_qpgf_v1(n, r, qpd, eps, out, ret)
        elif kind == "v2":
            out = np.zeros((n, 10), np.complex128)
            self.lib.rp_qpgf_v2(n, r, qpd, eps, out, ret)
        elif kind == "qG":
            out = np.zeros((n, 1), np.complex128)
            self.lib.rp_qpgf_qG(n, r, qpd, eps, out, ret)
        else:
            out = np.zeros((n, 3), np.complex128)
            self.lib.rp_qpgf_dqG(n, r, qpd, eps, out, ret)
        return out, ret

    def faddeeva(self, z: np.ndarray, relerr: float = 1e-15) -> np.ndarray:
        z = np.ascontiguousarray(z, dtype=np.complex128).ravel()
        w = np.zeros_like(z)
        self.lib.rp_faddeeva(len(z), z, relerr, w)
        return w

    # ---- solve, boundary values, fields ------------------------------------------------
    def solve_bieq(self, workdir: str) -> None:
        cwd = os.getcwd()
        os.chdir(workdir)
        try:
            self.lib.rp_solve_bieq()
        finally:
            os.chdir(cwd)

    def boundary_values(self, d: int):
        ne = self.info()["Ne_d"][d]
        U = np.zeros((ne + 1, 4, 4), np.complex128); dU = np.zeros_like(U)
        E = np.zeros((ne + 1, 4, 3), np.complex128); dE = np.zeros_like(E)
        H = np.zeros_like(E); dH = np.zeros_like(E)
        self.lib.rp_get_bv(d, U, dU, E, dE, H, dH)
        return dict(U=U, dU=dU, E=E, dE=dE, H=H, dH=dH)

    def set_boundary_values(self, d: int, bv: dict) -> None:
        a = {k: np.ascontiguousarray(v, dtype=np.complex128) for k, v in bv.items()}
        self.lib.rp_set_bv(d, a["U"], a["dU"], a["E"], a["dE"], a["H"], a["dH"])

    def EH(self, r: np.ndarray, type_: int = 0, total=True):
        """EH_s (total 0 / False), EH_t (1 / True) or EH_i (2) at points."""
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 3)
        E = np.zeros((len(r), 3), np.complex128); H = np.zeros_like(E)
        did = np.zeros(len(r), np.int32)
        self.lib.rp_EH(len(r), r, type_, int(total), E, H, did)
        return E, H, did

    def mEMP(self, r: np.ndarray, type_: int = 0, total=True):
        """mEMP_s / mEMP_t / mEMP_i (total 0, 1, 2): U[4] = (vector potential, scalar potential)."""
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 3)
        U = np.zeros((len(r), 4), np.complex128)
        did = np.zeros(len(r), np.int32)
        self.lib.rp_mEMP(len(r), r, type_, int(total), U, did)
        return U, did

    def EH_mEMP(self, r: np.ndarray, type_: int = 0, total=True):
        """EH_mEMP_s / _t / _i (total 0, 1, 2): fields from the potentials' derivatives."""
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 3)
        E = np.zeros((len(r), 3), np.complex128); H = np.zeros_like(E)
        did = np.zeros(len(r), np.int32)
        self.lib.rp_EH_mEMP(len(r), r, type_, int(total), E, H, did)
        return E, H, did

    def force(self, rc=(0.0, 0.0, 0.0), type_: int = 0):
        F = np.zeros(3); N = np.zeros(3)
        self.lib.rp_force(F, N, np.asarray(rc, np.float64), type_)
        return F, N

    def coef_rt(self, did: int, r, sd: int, type_: int) -> np.ndarray:
        """CC[9] of source element sd at point r (EH_s's per-element coefficients)."""
        out = np.zeros(9, np.complex128)
        self.lib.rp_coef_rt(did, np.ascontiguousarray(r, np.float64), sd, type_, out)
        return out

    def dcoef_rt_grad(self, did: int, r, sd: int, type_: int):
        """CC[9] and dC[3][9] of source element sd at point r (EH_mEMP_s's per-element values)."""
        cc = np.zeros(9, np.complex128)
        dc = np.zeros(27, np.complex128)
        self.lib.rp_dcoef_rt_grad(did, np.ascontiguousarray(r, np.float64), sd, type_, cc, dc)
        return cc, dc.reshape(3, 9)

    def domain_id(self, r) -> int:
        return int(self.lib.rp_domain_id(np.asarray(r, np.float64)))
