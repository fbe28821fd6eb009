"""Host-side problem description for the boundary-integral path (numpy).

This is the host mirror of the reference's set-up layer that produces the hot path's inputs:
the three text readers and the Gmsh 2.2 reader, element constants, sub-domain lists, the
quasi-periodic data and the incident field at the collocation nodes
(d3qd2_src/d3qd2_setup.c:3-139, 557-959, 1139-1349; d3qd2_src/m_ipw.c, d3qd2_src/ipw.c).
Arithmetic is written in the reference's order so that the element constants come out
bit-identical.  Nothing here is on the GPU path; it only prepares arrays for the C ABI.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List

import numpy as np

MEPS = 1.0e-15
OPENDID = 99
P44_N = 0.5773502691896257645091
P34_N0 = 0.2
P34_N1 = 0.3464101615137754587055


@dataclasses.dataclass
class PlaneWave:
    """One incident plane wave (Ipw, d3qd2_src/ipw.h:27-38) with its derived data (IpwD)."""
    lambda0: float
    ni: float
    power: float
    e0x: complex
    e0y: complex
    f: tuple
    theta: float
    phi: float

    def setup(self):
        # setup_ipw (d3qd2_src/ipw.c:121-145)
        cs = 1.0 / math.sqrt(abs(self.e0x) ** 2 + abs(self.e0y) ** 2)
        ex = self.e0x * cs
        ey = self.e0y * cs
        hx = -ey * self.ni
        hy = ex * self.ni
        self.E0 = math.sqrt(self.power * 2.0 / self.ni)
        self.ki = 2.0 * math.pi * self.ni / self.lambda0
        st, ct = math.sin(self.theta), math.cos(self.theta)
        sp, cp = math.sin(self.phi), math.cos(self.phi)
        self.sin_t, self.cos_t, self.sin_p, self.cos_p = st, ct, sp, cp
        self.ex = ex * (sp * sp + cp * cp * ct) + ey * (sp * cp * ct - sp * cp)
        self.ey = ex * (sp * cp * ct - sp * cp) + ey * (sp * sp * ct + cp * cp)
        self.ez = -(ex * cp + ey * sp) * st
        self.hx = hx * (sp * sp + cp * cp * ct) + hy * (sp * cp * ct - sp * cp)
        self.hy = hx * (sp * cp * ct - sp * cp) + hy * (sp * sp * ct + cp * cp)
        self.hz = -(hx * cp + hy * sp) * st

    def eh_dehdv(self, x: np.ndarray, n: np.ndarray):
        """Fields and directional derivatives (calc_ipw_dEHdv, d3qd2_src/ipw.c:229-257).
        x, n: [..., 3].  Returns e, h, de, dh of shape [..., 3] (complex)."""
        xc = x[..., 0] - self.f[0]
        yc = x[..., 1] - self.f[1]
        zc = x[..., 2] - self.f[2]
        te = self.ki * (xc * self.sin_t * self.cos_p + yc * self.sin_t * self.sin_p + zc * self.cos_t)
        Ee = np.cos(te) + 1j * np.sin(te)
        gcf = 1j * self.ki * (self.sin_t * self.cos_p * n[..., 0] + self.sin_t * self.sin_p * n[..., 1]
                              + self.cos_t * n[..., 2])
        e = np.stack([self.ex * Ee * self.E0, self.ey * Ee * self.E0, self.ez * Ee * self.E0], -1)
        h = np.stack([self.hx * Ee * self.E0, self.hy * Ee * self.E0, self.hz * Ee * self.E0], -1)
        return e, h, e * gcf[..., None], h * gcf[..., None]


def _data_lines(path: str) -> List[str]:
    with open(path) as f:
        return f.read().splitlines()


def read_planewaves(path: str) -> List[PlaneWave]:
    """read_data_mipw (d3qd2_src/m_ipw.c:9-106): 2 comment lines, count, 1 comment line, records."""
    lines = _data_lines(path)
    toks = " ".join(lines[2:]).split()
    n = int(toks[0])
    # the line after the count is a comment: skip its tokens
    rest = " ".join(lines[4:]).split()
    waves = []
    for i in range(n):
        v = [float(x) for x in rest[i * 12:(i + 1) * 12]]
        waves.append(PlaneWave(v[0], v[1], v[2], complex(v[3], v[4]), complex(v[5], v[6]), (v[7], v[8], v[9]),
                               v[10], v[11]))
    if not waves:
        raise ValueError("no plane wave defined")
    return waves


def read_periodicity(path: str):
    """read_periodicity_data (d3qd2_src/d3qd2_setup.c:557-587)."""
    toks = " ".join(_data_lines(path)[2:]).split()
    return int(toks[0]), (float(toks[1]), float(toks[2])), (float(toks[3]), float(toks[4]))


def read_media(path: str) -> List[complex]:
    """read_medium_data (d3qd2_src/d3qd2_setup.c:605-645): refractive indices of media 1..MN."""
    lines = _data_lines(path)
    mn = int(lines[2].split()[0])
    toks = " ".join(lines[4:]).split()
    return [complex(float(toks[2 * i]), float(toks[2 * i + 1])) for i in range(mn)]


def read_gmsh(path: str, MN: int):
    """read_mesh_data (d3qd2_src/d3qd2_setup.c:662-959).  Each surface element is written twice:
    ids 2i-1 (tag 1 = main domain) and 2i (tag 1 = the other domain, reversed node order).
    Returns rn [Nn+1,3], ed [Ne+1,4] (ed[:,3] = 0 for triangles), md, sd, gd [Ne+1]."""
    with open(path) as f:
        lines = f.read().splitlines()
    i = 0
    while lines[i].strip() != "$MeshFormat":
        i += 1
    ver, ftype, prec = lines[i + 1].split()
    if float(ver) < 2.2 or int(ftype) != 0 or int(prec) != 8:
        raise ValueError("mesh must be Gmsh 2.2 ASCII with 8-byte reals")
    while lines[i].strip() != "$Nodes":
        i += 1
    nn = int(lines[i + 1])
    rn = np.zeros((nn + 1, 3))
    for j in range(nn):
        p = lines[i + 2 + j].split()
        if int(p[0]) != j + 1:
            raise ValueError(f"bad node id {p[0]}")
        rn[j + 1] = [float(p[1]), float(p[2]), float(p[3])]
    while lines[i].strip() != "$Elements":
        i += 1
    ne2 = int(lines[i + 1])
    ne = ne2 // 2
    ed = np.zeros((ne + 1, 4), np.int32)
    md = np.zeros(ne + 1, np.int32)
    sd = np.zeros(ne + 1, np.int32)
    gd = np.zeros(ne + 1, np.int32)
    base = i + 2
    for e in range(1, ne + 1):
        a = [int(x) for x in lines[base + 2 * (e - 1)].split()]
        b = [int(x) for x in lines[base + 2 * (e - 1) + 1].split()]
        if a[0] != 2 * e - 1 or b[0] != 2 * e:
            raise ValueError(f"bad element id near {e}")
        etype = a[1]
        if etype not in (2, 3):
            raise ValueError("element type must be 2 (triangle) or 3 (quad)")
        ntag = a[2]
        tags = a[3:3 + ntag]
        m = 0 if tags[0] == OPENDID else tags[0]
        if m > MN:
            raise ValueError(f"domain id {m} is not defined in the medium data")
        md[e] = m
        if ntag > 1:
            gd[e] = tags[1]
        nodes = a[3 + ntag:]
        ed[e, :len(nodes)] = nodes
        ntag2 = b[2]
        m2 = 0 if b[3] == OPENDID else b[3]
        if m2 > MN:
            raise ValueError(f"domain id {m2} is not defined in the medium data")
        sd[e] = m2
        nodes2 = b[3 + ntag2:]
        want = [nodes[0], nodes[2], nodes[1]] if etype == 2 else [nodes[0], nodes[3], nodes[2], nodes[1]]
        if nodes2 != want:
            raise ValueError(f"node id mismatch in element {2 * e}")
        if sd[e] == 0:  # the open region becomes the main domain
            sd[e] = md[e]
            md[e] = 0
            if etype == 2:
                ed[e, 1], ed[e, 2] = ed[e, 2], ed[e, 1]
            else:
                ed[e, 3], ed[e, 1] = ed[e, 1], ed[e, 3]
    return rn, ed, md, sd, gd


def rotate_translate(rn: np.ndarray, rot) -> np.ndarray:
    """rotation_translation_obj (d3qd2_src/d3qd2_setup.c:1110-1137): Rodrigues' rotation of every
    node about the unit axis rv by th, then the translation tv, in the reference's operation order."""
    rv0, rv1, rv2, th, tv0, tv1, tv2 = rot
    a = math.sqrt(rv0 * rv0 + rv1 * rv1 + rv2 * rv2)
    n0, n1, n2 = rv0 / a, rv1 / a, rv2 / a
    st, ct = math.sin(th), math.cos(th)
    M = [ct + n0 * n0 * (1.0 - ct), n0 * n1 * (1.0 - ct) - n2 * st, n2 * n0 * (1.0 - ct) + n1 * st,
         n0 * n1 * (1.0 - ct) + n2 * st, ct + n1 * n1 * (1.0 - ct), n1 * n2 * (1.0 - ct) - n0 * st,
         n2 * n0 * (1.0 - ct) - n1 * st, n1 * n2 * (1.0 - ct) + n0 * st, ct + n2 * n2 * (1.0 - ct)]
    tv = (tv0, tv1, tv2)
    out = np.array(rn, dtype=np.float64, copy=True)
    for s in range(1, out.shape[0]):
        x, y, z = rn[s, 0], rn[s, 1], rn[s, 2]
        for i in range(3):
            out[s, i] = M[3 * i] * x + M[3 * i + 1] * y + M[3 * i + 2] * z + tv[i]
    return out


def element_constants(rn: np.ndarray, ed: np.ndarray):
    """init_elem_const (d3qd2_src/d3qd2_setup.c:1139-1186), in the reference's operation order."""
    ne = ed.shape[0] - 1
    cr = np.zeros((ne + 1, 3, 4))
    cw = np.zeros((ne + 1, 3, 3))
    for i in range(1, ne + 1):
        rc = [[rn[ed[i, j], d] for j in range(4)] for d in range(3)]
        if ed[i, 3] != 0:
            for d in range(3):
                r0, r1, r2, r3 = rc[d]
                cr[i, d, 0] = 0.25 * (r0 + r1 + r2 + r3)
                cr[i, d, 1] = 0.25 * (-r0 + r1 + r2 - r3)
                cr[i, d, 2] = 0.25 * (-r0 - r1 + r2 + r3)
                cr[i, d, 3] = 0.25 * (r0 - r1 + r2 - r3)
            for row, (a, b) in enumerate(((1, 2), (2, 0), (0, 1))):
                A, B = rc[a], rc[b]
                cw[i, row, 0] = 0.125 * ((A[0] - A[2]) * (B[1] - B[3]) - (A[1] - A[3]) * (B[0] - B[2]))
                cw[i, row, 1] = 0.125 * ((A[2] - A[3]) * (B[0] - B[1]) - (A[0] - A[1]) * (B[2] - B[3]))
                cw[i, row, 2] = 0.125 * ((A[1] - A[2]) * (B[0] - B[3]) - (A[0] - A[3]) * (B[1] - B[2]))
        else:
            for d in range(3):
                r0, r1, r2 = rc[d][0], rc[d][1], rc[d][2]
                cr[i, d, 0] = 1.0 / 3.0 * (r0 + r1 + r2)
                cr[i, d, 1] = 1.0 / 3.0 * (-r0 + 2.0 * r1 - r2)
                cr[i, d, 2] = 1.0 / math.sqrt(3.0) * (r2 - r0)
                cr[i, d, 3] = 0.0
            cw[i, 0, 0] = (rc[1][1] - rc[1][0]) * (rc[2][2] - rc[2][0]) - (rc[2][1] - rc[2][0]) * (rc[1][2] - rc[1][0])
            cw[i, 1, 0] = (rc[2][1] - rc[2][0]) * (rc[0][2] - rc[0][0]) - (rc[0][1] - rc[0][0]) * (rc[2][2] - rc[2][0])
            cw[i, 2, 0] = (rc[0][1] - rc[0][0]) * (rc[1][2] - rc[1][0]) - (rc[1][1] - rc[1][0]) * (rc[0][2] - rc[0][0])
    return cr, cw


ZT44 = (-P44_N, P44_N, P44_N, -P44_N)
ET44 = (-P44_N, -P44_N, P44_N, P44_N)
ZT34 = (-P34_N0, 2.0 * P34_N0, -P34_N0, 0.0)
ET34 = (-P34_N1, 0.0, P34_N1, 0.0)


class Problem:
    """A loaded problem: the inputs the reference's solver holds in DQD2 (d3qd2_elem.h:49-60)."""

    def __init__(self, waves, ps, vd1, vd2, media, rn, ed, md, sd, gd, rot=None):
        """rot = (rv0, rv1, rv2, th, tv0, tv1, tv2): the optional rotation about axis rv by th and
        translation tv that read_dqd2 takes from the command line (d3qd2_setup.c:16-38)."""
        self.rot = tuple(float(x) for x in rot) if rot is not None else (1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0)
        if self.rot[3] != 0.0 or any(x != 0.0 for x in self.rot[4:]):
            if self.rot[0] == 0.0 and self.rot[1] == 0.0 and self.rot[2] == 0.0:
                raise ValueError("the vector defining the rotation axis is zero")
            rn = rotate_translate(rn, self.rot)
        self.waves = waves
        self.ps = ps
        self.vd1, self.vd2 = vd1, vd2
        self.MN = len(media)
        self.rn, self.ed, self.md, self.sd, self.gd = rn, ed, md, sd, gd
        self.Ne = ed.shape[0] - 1
        self.nv = np.where(ed[:, 3] == 0, 3, 4).astype(np.int32)
        self.nv[0] = 4
        self.media = list(media)
        # initialize_dqd2 (d3qd2_src/d3qd2_setup.c:105-139)
        self._waves_setup(waves)
        self.cr, self.cw = element_constants(rn, ed)
        # sub-domains (init_sub_domain, d3qd2_setup.c:1290-1307)
        self.sid = []
        for d in range(self.MN + 1):
            lst = []
            for i in range(1, self.Ne + 1):
                if md[i] == d:
                    lst.append(i)
                elif sd[i] == d:
                    lst.append(-i)
            self.sid.append(np.array(lst, np.int32))
        # element node ids (read_mesh_data :806-820)
        self.eni = np.full((self.Ne + 1, 4), -1, np.int32)
        nc = 0
        for i in range(1, self.Ne + 1):
            for j in range(self.nv[i]):
                self.eni[i, j] = nc
                nc += 1
        self.NN = nc
        # collocation nodes and incident field (init_boundary_data, d3qd2_setup.c:1309-1349)
        self.ren = np.zeros((self.Ne + 1, 4, 3))
        self.wen = np.zeros((self.Ne + 1, 4, 3))
        for i in range(1, self.Ne + 1):
            c, w = self.cr[i], self.cw[i]
            for j in range(4):
                if self.nv[i] == 3:
                    z, e = ZT34[j], ET34[j]
                    r = c[:, 0] + c[:, 1] * z + c[:, 2] * e
                    wv = w[:, 0].copy()
                else:
                    z, e = ZT44[j], ET44[j]
                    r = c[:, 0] + c[:, 1] * z + c[:, 2] * e + c[:, 3] * z * e
                    wv = w[:, 0] + w[:, 1] * z + w[:, 2] * e
                self.ren[i, j] = r
                self.wen[i, j] = wv
        self._incident()

    def _waves_setup(self, waves):
        """Wave-dependent part of initialize_dqd2: check_mipw (d3qd2_setup.c:1078-1108), the QPGF
        data, the wave numbers of the media (:120-129)."""
        for w in waves:
            w.setup()
        self.waves = waves
        self.n0 = waves[0].ni
        self.lambda0 = waves[0].lambda0
        for w in waves[1:]:
            if w.ni != self.n0 or w.lambda0 != self.lambda0:
                raise ValueError("all plane waves must share ni and lambda0")
        if self.ps == 1:
            kx0 = waves[0].sin_t * waves[0].cos_p
            ky0 = waves[0].sin_t * waves[0].sin_p
            for w in waves:
                kxh, kyh, kzh = w.sin_t * w.cos_p, w.sin_t * w.sin_p, w.cos_t
                if kzh == 0.0:
                    raise ValueError("kz must not be equal to 0")
                if abs(kzh) == 1.0:
                    raise ValueError("kz must not be equal to the wave number (normal incidence)")
                if abs(kx0 - kxh) > MEPS * abs(kxh) or abs(ky0 - kyh) > MEPS * abs(kyh):
                    raise ValueError("all kx and ky must be the same")
        w0 = waves[0]
        k = w0.ki
        vk = [k * w0.sin_t * w0.cos_p, k * w0.sin_t * w0.sin_p, k * w0.cos_t]
        if vk[0] == 0.0:
            vk[0] = k * MEPS
        if vk[1] == 0.0:
            vk[1] = k * MEPS
        self.qpd = dict(k=k, vk=vk, vd1=self.vd1, vd2=self.vd2)
        self.n = [complex(self.n0)] + list(self.media)
        self.kn = [2.0 * math.pi / self.lambda0 * nd for nd in self.n]

    def with_incidence(self, waves) -> "Problem":
        """The same geometry and media under any other incident plane waves (wavelength,
        background index, angles, polarisation): the problem read_dqd2 + initialize_dqd2 would
        build from the same mesh and a different ipw file, without repeating the geometry."""
        import copy
        q = copy.copy(self)
        q._waves_setup(list(waves))
        q._incident()
        return q

    def _incident(self):
        nrm = self.wen / np.linalg.norm(self.wen, axis=-1, keepdims=True).clip(1e-300)
        self.Ui = np.zeros((self.Ne + 1, 4, 4), np.complex128)
        self.dUi = np.zeros((self.Ne + 1, 4, 4), np.complex128)
        for w in self.waves:
            e, h, de, dh = w.eh_dehdv(self.ren, nrm)
            self.Ui[..., :3] += e
            self.dUi[..., :3] += de
        self.Ui[0] = 0
        self.dUi[0] = 0

    def with_waves(self, waves) -> "Problem":
        """The same geometry and media under other incident plane waves with the same wavelength,
        background index and direction (so the same lattice phase and matrices)."""
        import copy
        for w in waves:
            w.setup()
            if (w.lambda0 != self.lambda0 or w.ni != self.n0 or w.theta != self.waves[0].theta
                    or w.phi != self.waves[0].phi):
                raise ValueError("a new incident field must keep the wavelength, index and direction")
        q = copy.copy(self)
        q.waves = list(waves)
        q._incident()
        return q

    def node_tangents(self):
        """Unit tangents t_zeta, t_eta at every collocation node (tz_te_bd_node,
        d3qd2_src/d3qd2_elem.c:122-143).  Returns two [(Ne+1), 4, 3] arrays (slot 0 zero)."""
        cr = self.cr
        quad = (self.nv == 4)[:, None, None]
        et = np.asarray(ET44)[None, :, None]
        zt = np.asarray(ZT44)[None, :, None]
        vtz = cr[:, None, :, 1] + np.where(quad, cr[:, None, :, 3] * et, 0.0)
        vte = cr[:, None, :, 2] + np.where(quad, cr[:, None, :, 3] * zt, 0.0)
        vtz = vtz / np.linalg.norm(vtz, axis=-1, keepdims=True).clip(1e-300)
        vte = vte / np.linalg.norm(vte, axis=-1, keepdims=True).clip(1e-300)
        vtz[0] = 0
        vte[0] = 0
        return vtz, vte

    def incident_tangent_derivatives(self):
        """dE_inc/dt_zeta and dE_inc/dt_eta at every collocation node, summed over the incident
        waves (calc_mipw_EH_dEHdv along tz_te_bd_node's tangents, as q1_solve_eh_bv does at
        d3qd2_src/d3qd2_solve_bieq.c:1003-1004).  Returns two [(Ne+1), 4, 3] complex arrays."""
        vtz, vte = self.node_tangents()
        dEz = np.zeros((self.Ne + 1, 4, 3), np.complex128)
        dEe = np.zeros_like(dEz)
        for w in self.waves:
            dEz += w.eh_dehdv(self.ren, vtz)[2]
            dEe += w.eh_dehdv(self.ren, vte)[2]
        dEz[0] = 0
        dEe[0] = 0
        return dEz, dEe

    @classmethod
    def from_files(cls, ipw: str, ped: str, med: str, msh: str, rot=None) -> "Problem":
        waves = read_planewaves(ipw)
        ps, vd1, vd2 = read_periodicity(ped)
        media = read_media(med)
        rn, ed, md, sd, gd = read_gmsh(msh, len(media))
        return cls(waves, ps, vd1, vd2, media, rn, ed, md, sd, gd, rot=rot)

    # ---- arrays for the C ABI ------------------------------------------------------------
    def flat_mesh(self):
        return (np.ascontiguousarray(self.cr), np.ascontiguousarray(self.cw), np.ascontiguousarray(self.ren),
                np.ascontiguousarray(self.wen), np.ascontiguousarray(self.nv, dtype=np.int32))

    def pairs_per_domain(self) -> List[int]:
        """Evaluations per domain as the reference's loop makes them: collocation nodes x sources."""
        out = []
        for d in range(self.MN + 1):
            s = self.sid[d]
            nodes = int(sum(self.nv[abs(t)] for t in s))
            out.append(nodes * len(s))
        return out


def problem_to_arrays(waves, ps, vd1, vd2, media, rn, ed, md, sd, gd, rot=None) -> dict:
    """Plain-array form of a problem's inputs (for fixtures and for meshes built in memory)."""
    wv = np.array([[w.lambda0, w.ni, w.power, w.e0x.real, w.e0x.imag, w.e0y.real, w.e0y.imag,
                    w.f[0], w.f[1], w.f[2], w.theta, w.phi] for w in waves])
    a = dict(waves=wv, ps=np.int32(ps), vd1=np.array(vd1, float), vd2=np.array(vd2, float),
             media=np.array(media, np.complex128), rn=rn, ed=ed, md=md, sd=sd, gd=gd)
    if rot is not None:
        a["rot"] = np.array(rot, np.float64)
    return a


def problem_from_arrays(a: dict) -> Problem:
    waves = [PlaneWave(v[0], v[1], v[2], complex(v[3], v[4]), complex(v[5], v[6]), (v[7], v[8], v[9]), v[10], v[11])
             for v in np.asarray(a["waves"])]
    return Problem(waves, int(a["ps"]), tuple(np.asarray(a["vd1"]).tolist()), tuple(np.asarray(a["vd2"]).tolist()),
                   [complex(x) for x in np.asarray(a["media"])], np.asarray(a["rn"]), np.asarray(a["ed"]),
                   np.asarray(a["md"]), np.asarray(a["sd"]), np.asarray(a["gd"]),
                   rot=np.asarray(a["rot"]).tolist() if "rot" in a else None)


def load_inputs(ipw: str, ped: str, med: str, msh: str, rot=None) -> dict:
    """Reads the four reference input files into the plain-array form; rot as Problem's."""
    waves = read_planewaves(ipw)
    ps, vd1, vd2 = read_periodicity(ped)
    media = read_media(med)
    rn, ed, md, sd, gd = read_gmsh(msh, len(media))
    return problem_to_arrays(waves, ps, vd1, vd2, media, rn, ed, md, sd, gd, rot)


def write_input_files(a: dict, outdir: str, mesh_name: str = "mesh.msh"):
    """Writes the plain-array form back as the reference's four input files (ipw, periodicity,
    medium, Gmsh 2.2 mesh with every element twice, read_mesh_data's convention) and returns
    their paths.  Reading them back with load_inputs gives the same arrays."""
    import os
    os.makedirs(outdir, exist_ok=True)
    wv = np.asarray(a["waves"])
    ipw = os.path.join(outdir, "ipw.txt")
    with open(ipw, "w") as f:
        f.write("## plane wave data\n# number of wave\n%d\n" % len(wv))
        f.write("# lambda ni power real(e0x) imag(e0x) real(e0y) imag(e0y) fx fy fz theta phi\n")
        for v in wv:
            f.write(" ".join("%.17g" % x for x in v) + "\n")
    ped = os.path.join(outdir, "periodicity_data.txt")
    d1, d2 = np.asarray(a["vd1"]), np.asarray(a["vd2"])
    with open(ped, "w") as f:
        f.write("## periodicity datafile\n# periodicity_setting d1_x d1_y d2_x d2_y\n")
        f.write("%d %.17g %.17g %.17g %.17g\n" % (int(a["ps"]), d1[0], d1[1], d2[0], d2[1]))
    med = os.path.join(outdir, "medium_data.txt")
    media = np.asarray(a["media"])
    with open(med, "w") as f:
        f.write("## medium datafile\n# number of medium\n%d\n# real imag\n" % len(media))
        for m in media:
            f.write("%.17g %.17g\n" % (m.real, m.imag))
    msh = os.path.join(outdir, mesh_name)
    rn, ed, md, sd, gd = (np.asarray(a[k]) for k in ("rn", "ed", "md", "sd", "gd"))
    ne = ed.shape[0] - 1
    with open(msh, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % (rn.shape[0] - 1))
        for i in range(1, rn.shape[0]):
            f.write("%d %.17g %.17g %.17g\n" % (i, rn[i, 0], rn[i, 1], rn[i, 2]))
        f.write("$EndNodes\n$Elements\n%d\n" % (2 * ne))
        for e in range(1, ne + 1):
            tri = ed[e, 3] == 0
            nodes = list(ed[e, :3]) if tri else list(ed[e])
            rev = [nodes[0], nodes[2], nodes[1]] if tri else [nodes[0], nodes[3], nodes[2], nodes[1]]
            et = 2 if tri else 3
            tag1 = OPENDID if md[e] == 0 else int(md[e])
            tag2 = OPENDID if sd[e] == 0 else int(sd[e])
            f.write("%d %d 2 %d %d %s\n" % (2 * e - 1, et, tag1, gd[e], " ".join(str(int(x)) for x in nodes)))
            f.write("%d %d 2 %d %d %s\n" % (2 * e, et, tag2, gd[e], " ".join(str(int(x)) for x in rev)))
        f.write("$EndElements\n")
    return ipw, ped, med, msh
