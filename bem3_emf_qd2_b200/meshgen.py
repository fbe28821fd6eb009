"""Seeded synthetic problems in the reference's input formats (Gmsh 2.2 + three text files).

The benchmark and test workloads are built here: equiangular cube-spheres (one or two
concentric surfaces of bilinear quads) and a triangulated cone with seeded node jitter.  The
writer follows the conventions read_mesh_data expects (d3qd2_src/d3qd2_setup.c:662-959): node
ids 1..Nn, every surface element written twice -- id 2i-1 tagged with the domain on the side
its normal W leaves, id 2i tagged with the other domain and the node order reversed (the
open region is physical id 99).
"""
from __future__ import annotations

import math
import os

import numpy as np

from .dqd2 import load_inputs, problem_from_arrays


class _Nodes:
    def __init__(self):
        self.pts = []
        self.index = {}

    def add(self, p, key=None):
        k = key if key is not None else tuple(np.round(p, 12))
        if k in self.index:
            return self.index[k]
        self.pts.append(np.asarray(p, float))
        self.index[k] = len(self.pts)
        return len(self.pts)


def _cw_center(pts):
    """Normal direction of an element the way init_elem_const computes it (d3qd2_setup.c:1162-1186)."""
    if len(pts) == 4:
        return np.cross(pts[0] - pts[2], pts[1] - pts[3])
    return np.cross(pts[1] - pts[0], pts[2] - pts[0])


def cube_sphere(nodes: _Nodes, radius: float, n: int, center=(0.0, 0.0, 0.0)):
    """Equiangular cube-sphere: 6 faces x n x n quads, node order giving an outward normal."""
    faces = []
    ang = np.linspace(-math.pi / 4, math.pi / 4, n + 1)
    c = np.asarray(center, float)
    # face frames: (normal axis, sign)
    for axis in range(3):
        for sgn in (1.0, -1.0):
            grid = np.zeros((n + 1, n + 1), int)
            for i, a in enumerate(ang):
                for j, b in enumerate(ang):
                    v = np.zeros(3)
                    u1, u2 = (axis + 1) % 3, (axis + 2) % 3
                    v[axis] = sgn
                    v[u1] = math.tan(a)
                    v[u2] = math.tan(b)
                    p = c + radius * v / np.linalg.norm(v)
                    # key on the unit direction so that shared cube edges merge exactly
                    key = tuple(np.round(v / np.linalg.norm(v), 12)) + (radius,)
                    grid[i, j] = nodes.add(p, key)
            for i in range(n):
                for j in range(n):
                    q = [grid[i, j], grid[i + 1, j], grid[i + 1, j + 1], grid[i, j + 1]]
                    pts = [nodes.pts[k - 1] for k in q]
                    cen = sum(pts) / 4.0
                    if np.dot(_cw_center(pts), cen - c) < 0:
                        q = [q[0], q[3], q[2], q[1]]
                    faces.append(q)
    return faces


def cone(nodes: _Nodes, radius: float, height: float, z0: float, rings: int, rows: int, sectors: int,
         jitter: float, seed: int):
    """Circular cone: base disk (rings x sectors) and lateral surface (rows x sectors), linear triangles
    with outward normals; interior nodes jittered by `jitter` x the local edge length (seeded)."""
    rng = np.random.default_rng(seed)
    apex = np.array([0.0, 0.0, z0 + height])
    cen = np.array([0.0, 0.0, z0])
    tris = []
    phis = 2 * math.pi * np.arange(sectors) / sectors

    def ring_point(r, z, k):
        return np.array([r * math.cos(phis[k]), r * math.sin(phis[k]), z])

    # base disk, rings of nodes (ring 0 = centre)
    h_disk = radius / rings
    disk = [[nodes.add(cen)]]
    for ri in range(1, rings + 1):
        r = radius * ri / rings
        row = []
        for k in range(sectors):
            p = ring_point(r, z0, k)
            if ri < rings:
                p = p + np.r_[rng.uniform(-1, 1, 2) * jitter * h_disk, 0.0]
            row.append(nodes.add(p, ("d", ri, k)))
        disk.append(row)
    # lateral rows from the base circle (row 0 shares the disk rim) to the apex
    lat = [disk[rings]]
    slant = math.hypot(radius, height)
    h_lat = slant / rows
    for li in range(1, rows):
        f = li / rows
        r, z = radius * (1 - f), z0 + height * f
        row = []
        for k in range(sectors):
            p = ring_point(r, z, k)
            tang = np.array([-math.sin(phis[k]), math.cos(phis[k]), 0.0])
            p = p + tang * rng.uniform(-1, 1) * jitter * h_lat
            row.append(nodes.add(p, ("l", li, k)))
        lat.append(row)
    top = nodes.add(apex)

    def add(tri, inside_ref):
        pts = [nodes.pts[k - 1] for k in tri]
        cc = sum(pts) / 3.0
        if np.dot(_cw_center(pts), cc - inside_ref) < 0:
            tri = [tri[0], tri[2], tri[1]]
        tris.append(tri)

    inside = np.array([0.0, 0.0, z0 + 0.25 * height])
    for k in range(sectors):
        k1 = (k + 1) % sectors
        add([disk[0][0], disk[1][k], disk[1][k1]], inside)
        for ri in range(1, rings):
            a, b, c, d = disk[ri][k], disk[ri][k1], disk[ri + 1][k1], disk[ri + 1][k]
            add([a, b, c], inside)
            add([a, c, d], inside)
        for li in range(rows - 1):
            a, b, c, d = lat[li][k], lat[li][k1], lat[li + 1][k1], lat[li + 1][k]
            add([a, b, c], inside)
            add([a, c, d], inside)
        add([lat[rows - 1][k], lat[rows - 1][k1], top], inside)
    return tris


def write_gmsh(path: str, nodes: _Nodes, surfaces):
    """surfaces: list of (elements, inner_id, outer_id); normals of `elements` leave `inner_id`."""
    elems = []
    for els, inner, outer in surfaces:
        for e in els:
            elems.append((e, inner, outer))
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(nodes.pts))
        for i, p in enumerate(nodes.pts, start=1):
            f.write("%d %.17g %.17g %.17g\n" % (i, p[0], p[1], p[2]))
        f.write("$EndNodes\n$Elements\n%d\n" % (2 * len(elems)))
        for i, (e, inner, outer) in enumerate(elems, start=1):
            et = 3 if len(e) == 4 else 2
            rev = [e[0], e[3], e[2], e[1]] if len(e) == 4 else [e[0], e[2], e[1]]
            f.write("%d %d 2 %d 1 %s\n" % (2 * i - 1, et, inner, " ".join(map(str, e))))
            f.write("%d %d 2 %d 1 %s\n" % (2 * i, et, outer, " ".join(map(str, rev))))
        f.write("$EndElements\n")


def write_inputs(d: str, lambda0: float, ni: float, power: float, e0, theta: float, phi: float,
                 d1, d2, media, ps: int = 1):
    os.makedirs(d, exist_ok=True)
    waves = e0 if isinstance(e0, list) else [e0]
    with open(os.path.join(d, "ipw.txt"), "w") as f:
        f.write("## plane wave data\n# number of wave\n%d\n" % len(waves))
        f.write("# lambda ni power real(e0x) imag(e0x) real(e0y) imag(e0y) fx fy fz theta phi\n")
        for e in waves:
            f.write("%.17g %.17g %.17g %.17g %.17g %.17g %.17g 0.0 0.0 0.0 %.17g %.17g\n"
                    % (lambda0, ni, power, e[0].real, e[0].imag, e[1].real, e[1].imag, theta, phi))
    with open(os.path.join(d, "periodicity_data.txt"), "w") as f:
        f.write("## periodicity datafile for bem3_emf_qd2\n")
        f.write("# periodicity_setting(0:non periodicity) d1_x d1_y d2_x d2_y\n")
        f.write("%d %.17g %.17g %.17g %.17g\n" % (ps, d1[0], d1[1], d2[0], d2[1]))
    with open(os.path.join(d, "medium_data.txt"), "w") as f:
        f.write("## medium datafile for bem3_emf_qd2\n# number of medium\n%d\n" % len(media))
        f.write("# real(refractive_index) imag(refractive_index)\n")
        for m in media:
            f.write("%.17g %.17g\n" % (complex(m).real, complex(m).imag))


CONFIGS = {
    # sphere r=0.3 um, n=1.59, 6x8x8 quads; square lattice 1.0 um in n=1.33; lambda0=0.6328,
    # x-polarised, amplitude 1 (power = ni/2).  theta = 1e-4 rad stands in for normal incidence,
    # which the reference rejects (kz == k, d3qd2_setup.c:1092-1095).
    "sphere384": dict(surfaces=[("sphere", 0.3, 8, 1, 99)], media=[1.59], lambda0=0.6328, ni=1.33,
                      theta=1e-4, phi=0.0, d1=(1.0, 0.0), d2=(0.0, 1.0), e0=[(1.0, 0.0)]),
    # two-layer sphere: core r=0.25 n=1.59 (medium 2), shell r=0.35 n=1.45+0.01i (medium 1),
    # 6x16x16 quads per surface; lambda0=0.532, theta=30 deg, phi=45 deg, TM and TE waves.
    "twolayer3072": dict(surfaces=[("sphere", 0.35, 16, 1, 99), ("sphere", 0.25, 16, 2, 1)],
                         media=[1.45 + 0.01j, 1.59], lambda0=0.532, ni=1.33, theta=math.pi / 6,
                         phi=math.pi / 4, d1=(1.0, 0.0), d2=(0.0, 1.0), e0=[(1.0, 0.0)]),
    # cone base r=0.3 at z=-0.3, height 0.6, n=2.0+0.1i, 12 rings x 48 + 24 rows x 48 triangles,
    # 1% seeded jitter; hexagonal lattice 0.9 um in n=1.0; lambda0=0.7, theta=10 deg.
    "cone3360": dict(surfaces=[("cone", 0.3, 0.6, -0.3, 12, 24, 48, 0.01, 12345, 1, 99)], media=[2.0 + 0.1j],
                     lambda0=0.7, ni=1.0, theta=math.radians(10.0), phi=0.0, d1=(0.9, 0.0), d2=(0.45, 0.7794),
                     e0=[(1.0, 0.0)]),
    # small cases for tests
    "sphere96": dict(surfaces=[("sphere", 0.3, 4, 1, 99)], media=[1.59], lambda0=0.6328, ni=1.33,
                     theta=0.3, phi=0.2, d1=(1.0, 0.0), d2=(0.0, 1.0), e0=[(1.0, 0.0)]),
    "twolayer192": dict(surfaces=[("sphere", 0.35, 4, 1, 99), ("sphere", 0.25, 4, 2, 1)],
                        media=[1.45 + 0.01j, 1.59], lambda0=0.532, ni=1.33, theta=math.pi / 6,
                        phi=math.pi / 4, d1=(1.0, 0.0), d2=(0.0, 1.0), e0=[(1.0, 0.0)]),
    "cone210": dict(surfaces=[("cone", 0.3, 0.6, -0.3, 3, 5, 12, 0.01, 12345, 1, 99)], media=[2.0 + 0.1j],
                    lambda0=0.7, ni=1.0, theta=math.radians(10.0), phi=0.0, d1=(0.9, 0.0), d2=(0.45, 0.7794),
                    e0=[(1.0, 0.0)]),
}


def make_config(name: str, outdir: str, **over):
    """Writes the four input files of a named synthetic configuration to `outdir` and returns
    their paths (ipw, periodicity, medium, mesh)."""
    cfg = dict(CONFIGS[name])
    cfg.update(over)
    return write_config(name, cfg, outdir)


def write_config(name: str, cfg: dict, outdir: str):
    """make_config for a configuration dictionary of the same form as CONFIGS' entries."""
    nodes = _Nodes()
    surfs = []
    for s in cfg["surfaces"]:
        if s[0] == "sphere":
            _, r, n, inner, outer = s
            surfs.append((cube_sphere(nodes, r, n), inner, outer))
        else:
            _, r, h, z0, rings, rows, sect, jit, seed, inner, outer = s
            surfs.append((cone(nodes, r, h, z0, rings, rows, sect, jit, seed), inner, outer))
    os.makedirs(outdir, exist_ok=True)
    msh = os.path.join(outdir, name + ".msh")
    write_gmsh(msh, nodes, surfs)
    e0 = [(complex(a), complex(b)) for a, b in cfg["e0"]]
    write_inputs(outdir, cfg["lambda0"], cfg["ni"], cfg["ni"] / 2.0, e0, cfg["theta"], cfg["phi"], cfg["d1"],
                 cfg["d2"], cfg["media"])
    return (os.path.join(outdir, "ipw.txt"), os.path.join(outdir, "periodicity_data.txt"),
            os.path.join(outdir, "medium_data.txt"), msh)


def problem(name: str, outdir: str, **over):
    """The named configuration, written to disk and read back through the reference-format readers."""
    files = make_config(name, outdir, **over)
    return problem_from_arrays(load_inputs(*files)), files
