"""Generates the golden fixtures in this directory from the reference (akohta/bem3_emf_qd2).

Run with the path of a checkout of the reference's sources, after ``make -C oracle ref REF=<it>``.
Every array stored here comes from the reference's own code, compiled from its sources by
oracle/Makefile and called through oracle/reforacle.py:

  gauleg.npz    the Gauss-Legendre tables of gauleg (com_src/gauleg.c) for n = 12, 64
  faddeeva.npz  Faddeeva_w (qgf2_src/Faddeeva.cc) at seeded points, relerr 1e-15
  qpgf.npz      d3hm_qpgf_d2_v1 / _qG / _dqG / _v2 (qgf2_src/d3_qpgf_d2.c) for 5 lattices
  rows_*.npz    inputs of a sample problem shipped with the reference (read by the reference's
                own readers) and complete rows of create_cmatrix_domain
                (d3qd2_src/d3qd2_solve_bieq.c:165-256) for selected collocation elements.
  bv_*.npz      boundary values (U, dU, E, H, dE, dH of every domain) stored in the result files
                the reference ships (verification/veri.dat, analysis_sample*/ex*.dat), read by its
                own dat_read, plus the reference's EH_t (d3qd2_field.c) at probe points and its
                force_FN (d3qd2_force.c) for those results, types 0 and 1.
  near_fields.npz  the reference's EH_t, types 0-3, at points just off the boundary of those
                results.
  potentials.npz  the reference's mEMP_s/_t/_i (types 0-3), EH_i and EH_mEMP_s/_t/_i (types
                0-2) at the probe points and the near-boundary points of those results.
  fullsize_rows.npz  rows of create_cmatrix_domain at the full sizes of the three plain
                configurations (sphere384, twolayer3072, cone3360), eight elements per domain: dF,
                and G, H (dG, dH on interior domains) at every 16th column and the element's own
                columns; for the cone's in-plane row block also the reference's rows with the
                collocation nodes moved by -4..4 ulps (see fullsize_rows).
  power.npz     incident, reflected and transmitted power through one unit cell for those
                results, from the reference's EH_t / EH_s on two planes.
  c1_sphere384.npz  plain configuration 1 end to end through the reference's own solver program
                (see c1_fixture).
  elem_const.npz  the reference's element constants and collocation nodes (cr, cw, ren, wen) for
                the shipped meshes of rows_*.npz and the rotated result file of bv_ex2.npz.
  example2_rows.npz  the reference's EH_t (type 1) on two rows of example2.c's first plane for the
                verification result, as the intensities that program writes.

Usage: python tests/golden/make_golden.py <reference_dir> [section ...]
       sections: gauleg faddeeva qpgf rows bv near potentials power fullsize c1 example2 elemconst
                 (default: all)
                 envelope (only the z-shifted rows of an existing fullsize_rows.npz)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, REPO)

from reforacle import RefOracle  # noqa: E402
from bem3_emf_qd2_b200.dqd2 import load_inputs  # noqa: E402

if len(sys.argv) < 2 or not os.path.isdir(os.path.join(sys.argv[1], "d3qd2_src")):
    sys.exit("usage: make_golden.py <checkout of akohta/bem3_emf_qd2> [section ...]")
REF = sys.argv[1]
SECTIONS = {a for a in sys.argv[2:] if "=" not in a} or {"gauleg", "faddeeva", "qpgf", "rows", "bv", "near",
                                                         "potentials", "power", "fullsize", "c1", "example2",
                                                         "elemconst"}
ONLY = {x for a in sys.argv[2:] if a.startswith("only=") for x in a[5:].split(",")}


def qpd_of(k, th, ph, d1, d2):
    vk = [k * np.sin(th) * np.cos(ph), k * np.sin(th) * np.sin(ph), k * np.cos(th)]
    if vk[0] == 0.0:
        vk[0] = k * 1e-15
    if vk[1] == 0.0:
        vk[1] = k * 1e-15
    return np.array([k, *vk, *d1, *d2])


LATTICES = {
    # config-1 lattice (square 1.0, n=1.33, lambda0=0.6328, near-normal incidence)
    "square1_c1": qpd_of(2 * np.pi * 1.33 / 0.6328, 1e-4, 0.0, (1.0, 0.0), (0.0, 1.0)),
    # the reference's verification lattice (hexagonal 2.0, lambda0=1, theta=0.2)
    "hex2_veri": qpd_of(2 * np.pi * 1.33 / 1.0, 0.2, 0.0, (2.0, 0.0), (1.0, 1.7320508075688772)),
    # config-3 lattice (hexagonal 0.9, n=1.0, lambda0=0.7, theta=10 deg)
    "hex09_c3": qpd_of(2 * np.pi * 1.0 / 0.7, np.radians(10.0), 0.0, (0.9, 0.0), (0.45, 0.7794)),
    # config-2 lattice (square 1.0, lambda0=0.532, theta=30 deg, phi=45 deg)
    "square1_c2": qpd_of(2 * np.pi * 1.33 / 0.532, np.pi / 6, np.pi / 4, (1.0, 0.0), (0.0, 1.0)),
    # analysis_sample3 lattice (hexagonal 0.75)
    "hex075": qpd_of(2 * np.pi * 1.33 / 1.0, 0.2, 0.0, (0.75, 0.0), (0.375, 0.649519052838329)),
}

CASES = {
    # name: (directory, mesh, {did: [1-based collocation elements]})
    "sphere_m4": ("verification", "sphere_m4.msh", {0: [1, 200], 1: [1, 100]}),
    "cone_m1": ("analysis_sample2", "cone_m1.msh", {0: [1, 300], 1: [5]}),
    "sphere_m2": ("analysis_sample1", "sphere_m2.msh", {0: [7], 1: [11], 2: [3]}),
}


def gauleg_tables(o):
    d = os.path.join(REF, "verification")
    o.load(*[os.path.join(d, f) for f in ("ipw.txt", "periodicity_data.txt", "medium_data.txt", "sphere_m4.msh")])
    g = o.geometry()
    np.savez_compressed(os.path.join(HERE, "gauleg.npz"), x12=g["xli"], w12=g["wli"], x64=g["xhi"], w64=g["whi"])


# result files shipped with the reference: name -> (directory, .dat, mesh, rotation given to the
# solver on its command line (d3qd2_bv_solver.log of each directory), probe points)
BV_CASES = {
    "veri": ("verification", "veri.dat", "sphere_m4.msh", None,
             [(0.3, 0.0, 1.1), (0.0, 0.0, 0.0), (0.15, -0.1, 0.2), (0.9, 0.4, 0.05), (-0.5, 0.3, 1.5),
              (0.1, -0.2, -1.3), (1.7, 1.2, 0.6)]),
    "ex2": ("analysis_sample2", "ex2.dat", "cone_m1.msh", (1.0, 0.0, 0.0, 3.1415926535, 0.0, 0.0, 0.0),
            [(0.3, 0.0, 1.1), (0.0, 0.0, 0.0), (0.3, 0.2, 1.2), (-0.4, 0.1, -1.0), (0.5, -0.6, 0.3)]),
}


def bv_fixtures(o):
    for name, (sub, dat, msh, rot, pts) in BV_CASES.items():
        if ONLY and name not in ONLY:
            continue
        d = os.path.join(REF, sub)
        o.load_dat(os.path.join(d, dat))
        files = [os.path.join(d, f) for f in ("ipw.txt", "periodicity_data.txt", "medium_data.txt", msh)]
        rec = {"in/" + k: v for k, v in load_inputs(*files, rot=rot).items()}
        rec["dat/rn"] = o.geometry()["rn"]  # the result file's (rotated) nodes, to pin the set-up
        info = o.info()
        for dd in range(info["MN"] + 1):
            for k, v in o.boundary_values(dd).items():
                rec[f"bv{dd}/{k}"] = v
        r = np.array(pts, np.float64)
        rec["probe/r"] = r
        for ty in (0, 1):
            E, H, did = o.EH(r, ty, total=True)
            rec[f"probe/E{ty}"] = E
            rec[f"probe/H{ty}"] = H
            rec[f"probe/did"] = did
            F, N = o.force((0.0, 0.0, 0.0), ty)
            rec[f"force/F{ty}"] = F
            rec[f"force/N{ty}"] = N
        np.savez_compressed(os.path.join(HERE, f"bv_{name}.npz"), **rec)
        print(name, "bv done", flush=True)


def near_fields(o):
    """EH_t of the reference, types 0-3, at points just off the boundary (both sides) of a few
    elements of each shipped result file."""
    out = {}
    for name, (sub, dat, msh, rot, pts) in BV_CASES.items():
        o.load_dat(os.path.join(REF, sub, dat))
        g = o.geometry()
        ne = g["cr"].shape[0] - 1
        pick = [1, ne // 3, (2 * ne) // 3]
        r = []
        for e in pick:
            c = g["cr"][e, :, 0]
            w = g["cw"][e, :, 0]
            h = np.sqrt(np.linalg.norm(w))
            n = w / np.linalg.norm(w)
            for f in (0.1, -0.1, 0.3):
                r.append(c + f * h * n)
        r = np.array(r)
        out[name + "/r"] = r
        for ty in (0, 1, 2, 3):
            E, H, did = o.EH(r, ty, total=True)
            out[f"{name}/E{ty}"] = E
            out[f"{name}/H{ty}"] = H
            out[f"{name}/did"] = did
        print(name, "near fields done", flush=True)
    np.savez_compressed(os.path.join(HERE, "near_fields.npz"), **out)


def potentials(o):
    """The reference's modified potentials (mEMP_s / _t / _i, types 0-3), incident field (EH_i) and
    fields from the potentials' derivatives (EH_mEMP_s / _t / _i, types 0-2) at the probe points of
    each shipped result file and at points just off its boundary (near_fields.npz)."""
    near = np.load(os.path.join(HERE, "near_fields.npz"))
    out = {}
    for name, (sub, dat, msh, rot, pts) in BV_CASES.items():
        o.load_dat(os.path.join(REF, sub, dat))
        r = np.concatenate([np.array(pts, float), near[name + "/r"]])
        out[name + "/r"] = r
        for ty in (0, 1, 2, 3):
            for mode in (0, 1, 2):
                U, did = o.mEMP(r, ty, mode)
                out[f"{name}/U{ty}_{mode}"] = U
                out[f"{name}/did"] = did
        E, H, _ = o.EH(r, 0, 2)
        out[name + "/Ei"], out[name + "/Hi"] = E, H
        for ty in (0, 1, 2):
            for mode in (0, 1, 2):
                E, H, did = o.EH_mEMP(r, ty, mode)
                out[f"{name}/mE{ty}_{mode}"], out[f"{name}/mH{ty}_{mode}"] = E, H
                out[f"{name}/mdid{ty}_{mode}"] = did
        print(name, "potentials done", flush=True)
    np.savez_compressed(os.path.join(HERE, "potentials.npz"), **out)


POWER = {"veri": (1.4, -1.4, 16), "ex2": (1.2, -1.2, 16)}  # z_top, z_bottom, grid


def power_balance(o):
    """Reflected, transmitted and incident power through one cell from the reference's EH_t/EH_s
    sampled on two planes (the same quadrature as bem3_emf_qd2_b200.plane_power)."""
    from bem3_emf_qd2_b200 import plane_power
    from bem3_emf_qd2_b200.dqd2 import problem_from_arrays
    out = {}
    for name, (sub, dat, msh, rot, pts) in BV_CASES.items():
        o.load_dat(os.path.join(REF, sub, dat))
        g = np.load(os.path.join(HERE, f"bv_{name}.npz"))
        p = problem_from_arrays({k[3:]: g[k] for k in g.files if k.startswith("in/")})
        zt, zb, n = POWER[name]

        def field(r, total):
            E, H, did = o.EH(r, 0, total=total)
            return E, H, did

        res = plane_power(field, p.vd1, p.vd2, p.waves[0].cos_t > 0, zt, zb, n)
        out[name + "/spec"] = np.array([zt, zb, n])
        for k, v in res.items():
            out[f"{name}/{k}"] = np.array(v)
        print(name, res, flush=True)
    np.savez_compressed(os.path.join(HERE, "power.npz"), **out)


# elements whose rows the full-size fixture holds (1-based positions in each domain's list): the
# rows where the double-layer identity F = 1/2 is least exact, the first element, and six more spread
# over the list; dG, dH are kept (interior domains; the open region's are zero) for every other one
FULLSIZE = {"sphere384": (1, 313), "twolayer3072": (1, 1536), "cone3360": (1, 69)}
FULLSIZE_SPREAD = 6
FULLSIZE_STRIDE = 16  # columns kept of each row (every 16th, plus the element's own four)
# rows whose sources lie in the plane of the collocation nodes to within one ulp: the reference's
# rows with those nodes moved by -4..4 ulps in z as well (its own spread there; the range over
# these nine rows is the same as over -8..8)
FULLSIZE_ENVELOPE = {"cone3360": {0: (1,)}}
ENVELOPE_ULPS = (-4, -3, -2, -1, 1, 2, 3, 4)


def fullsize_elements(name, ne):
    spread = np.unique(np.round(np.linspace(1, ne, FULLSIZE_SPREAD)).astype(int))
    return sorted({e for e in FULLSIZE[name] if e <= ne} | set(int(e) for e in spread))


def fullsize_rows(o):
    """Rows of create_cmatrix_domain at the three plain configurations' full sizes (meshes written
    by bem3_emf_qd2_b200.meshgen and read by the reference's own readers): dF in full, G and H (and
    for every other element of the interior domains dG, dH) at every FULLSIZE_STRIDE-th column and at
    the element's own four columns; for FULLSIZE_ENVELOPE's rows also G, H with the collocation
    nodes moved by ENVELOPE_ULPS."""
    import tempfile
    from bem3_emf_qd2_b200 import meshgen
    out = {}
    for name in FULLSIZE:
        d = tempfile.mkdtemp(prefix="bem3_full_")
        files = meshgen.make_config(name, d)
        cwd = os.getcwd()
        os.chdir(d)  # the reference keeps input file names in 64-byte buffers
        try:
            o.load(*[os.path.basename(f) for f in files])
        finally:
            os.chdir(cwd)
        info = o.info()
        for did in range(info["MN"] + 1):
            elems = fullsize_elements(name, info["Ne_d"][did])
            allrows = o.assemble_rows_list(did, elems)
            for j, t in enumerate(elems):
                G, H = allrows[0][4 * j:4 * j + 4], allrows[1][4 * j:4 * j + 4]
                dG, dH = allrows[2][8 * j:8 * j + 8], allrows[3][8 * j:8 * j + 8]
                dF = allrows[4][4 * j:4 * j + 4]
                N = G.shape[1]
                cols = np.union1d(np.arange(0, N, FULLSIZE_STRIDE), np.arange(4 * (t - 1), 4 * t))
                key = f"{name}/d{did}/t{t}"
                out[key + "/cols"] = cols.astype(np.int32)
                out[key + "/G"] = G[:, cols]
                out[key + "/H"] = H[:, cols]
                out[key + "/dF"] = dF
                if did > 0 and j % 2 == 0:
                    out[key + "/dG"] = dG[:, cols]
                    out[key + "/dH"] = dH[:, cols]
                if t in FULLSIZE_ENVELOPE.get(name, {}).get(did, ()):
                    out.update(envelope_rows(o, key, did, t, cols))
                print(name, did, t, "done", flush=True)
    np.savez_compressed(os.path.join(HERE, "fullsize_rows.npz"), **out)


def envelope_rows(o, key, did, t, cols):
    """G, H of element t's rows with its collocation nodes moved by ENVELOPE_ULPS in z (the
    reference loaded in `o`), at the columns `cols`."""
    out = {}
    for u in ENVELOPE_ULPS:
        Gs, Hs, _, _, _ = o.assemble_rows_zshift(did, t, t, u)
        out[f"{key}/zshift{u:+d}/G"] = Gs[:, cols]
        out[f"{key}/zshift{u:+d}/H"] = Hs[:, cols]
    return out


def fullsize_envelope(o):
    """Recomputes only the FULLSIZE_ENVELOPE rows of an existing fullsize_rows.npz (section
    "envelope"): the other entries are kept as they are."""
    import tempfile
    from bem3_emf_qd2_b200 import meshgen
    path = os.path.join(HERE, "fullsize_rows.npz")
    g = np.load(path)
    out = {k: g[k] for k in g.files if "/zshift" not in k}
    for name, per in FULLSIZE_ENVELOPE.items():
        d = tempfile.mkdtemp(prefix="bem3_env_")
        files = meshgen.make_config(name, d)
        cwd = os.getcwd()
        os.chdir(d)
        try:
            o.load(*[os.path.basename(f) for f in files])
        finally:
            os.chdir(cwd)
        for did, ts in per.items():
            for t in ts:
                key = f"{name}/d{did}/t{t}"
                out.update(envelope_rows(o, key, did, t, g[key + "/cols"]))
                print(key, "envelope done", flush=True)
    np.savez_compressed(path, **out)


# Plain configuration 1 end to end (sphere384): elements whose complete rows are stored (1-based
# positions in each domain's list, spread over the six cube faces), and the subset whose tangential
# derivative rows dG, dH are stored too (interior domain; the open domain's are zero).
C1_ROWS = [1 + 24 * i for i in range(16)]
C1_DROWS = C1_ROWS[::2]
C1_GRID = np.linspace(-0.5, 0.5, 21)  # probe grid on y = 0: x, z in [-0.5, 0.5] x period


def c1_fixture(o):
    """Plain configuration 1 (sphere384: cube-sphere r = 0.3 um of 384 quads, n = 1.59, square
    lattice 1.0 um in n = 1.33, lambda0 = 0.6328, theta = 1e-4 rad) through the reference's own
    programs: d3qd2_bv_solver (oracle/_ref, PARDISO replaced by a dense LU) writes the result
    file, example1.out prints its probe field and force, and the reference's EH_t, force_FN and
    create_cmatrix_domain give the rest.  Stored in c1_sphere384.npz:
      in/*        the problem's inputs as the reference-format readers return them
      bv{d}/*     boundary values of every domain (the result file's U, dU, E, H, dE, dH)
      grid/*      EH_t, types 0 and 1, on the 21 x 21 probe grid of the y = 0 plane
      force/*     force_FN types 0 and 1 about the origin
      power/*     incident, reflected and transmitted power through one cell (plane_power)
      rows/d{d}/t{t}/*  complete rows (G, H, dF; dG, dH for C1_DROWS of the interior domain)
      example1    the stdout of the reference's example1.out on the result file
    The solver run takes about half an hour on 8 cores; BEM3_C1_WORKDIR may name a directory that
    holds a finished run (c1.dat) to reuse."""
    import subprocess
    import tempfile
    from bem3_emf_qd2_b200 import meshgen, plane_power
    d = os.environ.get("BEM3_C1_WORKDIR") or tempfile.mkdtemp(prefix="bem3_c1_")
    files = meshgen.make_config("sphere384", d)
    names = [os.path.basename(f) for f in files]
    ref_bin = os.path.join(REPO, "oracle", "_ref")
    if not os.path.exists(os.path.join(d, "c1.dat")):
        with open(os.path.join(d, "solver.log"), "w") as log:
            subprocess.run([os.path.join(ref_bin, "d3qd2_bv_solver"), *names, "c1.dat"], cwd=d, check=True,
                           stdout=log, stderr=subprocess.STDOUT)
    ex1 = subprocess.run([os.path.join(ref_bin, "example1.out"), "c1.dat"], cwd=d, check=True,
                         capture_output=True, text=True).stdout
    rec = {"in/" + k: v for k, v in load_inputs(*files).items()}
    rec["example1"] = np.array(ex1)
    cwd = os.getcwd()
    os.chdir(d)  # the reference keeps file names in 64-byte buffers
    try:
        o.load_dat("c1.dat")
    finally:
        os.chdir(cwd)
    info = o.info()
    for dd in range(info["MN"] + 1):
        for k, v in o.boundary_values(dd).items():
            rec[f"bv{dd}/{k}"] = v
    X, Z = np.meshgrid(C1_GRID, C1_GRID, indexing="ij")
    r = np.c_[X.ravel(), np.zeros(X.size), Z.ravel()]
    rec["grid/r"] = r
    for ty in (0, 1):
        E, H, did = o.EH(r, ty, total=True)
        rec[f"grid/E{ty}"], rec[f"grid/H{ty}"], rec["grid/did"] = E, H, did
        F, N = o.force((0.0, 0.0, 0.0), ty)
        rec[f"force/F{ty}"], rec[f"force/N{ty}"] = F, N
    print("c1 grid and force done", flush=True)
    from bem3_emf_qd2_b200.dqd2 import problem_from_arrays
    p = problem_from_arrays({k[3:]: v for k, v in rec.items() if k.startswith("in/")})
    pw = plane_power(lambda x, total: o.EH(x, 0, total=total), p.vd1, p.vd2, p.waves[0].cos_t > 0, 0.6, -0.6, 16)
    for k, v in pw.items():
        rec[f"power/{k}"] = np.array(v)
    print("c1 power", pw, flush=True)
    for dd in range(info["MN"] + 1):
        for t in C1_ROWS:
            G, H, dG, dH, dF = o.assemble_rows(dd, t, t)
            key = f"rows/d{dd}/t{t}"
            rec[key + "/G"], rec[key + "/H"], rec[key + "/dF"] = G, H, dF
            if dd > 0 and t in C1_DROWS:
                rec[key + "/dG"], rec[key + "/dH"] = dG, dH
        print("c1 rows of domain", dd, "done", flush=True)
    np.savez_compressed(os.path.join(HERE, "c1_sphere384.npz"), **rec)


EX2_ROWS = (0, 100)  # rows i of example2.c's first plane (x = 0) held by example2_rows.npz


def example2_rows(o):
    """The reference's EH_t, type 1, at the points of rows EX2_ROWS of the first plane that the
    reference's example2.c evaluates (x = 0; y = -rang + i dr, z = -rang + j dr, rang = lambda_0,
    dr = 2 rang / 199, j = 0..199; example2.c:16-45) on its verification result (veri.dat), as the
    intensities |E|^2 and |H|^2 it writes to Ie_yz.txt / Ih_yz.txt."""
    sub, dat = BV_CASES["veri"][0], BV_CASES["veri"][1]
    o.load_dat(os.path.join(REF, sub, dat))
    lam = float(o.geometry()["lambda0"])
    rang, mx = 1.0 * lam, 200
    dr = rang * 2.0 / (mx - 1)
    out = {"rows": np.array(EX2_ROWS), "lambda0": np.array(lam)}
    for i in EX2_ROWS:
        r = np.array([[0.0, -rang + i * dr, -rang + j * dr] for j in range(mx)])
        E, H, _ = o.EH(r, 1, total=True)
        out[f"r{i}"] = r
        out[f"ie{i}"] = (np.abs(E) ** 2).sum(axis=1)
        out[f"ih{i}"] = (np.abs(H) ** 2).sum(axis=1)
        print("example2 row", i, "done", flush=True)
    np.savez_compressed(os.path.join(HERE, "example2_rows.npz"), **out)


def element_constants_fixture(o):
    """The reference's element constants and collocation nodes (init_elem_const and
    init_boundary_data, d3qd2_setup.c:1139-1186, 1309-1349) as it holds them after reading the
    shipped meshes (CASES) and the rotated result file of analysis_sample2 (BV_CASES["ex2"]):
    cr, cw, ren, wen per case, beside the inputs the host set-up reads."""
    out = {}
    for name, (sub, msh, _) in CASES.items():
        d = os.path.join(REF, sub)
        files = [os.path.join(d, f) for f in ("ipw.txt", "periodicity_data.txt", "medium_data.txt", msh)]
        o.load(*files)
        g = o.geometry()
        for k in ("cr", "cw", "ren", "wen"):
            out[f"{name}/{k}"] = g[k]
    sub, dat, msh, rot, _ = BV_CASES["ex2"]
    d = os.path.join(REF, sub)
    o.load_dat(os.path.join(d, dat))
    g = o.geometry()
    for k in ("cr", "cw", "ren", "wen"):
        out[f"ex2/{k}"] = g[k]
    np.savez_compressed(os.path.join(HERE, "elem_const.npz"), **out)


def main():
    o = RefOracle()
    if "elemconst" in SECTIONS:
        element_constants_fixture(o)
    if "c1" in SECTIONS:
        c1_fixture(o)
    if "example2" in SECTIONS:
        example2_rows(o)
    if "fullsize" in SECTIONS:
        fullsize_rows(o)
    if "envelope" in SECTIONS and "fullsize" not in SECTIONS:
        fullsize_envelope(o)
    if "power" in SECTIONS:
        power_balance(o)
    if "near" in SECTIONS:
        near_fields(o)
    if "potentials" in SECTIONS:
        potentials(o)
    if "gauleg" in SECTIONS:
        gauleg_tables(o)
    if "bv" in SECTIONS:
        bv_fixtures(o)
    if not SECTIONS & {"faddeeva", "qpgf", "rows"}:
        return
    rng = np.random.default_rng(20261203)

    # ---- Faddeeva -----------------------------------------------------------------------
    z = np.concatenate([
        rng.uniform(-12, 12, 3000) + 1j * rng.uniform(-10, 14, 3000),
        rng.uniform(-6, 6, 1000) + 1j * 10 ** rng.uniform(-12, 0.5, 1000) * rng.choice([-1, 1], 1000),
        rng.uniform(-0.5, 0.5, 500) + 1j * rng.uniform(-0.5, 0.5, 500),
    ])
    if "faddeeva" in SECTIONS:
        np.savez_compressed(os.path.join(HERE, "faddeeva.npz"), z=z, w=o.faddeeva(z))

    # ---- QPGF -----------------------------------------------------------------------------
    out = {}
    for name, p in LATTICES.items():
        r = np.concatenate([rng.uniform(-0.7, 0.7, (1200, 3)), rng.uniform(-0.04, 0.04, (300, 3)),
                            np.c_[rng.uniform(-1.5, 1.5, (300, 2)), rng.uniform(-2.5, 2.5, (300, 1))]])
        v1, rv1 = o.qpgf(r, p, "v1")
        g, rg = o.qpgf(r, p, "qG")
        d, rd = o.qpgf(r, p, "dqG")
        v2, rv2 = o.qpgf(r, p, "v2")
        out[name + "/v2"] = v2
        out[name + "/ret_v2"] = rv2
        out[name + "/qpd"] = p
        out[name + "/r"] = r
        out[name + "/v1"] = v1
        out[name + "/ret_v1"] = rv1
        out[name + "/qG"] = g[:, 0]
        out[name + "/dqG"] = d
    if "qpgf" in SECTIONS:
        np.savez_compressed(os.path.join(HERE, "qpgf.npz"), **out)

    # ---- rows of the assembly -----------------------------------------------------------
    if "rows" not in SECTIONS:
        return
    for name, (sub, msh, sel) in CASES.items():
        d = os.path.join(REF, sub)
        files = [os.path.join(d, f) for f in ("ipw.txt", "periodicity_data.txt", "medium_data.txt", msh)]
        o.load(*files)
        arr = load_inputs(*files)
        rec = {"in/" + k: v for k, v in arr.items()}
        for did, elems in sel.items():
            for t in elems:
                G, H, dG, dH, dF = o.assemble_rows(did, t, t)
                rec[f"d{did}/t{t}/G"] = G
                rec[f"d{did}/t{t}/H"] = H
                if did > 0:
                    rec[f"d{did}/t{t}/dG"] = dG
                    rec[f"d{did}/t{t}/dH"] = dH
                else:
                    rec[f"d{did}/t{t}/dGdH_absmax"] = np.array(max(np.abs(dG).max(), np.abs(dH).max()))
                rec[f"d{did}/t{t}/dF"] = dF
                print(name, did, t, "done", flush=True)
        np.savez_compressed(os.path.join(HERE, f"rows_{name}.npz"), **rec)


if __name__ == "__main__":
    main()
