"""CPU tests: the oracle against the committed golden vectors, the device math compiled for the
host against the same vectors, the host set-up, and the C-ABI library's exported symbols."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import REPO, golden


def _rel(a, b, floor=1e-300):
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


# ---- golden vectors pin the reference oracle (when it was built here) ------------------------
@pytest.mark.skipif(not os.path.exists(os.path.join(REPO, "oracle", "_ref", "libbem3ref.so")),
                    reason="reference oracle not built in this checkout")
def test_reference_oracle_reproduces_goldens():
    from reforacle import RefOracle
    o = RefOracle()
    f = golden("faddeeva.npz")
    assert np.array_equal(o.faddeeva(f["z"]), f["w"])
    q = golden("qpgf.npz")
    names = sorted({k.split("/")[0] for k in q.files})
    for n in names:
        out, ret = o.qpgf(q[n + "/r"][:300], q[n + "/qpd"], "v1")
        assert np.array_equal(out, q[n + "/v1"][:300]) and np.array_equal(ret, q[n + "/ret_v1"][:300])


# ---- device math compiled for the host ------------------------------------------------------
@pytest.mark.parametrize("fast", [False, True])
def test_faddeeva_host_build(devmath_host, fast):
    """Both forms of w(z): Smith-scaled reciprocals (the QPGF entry point) and the
    single-division reciprocals of the assembly kernels."""
    f = golden("faddeeva.npz")
    z = f["z"]
    zz = np.ascontiguousarray(np.stack([z.real, z.imag], 1).ravel())
    out = np.zeros_like(zz)
    (devmath_host.hm_faddeeva_fast if fast else devmath_host.hm_faddeeva)(len(z), zz.ctypes.data, out.ctypes.data)
    w = out[0::2] + 1j * out[1::2]
    # |w - w_ref| / |w_ref|: the reference itself targets 1e-15 relative error
    assert np.max(np.abs(w - f["w"]) / np.abs(f["w"])) < 1e-13


def test_erfcx_polynomial_against_mpmath(devmath_host):
    """The assembly's erfcx (polynomial form, csrc/erfcx_poly.h) against 50-digit mpmath over the
    arguments the spectral terms produce (and far beyond), negative ones included: 2e-15 relative."""
    import mpmath as mp
    mp.mp.dps = 50
    rng = np.random.default_rng(3)
    x = np.concatenate([np.linspace(0.0, 8.0, 801), np.geomspace(8.0, 1e9, 200), rng.uniform(0.0, 12.0, 400),
                        -rng.uniform(0.0, 3.0, 200)])
    out = np.zeros_like(x)
    devmath_host.hm_erfcx(len(x), x.ctypes.data, out.ctypes.data)
    for xi, vi in zip(x, out):
        ref = float(mp.exp(mp.mpf(float(xi)) ** 2) * mp.erfc(mp.mpf(float(xi))))
        assert abs(vi - ref) <= 2e-15 * abs(ref), (xi, vi, ref)


@pytest.mark.parametrize("mode", [0, 1])
def test_qpgf_host_build(devmath_host, mode):
    q = golden("qpgf.npz")
    names = sorted({k.split("/")[0] for k in q.files})
    for n in names:
        r = np.ascontiguousarray(q[n + "/r"])
        out = np.zeros(len(r) * 8)
        ret = np.zeros(len(r), np.int32)
        devmath_host.hm_qpgf(len(r), r.ctypes.data, np.ascontiguousarray(q[n + "/qpd"]).ctypes.data, mode,
                             out.ctypes.data, ret.ctypes.data)
        got = (out[0::2] + 1j * out[1::2]).reshape(-1, 4)
        assert np.all(ret > 0)
        if mode == 0:
            # same stop rules as d3hm_qpgf_d2_v1: identical term counts at every point
            assert np.array_equal(ret, q[n + "/ret_v1"]), n
            ref = q[n + "/v1"]
        else:
            ref = np.c_[q[n + "/qG"], q[n + "/dqG"]]
        scale = np.abs(ref).max(axis=1, keepdims=True)
        assert np.max(np.abs(got - ref) / scale) < 1e-10, n


def test_qpgf_second_derivatives_host_build(devmath_host):
    """qpgf_eval2 (the header code the field kernels run) against the reference's
    d3hm_qpgf_d2_v2: the same term counts at every point and G, grad G, d2G to 1e-10 of each
    point's largest component of that order."""
    q = golden("qpgf.npz")
    names = sorted({k.split("/")[0] for k in q.files})
    for n in names:
        r = np.ascontiguousarray(q[n + "/r"])
        out = np.zeros(len(r) * 20)
        ret = np.zeros(len(r), np.int32)
        devmath_host.hm_qpgf2(len(r), r.ctypes.data, np.ascontiguousarray(q[n + "/qpd"]).ctypes.data,
                              out.ctypes.data, ret.ctypes.data)
        got = (out[0::2] + 1j * out[1::2]).reshape(-1, 10)
        ref = q[n + "/v2"]
        assert np.array_equal(ret, q[n + "/ret_v2"]), n
        for lo, hi in ((0, 1), (1, 4), (4, 10)):
            scale = np.abs(ref[:, lo:hi]).max(axis=1, keepdims=True)
            assert np.max(np.abs(got[:, lo:hi] - ref[:, lo:hi]) / scale) < 1e-10, (n, lo)


def _pack(p):
    geo = np.zeros((p.Ne + 1, 48))
    geo[:, 0:12] = p.cr.reshape(-1, 12)
    geo[:, 12:21] = p.cw.reshape(-1, 9)
    geo[:, 21:33] = p.ren.reshape(-1, 12)
    geo[:, 33:45] = p.wen.reshape(-1, 12)
    geo[:, 45] = p.nv
    return np.ascontiguousarray(geo)


@pytest.mark.parametrize("case", ["sphere_m4", "cone_m1", "sphere_m2"])
def test_regular_pairs_host_build(devmath_host, case):
    """Regular (t != s) pairs of the golden rows, re-evaluated with the device element rules."""
    from bem3_emf_qd2_b200.dqd2 import problem_from_arrays
    import bem3_emf_qd2_b200 as B
    g = golden(f"rows_{case}.npz")
    p = problem_from_arrays({k[3:]: g[k] for k in g.files if k.startswith("in/")})
    geo = _pack(p)
    qpd = np.array([p.qpd["k"], *p.qpd["vk"], *p.qpd["vd1"], *p.qpd["vd2"]])
    xl, wl = _gl(12)
    xh, wh = _gl(64)
    rng = np.random.default_rng(7)
    keys = [k for k in g.files if k.endswith("/G") and k.startswith("d")]
    for key in keys:
        did = int(key.split("/")[0][1:])
        t = int(key.split("/")[1][1:])
        G, H = g[key], g[key.replace("/G", "/H")]
        ne = len(p.sid[did])
        td = int(p.sid[did][t - 1])
        for s in rng.choice(np.arange(1, ne + 1), size=12, replace=False):
            if s == t:
                continue
            sd = int(p.sid[did][s - 1])
            for tn in range(p.nv[abs(td)]):
                out = np.zeros(54)
                k = complex(p.kn[did])
                args = [geo.ctypes.data, td, tn, sd, 1 if did == 0 else 0, k.real, k.imag, qpd.ctypes.data]
                gh = devmath_host.hm_pair_regular(*args, 12, xl.ctypes.data, wl.ctypes.data, out.ctypes.data)
                if gh:
                    devmath_host.hm_pair_regular(*args, 64, xh.ctypes.data, wh.ctypes.data, out.ctypes.data)
                c = out[0::2] + 1j * out[1::2]
                ref_g = G[tn, 4 * (s - 1):4 * s]
                ref_h = H[tn, 4 * (s - 1):4 * s]
                sc = max(np.abs(ref_g).max(), np.abs(ref_h).max())
                assert np.abs(c[0:4] - ref_g).max() < 1e-12 * sc
                assert np.abs(c[4:8] - ref_h).max() < 1e-12 * sc


def _gl(n):
    """The library's Gauss-Legendre tables (the ones uploaded to the device)."""
    import bem3_emf_qd2_b200 as B
    x, w = B.gauss_legendre(n)
    return np.ascontiguousarray(x), np.ascontiguousarray(w)


# ---- host set-up mirrors the reference's readers ----------------------------------------------
def test_problem_setup_shapes():
    from bem3_emf_qd2_b200.dqd2 import problem_from_arrays
    g = golden("rows_sphere_m2.npz")
    p = problem_from_arrays({k[3:]: g[k] for k in g.files if k.startswith("in/")})
    assert p.MN == 2 and p.Ne == 1086 and p.NN == 4344
    assert [len(s) for s in p.sid] == [600, 486, 1086]
    # every element appears once in its main and once in its sub domain
    assert sum(len(s) for s in p.sid) == 2 * p.Ne


# ---- the C ABI ----------------------------------------------------------------------------------
def test_cabi_exports_every_declared_symbol():
    so = os.path.join(REPO, "bem3_emf_qd2_b200", "_lib", "libbem3qd2.so")
    if not os.path.exists(so):
        pytest.fail("CUDA library not built (run __graft_entry__.build())")
    hdrs = [os.path.join(REPO, "include", f) for f in os.listdir(os.path.join(REPO, "include")) if f.endswith(".h")]
    declared = set()
    for h in hdrs:
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        declared |= set(re.findall(r"\b(bem3_\w+|solve_bieq|EH_\w+|mEMP_\w+)\s*\(", txt))
    nm = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in nm.splitlines() if line.strip()}
    missing = sorted(declared - exported)
    assert not missing, missing


def test_entry_points_refuse_bad_arguments_before_device_work(cuda_lib_host, tmp_path):
    """Argument errors of the host-pointer and device set-up entry points come back as BEM3_ERR_ARG
    before any device call (these run on a machine without a GPU)."""
    import bem3_emf_qd2_b200 as B
    from bem3_emf_qd2_b200 import meshgen
    L = cuda_lib_host
    assert L.bem3_mesh_pack_dev(0, 10, None, None, None, None) == -1
    assert L.bem3_assemble_domains(None, 0, None, None, 0, None, None, None, None, None, None, None) == -1
    p, _ = meshgen.problem("sphere384", str(tmp_path))
    p.sid[1] = p.sid[1].copy()
    p.sid[1][5] = p.Ne + 3  # an element id past the mesh
    with pytest.raises(RuntimeError, match="invalid argument"):
        B.assemble_domains(p, derivatives=False)
    with pytest.raises(RuntimeError, match="invalid argument"):
        B.assemble_domain(p, 1, derivatives=False)


def test_cabi_library_loads():
    import bem3_emf_qd2_b200 as B
    L = B.lib()
    assert b"sm_100a" in L.bem3_version()


def test_gauss_legendre_tables_match_reference():
    """Near-singular pairs are sensitive to the last bit of the nodes: the device tables must be
    the reference's gauleg output exactly."""
    import bem3_emf_qd2_b200 as B
    g = golden("gauleg.npz")
    for n in (12, 64):
        x, w = B.gauss_legendre(n)
        assert np.array_equal(x, g[f"x{n}"]) and np.array_equal(w, g[f"w{n}"])


# ---- the C restatement oracle (oracle/qpgf_oracle.c) is pinned to the reference's vectors -------
def _port():
    import ctypes as C
    so = os.path.join(REPO, "oracle", "_build", "libqpgf_oracle.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), "port"], check=True, capture_output=True)
    L = C.CDLL(so)
    L.or_faddeeva_batch.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
    L.or_qpgf_batch.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return L


def test_restatement_oracle_pinned_to_reference_vectors():
    L = _port()
    f = golden("faddeeva.npz")
    z = f["z"]
    zz = np.ascontiguousarray(np.stack([z.real, z.imag], 1).ravel())
    o = np.zeros_like(zz)
    L.or_faddeeva_batch(len(z), zz.ctypes.data, o.ctypes.data)
    assert np.max(np.abs(o[0::2] + 1j * o[1::2] - f["w"]) / np.abs(f["w"])) < 1e-13
    q = golden("qpgf.npz")
    for n in sorted({k.split("/")[0] for k in q.files}):
        r = np.ascontiguousarray(q[n + "/r"])
        out = np.zeros(len(r) * 8)
        ret = np.zeros(len(r), np.int32)
        L.or_qpgf_batch(len(r), r.ctypes.data, np.ascontiguousarray(q[n + "/qpd"]).ctypes.data, out.ctypes.data,
                        ret.ctypes.data)
        got = (out[0::2] + 1j * out[1::2]).reshape(-1, 4)
        ref = q[n + "/v1"]
        assert np.array_equal(ret, q[n + "/ret_v1"]), n
        assert np.max(np.abs(got - ref) / np.abs(ref).max(axis=1, keepdims=True)) < 1e-12, n


@pytest.mark.parametrize("case", ["sphere_m4", "cone_m1", "sphere_m2"])
def test_self_pairs_host_build(devmath_host, case):
    """Self pairs (t == s) with the device polar / principal-value routines against the golden
    rows' self blocks (G, H) -- periodic and interior, quads and triangles."""
    from bem3_emf_qd2_b200.dqd2 import problem_from_arrays
    g = golden(f"rows_{case}.npz")
    p = problem_from_arrays({k[3:]: g[k] for k in g.files if k.startswith("in/")})
    geo = _pack(p)
    qpd = np.array([p.qpd["k"], *p.qpd["vk"], *p.qpd["vd1"], *p.qpd["vd2"]])
    xl, wl = _gl(12)
    xh, wh = _gl(64)
    for key in [k for k in g.files if k.endswith("/G") and k.startswith("d")]:
        did = int(key.split("/")[0][1:])
        t = int(key.split("/")[1][1:])
        sd = int(p.sid[did][t - 1])
        for tn in range(p.nv[abs(sd)]):
            out = np.zeros(54)
            if did == 0:
                rc = devmath_host.hm_self_periodic(geo.ctypes.data, sd, tn, qpd.ctypes.data, xl.ctypes.data,
                                                   wl.ctypes.data, xh.ctypes.data, wh.ctypes.data, out.ctypes.data)
                assert rc == 0
            else:
                k = complex(p.kn[did])
                devmath_host.hm_self_interior(geo.ctypes.data, sd, tn, k.real, k.imag, xl.ctypes.data, wl.ctypes.data,
                                              xh.ctypes.data, wh.ctypes.data, out.ctypes.data)
            c = out[0::2] + 1j * out[1::2]
            cols = slice(4 * (t - 1), 4 * t)
            ref_g = g[key][tn, cols]
            ref_h = g[key.replace("/G", "/H")][tn, cols].copy()
            ref_h[tn] -= g[key.replace("/G", "/dF")][tn, 0]  # the row sum (1+)F sits on the diagonal
            sc = max(np.abs(ref_g).max(), np.abs(ref_h).max())
            assert np.abs(c[0:4] - ref_g).max() < 1e-11 * sc, (case, did, t, tn)
            assert np.abs(c[4:8] - ref_h).max() < 1e-11 * sc, (case, did, t, tn)
            if did > 0:
                for name, dc in (("dG", c[9:13]), ("dH", c[13:17])):
                    ref = g[key.replace("/G", "/" + name)][2 * tn, cols]
                    assert np.abs(dc - ref).max() < 1e-11 * max(np.abs(ref).max(), 1e-300), (case, did, t, tn, name)


# ---- the result-file fixtures against the reference's published run log ----------------------
def test_veri_fixture_matches_reference_log():
    """verification/example1.log of the reference prints, for its veri.dat, the total field at
    (0.3, 0, 1.1) and the radiation force for types 0 and 1; the fixture (computed by the
    reference's own code from the same veri.dat) must agree to the printed 15 digits (5e-14)."""
    g = golden("bv_veri.npz")
    r = g["probe/r"]
    assert np.allclose(r[0], [0.3, 0.0, 1.1])
    log = {  # verification/example1.log, lines 29-41
        "E0": [-3.76208072827608e-02 - 2.85785594404603e-03j, 7.49983749571966e-03 + 7.41792296005539e-04j],
        "H0": -5.13555625232993e-02 - 3.84820633916324e-03j,
        "E1": [-3.76208144538066e-02 - 2.85786232985435e-03j, 7.49983744933408e-03 + 7.41786762174399e-04j],
        "H1": -5.13555629477514e-02 - 3.84820673327311e-03j,
        "F0": [2.26768049370030e-07, 1.53318582305794e-06],
        "F1": [2.28388853685501e-07, 1.54144035834764e-06],
        "N0y": -9.05416804491539e-11,
        "N1y": -9.09514287537933e-11,
    }
    for ty in (0, 1):
        E, H = g[f"probe/E{ty}"][0], g[f"probe/H{ty}"][0]
        assert abs(E[0] - log[f"E{ty}"][0]) <= 5e-14 * abs(E[0])
        assert abs(E[2] - log[f"E{ty}"][1]) <= 5e-14 * abs(E[2])
        assert abs(H[1] - log[f"H{ty}"]) <= 5e-14 * abs(H[1])
        F, N = g[f"force/F{ty}"], g[f"force/N{ty}"]
        assert abs(F[0] - log[f"F{ty}"][0]) <= 5e-14 * abs(F[0])
        assert abs(F[2] - log[f"F{ty}"][1]) <= 5e-14 * abs(F[2])
        # the torque is a small difference of large moments: 12 of its printed digits agree
        assert abs(N[1] - log[f"N{ty}y"]) <= 1e-11 * abs(N[1])


def test_ex2_fixture_matches_reference_log():
    """analysis_sample2/example1.log of the reference (cone_m1 triangles, rotated by pi about x
    on the solver's command line): total field at (0.3, 0, 1.1) and the radiation force."""
    g = golden("bv_ex2.npz")
    assert np.allclose(g["probe/r"][0], [0.3, 0.0, 1.1])
    log = {  # analysis_sample2/example1.log, lines 34-56
        "E0": [-5.84203979042922e-02 - 1.71331280017757e-02j, -1.59605270636755e-02 - 5.97684924605190e-03j],
        "H0": -7.70668013359473e-02 - 1.95100100680507e-02j,
        "E1": [-5.84233473949296e-02 - 1.71333199922096e-02j, -1.59568962146879e-02 - 5.95361410446437e-03j],
        "H1": -7.70672750262359e-02 - 1.95107411607629e-02j,
        "F0": [-2.26647784396326e-04, -1.51648727283879e-05],
        "F1": [-2.05481609738202e-04, -3.33790381045709e-05],
    }
    for ty in (0, 1):
        E, H = g[f"probe/E{ty}"][0], g[f"probe/H{ty}"][0]
        assert abs(E[0] - log[f"E{ty}"][0]) <= 5e-14 * abs(E[0])
        assert abs(E[2] - log[f"E{ty}"][1]) <= 5e-14 * abs(E[2])
        assert abs(H[1] - log[f"H{ty}"]) <= 5e-14 * abs(H[1])
        # the force sums singular boundary integrals whose last digits depend on the compiler that
        # produced the log (the reference's own build here agrees with it to 10 digits)
        F = g[f"force/F{ty}"]
        assert abs(F[0] - log[f"F{ty}"][0]) <= 1e-10 * abs(F[0])
        assert abs(F[2] - log[f"F{ty}"][1]) <= 1e-10 * abs(F[2])


@pytest.mark.parametrize("case", ["sphere_m4", "cone_m1", "sphere_m2", "ex2"])
def test_element_setup_equals_reference(case):
    """The host set-up's element constants and collocation nodes (dqd2.Problem) are the
    reference's init_elem_const / init_boundary_data output bit for bit, quads, triangles and a
    rotated mesh alike; the device set-up (bem3_mesh_pack_dev) is checked against the host set-up
    in tests/test_gpu_mesh.py."""
    from bem3_emf_qd2_b200.dqd2 import problem_from_arrays
    g = golden("elem_const.npz")
    src = golden("bv_ex2.npz" if case == "ex2" else f"rows_{case}.npz")
    p = problem_from_arrays({k[3:]: src[k] for k in src.files if k.startswith("in/")})
    assert np.array_equal(p.cr[1:], g[f"{case}/cr"][1:])
    assert np.array_equal(p.cw[1:], g[f"{case}/cw"][1:])
    nodes = [np.arange(p.nv[i]) for i in range(1, p.Ne + 1)]
    for k, mine in (("ren", p.ren), ("wen", p.wen)):
        ref = g[f"{case}/{k}"]
        for i, js in enumerate(nodes, start=1):
            if case == "ex2" and k == "ren":
                # dat_read takes the collocation nodes from the result file (d3qd2_setup.c:419), as
                # the build that wrote it computed them: they differ here in the last bit at most
                assert np.all(np.abs(mine[i, js] - ref[i, js]) <= 2.3e-16 * np.maximum(np.abs(ref[i, js]), 0.125)), i
            else:
                assert np.array_equal(mine[i, js], ref[i, js]), (case, k, i)


def test_rotation_reproduces_result_file_nodes():
    """Problem's rotation/translation (rotation_translation_obj) gives the node coordinates the
    reference stored in its result file, bit for bit."""
    from bem3_emf_qd2_b200.dqd2 import problem_from_arrays
    g = golden("bv_ex2.npz")
    p = problem_from_arrays({k[3:]: g[k] for k in g.files if k.startswith("in/")})
    assert np.array_equal(p.rn[1:], g["dat/rn"][1:])
