"""CPU checks of the field-evaluation element rules (field.cuh compiled for the host) against the
reference's own coef_rt / q0_coef_rt (compiled from its sources by oracle/Makefile), on seeded
synthetic meshes written in the reference's input formats and read by both sides.

Tolerance: |ours - ref| <= 1e-12 * max_n |ref CC[n]| per element (same rules, same Green's
function term counts; only the order of a few products differs).
"""
import os

import numpy as np
import pytest

from conftest import REPO, golden

HAVE_REF = os.path.exists(os.path.join(REPO, "oracle", "_ref", "libbem3ref.so"))


def _setup(name, tmp_path):
    from reforacle import RefOracle
    from bem3_emf_qd2_b200 import meshgen
    from bem3_emf_qd2_b200.dqd2 import Problem
    files = meshgen.make_config(name, str(tmp_path))
    o = RefOracle()
    # the reference keeps input file names in fixed 64-byte buffers: load by short relative names
    cwd = os.getcwd()
    os.chdir(str(tmp_path))
    try:
        o.load(*[os.path.basename(f) for f in files])
    finally:
        os.chdir(cwd)
    p = Problem.from_files(*files)
    return o, p


def _packed(p):
    # bem3_pack_geometry is host code: the library loads and packs without a GPU
    from bem3_emf_qd2_b200 import MeshArrays
    return np.ascontiguousarray(MeshArrays(p).packed())


@pytest.mark.skipif(not HAVE_REF, reason="reference oracle not built in this checkout")
@pytest.mark.parametrize("name", ["sphere96", "cone210"])
def test_field_coefficients_match_reference(devmath_host, tmp_path, name):
    o, p = _setup(name, tmp_path)
    geo = _packed(p)
    q = p.qpd
    qp = np.array([q["k"], *q["vk"], *q["vd1"], *q["vd2"]], np.float64)
    pts = np.array([[0.05, -0.02, 0.6], [0.3, 0.2, -0.45], [0.01, 0.03, 0.02], [-0.1, 0.12, -0.05]])
    gl = golden("gauleg.npz")
    tabs = np.ascontiguousarray(np.concatenate([gl["x12"], gl["w12"], gl["x64"], gl["w64"]]))
    for r in pts:
        for did in range(p.MN + 1):
            periodic = 1 if (did == 0 and p.ps == 1) else 0
            k = complex(p.kn[did])
            for sd in p.sid[did][::3]:
                # the 64 x 64 rule on a few elements only (4096 Green's functions each on the host)
                for ty in ((0, 1, 2, 3) if sd == p.sid[did][0] else (0, 1, 2)):
                    ref = o.coef_rt(did, r, int(sd), ty)
                    out = np.zeros(17)
                    st = devmath_host.hm_field_coef(geo.ctypes.data, int(sd), r.ctypes.data, periodic, k.real,
                                                    k.imag, ty, qp.ctypes.data, tabs.ctypes.data, out.ctypes.data)
                    assert st >= 0
                    got = out[0:16:2] + 1j * out[1:16:2]
                    scale = np.abs(ref[:8]).max()
                    assert np.abs(got - ref[:8]).max() <= 1e-12 * scale, (name, did, sd, ty)
                    assert abs(out[16] - ref[8].real) <= 1e-12 * max(abs(ref[8].real), 1e-3), (name, did, sd, ty)


@pytest.mark.skipif(not HAVE_REF, reason="reference oracle not built in this checkout")
@pytest.mark.parametrize("name", ["sphere96", "cone210"])
def test_coefficient_gradients_match_reference(devmath_host, tmp_path, name):
    """field_grad_coef (the rules of the far-field path) against the reference's q0_dcoef_rt_grad
    / dcoef_rt_grad, element by element: CC, dC/drt, F and dF/drt to 1e-11 of each part's
    largest entry (the QPGF's second derivatives agree with d3hm_qpgf_d2_v2 term for term)."""
    o, p = _setup(name, tmp_path)
    geo = _packed(p)
    q = p.qpd
    qp = np.array([q["k"], *q["vk"], *q["vd1"], *q["vd2"]], np.float64)
    pts = np.array([[0.05, -0.02, 0.6], [0.3, 0.2, -0.45], [0.01, 0.03, 0.02]])
    gl = golden("gauleg.npz")
    tabs = np.ascontiguousarray(np.concatenate([gl["x12"], gl["w12"], gl["x64"], gl["w64"]]))
    for r in pts:
        for did in range(p.MN + 1):
            periodic = 1 if (did == 0 and p.ps == 1) else 0
            k = complex(p.kn[did])
            for sd in p.sid[did][::5]:
                for ty in ((0, 1, 2, 3) if sd == p.sid[did][0] else (0, 1, 2)):
                    cc, dc = o.dcoef_rt_grad(did, r, int(sd), ty)
                    out = np.zeros(68)
                    st = devmath_host.hm_field_grad_coef(geo.ctypes.data, int(sd), r.ctypes.data, periodic, k.real,
                                                         k.imag, ty, qp.ctypes.data, tabs.ctypes.data,
                                                         out.ctypes.data)
                    assert st >= 0
                    got_cc = out[0:16:2] + 1j * out[1:16:2]
                    got_dc = (out[16:64:2] + 1j * out[17:64:2]).reshape(3, 8)
                    what = (name, did, int(sd), ty)
                    assert np.abs(got_cc - cc[:8]).max() <= 1e-11 * np.abs(cc[:8]).max(), what
                    assert np.abs(got_dc - dc[:, :8]).max() <= 1e-11 * np.abs(dc[:, :8]).max(), what
                    assert abs(out[64] - cc[8].real) <= 1e-11 * max(abs(cc[8].real), 1e-3), what
                    sf = max(np.abs(dc[:, 8].real).max(), 1e-3)
                    assert np.abs(out[65:68] - dc[:, 8].real).max() <= 1e-11 * sf, what


@pytest.mark.parametrize("name", ["sphere96", "cone210"])
def test_solid_angles_sum_to_the_enclosed_domain(devmath_host, tmp_path, name):
    """Over a closed surface the element solid angles add to 4 pi inside and 0 outside."""
    from bem3_emf_qd2_b200 import meshgen
    from bem3_emf_qd2_b200.dqd2 import Problem
    p = Problem.from_files(*meshgen.make_config(name, str(tmp_path)))
    rn = np.ascontiguousarray(p.rn)
    ed = np.ascontiguousarray(p.ed, dtype=np.int32)
    for r, want in (((0.01, 0.02, -0.03), 4 * np.pi), ((0.2, -0.1, 0.9), 0.0)):
        r = np.array(r)
        tot = 0.0
        flag = np.zeros(1, np.int32)
        for e in range(1, p.Ne + 1):
            om = devmath_host.hm_solid_angle(rn.ctypes.data, ed.ctypes.data, e, int(p.nv[e]), r.ctypes.data,
                                             flag.ctypes.data)
            assert flag[0] == 0
            # elements are listed with the open region as main domain: their normals point outward
            tot += om if p.md[e] == 0 else -om
        assert abs(abs(tot) - want) < 1e-9, (name, tot)
