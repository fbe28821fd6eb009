"""Plain configuration 1 (sphere384: cube-sphere r = 0.3 um of 6 x 8 x 8 quads, n = 1.59, square
lattice 1.0 um in n = 1.33, lambda0 = 0.6328 um, theta = 1e-4 rad standing in for normal incidence)
end to end against the reference's own programs on the same mesh (tests/golden/c1_sphere384.npz:
d3qd2_bv_solver's result file, its EH_t on the 21 x 21 probe grid of the y = 0 plane, force_FN,
plane powers, complete rows of create_cmatrix_domain).

  coefficient matrices (complete rows of 16 elements per domain, G, H, dF; dG, dH on 8 interior
  elements): |ours - ref| <= 1e-10 x the row's largest |entry| of the same matrix
  boundary values of our solve:                1e-8 x max |ref| per array and domain
  fields on the grid, types 0 and 1:            1e-8 x max |ref| over the grid, with the reference's
                                                boundary values and end to end
  force and torque, types 0 and 1:              1e-8 x the vector's largest component
  power balance of the lossless sphere:         ours equals the reference's to 1e-8 (both carry the
                                                same discretisation error, 1 - balance ~ 1e-3)
The four grid points that coincide with mesh nodes ((+-0.3, 0, 0), (0, 0, +-0.3)) lie on the boundary
itself, where the boundary-integral representation of the field is singular; they are left out.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

BV = ("U", "dU", "E", "dE", "H", "dH")


def _fixture():
    from bem3_emf_qd2_b200.dqd2 import problem_from_arrays
    g = golden("c1_sphere384.npz")
    return g, problem_from_arrays({k[3:]: g[k] for k in g.files if k.startswith("in/")})


def _grid_mask(g):
    r = g["grid/r"]
    on_node = np.isclose(np.abs(r).sum(axis=1), 0.3, atol=1e-12) & (np.sum(np.abs(r) > 0, axis=1) == 1)
    return ~on_node


def test_c1_rows_match_reference(cuda_lib):
    g, p = _fixture()
    rows = sorted({int(k.split("/")[2][1:]) for k in g.files if k.startswith("rows/d0/")})
    for did in range(p.MN + 1):
        M = cuda_lib.assemble_domain(p, did)
        for t in rows:
            key = f"rows/d{did}/t{t}"
            sl = slice(4 * (t - 1), 4 * t)
            for name in ("G", "H"):
                ref, got = g[f"{key}/{name}"], M[name][sl]
                sc = np.abs(ref).max(axis=1, keepdims=True)
                assert (np.abs(got - ref) <= 1e-10 * sc).all(), (did, t, name, (np.abs(got - ref) / sc).max())
            ref, got = g[f"{key}/dF"], M["dF"][sl]
            assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max(), (did, t, "dF")
            if f"{key}/dG" in g.files:
                for name in ("dG", "dH"):
                    ref, got = g[f"{key}/{name}"], M[name][2 * (t - 1) * 4:2 * t * 4]
                    sc = np.abs(ref).max(axis=1, keepdims=True)
                    assert (np.abs(got - ref) <= 1e-10 * sc).all(), (did, t, name)


def _check_fields(g, ctx, tol):
    m = _grid_mask(g)
    r = g["grid/r"][m]
    for ty in (0, 1):
        E, H, did = ctx.field(r, ty, True)
        assert np.array_equal(did, g["grid/did"][m])
        for name, got in (("E", E), ("H", H)):
            ref = g[f"grid/{name}{ty}"][m]
            assert np.abs(got - ref).max() <= tol * np.abs(ref).max(), (ty, name, np.abs(got - ref).max())


def _check_force(g, ctx, tol):
    for ty in (0, 1):
        F, N = ctx.force((0.0, 0.0, 0.0), ty)
        for got, ref in ((F, g[f"force/F{ty}"]), (N, g[f"force/N{ty}"])):
            assert np.abs(got - ref).max() <= tol * np.abs(ref).max(), (ty, got, ref)


def test_c1_fields_and_force_from_reference_boundary_values(cuda_lib):
    g, p = _fixture()
    ctx = cuda_lib.Context(p)
    ctx.set_boundary_values([{k: g[f"bv{d}/{k}"] for k in BV} for d in range(p.MN + 1)])
    _check_fields(g, ctx, 1e-9)
    _check_force(g, ctx, 1e-9)
    ctx.close()


def test_c1_end_to_end(cuda_lib):
    g, p = _fixture()
    ctx = cuda_lib.Context(p)
    ctx.solve()
    bv = ctx.boundary_values()
    for d in range(p.MN + 1):
        for k in BV:
            ref = g[f"bv{d}/{k}"]
            assert np.abs(bv[d][k] - ref).max() <= 1e-8 * np.abs(ref).max(), (d, k)
    _check_fields(g, ctx, 1e-8)
    _check_force(g, ctx, 1e-8)
    got = ctx.power(0.6, -0.6, 16)
    for k in ("P_inc", "P_ref", "P_tra", "balance"):
        ref = float(g[f"power/{k}"])
        assert abs(got[k] - ref) <= 1e-8 * abs(ref), (k, got[k], ref)
    ctx.close()
