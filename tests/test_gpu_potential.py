"""Modified electromagnetic potentials (bem3_ctx_potential: mEMP_s / mEMP_t / mEMP_i) and the
incident field alone (bem3_ctx_field with total 2: EH_i) against the reference.

tests/golden/potentials.npz holds the reference's own values (d3qd2_field.c:10-87, 287-300) for
its shipped result files veri.dat (sphere_m4 quads, hexagonal lattice) and ex2.dat (cone_m1
triangles) at probe points inside and outside the particle and just off its boundary, types 0-3.
With the reference's boundary values loaded:

  |U - U_ref| <= 1e-10 * max |U_ref|   per (type, mode) over the points, and the same domains;
  |E_i - E_i,ref| <= 1e-13 * max |E_i,ref| (a closed form).
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

CASES = ["veri", "ex2"]
TOL = 1e-10


def _ctx(B, name):
    from bem3_emf_qd2_b200.dqd2 import problem_from_arrays
    g = golden(f"bv_{name}.npz")
    p = problem_from_arrays({k[3:]: g[k] for k in g.files if k.startswith("in/")})
    ctx = B.Context(p)
    ctx.set_boundary_values([{k: g[f"bv{d}/{k}"] for k in ("U", "dU", "E", "dE", "H", "dH")}
                             for d in range(p.MN + 1)])
    return ctx


@pytest.mark.parametrize("name", CASES)
def test_potentials_match_reference(cuda_lib, name):
    g = golden("potentials.npz")
    ctx = _ctx(cuda_lib, name)
    r = g[f"{name}/r"]
    for ty in (0, 1, 2, 3):
        for mode in (0, 1, 2):
            U, did = ctx.potential(r, ty, mode)
            assert np.array_equal(did, g[f"{name}/did"]), (ty, mode)
            ref = g[f"{name}/U{ty}_{mode}"]
            scale = np.abs(ref).max()
            err = np.abs(U - ref).max()
            assert err <= TOL * scale, (name, ty, mode, err, scale)
    ctx.close()


@pytest.mark.parametrize("name", CASES)
def test_incident_field_alone(cuda_lib, name):
    g = golden("potentials.npz")
    ctx = _ctx(cuda_lib, name)
    r = g[f"{name}/r"]
    E, H, did = ctx.field(r, 0, 2)
    for got, key in ((E, "Ei"), (H, "Hi")):
        ref = g[f"{name}/{key}"]
        assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max(), key
    # the vector potential of the incident wave is its electric field
    U, _ = ctx.potential(r, 0, 2)
    assert np.array_equal(U[:, :3], E) and not U[:, 3].any()
    ctx.close()


@pytest.mark.parametrize("name", CASES)
def test_fields_from_potential_derivatives_match_reference(cuda_lib, name):
    """bem3_ctx_field_memp (EH_mEMP_s / _t / _i) against the reference, types 0-2: the same domain
    of every point (negative where the point is too close to the boundary for these rules) and
    |E - E_ref|, |H - H_ref| <= 1e-10 of the largest reference value."""
    g = golden("potentials.npz")
    ctx = _ctx(cuda_lib, name)
    r = g[f"{name}/r"]
    for ty in (0, 1, 2):
        for mode in (0, 1, 2):
            E, H, did = ctx.field_memp(r, ty, mode)
            assert np.array_equal(did, g[f"{name}/mdid{ty}_{mode}"]), (ty, mode, did)
            for got, key in ((E, "mE"), (H, "mH")):
                ref = g[f"{name}/{key}{ty}_{mode}"]
                scale = np.abs(ref).max()
                err = np.abs(got - ref).max()
                assert err <= TOL * scale, (name, key, ty, mode, err, scale)
    ctx.close()
