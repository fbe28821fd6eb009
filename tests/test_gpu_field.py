"""GPU field evaluation (bem3_ctx_field) against the reference's EH_t at probe points.

The fixtures hold, for the reference's shipped result files (veri.dat: sphere_m4 quads on a
hexagonal lattice; ex2.dat: cone_m1 triangles), the boundary values the reference's solver wrote
and the reference's own EH_t at probe points inside and outside the particle, types 0 and 1.

  with the reference's boundary values:  |E - E_ref| <= 1e-10 * max|E_ref| over the points
  end to end (our solve, then fields):   |E - E_ref| <= 1e-8  * max|E_ref|
and the same for H; the domain of every point must match.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

CASES = ["veri", "ex2"]


def _case(name):
    from bem3_emf_qd2_b200.dqd2 import problem_from_arrays
    g = golden(f"bv_{name}.npz")
    return g, problem_from_arrays({k[3:]: g[k] for k in g.files if k.startswith("in/")})


def _ref_bv(g, p):
    return [{k: g[f"bv{d}/{k}"] for k in ("U", "dU", "E", "dE", "H", "dH")} for d in range(p.MN + 1)]


def _check(g, E, H, did, ty, tol):
    assert np.array_equal(did, g["probe/did"])
    for got, key in ((E, f"probe/E{ty}"), (H, f"probe/H{ty}")):
        ref = g[key]
        scale = np.abs(ref).max()
        err = np.abs(got - ref).max()
        assert err <= tol * scale, (key, err, scale)


@pytest.mark.parametrize("name", CASES)
def test_fields_from_reference_boundary_values(cuda_lib, name):
    g, p = _case(name)
    ctx = cuda_lib.Context(p)
    ctx.set_boundary_values(_ref_bv(g, p))
    r = g["probe/r"]
    assert np.array_equal(ctx.domain_id(r), g["probe/did"])
    for ty in (0, 1):
        E, H, did = ctx.field(r, ty, total=True)
        _check(g, E, H, did, ty, 1e-10)
    ctx.close()


@pytest.mark.parametrize("name", CASES)
def test_fields_end_to_end(cuda_lib, name):
    g, p = _case(name)
    ctx = cuda_lib.Context(p)
    ctx.solve()
    r = g["probe/r"]
    for ty in (0, 1):
        E, H, did = ctx.field(r, ty, total=True)
        _check(g, E, H, did, ty, 1e-8)
    ctx.close()


def test_scattered_plus_incident_is_total(cuda_lib):
    g, p = _case("veri")
    ctx = cuda_lib.Context(p)
    ctx.set_boundary_values(_ref_bv(g, p))
    r = g["probe/r"]
    Et, Ht, did = ctx.field(r, 0, total=True)
    Es, Hs, _ = ctx.field(r, 0, total=False)
    out = did == 0
    assert out.any() and (~out).any()
    # inside the particle the two agree; outside they differ by the incident wave
    assert np.array_equal(Et[~out], Es[~out])
    e_inc = np.zeros((out.sum(), 3), np.complex128)
    for w in p.waves:
        e_inc += w.eh_dehdv(r[out], np.zeros_like(r[out]))[0]
    assert np.abs(Et[out] - Es[out] - e_inc).max() <= 1e-13 * np.abs(e_inc).max()
    ctx.close()


@pytest.mark.parametrize("name", CASES)
def test_near_boundary_fields_all_rules(cuda_lib, name):
    """Points at 0.1 and 0.3 element sizes off the boundary, rules of types 0-3, against the
    reference's EH_t with the same boundary values: |E - E_ref| <= 1e-9 * max|E_ref|."""
    g, p = _case(name)
    near = golden("near_fields.npz")
    r = near[f"{name}/r"]
    ctx = cuda_lib.Context(p)
    ctx.set_boundary_values(_ref_bv(g, p))
    for ty in (0, 1, 2, 3):
        E, H, did = ctx.field(r, ty, total=True)
        assert np.array_equal(did, near[f"{name}/did"])
        for got, key in ((E, f"{name}/E{ty}"), (H, f"{name}/H{ty}")):
            ref = near[key]
            assert np.abs(got - ref).max() <= 1e-9 * np.abs(ref).max(), (ty, key)
    ctx.close()
