"""Incident, reflected and transmitted power through one unit cell (Context.power) against the
same quadrature applied to the reference's EH_t / EH_s (tests/golden/power.npz).

  with the reference's boundary values: each power within 1e-9 relative
  end to end (our solve):                each power within 1e-8 relative
veri.dat's sphere is lossless: its balance (P_ref + P_tra) / P_inc is 1 up to the boundary-element
discretisation (1 + 2.5e-5 for the reference itself); our balance must equal the reference's to
1e-8.  ex2.dat's cone absorbs (balance 0.985)."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _case(name):
    from bem3_emf_qd2_b200.dqd2 import problem_from_arrays
    g = golden(f"bv_{name}.npz")
    return g, problem_from_arrays({k[3:]: g[k] for k in g.files if k.startswith("in/")})


def _check(ctx, name, tol):
    pw = golden("power.npz")
    zt, zb, n = pw[name + "/spec"]
    got = ctx.power(float(zt), float(zb), int(n))
    for k in ("P_inc", "P_ref", "P_tra", "balance"):
        ref = float(pw[f"{name}/{k}"])
        assert abs(got[k] - ref) <= tol * abs(ref), (name, k, got[k], ref)
    return got


@pytest.mark.parametrize("name", ["veri", "ex2"])
def test_power_from_reference_boundary_values(cuda_lib, name):
    g, p = _case(name)
    ctx = cuda_lib.Context(p)
    ctx.set_boundary_values([{k: g[f"bv{d}/{k}"] for k in ("U", "dU", "E", "dE", "H", "dH")}
                             for d in range(p.MN + 1)])
    got = _check(ctx, name, 1e-9)
    if name == "veri":
        assert abs(got["balance"] - 1.0) < 1e-4
    ctx.close()


@pytest.mark.parametrize("name", ["veri", "ex2"])
def test_power_end_to_end(cuda_lib, name):
    g, p = _case(name)
    ctx = cuda_lib.Context(p)
    ctx.solve()
    _check(ctx, name, 1e-8)
    ctx.close()
