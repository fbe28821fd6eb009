"""GPU radiation force and torque (bem3_ctx_force) against the reference's force_FN for its shipped
result files (veri.dat: quads; ex2.dat: rotated triangles), types 0 and 1.

  with the reference's boundary values:  |F - F_ref| <= 1e-9 * max|F_ref|, same for N
  end to end (our solve, then force):    1e-8 (the parity tolerance for fields and forces)
Components far below the largest (e.g. Fy ~ 1e-20 against Fx ~ 1e-7 on the symmetric cases) are
compared in that absolute sense.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _case(name):
    from bem3_emf_qd2_b200.dqd2 import problem_from_arrays
    g = golden(f"bv_{name}.npz")
    return g, problem_from_arrays({k[3:]: g[k] for k in g.files if k.startswith("in/")})


def _ref_bv(g, p):
    return [{k: g[f"bv{d}/{k}"] for k in ("U", "dU", "E", "dE", "H", "dH")} for d in range(p.MN + 1)]


def _check(g, ctx, tol):
    for ty in (0, 1):
        F, N = ctx.force((0.0, 0.0, 0.0), ty)
        Fr, Nr = g[f"force/F{ty}"], g[f"force/N{ty}"]
        assert np.abs(F - Fr).max() <= tol * np.abs(Fr).max(), (ty, F, Fr)
        assert np.abs(N - Nr).max() <= tol * np.abs(Nr).max(), (ty, N, Nr)


@pytest.mark.parametrize("name", ["veri", "ex2"])
def test_force_from_reference_boundary_values(cuda_lib, name):
    g, p = _case(name)
    ctx = cuda_lib.Context(p)
    ctx.set_boundary_values(_ref_bv(g, p))
    _check(g, ctx, 1e-9)
    ctx.close()


@pytest.mark.parametrize("name", ["veri", "ex2"])
def test_force_end_to_end(cuda_lib, name):
    g, p = _case(name)
    ctx = cuda_lib.Context(p)
    ctx.solve()
    _check(g, ctx, 1e-8)
    ctx.close()
