"""Resident factorisations: a new polarisation on a solved context (bem3_ctx_set_incident +
bem3_ctx_resolve, right-hand sides only) must give what a fresh solve of the new problem gives.

  |resolved - fresh| <= 1e-10 * max|fresh| per array and domain
(both use the same matrices and factorisations; the fresh solve repeats them)."""
import dataclasses

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _case(name):
    from bem3_emf_qd2_b200.dqd2 import problem_from_arrays
    g = golden(f"bv_{name}.npz")
    return problem_from_arrays({k[3:]: g[k] for k in g.files if k.startswith("in/")})


def _other_polarisation(p):
    out = []
    for w in p.waves:
        out.append(dataclasses.replace(w, e0x=complex(0.3), e0y=complex(0.0, 0.9)))
    return out


def _close(a, b, tol):
    for d in range(len(b)):
        for k in ("U", "dU", "E", "H", "dE", "dH"):
            scale = np.abs(b[d][k]).max()
            assert np.abs(a[d][k] - b[d][k]).max() <= tol * scale, (d, k)


@pytest.mark.parametrize("name,method", [("veri", 2), ("ex2", 1)])
def test_resolve_matches_fresh_solve(cuda_lib, name, method):
    p = _case(name)
    ctx = cuda_lib.Context(p)
    ctx.solve(method)
    first = ctx.boundary_values()
    assert ctx.device_bytes() > 0
    waves = _other_polarisation(p)
    ctx.set_incident(waves)
    ctx.resolve()
    resolved = ctx.boundary_values()
    fresh_ctx = cuda_lib.Context(p.with_waves(waves))
    fresh_ctx.solve(method)
    _close(resolved, fresh_ctx.boundary_values(), 1e-10)
    fresh_ctx.close()
    # and back to the first polarisation
    ctx.set_incident(p.waves)
    ctx.resolve()
    _close(ctx.boundary_values(), first, 1e-12)
    ctx.release()
    assert ctx.device_bytes() == 0
    ctx.close()
