"""The reference's own solver program, relinked on libbem3qd2 (bem3_emf_qd2_b200/dropin), run on the
reference's verification inputs: its result file must hold the boundary values the reference wrote
in its own result file for the same inputs (veri.dat), to 1e-8 * max|ref| per array and domain.

The relinked program is built where the reference sources are present (build() in
__graft_entry__); the result file is read back with the reference's dat_read through the oracle.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO, golden

pytestmark = pytest.mark.gpu

SOLVER = os.path.join(REPO, "bem3_emf_qd2_b200", "dropin", "_build", "d3qd2_bv_solver")
ORACLE = os.path.join(REPO, "oracle", "_ref", "libbem3ref.so")


@pytest.mark.skipif(not (os.path.exists(SOLVER) and os.path.exists(ORACLE)),
                    reason="relinked reference program or oracle not built in this checkout")
def test_relinked_bv_solver_reproduces_reference_result(cuda_lib, tmp_path):
    from reforacle import RefOracle
    from bem3_emf_qd2_b200.dqd2 import write_input_files
    g = golden("bv_veri.npz")
    files = write_input_files({k[3:]: g[k] for k in g.files if k.startswith("in/")}, str(tmp_path), "sphere_m4.msh")
    out = os.path.join(str(tmp_path), "gpu.dat")
    r = subprocess.run([SOLVER, *[os.path.basename(f) for f in files], out], cwd=str(tmp_path),
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "finished" in r.stdout
    assert not [f for f in os.listdir(str(tmp_path)) if f.startswith("tmp")], "no temporary matrix files"
    o = RefOracle()
    o.load_dat(out)
    for d in range(o.info()["MN"] + 1):
        bv = o.boundary_values(d)
        for k in ("U", "dU", "E", "H", "dE", "dH"):
            ref = g[f"bv{d}/{k}"]
            err = np.abs(bv[k] - ref).max()
            assert err <= 1e-8 * np.abs(ref).max(), (d, k, err)
