"""The reference's example1.c and example2.c relinked on the GPU drop-ins of d3qd2_field.o and
d3qd2_force.o (bem3_emf_qd2_b200/dropin/d3qd2_field_b200.c), run unchanged on the verification
result of the reference (its veri.dat: the boundary values it ships, bv_veri.npz, written to a result
file by the reference's own set-up and dat_write through the oracle).

example1: total field at (0.3, 0, 1.1) with types 0 and 1, force and torque with types 0 and 1, as
printed, against the reference's EH_t / force_FN on the same result (1e-8 of each vector's largest
component; the printed 15 significant digits are far below that).
example2: the field intensities it writes on its first plane, rows 0 and 100 of 200, against the
reference's EH_t (type 1) at the same points (1e-8 relative), while its OpenMP threads call EH_t
concurrently through the drop-in's shared queue.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import REPO, golden

pytestmark = pytest.mark.gpu

BUILD = os.path.join(REPO, "bem3_emf_qd2_b200", "dropin", "_build")
ORACLE = os.path.join(REPO, "oracle", "_ref", "libbem3ref.so")
NUM = r"[-+]?\d\.\d+e[-+]\d+"


def _veri_dat(tmp):
    """veri.dat rebuilt from the shipped boundary values by the reference's set-up and dat_write."""
    from reforacle import RefOracle
    from bem3_emf_qd2_b200.dqd2 import write_input_files
    g = golden("bv_veri.npz")
    files = write_input_files({k[3:]: g[k] for k in g.files if k.startswith("in/")}, tmp, "sphere_m4.msh")
    o = RefOracle()
    cwd = os.getcwd()
    os.chdir(tmp)  # the reference keeps file names in 64-byte buffers
    try:
        o.load(*[os.path.basename(f) for f in files])
        for d in range(o.info()["MN"] + 1):
            o.set_boundary_values(d, {k: g[f"bv{d}/{k}"] for k in ("U", "dU", "E", "H", "dE", "dH")})
        o.write_dat("veri.dat")
    finally:
        os.chdir(cwd)
    return g


def _close(a, b, tol=1e-8):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() <= tol * np.abs(b).max()


@pytest.mark.skipif(not (os.path.exists(os.path.join(BUILD, "example1.out")) and os.path.exists(ORACLE)),
                    reason="relinked reference programs or oracle not built in this checkout")
def test_relinked_example1_prints_reference_fields_and_force(cuda_lib, tmp_path):
    tmp = str(tmp_path)
    g = _veri_dat(tmp)
    r = subprocess.run([os.path.join(BUILD, "example1.out"), "veri.dat"], cwd=tmp, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    comp = [complex(float(a), float(b)) for a, b in re.findall(rf"[EH][xyz] = \s*({NUM})\s*({NUM}) I", r.stdout)]
    assert len(comp) == 12, r.stdout[-3000:]
    vec = [[float(x) for x in m] for m in re.findall(rf"[FN] = \(\s*({NUM}),\s*({NUM}),\s*({NUM})\)", r.stdout)]
    assert len(vec) == 4, r.stdout[-3000:]
    assert _close(comp[0:3], g["probe/E0"][0]) and _close(comp[3:6], g["probe/H0"][0])
    assert _close(comp[6:9], g["probe/E1"][0]) and _close(comp[9:12], g["probe/H1"][0])
    assert _close(vec[0], g["force/F0"]) and _close(vec[1], g["force/N0"])
    assert _close(vec[2], g["force/F1"]) and _close(vec[3], g["force/N1"])


def _blocks(path):
    """example2.c's output: one block of 200 lines (a, b, value) per row, blank-line separated."""
    rows, cur = [], []
    with open(path) as f:
        next(f)
        for line in f:
            if not line.strip():
                rows.append(np.array(cur))
                cur = []
            else:
                cur.append([float(x) for x in line.split()])
    return rows


@pytest.mark.skipif(not (os.path.exists(os.path.join(BUILD, "example2.out")) and os.path.exists(ORACLE)),
                    reason="relinked reference programs or oracle not built in this checkout")
def test_relinked_example2_plane_matches_reference(cuda_lib, tmp_path):
    tmp = str(tmp_path)
    _veri_dat(tmp)
    x = golden("example2_rows.npz")
    env = dict(os.environ, OMP_NUM_THREADS=str(min(16, os.cpu_count() or 1)))
    r = subprocess.run([os.path.join(BUILD, "example2.out"), "veri.dat"], cwd=tmp, capture_output=True, text=True,
                       timeout=1200, env=env)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "Intensity plot is finished" in r.stdout
    ie, ih = _blocks(os.path.join(tmp, "Ie_yz.txt")), _blocks(os.path.join(tmp, "Ih_yz.txt"))
    assert len(ie) == 200 and len(ih) == 200 and all(len(b) == 200 for b in ie)
    for name in ("Ie_xz.txt", "Ih_xz.txt", "Ie_xy.txt", "Ih_xy.txt"):
        assert len(_blocks(os.path.join(tmp, name))) == 200
    for i in x["rows"]:
        pts = x[f"r{i}"]
        assert np.allclose(ie[i][:, 0], pts[:, 1], atol=1e-5) and np.allclose(ie[i][:, 1], pts[:, 2], atol=1e-5)
        assert _close(ie[i][:, 2], x[f"ie{i}"]), i
        assert _close(ih[i][:, 2], x[f"ih{i}"]), i
