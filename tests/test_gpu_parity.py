"""GPU parity: the CUDA path (through the C ABI) against the reference's golden outputs.

Tolerances (FP64 throughout):
  Green's function        |got - ref| <= 1e-10 * max_j |ref_j|   per point
  coefficient matrices    |got - ref| <= 1e-10 * max |ref row block|  (matrix entries, 1e-10 rel)
  dF row sums             |got - ref| <= 1e-10 * (1 + |ref|)
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def test_qpgf_gpu_matches_reference(cuda_lib):
    B = cuda_lib
    q = golden("qpgf.npz")
    names = sorted({k.split("/")[0] for k in q.files})
    for n in names:
        p = q[n + "/qpd"]
        qpd = dict(k=p[0], vk=p[1:4], vd1=p[4:6], vd2=p[6:8])
        out, ret = B.qpgf(qpd, q[n + "/r"], mode=0)
        assert np.all(ret > 0), n
        assert np.array_equal(ret, q[n + "/ret_v1"]), n  # same stop rules, same term counts
        ref = q[n + "/v1"]
        assert np.max(np.abs(out - ref) / np.abs(ref).max(axis=1, keepdims=True)) < 1e-10, n
        out2, ret2 = B.qpgf(qpd, q[n + "/r"], mode=1)
        ref2 = np.c_[q[n + "/qG"], q[n + "/dqG"]]
        assert np.max(np.abs(out2 - ref2) / np.abs(ref2).max(axis=1, keepdims=True)) < 1e-10, n


def _problem(case):
    from bem3_emf_qd2_b200.dqd2 import problem_from_arrays
    g = golden(f"rows_{case}.npz")
    return g, problem_from_arrays({k[3:]: g[k] for k in g.files if k.startswith("in/")})


_cache = {}


def _assembled(B, case, did):
    key = (case, did)
    if key not in _cache:
        g, p = _problem(case)
        _cache[key] = (g, p, B.assemble_domain(p, did))
    return _cache[key]


CASE_DOMAINS = [("sphere_m4", 0), ("sphere_m4", 1), ("cone_m1", 0), ("cone_m1", 1),
                ("sphere_m2", 0), ("sphere_m2", 1), ("sphere_m2", 2)]


@pytest.mark.parametrize("case,did", CASE_DOMAINS)
def test_assembly_rows_match_reference(cuda_lib, case, did):
    g, p, M = _assembled(cuda_lib, case, did)
    elems = sorted({int(k.split("/")[1][1:]) for k in g.files if k.startswith(f"d{did}/")})
    assert elems
    for t in elems:
        rows = slice(4 * (t - 1), 4 * t)
        drows = slice(8 * (t - 1), 8 * t)
        G, H, dF = g[f"d{did}/t{t}/G"], g[f"d{did}/t{t}/H"], g[f"d{did}/t{t}/dF"]
        for name, got, ref in (("G", M["G"][rows], G), ("H", M["H"][rows], H)):
            sc = np.abs(ref).max()
            err = np.abs(got - ref).max() / sc
            assert err < 1e-10, (case, did, t, name, err)
        assert np.abs(M["dF"][rows] - dF).max() < 1e-10 * (1 + np.abs(dF).max()), (case, did, t)
        if did == 0:
            assert np.abs(M["dG"][drows]).max() == 0 and np.abs(M["dH"][drows]).max() == 0
        else:
            for name in ("dG", "dH"):
                ref = g[f"d{did}/t{t}/{name}"]
                sc = np.abs(ref).max()
                err = np.abs(M[name][drows] - ref).max() / sc
                assert err < 1e-10, (case, did, t, name, err)


def test_assembly_is_deterministic(cuda_lib):
    B = cuda_lib
    g, p = _problem("sphere_m4")
    a = B.assemble_domain(p, 0)
    b = B.assemble_domain(p, 0)
    assert np.array_equal(a["G"], b["G"]) and np.array_equal(a["H"], b["H"]) and np.array_equal(a["dF"], b["dF"])


def test_triangle_rows_tn3_are_empty(cuda_lib):
    g, p, M = _assembled(cuda_lib, "cone_m1", 1)
    for t, sd in enumerate(p.sid[1], start=1):
        if p.nv[abs(sd)] == 3:
            r = 4 * (t - 1) + 3
            assert np.abs(M["G"][r]).max() == 0 and np.abs(M["H"][r]).max() == 0 and np.abs(M["dF"][r]).max() == 0
            break


@pytest.mark.parametrize("case", ["sphere_m4", "cone_m1", "sphere_m2"])
def test_all_domains_call_equals_one_domain_calls(cuda_lib, case):
    """bem3_assemble_domains (every domain in one call, copies overlapping the later domains'
    kernels) gives each domain's matrices exactly as bem3_assemble_domain does, and the same number
    of near-singular pairs."""
    B = cuda_lib
    g, p = _problem(case)
    one, gh = {}, 0
    for d in range(p.MN + 1):
        one[d] = B.assemble_domain(p, d)
        gh += one[d]["gh_pairs"]
    allm = B.assemble_domains(p)
    assert B.last_stats()["gh_pairs"] == gh
    for d in range(p.MN + 1):
        for k in ("G", "H", "dG", "dH", "dF"):
            assert np.array_equal(allm[d][k], one[d][k]), (case, d, k)
    part = B.assemble_domains(p, derivatives=False)  # the derivative matrices skipped
    for d in range(p.MN + 1):
        assert part[d]["dG"] is None and np.array_equal(part[d]["G"], one[d]["G"])
