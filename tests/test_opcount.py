"""The roofline numerator: algorithmic FP64 operations per lattice-sum term (oracle/opcount.py).

The counted special functions must be accurate to the stated level (their counts are only
meaningful for methods that compute the function), the counted lattice sums must give the reference's
Green's function, and bench.py's frozen operations per term must be what the restatement counts on
the bench workload (a smaller seeded sample here: within 3 %).
"""
import numpy as np

from conftest import golden


def _oc():
    import opcount
    return opcount, opcount.OpCount()


def test_counted_special_functions_are_accurate():
    _, oc = _oc()
    r = oc.check_special_functions()
    assert r["exp"][0] < 1e-15 and r["sincos"][0] < 1e-15
    assert r["erfc"][0] < 5e-15
    assert r["w"][0] < 5e-14
    assert r["exp"][1] > 0 and r["w"][1] > r["erfc"][1] > r["exp"][1]


def test_counted_lattice_sums_match_reference_green_function():
    """oc_point (the restatement on the counting type) against the reference's d3hm_qpgf_d2_v1, with
    the reference's method choice (term counts identical) and with the assembly's cost rule."""
    opcount, oc = _oc()
    q = golden("qpgf.npz")
    for name in ("square1_c2", "hex09_c3"):
        p, r, ref, rret = q[name + "/qpd"], q[name + "/r"], q[name + "/v1"], q[name + "/ret_v1"]
        for i in range(0, len(r), 97):
            for zfac in (0.0, opcount.ZFAC):
                ret, out, terms, ops, fd = oc.point(p, r[i], zfac)
                v = out[0::2] + 1j * out[1::2]
                assert ret > 0 and ops > 0
                if zfac == 0.0:
                    assert ret == rret[i]
                err = np.abs(v - ref[i]).max() / np.abs(ref[i]).max()
                assert err < 1e-11, (name, i, zfac, err)


def test_bench_frozen_ops_per_term_reproduced():
    import bench
    opcount, _ = _oc()
    r = opcount.workload_ops("twolayer3072", pairs=6, seed=11)
    frozen = bench.ALG_OPS_PER_TERM["twolayer3072"]
    assert abs(r["ops_per_term"] / frozen - 1.0) < 0.03, (r, frozen)
