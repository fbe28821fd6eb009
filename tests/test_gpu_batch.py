"""Batched assembly (bem3_batch_*) on the GPU.

A batch of five small instances of different kinds (quads and triangles; one, two and three
domains; each its own lattice, wavelength, incidence and materials) is assembled in one run and
checked domain by domain:

  * against bem3_assemble_domain_dev on the same inputs (the one-domain path, itself checked
    against the reference in test_gpu_parity.py):  |batch - single| <= 1e-13 * max |single|
    per matrix (same device functions; the compiler may contract them differently in the
    batched kernels);
  * alone (a batch of one) against in the mix, and under another launch shape: bit-identical,
    because every pair is computed by the same kernel code whatever else is in the batch and
    however the work is split.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13
KEYS = ("G", "H", "dG", "dH", "dF")


def _instances(tmp_path):
    from bem3_emf_qd2_b200 import batch, meshgen
    from bem3_emf_qd2_b200.dqd2 import Problem
    specs = [batch.InstanceSpec("sphere", 4, 1.0, 1.1, 0.63, 0.3, 0.2, 1.59 + 0j),
             batch.InstanceSpec("twolayer", 3, 0.9, 1.3, 0.53, math.radians(30), math.radians(45), 1.8 + 0.05j),
             batch.InstanceSpec("sphere", 3, 1.4, 0.85, 0.45, math.radians(55), 4.0, 2.1 + 0.1j),
             batch.InstanceSpec("twolayer", 2, 1.2, 1.2, 0.75, 0.05, 2.5, 1.45 + 0.0j)]
    probs = batch.build_problems(specs, str(tmp_path))
    # a small triangulated cone (hexagonal lattice, 210 triangles)
    files = meshgen.make_config("cone210", str(tmp_path / "cone"))
    probs.append(Problem.from_files(*files))
    return probs


def _snapshot(inst):
    return [{k: o[k].detach().clone() for k in KEYS} for o in inst.out]


def _fill_nan(inst):
    for o in inst.out:
        for k in KEYS:
            o[k].fill_(float("nan"))


def test_batch_matches_single_domain_and_is_independent_of_the_mix(cuda_lib, tmp_path):
    import torch
    from bem3_emf_qd2_b200 import batch
    probs = _instances(tmp_path)
    insts = [batch.InstanceDevice(p) for p in probs]
    for i in insts:
        _fill_nan(i)
    b = batch.Batch(insts)
    b.run()
    st = b.wait()
    assert st == [0] * len(st)
    launches, nbytes = b.info()
    assert launches >= 5 and nbytes > 0
    mixed = [_snapshot(i) for i in insts]

    # the same batch again (counters and work lists reset by the graph itself)
    b.run()
    assert b.wait() == [0] * len(st)
    for i, inst in enumerate(insts):
        for d, o in enumerate(inst.out):
            for k in KEYS:
                assert torch.equal(o[k], mixed[i][d][k]), ("rerun", i, d, k)
    b.close()

    for i, p in enumerate(probs):
        # alone: a batch of one
        alone = batch.InstanceDevice(p)
        _fill_nan(alone)
        b1 = batch.Batch([alone])
        b1.run()
        assert b1.wait() == [0] * (p.MN + 1)
        b1.close()
        for d in range(p.MN + 1):
            for k in KEYS:
                assert torch.equal(alone.out[d][k], mixed[i][d][k]), ("alone", i, d, k)
        # one domain at a time through bem3_assemble_domain_dev
        _fill_nan(alone)
        alone.assemble_sequential()
        torch.cuda.synchronize()
        for d in range(p.MN + 1):
            for k in KEYS:
                ref = alone.out[d][k]
                got = mixed[i][d][k]
                assert bool(torch.isfinite(ref).all()), (i, d, k)
                scale = float(ref.abs().max())
                err = float((got - ref).abs().max())
                assert err <= TOL * max(scale, 1e-300), (i, d, k, err, scale)
        del alone
    torch.cuda.empty_cache()


def test_launch_shape_does_not_change_results(cuda_lib, tmp_path):
    import torch
    from bem3_emf_qd2_b200 import batch
    probs = _instances(tmp_path)[:3]
    insts = [batch.InstanceDevice(p) for p in probs]
    out = []
    for t in (batch.Tuning(), batch.Tuning(1, 1, 2), batch.Tuning(64, 2, 8)):
        for i in insts:
            _fill_nan(i)
        b = batch.Batch(insts, t)
        b.run()
        assert b.wait() == [0] * b.n
        b.close()
        out.append([_snapshot(i) for i in insts])
    for r in out[1:]:
        for i in range(len(insts)):
            for d in range(len(r[i])):
                for k in KEYS:
                    assert torch.equal(r[i][d][k], out[0][i][d][k]), (i, d, k)


def test_batch_rejects_bad_arguments(cuda_lib):
    import ctypes as C
    from bem3_emf_qd2_b200 import bem3_batch_domain, bem3_batch_tuning, lib
    h = C.c_void_p()
    e = bem3_batch_domain()  # null pointers
    arr = (bem3_batch_domain * 1)(e)
    assert lib().bem3_batch_create(arr, 1, None, C.byref(h)) == -1
    assert lib().bem3_batch_create(arr, 0, None, C.byref(h)) == -1
    t = bem3_batch_tuning(0, 2, 4)
    assert lib().bem3_batch_create(arr, 1, C.byref(t), C.byref(h)) == -1
    assert lib().bem3_batch_run(None, None) == -1
