"""CPU tests of the batched assembly's host logic (bem3_emf_qd2_b200/batch.py): wave planning
under the HBM budget, size classes, the seeded instance mix, the autotuner's coordinate search,
and the byte estimates against the library's own (bem3_batch_scratch_bytes needs no GPU)."""
import ctypes as C
import math

import numpy as np
import pytest


def test_plan_waves_respects_budget_and_covers_every_item():
    from bem3_emf_qd2_b200 import batch
    rng = np.random.default_rng(0)
    sizes = [int(x) for x in rng.integers(1, 100, size=200)]
    waves = batch.plan_waves(sizes, 250)
    seen = sorted(i for w in waves for i in w)
    assert seen == list(range(len(sizes)))
    assert all(sum(sizes[i] for i in w) <= 250 for w in waves)
    # first fit largest first never needs more than twice the lower bound here
    assert len(waves) <= 2 * math.ceil(sum(sizes) / 250)
    with pytest.raises(ValueError):
        batch.plan_waves([10, 300], 250)


def test_mix_is_seeded_and_within_ranges():
    from bem3_emf_qd2_b200 import batch
    a = batch.mix_specs(64, seed=5)
    b = batch.mix_specs(64, seed=5)
    assert a == b and len(a) == 64
    assert a != batch.mix_specs(64, seed=6)
    for s in a:
        assert s.kind in ("sphere", "twolayer", "cone")
        assert (s.k in (8, 12, 16, 20)) if s.kind != "cone" else s.k == 0
        assert 0.8 <= s.d1 <= 1.5 and 0.8 <= s.d2 <= 1.5
        assert 0.4 <= s.lambda0 <= 0.8
        assert 0.0 < s.theta < math.radians(60.0)
        assert 0.0 <= s.phi < 2 * math.pi
        assert 1.4 <= s.n_particle.real <= 2.2 and 0.0 <= s.n_particle.imag <= 0.1
    assert {s.kind for s in a} == {"sphere", "twolayer", "cone"}


def test_mix_instances_build_with_expected_element_counts(tmp_path):
    from bem3_emf_qd2_b200 import batch
    specs = [batch.InstanceSpec("sphere", 3, 1.0, 1.2, 0.5, 0.3, 1.0, 1.6 + 0.01j),
             batch.InstanceSpec("twolayer", 2, 0.9, 1.4, 0.7, 0.5, 4.0, 2.0 + 0.0j)]
    probs = batch.build_problems(specs, str(tmp_path))
    assert probs[0].Ne == 6 * 9 and probs[0].MN == 1
    assert probs[1].Ne == 2 * 6 * 4 and probs[1].MN == 2
    assert [len(s) for s in probs[1].sid] == [24, 48, 24]
    assert probs[0].qpd["vd1"][0] == pytest.approx(1.0) and probs[0].qpd["vd2"][1] == pytest.approx(1.2)


def test_plan_groups_by_size_class(tmp_path):
    from bem3_emf_qd2_b200 import batch
    specs = [batch.InstanceSpec("sphere", k, 1.0, 1.0, 0.6, 0.2, 0.0, 1.5 + 0j) for k in (2, 3, 2, 3)]
    probs = batch.build_problems(specs, str(tmp_path))
    per = [batch.instance_bytes(p) for p in probs]
    waves = batch.plan(probs, 2 * max(per))
    assert sorted(i for _, w in waves for i in w) == [0, 1, 2, 3]
    for cls, w in waves:
        assert all(batch.size_class(probs[i]) == cls for i in w)
        assert sum(per[i] for i in w) <= 2 * max(per)


def test_coordinate_search_finds_the_best_shape_on_its_path():
    from bem3_emf_qd2_b200 import batch
    calls = []

    def cost(t):
        calls.append(t)
        return abs(t.grab_units - 16) + 3 * (t.regp_blocks_per_sm != 2) + 0.5 * abs(t.gh_blocks_per_sm - 8)

    best, table = batch.coordinate_search(cost)
    assert best == batch.Tuning(16, 2, 8)
    assert len(calls) == len(set(calls)) == len(table)   # each shape measured once
    assert min(v for _, v in table) == cost(best)


def test_scratch_estimate_bounds_the_library(cuda_lib_host):
    """The planner's per-domain scratch estimate is at least what bem3_batch_create allocates."""
    from bem3_emf_qd2_b200 import bem3_batch_domain, batch
    doms = []
    ests = 0
    for ne, per in ((96, True), (384, False), (1000, True), (4800, False)):
        e = bem3_batch_domain()
        e.Ne_d, e.Ne, e.periodic = ne, ne, 1 if per else 0
        doms.append(e)
        ests += batch.domain_scratch_bytes(ne, per)
    arr = (bem3_batch_domain * len(doms))(*doms)
    lib_bytes = cuda_lib_host.bem3_batch_scratch_bytes(arr, len(doms))
    table = 64 * 1024  # descriptor table and segments (bounded by the library's own formula)
    assert lib_bytes <= ests + table
    assert lib_bytes >= sum(24 * 4 * ne * ne for ne, _ in ((96, 0), (384, 0), (1000, 0), (4800, 0)))
