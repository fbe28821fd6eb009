"""The solve service on the GPU: every request's answer in the concurrent mix (with resident
factorisations reused for polarisation-only repeats) equals its answer solved alone by the plain
path (create, solve, evaluate, destroy):

  fields at the probe points and force/torque: |mix - alone| <= 1e-9 * max|alone|
(the reused factorisations and the fresh ones are the same numbers; only the order in which the
GPU interleaves independent work changes)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pool(tmp_path_factory):
    from bem3_emf_qd2_b200 import serve
    return serve.mesh_pool(str(tmp_path_factory.mktemp("pool")), sizes=(3, 4), layers=(3,))


def test_mix_equals_alone(cuda_lib, pool):
    from bem3_emf_qd2_b200 import serve
    meshes, probes = pool
    be = serve.GpuBackend(probes)
    reqs = serve.request_stream(meshes, 12, rate=None, reuse=0.4, seed=21)
    alone = serve.run_sequential(meshes, be, reqs)
    srv = serve.SolveServer(meshes, be, int(20e9), workers=3)
    mix = srv.run(reqs)
    srv.close()
    assert not srv.errors
    assert [r.rid for r in mix] == [r.rid for r in reqs]
    assert sum(r.reused for r in mix) > 0
    for a, m in zip(alone, mix):
        for x, y in ((a.E, m.E), (a.H, m.H), (a.F, m.F), (a.N, m.N)):
            assert np.abs(x - y).max() <= 1e-9 * np.abs(x).max(), (a.rid, m.reused)
        assert np.array_equal(a.did, m.did)


def test_batched_waves_equal_alone(cuda_lib, pool):
    """The service with batched assembly (BatchingGpuBackend: new problems admitted together are
    assembled by one bem3_batch graph launch, then factorised per worker) gives every request the
    answer of the plain path, within the same tolerance, and did assemble at least one wave of
    several problems."""
    from bem3_emf_qd2_b200 import serve
    meshes, probes = pool
    plain = serve.GpuBackend(probes)
    reqs = serve.request_stream(meshes, 12, rate=None, reuse=0.3, seed=5)
    alone = serve.run_sequential(meshes, plain, reqs)
    be = serve.BatchingGpuBackend(probes, gather_s=0.02)
    srv = serve.SolveServer(meshes, be, int(20e9), workers=4)
    mix = srv.run(reqs)
    srv.close()
    assert not srv.errors
    assert [r.rid for r in mix] == [r.rid for r in reqs]
    assert be.waves and max(be.waves) >= 2, be.waves
    for a, m in zip(alone, mix):
        for x, y in ((a.E, m.E), (a.H, m.H), (a.F, m.F), (a.N, m.N)):
            assert np.abs(x - y).max() <= 1e-9 * np.abs(x).max(), (a.rid, m.reused)
        assert np.array_equal(a.did, m.did)
