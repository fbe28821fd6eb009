"""CPU tests of the solve service's scheduling (bem3_emf_qd2_b200/serve.py) with a stand-in
backend: every request answered once, polarisation-only repeats served from resident
factorisations, the HBM budget never exceeded, idle problems evicted least recently used first,
no context driven by two threads at once."""
import threading
import time

import numpy as np
import pytest


class FakeBackend:
    def __init__(self, probes, per_bytes):
        self.probes = probes
        self.per_bytes = per_bytes
        self.lock = threading.Lock()
        self.open_handles = 0
        self.max_open = 0
        self.busy = set()
        self.violations = 0
        self.solves = 0
        self.resolves = 0

    class H:
        def __init__(self, p):
            self.p = p

    def _enter(self, h):
        with self.lock:
            if id(h) in self.busy:
                self.violations += 1
            self.busy.add(id(h))

    def _leave(self, h):
        with self.lock:
            self.busy.discard(id(h))

    def open(self, problem):
        with self.lock:
            self.open_handles += 1
            self.max_open = max(self.max_open, self.open_handles)
        return FakeBackend.H(problem)

    def solve(self, h):
        self._enter(h)
        time.sleep(0.01)
        with self.lock:
            self.solves += 1
        self._leave(h)

    def set_incident(self, h, problem):
        h.p = problem

    def resolve(self, h):
        self._enter(h)
        time.sleep(0.002)
        with self.lock:
            self.resolves += 1
        self._leave(h)

    def evaluate(self, h, mesh):
        w = h.p.waves[0]
        v = np.array([w.lambda0, w.theta, w.phi, abs(w.e0x), abs(w.e0y)])
        E = np.tile(v[:3], (len(self.probes[mesh]), 1)).astype(complex)
        return E, 2 * E, np.zeros(len(E), np.int32), v[:3], v[2:]

    def resident_bytes(self, h):
        from bem3_emf_qd2_b200 import serve
        return int(0.9 * serve.estimate_bytes(h.p))  # a solve holds less than its estimate

    def close(self, h):
        with self.lock:
            self.open_handles -= 1


@pytest.fixture(scope="module")
def pool(tmp_path_factory):
    from bem3_emf_qd2_b200 import serve
    return serve.mesh_pool(str(tmp_path_factory.mktemp("pool")), sizes=(3, 4), layers=(3,))


def _server(pool, budget_units, workers=3):
    from bem3_emf_qd2_b200 import serve
    meshes, probes = pool
    per = max(serve.estimate_bytes(m) for m in meshes.values())
    be = FakeBackend(probes, per)
    return serve.SolveServer(meshes, be, budget_units * per, workers), be, per


def test_every_request_answered_and_repeats_reuse(pool):
    from bem3_emf_qd2_b200 import serve
    meshes, _ = pool
    reqs = serve.request_stream(meshes, 30, rate=400.0, reuse=0.4, seed=3)
    srv, be, _ = _server(pool, 100)
    res = srv.run(reqs)
    assert [r.rid for r in res] == [r.rid for r in reqs]
    assert be.violations == 0
    keys = {r.key for r in reqs}
    assert be.solves == len(keys)           # one factorisation per distinct problem
    assert be.resolves == len(reqs) - len(keys)
    assert sum(r.reused for r in res) == be.resolves
    for q, r in zip(reqs, res):             # each answer belongs to its own request
        assert np.allclose(r.E[0].real, [q.lambda0, q.theta, q.phi])
    srv.close()
    assert be.open_handles == 0


def test_budget_bounds_memory_and_evicts(pool):
    from bem3_emf_qd2_b200 import serve
    meshes, _ = pool
    reqs = serve.request_stream(meshes, 24, rate=None, reuse=0.0, seed=5)
    srv, be, per = _server(pool, 2)
    res = srv.run(reqs)
    assert len(res) == len(reqs)
    assert srv.peak_bytes <= srv.budget
    smallest = min(serve.estimate_bytes(m) for m in meshes.values())
    assert srv.evictions > 0
    assert be.max_open <= srv.budget // smallest
    srv.close()


def test_oversized_request_is_refused(pool):
    from bem3_emf_qd2_b200 import serve
    meshes, _ = pool
    reqs = serve.request_stream(meshes, 1, rate=None, seed=1)
    srv, _, per = _server(pool, 1)
    srv.budget = per // 10
    with pytest.raises(ValueError):
        srv.run(reqs)


def test_queued_repeats_reuse_under_a_tight_budget(pool):
    """All requests queued at once, room for two problems: the problems that queued requests ask
    for are evicted last and their requests admitted first, so every polarisation repeat is served
    from its resident factorisation although the budget forces evictions."""
    from bem3_emf_qd2_b200 import serve
    meshes, _ = pool
    reqs = serve.request_stream(meshes, 30, rate=None, reuse=0.4, seed=9)
    keys = {r.key for r in reqs}
    assert len(reqs) - len(keys) >= 5
    srv, be, _ = _server(pool, 2)
    res = srv.run(reqs)
    assert len(res) == len(reqs) and be.violations == 0
    assert srv.peak_bytes <= srv.budget and srv.evictions > 0
    assert be.solves == len(keys)
    assert be.resolves == len(reqs) - len(keys)
    srv.close()
