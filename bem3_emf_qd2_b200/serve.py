"""Continuous-batching solve service on one GPU.

A request asks for the solution of one problem of the reference's kind: a mesh from a resident
pool, a wavelength, incidence angles and a polarisation.  The answer is the total field at the
mesh's probe points (EH_t, d3qd2_field.c:272-285) and the radiation force and torque (force_FN,
d3qd2_force.c:10-54), computed from the boundary values of solve_bieq (d3qd2_solve_bieq.c:36-84).

The server keeps solved problems resident on the device (a bem3 context holds the matrices and
their factorisations), keyed by (mesh, wavelength, angles): a request that differs from a
resident problem only in polarisation (or amplitude) reuses its factorisations and costs only
right-hand sides.  New problems are admitted while their estimated device memory fits the HBM
budget, evicting idle resident problems (least recently used first); requests that arrive while
others are running are admitted as soon as memory and a worker free up, and run concurrently
(each worker thread drives its contexts on its own CUDA stream).

    python -m bem3_emf_qd2_b200.serve [--requests 48] [--workers 8] [--budget-gb 120] ...

prints one JSON line: served solves/s at saturation, p50/p99 latency under a Poisson stream at
80 % of that capacity, and the same requests solved one at a time by the plain drop-in path
(create, solve, evaluate, destroy; no reuse), on the same GPU.
"""
import argparse
import dataclasses
import heapq
import json
import math
import threading
import time
from collections import OrderedDict
from concurrent.futures import ThreadPoolExecutor
from typing import Dict, List, Optional, Tuple

import numpy as np


@dataclasses.dataclass
class SolveRequest:
    rid: int
    mesh: str
    lambda0: float
    theta: float
    phi: float
    e0: Tuple[complex, complex]
    arrival: float = 0.0  # seconds after the start of the run

    @property
    def key(self):
        return (self.mesh, self.lambda0, self.theta, self.phi)


@dataclasses.dataclass
class SolveResult:
    rid: int
    E: np.ndarray       # [probes, 3] total electric field
    H: np.ndarray       # [probes, 3] total magnetic field
    did: np.ndarray     # [probes] domain of each probe point
    F: np.ndarray       # radiation force (type 0)
    N: np.ndarray       # torque about the origin (type 0)
    reused: bool        # served from a resident factorisation
    t_arrival: float
    t_start: float
    t_done: float

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrival


def request_waves(base, req: SolveRequest):
    """The request's incident plane wave on the mesh's background (ipw.txt's fields)."""
    from .dqd2 import PlaneWave
    w0 = base.waves[0]
    return [PlaneWave(req.lambda0, w0.ni, w0.power, complex(req.e0[0]), complex(req.e0[1]), (0.0, 0.0, 0.0),
                      req.theta, req.phi)]


def estimate_bytes(problem) -> int:
    """Device memory a solve of `problem` holds (matrices, factorisations, reduced system) plus
    its largest temporaries, from the mesh sizes alone."""
    nodes = [int(sum(problem.nv[abs(t)] for t in s)) for s in problem.sid]
    mats = sum(96 * (4 * len(s)) ** 2 + 24 * 4 * len(s) for s in problem.sid)
    gc = sum(16 * n * n for n in nodes)
    NN = problem.NN
    red = 16 * (4 * NN) ** 2
    temps = max(3 * 16 * n * NN + 16 * n * n for n in nodes)
    return int(1.1 * (mats + 2 * gc + red + temps)) + (64 << 20)


class GpuBackend:
    """The server's operations on bem3 contexts (one context is used by one thread at a time)."""

    def __init__(self, probes: Dict[str, np.ndarray]):
        from . import lib
        lib()  # fail loudly here if the CUDA library is missing
        self.probes = probes

    def open(self, problem):
        from . import Context
        return Context(problem)

    def solve(self, h):
        h.solve()

    def set_incident(self, h, problem):
        h.set_incident(problem.waves)

    def resolve(self, h):
        h.resolve()

    def evaluate(self, h, mesh):
        E, H, did = h.field(self.probes[mesh], 0, total=True)
        F, N = h.force((0.0, 0.0, 0.0), 0)
        return E, H, did, F, N

    def resident_bytes(self, h) -> int:
        return h.device_bytes()

    def close(self, h):
        h.close()


class BatchingGpuBackend(GpuBackend):
    """GpuBackend whose first solves of new problems assemble together.  Workers that reach solve()
    while an assembly is being gathered join it: the first of them waits `gather_s` for the others
    of its admission wave, then one batch (one CUDA graph launch, bem3_batch_*) assembles every
    domain of every problem in the wave; each worker then factorises and solves its own problem
    (bem3_ctx_solve_prepared) concurrently with the others.  Results are those of GpuBackend: the
    batched kernels run the same per-pair device code."""

    def __init__(self, probes: Dict[str, np.ndarray], gather_s: float = 0.003):
        super().__init__(probes)
        self.gather_s = gather_s
        self.cv = threading.Condition()
        self.queue: list = []
        self.gathering = False
        self.waves: List[int] = []

    def solve(self, h):
        from .batch import assemble_entries
        entries = h.prepare()
        slot = {"done": False, "err": None}
        with self.cv:
            self.queue.append((entries, slot))
            while not slot["done"]:
                if self.gathering:
                    self.cv.wait()
                    continue
                self.gathering = True
                self.cv.wait(timeout=self.gather_s)  # the rest of the wave joins meanwhile
                wave, self.queue = self.queue, []
                self.cv.release()
                err = None
                try:
                    assemble_entries([e for ents, _ in wave for e in ents])
                except Exception as ex:  # every member of the wave reports it
                    err = ex
                finally:
                    self.cv.acquire()
                for _, sl in wave:
                    sl["done"], sl["err"] = True, err
                self.waves.append(len(wave))
                self.gathering = False
                self.cv.notify_all()
        if slot["err"] is not None:
            raise slot["err"]
        h.solve_prepared()


@dataclasses.dataclass
class _Resident:
    handle: object
    problem: object
    bytes: int
    busy: bool = False


class SolveServer:
    def __init__(self, meshes: Dict[str, object], backend, hbm_budget: int, workers: int = 4):
        self.meshes = meshes
        self.backend = backend
        self.budget = int(hbm_budget)
        self.workers = workers
        self.lock = threading.Condition()
        self.resident: "OrderedDict[tuple, _Resident]" = OrderedDict()  # LRU order, oldest first
        self.wanted: set = set()  # keys that queued requests ask for (kept resident when possible)
        self.reserved = 0        # estimates of problems being solved for the first time
        self.peak_bytes = 0
        self.evictions = 0
        self.errors: List[str] = []

    # -- memory accounting (under self.lock) -------------------------------------------------
    def _in_use(self) -> int:
        return self.reserved + sum(r.bytes for r in self.resident.values())

    def _make_room(self, need: int) -> bool:
        """Evicts idle resident problems, least recently used first among those no queued request
        asks for, then among the rest, until `need` more bytes fit the budget."""
        while self._in_use() + need > self.budget:
            idle = [k for k, r in self.resident.items() if not r.busy]
            if not idle:
                return False
            idle.sort(key=lambda k: k in self.wanted)  # stable: LRU order within each group
            r = self.resident.pop(idle[0])
            self.backend.close(r.handle)
            self.evictions += 1
        return True

    def _admit(self, req: SolveRequest):
        """Returns ("reuse", resident) / ("new", estimate) / None (not now)."""
        r = self.resident.get(req.key)
        if r is not None:
            if r.busy:
                return None
            r.busy = True
            self.resident.move_to_end(req.key)
            return ("reuse", r)
        if any(k == req.key for k in self._starting):
            return None  # the same problem is being solved right now: wait and reuse it
        base = self.meshes[req.mesh]
        need = estimate_bytes(base)
        if need > self.budget:
            raise ValueError(f"request {req.rid}: {need / 1e9:.1f} GB does not fit the budget")
        if not self._make_room(need):
            return None
        self.reserved += need
        self._starting.add(req.key)
        self.peak_bytes = max(self.peak_bytes, self._in_use())
        return ("new", need)

    # -- one request on a worker thread --------------------------------------------------------
    def _run(self, req: SolveRequest, how, t0: float) -> SolveResult:
        t_start = time.perf_counter() - t0
        base = self.meshes[req.mesh]
        problem = base.with_incidence(request_waves(base, req))
        kind, what = how
        h = None
        try:
            if kind == "reuse":
                h = what.handle
                self.backend.set_incident(h, problem)
                self.backend.resolve(h)
            else:
                h = self.backend.open(problem)
                self.backend.solve(h)
            E, H, did, F, N = self.backend.evaluate(h, req.mesh)
        except Exception as ex:  # keep the server alive; the request reports the failure
            if kind == "new" and h is not None:
                self.backend.close(h)  # a failed first solve keeps nothing on the device
            with self.lock:
                self.errors.append(f"request {req.rid}: {ex}")
                if kind == "new":
                    self.reserved -= what
                    self._starting.discard(req.key)
                else:
                    what.busy = False
                self.lock.notify_all()
            raise
        t_done = time.perf_counter() - t0
        with self.lock:
            if kind == "new":
                self.reserved -= what
                self._starting.discard(req.key)
                self.resident[req.key] = _Resident(h, problem, self.backend.resident_bytes(h))
                self._make_room(0)  # should a solve hold more than its estimate
                self.peak_bytes = max(self.peak_bytes, self._in_use())
            else:
                what.busy = False
            self.lock.notify_all()
        return SolveResult(req.rid, E, H, did, F, N, kind == "reuse", req.arrival, t_start, t_done)

    def run(self, requests: List[SolveRequest]) -> List[SolveResult]:
        """Serves the requests, each released at its arrival time; returns results by rid."""
        self._starting = set()
        pending: List[SolveRequest] = []
        future = [(r.arrival, r.rid, r) for r in requests]
        heapq.heapify(future)
        results: Dict[int, SolveResult] = {}
        running = 0
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=self.workers) as pool:
            def done(fut, rid):
                nonlocal running
                with self.lock:
                    running -= 1
                    if fut.exception() is None:
                        results[rid] = fut.result()
                    self.lock.notify_all()

            with self.lock:
                while future or pending or running:
                    now = time.perf_counter() - t0
                    while future and future[0][0] <= now:
                        pending.append(heapq.heappop(future)[2])
                    # admit requests for idle resident problems first, then the rest in arrival
                    # order; a request that cannot start now does not block later ones
                    # (continuous batching); problems that queued requests ask for are evicted last
                    self.wanted = {r.key for r in pending}
                    for reuse_pass in (True, False):
                        i = 0
                        while i < len(pending) and running < self.workers:
                            r0 = self.resident.get(pending[i].key)
                            if reuse_pass and (r0 is None or r0.busy):
                                i += 1
                                continue
                            how = self._admit(pending[i])
                            if how is None:
                                i += 1
                                continue
                            req = pending.pop(i)
                            running += 1
                            fut = pool.submit(self._run, req, how, t0)
                            fut.add_done_callback(lambda f, rid=req.rid: done(f, rid))
                    if not (future or pending or running):
                        break
                    wait = (future[0][0] - now) if future else 0.5
                    self.lock.wait(timeout=max(1e-4, min(wait, 0.5)))
                    if self.errors and not running and not future and pending:
                        break  # nothing will change any more
        return [results[r.rid] for r in requests if r.rid in results]

    def close(self):
        with self.lock:
            for r in self.resident.values():
                self.backend.close(r.handle)
            self.resident.clear()


def run_sequential(meshes, backend, requests: List[SolveRequest]) -> List[SolveResult]:
    """The plain drop-in one request at a time: create, solve, evaluate, destroy (no reuse)."""
    out = []
    t0 = time.perf_counter()
    for req in requests:
        ts = time.perf_counter() - t0
        base = meshes[req.mesh]
        h = backend.open(base.with_incidence(request_waves(base, req)))
        backend.solve(h)
        E, H, did, F, N = backend.evaluate(h, req.mesh)
        backend.close(h)
        out.append(SolveResult(req.rid, E, H, did, F, N, False, ts, ts, time.perf_counter() - t0))
    return out


# ---------------------------------------------------------------------------------------------
# The served workload: a resident mesh pool and a seeded request stream
# The served configuration's pool at the sizes one B200 can hold resident: cube-spheres 6 n^2 and
# two-layer cube-spheres 2 x 6 n^2 from 384 elements up to 3072 (two-layer n = 16, whose resident
# solve takes ~85 GB of the 120 GB budget by estimate_bytes; n = 18, 3888 elements, would need ~136 GB,
# and the 12288-element two-layer meshes ~2.5 TB in this dense form).
C5_SPHERES = (8, 10, 12, 14, 16, 18, 20)
C5_LAYERS = (8, 9, 10, 11, 12, 13, 14, 16)


def mesh_pool(outdir: str, sizes=(4, 5, 6, 7, 8), layers=(4, 5, 6), seed: int = 7):
    """Cube-spheres (6 n^2 quads) and two-layer cube-spheres (2 x 6 n^2) on seeded rectangular
    lattices, written in the reference's input formats and read back; returns (meshes, probes)."""
    import os
    from . import meshgen
    from .dqd2 import Problem
    rng = np.random.default_rng(seed)
    meshes, probes = {}, {}
    specs = [("sphere", n) for n in sizes] + [("twolayer", n) for n in layers]
    for kind, n in specs:
        d1 = float(rng.uniform(0.8, 1.5))
        d2 = float(rng.uniform(0.8, 1.5))
        nre, nim = float(rng.uniform(1.4, 2.2)), float(rng.uniform(0.0, 0.1))
        if kind == "sphere":
            r = 0.25 * min(d1, d2)
            surfaces = [("sphere", r, n, 1, 99)]
            media = [complex(nre, nim)]
        else:
            r = 0.3 * min(d1, d2)
            surfaces = [("sphere", r, n, 1, 99), ("sphere", 0.7 * r, n, 2, 1)]
            media = [complex(1.45, 0.01), complex(nre, nim)]
        name = f"{kind}{6 * n * n * len(surfaces)}"
        cfg = dict(surfaces=surfaces, media=media, lambda0=0.6, ni=1.33, theta=0.3, phi=0.2, d1=(d1, 0.0),
                   d2=(0.0, d2), e0=[(1.0, 0.0)])
        files = meshgen.write_config(name, cfg, os.path.join(outdir, name))
        meshes[name] = Problem.from_files(*files)
        zt = 1.3 * r
        probes[name] = np.array([[0.0, 0.0, zt], [0.1 * d1, -0.05 * d2, -zt], [0.0, 0.0, 0.0], [0.3 * d1, 0.2 * d2, 0.9]])
    return meshes, probes


def request_stream(meshes, n: int, rate: Optional[float], reuse: float = 0.3, seed: int = 11) -> List[SolveRequest]:
    """n requests; a fraction `reuse` repeats an earlier request's mesh, wavelength and angles with
    another polarisation; Poisson arrivals at `rate` per second (all at t = 0 when rate is None)."""
    rng = np.random.default_rng(seed)
    names = sorted(meshes)
    out: List[SolveRequest] = []
    t = 0.0
    for i in range(n):
        if out and rng.random() < reuse:
            prev = out[int(rng.integers(len(out)))]
            mesh, lam, th, ph = prev.mesh, prev.lambda0, prev.theta, prev.phi
        else:
            mesh = names[int(rng.integers(len(names)))]
            lam = float(rng.uniform(0.4, 0.8))
            th = float(rng.uniform(math.radians(2.0), math.radians(60.0)))
            ph = float(rng.uniform(0.0, 2.0 * math.pi))
        a = float(rng.uniform(0.0, 2.0 * math.pi))
        e0 = (complex(math.cos(a), 0.0), complex(0.0, math.sin(a)))
        if rate is not None and i > 0:
            t += float(rng.exponential(1.0 / rate))
        out.append(SolveRequest(i, mesh, lam, th, ph, e0, t))
    return out


def _pct(x, q):
    return float(np.percentile(np.asarray(x), q)) if len(x) else float("nan")


def measure(meshes, probes, requests: int = 48, workers: int = 8, budget_gb: float = 120.0, load: float = 0.8,
            sequential: bool = True, batched: bool = True) -> dict:
    """Served solves/s at saturation (every request queued at t = 0), p50/p99 latency under a
    Poisson stream at `load` x that capacity, and the same requests solved one at a time by the plain
    drop-in path (create, solve, evaluate, destroy; no reuse), on the current GPU.  batched: the
    service's new problems assemble in batches (BatchingGpuBackend); the sequential path never does."""
    plain = GpuBackend(probes)
    backend = BatchingGpuBackend(probes) if batched else plain
    budget = int(budget_gb * 1e9)
    # warm-up: one solve per pooled mesh loads the library's kernels and the solver libraries'
    # kernels for every system size the pool reaches (modules load lazily, on first launch)
    for name in sorted(meshes):
        run_sequential(meshes, plain, request_stream({name: meshes[name]}, 1, None))
    seq = None
    reqs0 = request_stream(meshes, requests, None)
    if sequential:
        t = time.perf_counter()
        run_sequential(meshes, plain, reqs0)
        seq = requests / (time.perf_counter() - t)
    srv = SolveServer(meshes, backend, budget, workers)
    t = time.perf_counter()
    res = srv.run(reqs0)
    cap = len(res) / (time.perf_counter() - t)
    cap_stats = {"reused": sum(r.reused for r in res), "evictions": srv.evictions,
                 "peak_reserved_gb": srv.peak_bytes / 1e9}
    srv.close()
    reqs = request_stream(meshes, requests, load * cap, seed=13)
    srv = SolveServer(meshes, backend, budget, workers)
    t = time.perf_counter()
    res2 = srv.run(reqs)
    wall = time.perf_counter() - t
    lat = [r.latency for r in res2]
    line = {
        "metric": "served solves/s", "value": cap, "unit": "solves/s", "higher_is_better": True,
        "sequential_dropin_solves_per_s": seq, "speedup_vs_sequential": (cap / seq) if seq else None,
        "capacity_run": cap_stats,
        "poisson": {"rate": load * cap, "solves_per_s": len(res2) / wall, "p50_s": _pct(lat, 50),
                    "p99_s": _pct(lat, 99), "reused": sum(r.reused for r in res2), "requests": len(reqs),
                    "completed": len(res2)},
        "workers": workers, "hbm_budget_gb": budget_gb, "peak_reserved_gb": srv.peak_bytes / 1e9,
        "evictions": srv.evictions, "errors": srv.errors[:3],
        "pool": {k: int(m.Ne) for k, m in sorted(meshes.items())},
        "batched_assembly": batched,
        "assembly_waves": (len(backend.waves), max(backend.waves) if backend.waves else 0) if batched else None,
    }
    srv.close()
    return line


def main():
    import tempfile
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=48)
    ap.add_argument("--workers", type=int, default=8)
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--load", type=float, default=0.8, help="Poisson rate as a fraction of the measured capacity")
    ap.add_argument("--no-sequential", action="store_true")
    ap.add_argument("--unbatched", action="store_true", help="each new problem assembles on its own")
    ap.add_argument("--pool", default="small", choices=["small", "c5"],
                    help="small: 96-432 elements; c5: 384-3072 elements (the largest resident under 120 GB)")
    args = ap.parse_args()
    if args.pool == "c5":
        meshes, probes = mesh_pool(tempfile.mkdtemp(prefix="bem3_pool_"), C5_SPHERES, C5_LAYERS)
    else:
        meshes, probes = mesh_pool(tempfile.mkdtemp(prefix="bem3_pool_"))
    line = measure(meshes, probes, args.requests, args.workers, args.budget_gb, args.load, not args.no_sequential,
                   not args.unbatched)
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
