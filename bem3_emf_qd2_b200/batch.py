"""Batched assembly of many instances of uneven size (C ABI ``bem3_batch_*``).

An instance is one problem: its own mesh, wavelength, incidence angles, lattice and materials.
A batch holds every domain of several instances; one run assembles all of their coefficient
matrices with one launch per pair class, the regular periodic pairs by a persistent kernel fed
from a device work counter (csrc/batch.cu), replayed as one CUDA graph.

What does not fit in HBM at once runs in waves.  The planner groups instances by size class,
packs each class into waves that fit the byte budget (outputs plus the batch's scratch), and the
autotuner picks the launch shape of each class (units a warp takes per grab, resident CTAs per SM
of the persistent kernel, CTAs per SM of the near-singular kernels) by timing candidates on an
element-subsampled probe of the class.

The seeded 64-instance mix (``mix``) follows the batched benchmark configuration: cube-spheres
6k^2 with k in {8, 12, 16, 20}, two-layer cube-spheres, or the jittered cone (3,360 triangles);
rectangular lattice periods in [0.8, 1.5] um; lambda0 in [0.4, 0.8] um; theta in [0, 60) deg
(theta = 0 exactly is redrawn: the reference rejects normal incidence); phi in [0, 360) deg;
particle index n_re in [1.4, 2.2], n_im in [0, 0.1].

  python -m bem3_emf_qd2_b200.batch [--preset c4|small] [--instances N] [--budget-gb B]

prints one JSON line: pairs/s batched and one domain at a time (bem3_assemble_domain_dev, the
plain drop-in's assembly), the speed-up, the waves and the launch shapes picked.
"""
import argparse
import ctypes as C
import json
import math
import os
import tempfile
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

# output bytes of a domain with ne elements: G, H (16 N^2 each) and dG, dH (32 N^2 each), N = 4 ne,
# plus dF (24 N)
def domain_output_bytes(ne: int) -> int:
    n = 4 * ne
    return 96 * n * n + 24 * n


# scratch the batch allocates for a domain (bem3_batch_scratch_bytes, per domain): per-pair F
# terms (24 B per pair), self-pair terms, the near-singular list, the propagating-order list
PROP_LIST_BYTES = 32 * 2048


def domain_scratch_bytes(ne: int, periodic: bool) -> int:
    np_ = 4 * ne * ne
    b = 24 * np_ + 96 * ne + 4 * (np_ // 8 + 4096) + 4 * 256
    return b + (PROP_LIST_BYTES if periodic else 0)


def instance_domains(p) -> List[Tuple[int, int, bool]]:
    """(did, ne, periodic) of every domain of a problem."""
    return [(d, len(p.sid[d]), d == 0 and p.ps == 1) for d in range(p.MN + 1)]


def instance_bytes(p) -> int:
    return sum(domain_output_bytes(ne) + domain_scratch_bytes(ne, per) for _, ne, per in instance_domains(p))


def size_class(p) -> str:
    """Launch-shape class of an instance by its largest domain."""
    ne = max(len(s) for s in p.sid)
    return "small" if ne < 1000 else ("medium" if ne < 2600 else "large")


def plan_waves(sizes: Sequence[int], budget: int) -> List[List[int]]:
    """Packs items (bytes each) into waves of at most `budget` bytes: first fit, largest first.
    Returns lists of item indices; raises ValueError for an item larger than the budget."""
    order = sorted(range(len(sizes)), key=lambda i: -sizes[i])
    waves: List[List[int]] = []
    room: List[int] = []
    for i in order:
        if sizes[i] > budget:
            raise ValueError(f"instance {i}: {sizes[i] / 1e9:.1f} GB does not fit the {budget / 1e9:.1f} GB budget")
        for w in range(len(waves)):
            if sizes[i] <= room[w]:
                waves[w].append(i)
                room[w] -= sizes[i]
                break
        else:
            waves.append([i])
            room.append(budget - sizes[i])
    return waves


def plan(problems: Sequence, budget: int) -> List[Tuple[str, List[int]]]:
    """Waves per size class: [(class, instance indices)], classes in a fixed order."""
    out = []
    for cls in ("large", "medium", "small"):
        idx = [i for i, p in enumerate(problems) if size_class(p) == cls]
        if not idx:
            continue
        for w in plan_waves([instance_bytes(problems[i]) for i in idx], budget):
            out.append((cls, [idx[j] for j in w]))
    return out


# ---------------------------------------------------------------------------------------------
# The seeded instance mix
@dataclass
class InstanceSpec:
    kind: str          # "sphere", "twolayer" or "cone"
    k: int             # cube-sphere subdivision (6 k^2 quads per surface); 0 for the cone
    d1: float
    d2: float
    lambda0: float
    theta: float
    phi: float
    n_particle: complex

    def config(self) -> dict:
        if self.kind == "cone":
            return dict(surfaces=[("cone", 0.3, 0.6, -0.3, 12, 24, 48, 0.01, 12345, 1, 99)],
                        media=[self.n_particle], lambda0=self.lambda0, ni=1.0, theta=self.theta, phi=self.phi,
                        d1=(self.d1, 0.0), d2=(0.0, self.d2), e0=[(1.0, 0.0)])
        r = 0.3 * min(self.d1, self.d2)
        if self.kind == "sphere":
            surfaces = [("sphere", r, self.k, 1, 99)]
            media = [self.n_particle]
        else:
            surfaces = [("sphere", r, self.k, 1, 99), ("sphere", 0.7 * r, self.k, 2, 1)]
            media = [complex(1.45, 0.01), self.n_particle]
        return dict(surfaces=surfaces, media=media, lambda0=self.lambda0, ni=1.33, theta=self.theta, phi=self.phi,
                    d1=(self.d1, 0.0), d2=(0.0, self.d2), e0=[(1.0, 0.0)])


def mix_specs(n: int = 64, seed: int = 2024, ks: Sequence[int] = (8, 12, 16, 20),
              kinds: Sequence[str] = ("sphere", "twolayer", "cone")) -> List[InstanceSpec]:
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        kind = kinds[int(rng.integers(len(kinds)))]
        k = int(ks[int(rng.integers(len(ks)))]) if kind != "cone" else 0
        d1, d2 = float(rng.uniform(0.8, 1.5)), float(rng.uniform(0.8, 1.5))
        lam = float(rng.uniform(0.4, 0.8))
        th = 0.0
        while th == 0.0:
            th = float(rng.uniform(0.0, math.radians(60.0)))
        ph = float(rng.uniform(0.0, 2.0 * math.pi))
        nre, nim = float(rng.uniform(1.4, 2.2)), float(rng.uniform(0.0, 0.1))
        out.append(InstanceSpec(kind, k, d1, d2, lam, th, ph, complex(nre, nim)))
    return out


def build_problems(specs: Sequence[InstanceSpec], outdir: str):
    """Writes every instance in the reference's input formats and reads it back."""
    from . import meshgen
    from .dqd2 import Problem
    probs = []
    for i, s in enumerate(specs):
        name = f"inst{i:03d}_{s.kind}{s.k or ''}"
        files = meshgen.write_config(name, s.config(), os.path.join(outdir, name))
        probs.append(Problem.from_files(*files))
    return probs


# ---------------------------------------------------------------------------------------------
# Device side
class InstanceDevice:
    """An instance's geometry and per-domain output matrices in HBM (torch tensors used as device
    allocations)."""

    def __init__(self, problem, device="cuda", derivatives: bool = True):
        import torch
        from . import MeshArrays, make_qpd
        self.p = problem
        self.geo = torch.from_numpy(MeshArrays(problem).packed()).to(device)
        self.sids = [torch.from_numpy(np.ascontiguousarray(s, dtype=np.int32)).to(device) for s in problem.sid]
        self.q = make_qpd(problem.qpd)
        self.out = []
        for d in range(problem.MN + 1):
            n = 4 * len(problem.sid[d])
            o = dict(G=torch.empty((n, n), dtype=torch.complex128, device=device),
                     H=torch.empty((n, n), dtype=torch.complex128, device=device),
                     dF=torch.empty((n, 3), dtype=torch.float64, device=device))
            if derivatives:
                o["dG"] = torch.empty((2 * n, n), dtype=torch.complex128, device=device)
                o["dH"] = torch.empty((2 * n, n), dtype=torch.complex128, device=device)
            self.out.append(o)

    def domain_entries(self):
        from . import bem3_batch_domain
        out = []
        for d in range(self.p.MN + 1):
            k = complex(self.p.kn[d])
            o = self.out[d]
            e = bem3_batch_domain()
            e.geo = self.geo.data_ptr()
            e.Ne = self.p.Ne
            e.sid = self.sids[d].data_ptr()
            e.Ne_d = len(self.p.sid[d])
            e.did = d
            e.periodic = 1 if (d == 0 and self.p.ps == 1) else 0
            e.qd = self.q
            e.kre, e.kim = k.real, k.imag
            e.G, e.H, e.dF = o["G"].data_ptr(), o["H"].data_ptr(), o["dF"].data_ptr()
            e.dG = o["dG"].data_ptr() if "dG" in o else None
            e.dH = o["dH"].data_ptr() if "dH" in o else None
            out.append(e)
        return out

    def assemble_sequential(self, stream=None) -> None:
        """Every domain through bem3_assemble_domain_dev, one after the other."""
        from . import check, lib
        for e in self.domain_entries():
            rc = lib().bem3_assemble_domain_dev(e.geo, e.Ne, e.sid, e.Ne_d, e.did, e.periodic, C.byref(e.qd), e.kre,
                                                e.kim, e.G, e.H, e.dG, e.dH, e.dF, stream)
            check(rc, "bem3_assemble_domain_dev")


@dataclass(frozen=True)
class Tuning:
    grab_units: int = 8
    regp_blocks_per_sm: int = 2
    gh_blocks_per_sm: int = 4

    def c(self):
        from . import bem3_batch_tuning
        return bem3_batch_tuning(self.grab_units, self.regp_blocks_per_sm, self.gh_blocks_per_sm)


class Batch:
    """Every domain of `instances` (InstanceDevice) as one bem3_batch, or the given bem3_batch_domain
    `entries` (e.g. from Context.prepare)."""

    def __init__(self, instances: Sequence[InstanceDevice] = (), tuning: Optional[Tuning] = None, entries=None):
        from . import bem3_batch_domain, check, lib
        self.instances = list(instances)
        if entries is None:
            entries = [e for inst in self.instances for e in inst.domain_entries()]
        self.n = len(entries)
        self._arr = (bem3_batch_domain * self.n)(*entries)
        self.h = C.c_void_p()
        t = (tuning or Tuning()).c()
        check(lib().bem3_batch_create(self._arr, self.n, C.byref(t), C.byref(self.h)), "bem3_batch_create")

    def run(self, stream=None) -> None:
        from . import check, lib
        check(lib().bem3_batch_run(self.h, stream), "bem3_batch_run")

    def wait(self, stream=None) -> List[int]:
        from . import lib
        st = (C.c_int * self.n)()
        rc = lib().bem3_batch_wait(self.h, stream, st)
        if rc == -2:
            raise RuntimeError("bem3_batch_wait failed: CUDA failure")
        return list(st)

    def info(self) -> Tuple[int, int]:
        from . import lib
        n, b = C.c_int(), C.c_size_t()
        lib().bem3_batch_info(self.h, C.byref(n), C.byref(b))
        return n.value, b.value

    def close(self) -> None:
        """Frees the batch's scratch and drops its references to the instances (whose matrices the
        caller may then release)."""
        from . import lib
        if self.h:
            lib().bem3_batch_destroy(self.h)
            self.h = C.c_void_p()
        self.instances = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def assemble_entries(entries, tuning: Optional[Tuning] = None, stream=None) -> None:
    """Assembles the matrices of the given bem3_batch_domain entries in one batch run (one graph
    launch) and waits for it; raises if any domain fails."""
    b = Batch(entries=list(entries), tuning=tuning)
    try:
        b.run(stream)
        st = b.wait(stream)
        bad = [x for x in st if x != 0]
        if bad:
            raise RuntimeError(f"batched assembly failed: status {bad[0]}")
    finally:
        b.close()


# ---------------------------------------------------------------------------------------------
# Autotuner
CANDIDATES = {
    "grab_units": (1, 4, 16, 64),
    "regp_blocks_per_sm": (2, 1),
    "gh_blocks_per_sm": (4, 2, 8),
}


def coordinate_search(measure: Callable[[Tuning], float], start: Tuning = Tuning(),
                      candidates: Dict[str, Sequence[int]] = CANDIDATES) -> Tuple[Tuning, List[Tuple[Tuning, float]]]:
    """One pass of coordinate descent over the launch-shape parameters: each parameter in turn
    takes the candidate value with the smallest measured time, the others held.  Returns the
    best shape and every (shape, seconds) measured."""
    best = start
    seen: Dict[Tuning, float] = {}

    def timed(t: Tuning) -> float:
        if t not in seen:
            seen[t] = float(measure(t))
        return seen[t]

    timed(best)
    for name, values in candidates.items():
        for v in values:
            t = Tuning(**{**best.__dict__, name: v})
            if timed(t) < timed(best):
                best = t
    return best, list(seen.items())


def probe_problems(problems: Sequence, stride: int):
    """Element-subsampled copies (every `stride`-th element of every domain): the same lattices,
    wavelengths, element sizes and pair mix at 1/stride^2 of the pairs."""
    import copy
    out = []
    for p in problems:
        q = copy.copy(p)
        q.sid = [np.ascontiguousarray(s[::stride]) for s in p.sid]
        out.append(q)
    return out


def autotune(problems: Sequence, stride: int = 4, repeats: int = 1, device="cuda"):
    """Launch shape for these instances, timed on their element-subsampled probe (CUDA events,
    one warm-up run per shape)."""
    import torch
    insts = [InstanceDevice(p, device) for p in probe_problems(problems, stride)]

    def measure(t: Tuning) -> float:
        b = Batch(insts, t)
        try:
            b.run()
            b.wait()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(repeats):
                b.run()
            e1.record()
            st = b.wait()
            if any(st):
                raise RuntimeError(f"batch status {st}")
            return e0.elapsed_time(e1) * 1e-3 / repeats
        finally:
            b.close()

    best, table = coordinate_search(measure)
    del insts
    return best, table


# ---------------------------------------------------------------------------------------------
def _pairs(problems) -> int:
    return int(sum(sum(p.pairs_per_domain()) for p in problems))


def run_mix(problems, budget: int, tune: bool = True, sequential: bool = True, device="cuda") -> dict:
    """Assembles every instance batched (wave by wave) and, if asked, one domain at a time; returns
    the figures of the JSON line."""
    import torch
    waves = plan(problems, budget)
    tunings: Dict[str, Tuning] = {}
    tune_table = {}
    if tune:
        for cls in sorted({c for c, _ in waves}):
            members = [problems[i] for c, w in waves if c == cls for i in w][:4]
            best, table = autotune(members)
            tunings[cls] = best
            tune_table[cls] = {"picked": best.__dict__, "candidates": len(table)}
    t_batched = 0.0
    t_seq = 0.0
    launches = 0
    bad = []
    import sys
    for iw, (cls, w) in enumerate(waves):
        insts = [InstanceDevice(problems[i], device) for i in w]
        b = Batch(insts, tunings.get(cls))
        if iw == 0:                 # warm-up: the first graph launch loads the kernels' modules
            b.run()
            b.wait()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b.run()
        e1.record()
        st = b.wait()
        t_batched += e0.elapsed_time(e1) * 1e-3
        bad += [(w, s) for s in st if s]
        launches += b.info()[0]
        b.close()
        del b
        if sequential:
            torch.cuda.synchronize()
            e0.record()
            for inst in insts:
                inst.assemble_sequential()
            del inst
            e1.record()
            torch.cuda.synchronize()
            t_seq += e0.elapsed_time(e1) * 1e-3
        print(f"wave {iw + 1}/{len(waves)} ({cls}, {len(w)} instances): batched {t_batched:.1f} s, "
              f"one domain at a time {t_seq:.1f} s so far", file=sys.stderr, flush=True)
        del insts
        torch.cuda.empty_cache()
    pairs = _pairs(problems)
    out = {
        "pairs": pairs, "batched_s": t_batched, "batched_pairs_per_s": pairs / t_batched,
        "waves": [{"class": c, "instances": len(w)} for c, w in waves], "launches": launches,
        "tuning": tune_table, "errors": [str(x) for x in bad[:3]],
    }
    if sequential:
        out.update({"sequential_s": t_seq, "sequential_pairs_per_s": pairs / t_seq, "speedup": t_seq / t_batched})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--preset", default="c4", choices=["c4", "small"],
                    help="c4: the 64-instance mix as configured; small: k in {4, 6, 8}, cones left out")
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--no-sequential", action="store_true")
    args = ap.parse_args()
    if args.preset == "c4":
        specs = mix_specs(args.instances, args.seed)
    else:
        specs = mix_specs(args.instances, args.seed, ks=(4, 6, 8), kinds=("sphere", "twolayer"))
    problems = build_problems(specs, tempfile.mkdtemp(prefix="bem3_mix_"))
    res = run_mix(problems, int(args.budget_gb * 1e9), tune=not args.no_tune, sequential=not args.no_sequential)
    line = {"metric": "batched assembly element-pair evals/s", "value": res["batched_pairs_per_s"], "unit": "pairs/s",
            "preset": args.preset, "instances": len(problems), "seed": args.seed,
            "elements": [int(p.Ne) for p in problems], **res}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
