"""Benchmark: element-pair evaluations/s of the coefficient-matrix assembly (FP64).

Workload: the two-layer cube-sphere of the larger plain configuration (3072 bilinear quads over
two interfaces, square lattice 1.0 um in n=1.33, lambda0=0.532 um, theta=30 deg, phi=45 deg;
core r=0.25 n=1.59, shell r=0.35 n=1.45+0.01i).  One step assembles every domain's coefficient
matrices (G, H, dG, dH, dF; the reference's create_cmatrix_domain for did = 0, 1, 2), i.e.
56,623,104 (collocation node, source element) evaluations.  Synthetic seeded geometry.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config NAME]

`value`  : pairs/s with geometry resident in HBM (device-timed, max over ranks, weak scaling:
           every rank assembles its own instance).
`e2e`    : the same through the host-pointer C ABI (bem3_assemble_domains, every domain in one call,
           the reference's create_cmatrix): geometry uploaded and
           all matrices copied back to host memory inside the timed region.
`--impl reference`: the reference's own CPU code (compiled from its sources into oracle/_ref)
           on a bounded, class-stratified sample of the same pairs using all host threads,
           extrapolated to pairs/s.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "QPGF element-pair evals/s"
UNIT = "pairs/s"
# Algorithmic FP64 operations per lattice-sum term of the regular periodic pairs, per workload:
# oracle/opcount.py (the CPU restatement of the lattice sums on an operation-counting number type,
# special functions at the counts of compact published methods, per-point element work included)
# over a seeded sample of 96 of the workload's regular periodic pairs, with the assembly's method
# choice.  Fixed: the kernel's own instruction count is reported beside it, not in its place.
ALG_OPS_PER_TERM = {"twolayer3072": 378.23, "sphere384": 377.03, "cone3360": 398.91}
# FP64 operations per term the hardware executed in k_reg_periodic (ncu: 2 x DFMA + DADD + DMUL,
# thread level, over the kernel's own term counter), from the capture of the workload's /stride8
# subsample in profiles/; None where no capture of the current kernel exists.
HW_OPS_PER_TERM = {"twolayer3072": 253.6}
# DRAM bytes (read + write) of one k_reg_periodic launch, from the same capture scaled by the
# pairs processed (64x for stride 8).
TRAFFIC_PER_LAUNCH = {"twolayer3072": 35.1e9}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="twolayer3072")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU baseline sampling")
    ap.add_argument("--e2e-steps", type=int, default=None, help="steps of the e2e leg (default: --steps)")
    ap.add_argument("--no-solve-stage", action="store_true", help="skip the separately timed solve stage")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-requests leg")
    ap.add_argument("--serve-requests", type=int, default=40)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--element-stride", type=int, default=1,
                    help="keep every S-th element of each domain's list: a smaller workload with the "
                         "same lattice, wavelength and element size, for profiler captures")
    return ap.parse_args()


# ---------------------------------------------------------------------------------------------
def class_counts(p):
    """Pairs per class as the reference's loop makes them (self pairs are t == s)."""
    out = {}
    for d in range(p.MN + 1):
        nodes = int(sum(p.nv[abs(t)] for t in p.sid[d]))
        total = nodes * len(p.sid[d])
        kind = "periodic" if (d == 0 and p.ps == 1) else "interior"
        out[(d, kind, "self")] = nodes
        out[(d, kind, "regular")] = total - nodes
    return out


def cpu_sample(files, p, budget, nthreads, seed=1234):
    """Times the reference on a stratified sample; returns (pairs/s extrapolated, description)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import reforacle
    if reforacle.have_ref():
        o = reforacle.RefOracle().load(*files)
        kind = "reference"
    else:
        raise RuntimeError("reference oracle library missing (oracle/_ref); run __graft_entry__.build()")
    rng = np.random.default_rng(seed)
    counts = class_counts(p)
    # budget split: most of the time goes where the work is
    share = {"regular": 0.7, "self": 0.3}
    per_pair = {}
    sampled = {}
    for (d, kd, cls), n in counts.items():
        if n == 0:
            continue
        ne = len(p.sid[d])
        b = budget * share[cls] * (0.8 if kd == "periodic" else 0.2) / (1 if p.MN == 0 else 1)
        m = max(nthreads, 8)
        done, spent = 0, 0.0
        while spent < b and done < 200000:
            quads = []
            for _ in range(m):
                t = int(rng.integers(1, ne + 1))
                tn = int(rng.integers(0, p.nv[abs(p.sid[d][t - 1])]))
                s = t if cls == "self" else int(rng.integers(1, ne + 1))
                while cls == "regular" and s == t:
                    s = int(rng.integers(1, ne + 1))
                quads.append((d, t, tn, s))
            t0 = time.perf_counter()
            o.pairs(np.array(quads, np.int32), nthreads)
            spent += time.perf_counter() - t0
            done += m
            if cls == "regular" and kd == "interior":
                m = min(m * 2, 65536)
        per_pair[(d, kd, cls)] = spent / done
        sampled[(d, kd, cls)] = done
    total_pairs = sum(counts.values())
    est = sum(counts[k] * per_pair[k] for k in per_pair)
    desc = "; ".join(f"d{d} {kd} {cls}: {sampled[(d, kd, cls)]} pairs, {per_pair[(d, kd, cls)] * 1e3:.4f} ms/pair"
                     for (d, kd, cls) in per_pair)
    return total_pairs / est, kind, desc, est


# ---------------------------------------------------------------------------------------------
class ClockSampler:
    def __init__(self, path):
        self.path = path
        self.proc = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self, gpu_index=0):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9 or c[0] != str(gpu_index):
                continue
            try:
                sm.append(float(c[1]))
                mx = max(mx, float(c[2]))
            except ValueError:
                continue
            for n, v in zip(names, c[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------------------------
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from bem3_emf_qd2_b200 import meshgen
    tmp = tempfile.mkdtemp(prefix="bem3ref_")
    p, files = meshgen.problem(args.config, tmp)
    nthreads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_sample(files, p, 0.5, nthreads, seed=7)
    vals, t_total = [], 0.0
    per_step = max(args.cpu_budget / max(args.steps, 1), 2.0)
    desc = kind = ""
    for k in range(args.steps):
        t0 = time.perf_counter()
        v, kind, desc, _ = cpu_sample(files, p, per_step, nthreads, seed=100 + k)
        t_total += time.perf_counter() - t0
        vals.append(v)
    value = float(np.mean(vals))
    pairs = sum(p.pairs_per_domain())
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": pairs / value * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": args.config, "pairs_per_step": pairs, "sample": "stratified by pair class"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": kind,
                         "sample": f"per step ~{per_step:.0f} s of sampled pairs ({desc})"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def ranks_timed(step, steps, warmup, dist, timer, device="cpu"):
    """W untimed steps, a barrier, then K timed steps on every rank; returns the time in ms, the
    maximum over ranks (the slowest rank bounds the whole job).  `timer(fn)` runs fn and returns
    its duration in ms (CUDA events on the GPU)."""
    import torch
    for _ in range(warmup):
        step()
    if dist:
        dist.barrier()
    ms = timer(lambda: [step() for _ in range(steps)])
    if dist:
        dist.barrier()
        t = torch.tensor([ms], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms


def whole_job_value(pairs_per_step, steps, world, ms):
    """Pairs per second of the whole job: every rank assembles its own instance."""
    return pairs_per_step * steps * world / (ms * 1e-3)


def hbm_peak_gbs():
    """The measured HBM copy bandwidth of this pool's B200s (MEASURED_PEAKS.json), else the stated
    fallback; returns (GB/s, source)."""
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            v = json.load(f).get("hbm_gbs")
        if v:
            return float(v), "MEASURED_PEAKS.json hbm_gbs"
    except (OSError, ValueError):
        pass
    return 6650.0, "fallback (earlier measurement on this pool)"


def solve_stage(B, meshgen, configs=("sphere384", "twolayer3072")):
    """The solve stage timed on its own (device time of bem3_ctx_solve's phases, CUDA events): the
    coefficient matrices of every domain, the factorisations (each domain's compacted G and the
    system of the potentials, dense LU in cuSOLVER), the right-hand sides with the boundary fields."""
    out = {}
    for name in configs:
        p, _ = meshgen.problem(name, tempfile.mkdtemp(prefix="bem3_solve_"))
        ctx = B.Context(p)
        ctx.solve()  # first solve loads the solver libraries' kernels; timed below
        ctx.solve()
        ph = ctx.phase_times()
        ctx.close()
        out[name] = {"unknowns_reduced_system": 4 * int(p.NN), **{k: round(v, 2) for k, v in ph.items()},
                     "solver": "reduced 4 NN system (Dirichlet-to-Neumann elimination), dense LU"}
    return out


def served(requests):
    """Served solves/s and p50/p99 latency (bem3_emf_qd2_b200.serve) on its seeded pool, against the
    same requests solved one at a time by the plain drop-in path."""
    from bem3_emf_qd2_b200 import serve
    pool_dir = tempfile.mkdtemp(prefix="bem3_pool_")
    meshes, probes = serve.mesh_pool(pool_dir)
    return serve.measure(meshes, probes, requests=requests, workers=8, budget_gb=120.0, load=0.8)


def run_ours(args):
    import torch
    import bem3_emf_qd2_b200 as B
    from bem3_emf_qd2_b200 import meshgen

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    tmp = tempfile.mkdtemp(prefix=f"bem3_{rank}_")
    p, files = meshgen.problem(args.config, tmp)
    workload = args.config
    if args.element_stride > 1:
        p.sid = [s[::args.element_stride].copy() for s in p.sid]
        workload = f"{args.config}/stride{args.element_stride}"
    dev = B.DeviceProblem(p)
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    domains = list(range(p.MN + 1))
    pairs = sum(p.pairs_per_domain())

    def step():
        for d in domains:
            dev.assemble(d, sptr)

    def cuda_timer(fn):
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        fn()
        ev1.record(stream)
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1)

    for _ in range(args.warmup):
        step()
    clocks = ClockSampler(os.path.join(tmp, "clocks.csv"))  # samples the timed steps only
    clocks.start()
    ms = ranks_timed(step, args.steps, 0, dist, cuda_timer, device="cuda")
    clk = clocks.stop(local)
    value = whole_job_value(pairs, args.steps, world, ms)

    # kernel launches per step and the roofline of the dominant kernel (profiling pass, not timed above)
    B.set_profiling(True)
    reg_ms, reg_launches, terms, per_step_launches, gh = 0.0, 0, 0, 0, 0
    counts = class_counts(p)
    classes = {}
    for d in domains:
        dev.assemble(d, sptr)
        st = B.last_stats()
        reg_ms += st["reg_periodic_ms"]
        reg_launches += st["reg_periodic_launches"]
        terms += st["qpgf_terms"]
        per_step_launches += st["launches"]
        gh += st["gh_pairs"]
        kd = "periodic" if (d == 0 and p.ps == 1) else "interior"
        ms_self, ms_reg, ms_gh, ms_sum = st["class_ms"]
        n_self = counts[(d, kd, "self")]
        n_reg = counts[(d, kd, "regular")]
        for cls, n, cms in ((f"{kd}_self", n_self, ms_self), (f"{kd}_regular", n_reg - st["gh_pairs"], ms_reg),
                            (f"{kd}_near_singular", st["gh_pairs"], ms_gh), ("row_sums", 0, ms_sum)):
            c = classes.setdefault(cls, {"pairs": 0, "ms": 0.0})
            c["pairs"] += int(n)
            c["ms"] += cms
    for c in classes.values():
        c["pairs_per_s"] = c["pairs"] / (c["ms"] * 1e-3) if c["pairs"] and c["ms"] > 0 else None
    B.set_profiling(False)
    peak = B.fp64_peak_tflops()
    roof = None
    if reg_launches:
        per_launch_ms = reg_ms / reg_launches
        terms_per_launch = terms / reg_launches
        ops = ALG_OPS_PER_TERM.get(args.config)
        hw = HW_OPS_PER_TERM.get(args.config)
        achieved = terms_per_launch * ops / (per_launch_ms * 1e-3) / 1e12 if ops else None
        roof = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak if achieved else None,
                "traffic": TRAFFIC_PER_LAUNCH.get(args.config), "kernel": "k_reg_periodic",
                "peak_source": "measured DFMA probe on this GPU (MEASURED_PEAKS.json has no FP64 entry)",
                "alg_ops_per_term": ops, "ops_basis": "oracle/opcount.py: restatement op count, seeded sample",
                "hw_ops_per_term": hw,
                "hw_frac": terms_per_launch * hw / (per_launch_ms * 1e-3) / 1e12 / peak if hw else None,
                "terms_per_s": terms_per_launch / (per_launch_ms * 1e-3)}
        roof["launch_ms"] = per_launch_ms
        roof["terms_per_launch"] = terms_per_launch

    # end to end through the host-pointer C ABI
    e2e = None
    if args.e2e_steps is None:
        args.e2e_steps = args.steps
    if args.e2e_steps > 0:
        h2d = d2h = 0
        # the caller's result arrays, page-locked, allocated once (outside the timed region)
        outs = {d: B.domain_outputs(p, d, pinned=True) for d in domains}
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.e2e_steps):
            # every domain in one call (the reference's create_cmatrix): each domain's copies overlap
            # the later domains' kernels
            M = B.assemble_domains(p, out=outs)
            if _ == 0:
                h2d += (p.Ne + 1) * 48 * 8
                for d in domains:
                    d2h += sum(M[d][k].nbytes for k in ("G", "H", "dG", "dH", "dF"))
                    h2d += len(p.sid[d]) * 4
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1)
        e2e = {"value": pairs * args.e2e_steps / (ems * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h}

    # the matrix write-out: bytes the assembly stores per step (G, H, dG, dH, dF of every domain, the
    # reference's layout) over the step's device time, against the HBM roofline
    peak_hbm, hbm_src = hbm_peak_gbs()
    wbytes = sum(16 * 6 * (4 * len(s)) ** 2 + 24 * 4 * len(s) for s in p.sid)
    wgbs = wbytes / (ms / args.steps * 1e-3) / 1e9
    matrix_write = {"bytes_per_step": wbytes, "gbs": wgbs, "peak_gbs": peak_hbm, "frac": wgbs / peak_hbm,
                    "peak_source": hbm_src,
                    "note": "average over the step; the assembly is FP64-bound, the write-out is not the limit"}

    solve = None
    if rank == 0 and not args.no_solve_stage and args.element_stride == 1:
        try:
            solve = solve_stage(B, meshgen)
        except Exception as ex:  # reported, never required
            solve = {"error": str(ex)[:300]}
    serve_line = None
    if rank == 0 and world == 1 and not args.no_serve and args.element_stride == 1:
        try:
            serve_line = served(args.serve_requests)
        except Exception as ex:
            serve_line = {"error": str(ex)[:300]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            nth = os.cpu_count() or 1
            v, kind, desc, _ = cpu_sample(files, p, args.cpu_budget, nth)
            cpu = {"value": v, "unit": UNIT, "cores": nth, "kind": kind,
                   "sample": f"~{args.cpu_budget:.0f} s stratified sample of the same pairs ({desc})"}
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"unavailable: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded cube-sphere meshes)",
            "config": {"workload": workload, "pairs_per_step": pairs, "domains": len(domains),
                       "elements": int(p.Ne), "gh_pairs_per_step": gh,
                       "l2": "each step writes %.1f GB of matrices (> 126 MB L2); no state carried in L2"
                             % (sum(16 * 6 * (4 * len(s)) ** 2 for s in p.sid) / 1e9),
                       "parallelism": f"{world} independent instances (one per GPU)"},
            "gpu_launches": per_step_launches * args.steps,
            "roofline": roof, "e2e": e2e, "cpu_baseline": cpu, "clocks": clk,
            "classes": classes, "matrix_write": matrix_write, "solve_stage": solve, "served": serve_line,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)
