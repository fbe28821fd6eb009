"""bem3_emf_qd2_b200 -- B200 (sm_100a, FP64) boundary-integral hot path of bem3_emf_qd2.

The compute runs in the CUDA library ``_lib/libbem3qd2.so`` (sources in ``csrc/``, C ABI in
``include/bem3_qd2_b200.h``).  This module loads it with ctypes and offers numpy-level calls
that mirror the reference's operator interface for the path:

* ``qpgf(qd, r)``                       -- d3hm_qpgf_d2_v1 over many points (qgf2_src/d3_qpgf_d2.c:124)
* ``assemble_domain(problem, did)``      -- create_cmatrix_domain (d3qd2_src/d3qd2_solve_bieq.c:165)

There is no CPU fallback: if the library is missing or no CUDA device is present the calls
raise ``RuntimeError``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from .dqd2 import Problem  # noqa: F401  (re-exported)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libbem3qd2.so")
REPO = os.path.dirname(HERE)

# --default-stream per-thread: work the library issues without an explicit stream goes to the calling
# host thread's own default stream, so contexts driven from different threads overlap on the GPU.
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "--default-stream", "per-thread", "-diag-suppress", "20091", "-Xcompiler", "-fPIC", "-shared"]

ERRORS = {
    -1: "invalid argument", -2: "CUDA failure", -3: "scratch too small", -4: "degenerate lattice",
    -5: "singular system", -900: "near-singular work list overflow",
}


def build(verbose: bool = False) -> str:
    """Compile the CUDA library in-tree for sm_100a (nvcc cross-compiles without a GPU)."""
    os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
    src = os.path.join(HERE, "csrc", "bem3_lib.cu")
    cmd = ["nvcc", *NVCC_FLAGS, "-I" + os.path.join(REPO, "include"), "-I" + os.path.join(HERE, "csrc"),
           src, "-o", LIB_PATH, "-lcusolver", "-lcublas"]
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + out.stdout[-6000:] + out.stderr[-6000:])
    if verbose:
        print(out.stdout + out.stderr)
    return LIB_PATH


class bem3_qpd2(C.Structure):
    _fields_ = [("k", C.c_double), ("vk", C.c_double * 3), ("vd1", C.c_double * 2), ("vd2", C.c_double * 2)]


class bem3_mesh(C.Structure):
    _fields_ = [("Ne", C.c_int), ("cr", C.c_void_p), ("cw", C.c_void_p), ("ren", C.c_void_p),
                ("wen", C.c_void_p), ("nv", C.c_void_p)]


class bem3_wave(C.Structure):
    _fields_ = [("E0", C.c_double), ("ki", C.c_double), ("cos_t", C.c_double), ("sin_t", C.c_double),
                ("cos_p", C.c_double), ("sin_p", C.c_double), ("f", C.c_double * 3), ("e", C.c_double * 6),
                ("h", C.c_double * 6)]


class bem3_problem(C.Structure):
    _fields_ = [("MN", C.c_int), ("Ne", C.c_int), ("NN", C.c_int), ("ps", C.c_int), ("mesh", bem3_mesh),
                ("md", C.c_void_p), ("sd", C.c_void_p), ("eni", C.c_void_p), ("Ne_d", C.c_void_p),
                ("sid", C.c_void_p), ("kn", C.c_void_p), ("qd", bem3_qpd2), ("lambda0", C.c_double),
                ("Ui", C.c_void_p), ("dUi", C.c_void_p), ("dEiz", C.c_void_p), ("dEie", C.c_void_p),
                ("Nn", C.c_int), ("rn", C.c_void_p), ("ed", C.c_void_p), ("nwaves", C.c_int),
                ("waves", C.c_void_p)]


class bem3_bv(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("U", "dU", "E", "dE", "H", "dH")]


class bem3_stats(C.Structure):
    _fields_ = [("gh_pairs", C.c_ulonglong), ("qpgf_terms", C.c_ulonglong), ("launches", C.c_int),
                ("reg_periodic_launches", C.c_int), ("reg_periodic_ms", C.c_double),
                ("class_ms", C.c_double * 4)]


class bem3_batch_domain(C.Structure):
    _fields_ = [("geo", C.c_void_p), ("Ne", C.c_int), ("sid", C.c_void_p), ("Ne_d", C.c_int), ("did", C.c_int),
                ("periodic", C.c_int), ("qd", bem3_qpd2), ("kre", C.c_double), ("kim", C.c_double),
                ("G", C.c_void_p), ("H", C.c_void_p), ("dG", C.c_void_p), ("dH", C.c_void_p), ("dF", C.c_void_p)]


class bem3_batch_tuning(C.Structure):
    _fields_ = [("grab_units", C.c_int), ("regp_blocks_per_sm", C.c_int), ("gh_blocks_per_sm", C.c_int)]


_lib = None


def lib():
    """The loaded CUDA library (raises if it is not built)."""
    global _lib
    if _lib is None:
        # BEM3_QD2_LIB: another build of the same library (e.g. a variant compiled with other -D options)
        path = os.environ.get("BEM3_QD2_LIB", LIB_PATH)
        if not os.path.exists(path):
            raise RuntimeError(f"CUDA library not built: {path} (run bem3_emf_qd2_b200.build())")
        L = C.CDLL(path)
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        L.bem3_qpgf.argtypes = [C.POINTER(bem3_qpd2), i, vp, vp, vp, i]
        L.bem3_qpgf_dev.argtypes = [C.POINTER(bem3_qpd2), i, vp, vp, vp, i, vp]
        L.bem3_assemble_domain.argtypes = [C.POINTER(bem3_mesh), vp, i, i, i, C.POINTER(bem3_qpd2), d, d,
                                           vp, vp, vp, vp, vp]
        L.bem3_assemble_domain_dev.argtypes = [vp, i, vp, i, i, i, C.POINTER(bem3_qpd2), d, d, vp, vp, vp, vp, vp, vp]
        L.bem3_pack_geometry.argtypes = [C.POINTER(bem3_mesh), vp]
        L.bem3_mesh_pack_dev.argtypes = [i, i, vp, vp, vp, vp]
        L.bem3_assemble_domains.argtypes = [C.POINTER(bem3_mesh), i, vp, vp, i, C.POINTER(bem3_qpd2), vp, vp, vp, vp,
                                            vp, vp]
        L.bem3_solve_bieq_arrays.argtypes = [C.POINTER(bem3_problem), C.POINTER(bem3_bv)]
        L.bem3_ctx_create.argtypes = [C.POINTER(bem3_problem), C.POINTER(C.c_void_p)]
        L.bem3_ctx_destroy.argtypes = [vp]
        L.bem3_ctx_destroy.restype = None
        L.bem3_ctx_solve.argtypes = [vp]
        L.bem3_ctx_set_solver.argtypes = [vp, i]
        L.bem3_ctx_set_incident.argtypes = [vp, i, vp, vp, vp, vp, vp]
        L.bem3_ctx_resolve.argtypes = [vp]
        L.bem3_ctx_phase_times.argtypes = [vp, vp]
        L.bem3_ctx_prepare.argtypes = [vp, vp]
        L.bem3_ctx_solve_prepared.argtypes = [vp]
        L.bem3_ctx_release.argtypes = [vp]
        L.bem3_ctx_device_bytes.argtypes = [vp]
        L.bem3_ctx_device_bytes.restype = C.c_size_t
        L.bem3_ctx_get_bv.argtypes = [vp, C.POINTER(bem3_bv)]
        L.bem3_ctx_set_bv.argtypes = [vp, C.POINTER(bem3_bv)]
        L.bem3_ctx_domain_id.argtypes = [vp, i, vp, vp]
        L.bem3_ctx_field.argtypes = [vp, i, vp, i, i, vp, vp, vp]
        L.bem3_ctx_potential.argtypes = [vp, i, vp, i, i, vp, vp]
        L.bem3_ctx_field_memp.argtypes = [vp, i, vp, i, i, vp, vp, vp]
        L.bem3_ctx_force.argtypes = [vp, vp, i, vp, vp]
        L.bem3_geo_stride.restype = i
        L.bem3_last_gh_pairs.restype = C.c_ulonglong
        L.bem3_gauss_legendre.argtypes = [i, vp, vp]
        L.bem3_version.restype = C.c_char_p
        L.bem3_set_profiling.argtypes = [i]
        L.bem3_last_stats.argtypes = [C.POINTER(bem3_stats)]
        L.bem3_fp64_peak_tflops.restype = d
        L.bem3_batch_scratch_bytes.argtypes = [C.POINTER(bem3_batch_domain), i]
        L.bem3_batch_scratch_bytes.restype = C.c_size_t
        L.bem3_batch_create.argtypes = [C.POINTER(bem3_batch_domain), i, C.POINTER(bem3_batch_tuning),
                                        C.POINTER(C.c_void_p)]
        L.bem3_batch_run.argtypes = [vp, vp]
        L.bem3_batch_wait.argtypes = [vp, vp, vp]
        L.bem3_batch_info.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_size_t)]
        L.bem3_batch_destroy.argtypes = [vp]
        _lib = L
    return _lib


def check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what} failed: {rc} ({ERRORS.get(rc, 'quasi-periodic Green function failure')})")


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def make_qpd(qpd: dict) -> bem3_qpd2:
    q = bem3_qpd2()
    q.k = qpd["k"]
    for j in range(3):
        q.vk[j] = qpd["vk"][j]
    for j in range(2):
        q.vd1[j] = qpd["vd1"][j]
        q.vd2[j] = qpd["vd2"][j]
    return q


def qpgf(qpd: dict, r: np.ndarray, mode: int = 0):
    """Green's function and gradient at points r[n,3].  Returns (out[n,4] complex, ret[n])."""
    r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 3)
    n = len(r)
    out = np.zeros((n, 4), np.complex128)
    ret = np.zeros(n, np.int32)
    q = make_qpd(qpd)
    check(lib().bem3_qpgf(C.byref(q), n, _ptr(r), _ptr(out), _ptr(ret), mode), "bem3_qpgf")
    return out, ret


class MeshArrays:
    """Keeps the flattened mesh arrays alive while a bem3_mesh points at them."""

    def __init__(self, problem: Problem):
        self.cr, self.cw, self.ren, self.wen, self.nv = problem.flat_mesh()
        self.m = bem3_mesh(problem.Ne, _ptr(self.cr), _ptr(self.cw), _ptr(self.ren), _ptr(self.wen), _ptr(self.nv))

    def packed(self) -> np.ndarray:
        stride = lib().bem3_geo_stride()
        geo = np.zeros((self.m.Ne + 1) * stride)
        check(lib().bem3_pack_geometry(C.byref(self.m), _ptr(geo)), "bem3_pack_geometry")
        return geo


def mesh_pack_dev(rn, ed, stream=None):
    """Geometry records of a mesh computed on the device (bem3_mesh_pack_dev): rn [Nn + 1, 3] float64
    and ed [Ne + 1, 4] int32 torch tensors on the GPU (the reference's node table and element vertex
    lists); returns the [(Ne + 1) * stride] float64 device tensor that bem3_pack_geometry would give."""
    import torch
    if rn.dtype != torch.float64 or ed.dtype != torch.int32 or not rn.is_cuda or not ed.is_cuda:
        raise ValueError("rn must be float64 and ed int32, both on the GPU")
    rn, ed = rn.contiguous(), ed.contiguous()
    ne, nn = ed.shape[0] - 1, rn.shape[0] - 1
    geo = torch.empty((ne + 1) * lib().bem3_geo_stride(), dtype=torch.float64, device=rn.device)
    st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    check(lib().bem3_mesh_pack_dev(ne, nn, C.c_void_p(rn.data_ptr()), C.c_void_p(ed.data_ptr()),
                                   C.c_void_p(geo.data_ptr()), C.c_void_p(st)), "bem3_mesh_pack_dev")
    return geo


def domain_outputs(problem: Problem, did: int, derivatives: bool = True, pinned: bool = False) -> dict:
    """Host arrays for assemble_domain's outputs (page-locked when `pinned`, through torch, so that
    the library's row-chunk copies run asynchronously)."""
    N = 4 * len(problem.sid[did])
    shapes = dict(G=(N, N), H=(N, N), dF=(N, 3))
    if derivatives:
        shapes.update(dG=(2 * N, N), dH=(2 * N, N))
    out = {}
    for k, shp in shapes.items():
        dt = np.float64 if k == "dF" else np.complex128
        if pinned:
            import torch
            t = torch.empty(shp, dtype=torch.float64 if k == "dF" else torch.complex128, pin_memory=True)
            out[k] = t.numpy()
            out["_" + k] = t  # keeps the page-locked allocation alive
        else:
            out[k] = np.zeros(shp, dt)
    if not derivatives:
        out["dG"] = out["dH"] = None
    return out


def assemble_domain(problem: Problem, did: int, derivatives: bool = True, out: dict = None):
    """Coefficient matrices of domain `did` on the GPU (host in, host out).

    Returns dict G, H [N,N], dG, dH [2N,N] (complex), dF [N,3] with N = 4 Ne_d, in the layout of
    the reference's temp files (d3qd2_solve_bieq.c:213-236).  `out` (from domain_outputs) supplies
    the arrays to fill instead of new ones."""
    sid = np.ascontiguousarray(problem.sid[did], dtype=np.int32)
    ne = len(sid)
    o = out if out is not None else domain_outputs(problem, did, derivatives)
    G, H, dG, dH, dF = o["G"], o["H"], o["dG"], o["dH"], o["dF"]
    ma = MeshArrays(problem)
    q = make_qpd(problem.qpd)
    periodic = 1 if (did == 0 and problem.ps == 1) else 0
    k = complex(problem.kn[did])
    rc = lib().bem3_assemble_domain(C.byref(ma.m), _ptr(sid), ne, did, periodic, C.byref(q), k.real, k.imag,
                                    _ptr(G), _ptr(H), _ptr(dG) if dG is not None else None,
                                    _ptr(dH) if dH is not None else None, _ptr(dF))
    check(rc, "bem3_assemble_domain")
    return dict(G=G, H=H, dG=dG, dH=dH, dF=dF, gh_pairs=int(lib().bem3_last_gh_pairs()))


def assemble_domains(problem: Problem, derivatives: bool = True, out: dict = None):
    """Coefficient matrices of every domain in one call (bem3_assemble_domains: the reference's
    create_cmatrix, the loop of create_cmatrix_domain over the domains), the copies of each domain's
    matrices overlapping the later domains' kernels.  Returns {did: dict as assemble_domain};
    `out` maps did to arrays from domain_outputs."""
    nd = problem.MN + 1
    outs = out if out is not None else {d: domain_outputs(problem, d, derivatives) for d in range(nd)}
    sids = [np.ascontiguousarray(problem.sid[d], dtype=np.int32) for d in range(nd)]
    ne = np.array([len(s) for s in sids], np.int32)
    kn = np.array([[complex(problem.kn[d]).real, complex(problem.kn[d]).imag] for d in range(nd)], np.float64)
    P = C.c_void_p * nd

    def ptrs(key):
        return P(*[(_ptr(outs[d][key]).value if outs[d][key] is not None else None) for d in range(nd)])

    ma = MeshArrays(problem)
    q = make_qpd(problem.qpd)
    sid_p = P(*[_ptr(s).value for s in sids])
    G, H, dG, dH, dF = ptrs("G"), ptrs("H"), ptrs("dG"), ptrs("dH"), ptrs("dF")
    rc = lib().bem3_assemble_domains(C.byref(ma.m), problem.MN, sid_p, _ptr(ne), 1 if problem.ps == 1 else 0,
                                     C.byref(q), _ptr(kn), G, H, dG, dH, dF)
    check(rc, "bem3_assemble_domains")
    return {d: dict(G=outs[d]["G"], H=outs[d]["H"], dG=outs[d]["dG"], dH=outs[d]["dH"], dF=outs[d]["dF"])
            for d in range(nd)}


class ProblemArrays:
    """A bem3_problem over arrays kept alive by this object."""

    def __init__(self, problem: Problem):
        p = problem
        self.ma = MeshArrays(p)
        self.md = np.ascontiguousarray(p.md, dtype=np.int32)
        self.sd = np.ascontiguousarray(p.sd, dtype=np.int32)
        self.eni = np.ascontiguousarray(p.eni, dtype=np.int32)
        self.ne_d = np.array([len(s) for s in p.sid], np.int32)
        self.sids = [np.ascontiguousarray(s, dtype=np.int32) for s in p.sid]
        self.sid_ptrs = (C.c_void_p * len(self.sids))(*[s.ctypes.data for s in self.sids])
        self.kn = np.ascontiguousarray(np.array(p.kn, np.complex128))
        self.Ui = np.ascontiguousarray(p.Ui)
        self.dUi = np.ascontiguousarray(p.dUi)
        dEz, dEe = p.incident_tangent_derivatives()
        self.dEiz = np.ascontiguousarray(dEz)
        self.dEie = np.ascontiguousarray(dEe)
        self.rn = np.ascontiguousarray(p.rn, dtype=np.float64)
        self.ed = np.ascontiguousarray(p.ed, dtype=np.int32)
        self.waves = (bem3_wave * len(p.waves))()
        for j, w in enumerate(p.waves):
            W = self.waves[j]
            W.E0, W.ki, W.cos_t, W.sin_t, W.cos_p, W.sin_p = w.E0, w.ki, w.cos_t, w.sin_t, w.cos_p, w.sin_p
            for l in range(3):
                W.f[l] = w.f[l]
            for l, (ev, hv) in enumerate(((w.ex, w.hx), (w.ey, w.hy), (w.ez, w.hz))):
                W.e[2 * l], W.e[2 * l + 1] = complex(ev).real, complex(ev).imag
                W.h[2 * l], W.h[2 * l + 1] = complex(hv).real, complex(hv).imag
        self.s = bem3_problem(p.MN, p.Ne, p.NN, p.ps, self.ma.m, _ptr(self.md), _ptr(self.sd), _ptr(self.eni),
                              _ptr(self.ne_d), C.cast(self.sid_ptrs, C.c_void_p), _ptr(self.kn), make_qpd(p.qpd),
                              p.lambda0, _ptr(self.Ui), _ptr(self.dUi), _ptr(self.dEiz), _ptr(self.dEie),
                              self.rn.shape[0] - 1, _ptr(self.rn), _ptr(self.ed), len(p.waves),
                              C.cast(self.waves, C.c_void_p))


def _bv_arrays(problem: Problem):
    out = []
    bvs = (bem3_bv * (problem.MN + 1))()
    for d in range(problem.MN + 1):
        ne = len(problem.sid[d])
        r = dict(U=np.zeros((ne + 1, 4, 4), np.complex128), dU=np.zeros((ne + 1, 4, 4), np.complex128))
        for k in ("E", "dE", "H", "dH"):
            r[k] = np.zeros((ne + 1, 4, 3), np.complex128)
        for k, v in r.items():
            setattr(bvs[d], k, v.ctypes.data)
        out.append(r)
    return out, bvs


def plane_power(field, vd1, vd2, upward: bool, z_top: float, z_bottom: float, n: int = 16):
    """Time-averaged power through one unit cell of the lattice, from the fields on the planes
    z = z_top (above the objects) and z = z_bottom (below), each sampled on an n x n grid of the
    cell and integrated with the midpoint rule (spectrally accurate: Re(E x H*) is periodic and
    smooth away from the objects).  field(r, total) -> (E, H, did) evaluates EH_t (total) or EH_s.
    Returns P_inc (incident field through the entry plane), P_ref (scattered field leaving
    through the entry plane), P_tra (total field leaving through the other plane) and
    balance = (P_ref + P_tra) / P_inc, which is 1 for lossless objects.  The Poynting vector is
    Re(E x H*) / 2 in the units of E and H."""
    d1 = np.array([vd1[0], vd1[1], 0.0])
    d2 = np.array([vd2[0], vd2[1], 0.0])
    u = (np.arange(n) + 0.5) / n
    grid = (u[:, None, None] * d1 + u[None, :, None] * d2).reshape(-1, 3)
    area = abs(d1[0] * d2[1] - d1[1] * d2[0])

    def fields(z, total):
        E, H, did = field(grid + np.array([0.0, 0.0, z]), total)
        if np.any(np.asarray(did) != 0):
            raise ValueError("the planes must lie in the open region")
        return E, H

    def flux(E, H):
        return (0.5 * (E[:, 0] * np.conj(H[:, 1]) - E[:, 1] * np.conj(H[:, 0])).real).mean() * area

    up = 1.0 if upward else -1.0  # the incident wave travels along +z or -z
    zin, zout = (z_bottom, z_top) if upward else (z_top, z_bottom)
    Et, Ht = fields(zin, True)
    Es, Hs = fields(zin, False)
    P_inc = up * flux(Et - Es, Ht - Hs)
    P_ref = -up * flux(Es, Hs)
    P_tra = up * flux(*fields(zout, True))
    return dict(P_inc=P_inc, P_ref=P_ref, P_tra=P_tra, balance=(P_ref + P_tra) / P_inc)


class Context:
    """A problem resident on the current CUDA device (bem3_ctx): solve, boundary values, fields."""

    def __init__(self, problem: Problem):
        self.p = problem
        self.pa = ProblemArrays(problem)
        self.h = C.c_void_p()
        check(lib().bem3_ctx_create(C.byref(self.pa.s), C.byref(self.h)), "bem3_ctx_create")

    def close(self) -> None:
        if self.h:
            lib().bem3_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, method: int = 0) -> None:
        """method 0: reduced 4 NN system where applicable, 1: the full 8 NN system, 2: reduced only."""
        check(lib().bem3_ctx_set_solver(self.h, method), "bem3_ctx_set_solver")
        check(lib().bem3_ctx_solve(self.h), "bem3_ctx_solve")

    def prepare(self) -> list:
        """Allocates this context's matrices for an assembly outside the solve (bem3_ctx_prepare) and
        returns every domain's bem3_batch_domain entry, to be assembled by a batch; then
        solve_prepared() finishes the solve."""
        arr = (bem3_batch_domain * (self.p.MN + 1))()
        check(lib().bem3_ctx_prepare(self.h, arr), "bem3_ctx_prepare")
        return [arr[i] for i in range(self.p.MN + 1)]

    def solve_prepared(self) -> None:
        """The solve after an external assembly of prepare()'s entries -- bem3_ctx_solve_prepared."""
        check(lib().bem3_ctx_solve_prepared(self.h), "bem3_ctx_solve_prepared")

    def phase_times(self) -> dict:
        """Device time (ms) of the last solve's phases -- bem3_ctx_phase_times: the coefficient
        matrices, the factorisations, the right-hand sides with the boundary fields."""
        ms = (C.c_double * 3)()
        check(lib().bem3_ctx_phase_times(self.h, ms), "bem3_ctx_phase_times")
        return dict(assembly_ms=ms[0], factor_ms=ms[1], rhs_fields_ms=ms[2])

    def set_incident(self, waves) -> None:
        """Replace the incident plane waves (same wavelength and direction as the solved ones; the
        matrices and factorisations stay valid) -- bem3_ctx_set_incident."""
        q = self.p.with_waves(waves)
        pa = ProblemArrays(q)
        check(lib().bem3_ctx_set_incident(self.h, len(q.waves), C.cast(pa.waves, C.c_void_p), _ptr(pa.Ui),
                                          _ptr(pa.dUi), _ptr(pa.dEiz), _ptr(pa.dEie)), "bem3_ctx_set_incident")
        self.p = q

    def resolve(self) -> None:
        """Boundary values for the current incident field with the resident factorisations."""
        check(lib().bem3_ctx_resolve(self.h), "bem3_ctx_resolve")

    def release(self) -> None:
        check(lib().bem3_ctx_release(self.h), "bem3_ctx_release")

    def device_bytes(self) -> int:
        return int(lib().bem3_ctx_device_bytes(self.h))

    def boundary_values(self):
        out, bvs = _bv_arrays(self.p)
        check(lib().bem3_ctx_get_bv(self.h, bvs), "bem3_ctx_get_bv")
        return out

    def set_boundary_values(self, bv) -> None:
        keep, bvs = [], (bem3_bv * (self.p.MN + 1))()
        for d in range(self.p.MN + 1):
            for k in ("U", "dU", "E", "dE", "H", "dH"):
                a = np.ascontiguousarray(bv[d][k], dtype=np.complex128)
                keep.append(a)
                setattr(bvs[d], k, a.ctypes.data)
        check(lib().bem3_ctx_set_bv(self.h, bvs), "bem3_ctx_set_bv")

    def domain_id(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 3)
        did = np.zeros(len(r), np.int32)
        check(lib().bem3_ctx_domain_id(self.h, len(r), _ptr(r), _ptr(did)), "bem3_ctx_domain_id")
        return did

    def force(self, rc=(0.0, 0.0, 0.0), type_: int = 0):
        """Radiation force F[3] and torque N[3] about rc (force_FN)."""
        rc = np.ascontiguousarray(rc, dtype=np.float64)
        F = np.zeros(3)
        N = np.zeros(3)
        check(lib().bem3_ctx_force(self.h, _ptr(rc), type_, _ptr(F), _ptr(N)), "bem3_ctx_force")
        return F, N

    def power(self, z_top: float, z_bottom: float, n: int = 16, type_: int = 0):
        """Reflected and transmitted power through one unit cell (plane_power) from this context's
        fields."""
        p = self.p
        return plane_power(lambda r, total: self.field(r, type_, total), p.vd1, p.vd2, p.waves[0].cos_t > 0,
                           z_top, z_bottom, n)

    def field(self, r, type_: int = 0, total=True):
        """E, H [n,3] complex and the domain of each point: EH_t (total True / 1), EH_s (False / 0)
        or EH_i (2, the incident field alone)."""
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 3)
        E = np.zeros((len(r), 3), np.complex128)
        H = np.zeros((len(r), 3), np.complex128)
        did = np.zeros(len(r), np.int32)
        check(lib().bem3_ctx_field(self.h, len(r), _ptr(r), type_, int(total), _ptr(E), _ptr(H), _ptr(did)),
              "bem3_ctx_field")
        return E, H, did

    def field_memp(self, r, type_: int = 0, total=True):
        """E, H [n,3] from the derivatives of the potentials (EH_mEMP_t / _s / _i for total
        True or 1 / 0 / 2) and the domain of each point (negative where the point is too close
        to the boundary for these rules)."""
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 3)
        E = np.zeros((len(r), 3), np.complex128)
        H = np.zeros((len(r), 3), np.complex128)
        did = np.zeros(len(r), np.int32)
        check(lib().bem3_ctx_field_memp(self.h, len(r), _ptr(r), type_, int(total), _ptr(E), _ptr(H), _ptr(did)),
              "bem3_ctx_field_memp")
        return E, H, did

    def potential(self, r, type_: int = 0, total=True):
        """Modified electromagnetic potentials U [n,4] complex (vector potential, scalar potential)
        and the domain of each point: mEMP_t (total True / 1), mEMP_s (0) or mEMP_i (2)."""
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 3)
        U = np.zeros((len(r), 4), np.complex128)
        did = np.zeros(len(r), np.int32)
        check(lib().bem3_ctx_potential(self.h, len(r), _ptr(r), type_, int(total), _ptr(U), _ptr(did)),
              "bem3_ctx_potential")
        return U, did


def solve_bieq(problem: Problem):
    """Boundary values of every domain (solve_bieq, d3qd2_src/d3qd2_solve_bieq.c:36-84) on the GPU.

    Returns a list over domains 0..MN of dicts U, dU [(Ne_d+1),4,4] and E, H, dE, dH
    [(Ne_d+1),4,3] (complex, slot 0 unused), the arrays SUBD holds (d3qd2_elem.h:13-20)."""
    pa = ProblemArrays(problem)
    out, bvs = _bv_arrays(problem)
    check(lib().bem3_solve_bieq_arrays(C.byref(pa.s), bvs), "bem3_solve_bieq_arrays")
    return out


def gauss_legendre(n: int):
    x = np.zeros(n)
    w = np.zeros(n)
    lib().bem3_gauss_legendre(n, _ptr(x), _ptr(w))
    return x, w


def last_stats() -> dict:
    st = bem3_stats()
    lib().bem3_last_stats(C.byref(st))
    out = {f: getattr(st, f) for f, _ in bem3_stats._fields_}
    out["class_ms"] = list(out["class_ms"])
    return out


def set_profiling(on: bool) -> None:
    lib().bem3_set_profiling(1 if on else 0)


def fp64_peak_tflops() -> float:
    return float(lib().bem3_fp64_peak_tflops())


class DeviceProblem:
    """Geometry resident in HBM plus output buffers sized for the largest domain (torch tensors
    used as device allocations only).  ``assemble(did, stream)`` runs one domain through
    bem3_assemble_domain_dev."""

    def __init__(self, problem: Problem, device="cuda"):
        import torch
        self.p = problem
        ma = MeshArrays(problem)
        self.geo = torch.from_numpy(ma.packed()).to(device)
        self.sids = [torch.from_numpy(np.ascontiguousarray(s, dtype=np.int32)).to(device) for s in problem.sid]
        nmax = max(4 * len(s) for s in problem.sid)
        self.G = torch.empty((nmax, nmax), dtype=torch.complex128, device=device)
        self.H = torch.empty_like(self.G)
        self.dG = torch.empty((2 * nmax, nmax), dtype=torch.complex128, device=device)
        self.dH = torch.empty_like(self.dG)
        self.dF = torch.empty((nmax, 3), dtype=torch.float64, device=device)
        self.q = make_qpd(problem.qpd)

    def assemble(self, did: int, stream=None) -> None:
        k = complex(self.p.kn[did])
        ne = len(self.p.sid[did])
        periodic = 1 if (did == 0 and self.p.ps == 1) else 0
        rc = lib().bem3_assemble_domain_dev(self.geo.data_ptr(), self.p.Ne, self.sids[did].data_ptr(), ne, did,
                                            periodic, C.byref(self.q), k.real, k.imag, self.G.data_ptr(),
                                            self.H.data_ptr(), self.dG.data_ptr(), self.dH.data_ptr(),
                                            self.dF.data_ptr(), stream)
        check(rc, "bem3_assemble_domain_dev")
