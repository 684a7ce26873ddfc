"""voluma_b200 — B200-native pressure-equation hot path of Voluma behind its FvMatrix::solve /
solver-dictionary interface.

The product is the C-ABI library built from voluma_b200/csrc (include/voluma_b200.h).  This
module is the Python host side over that ABI, with the reference's names:

    SolverControls      <- cfd::SolverControls      (src/fvm/linalg/LinearSolver.h:15-23)
    SolverPerformance   <- cfd::SolverPerformance   (src/fvm/linalg/LinearSolver.h:25-31)
    Mesh                <- the cfd::Mesh arrays the solver needs, registered on the device
    solve_ldu           <- cfd::solveLdu            (src/fvm/linalg/LinearSolver.cpp:135)
    amul                <- cfd::amul                (src/fvm/linalg/LinearSolver.cpp:121)

Errors follow the reference: an unknown solver/preconditioner or PCG on an asymmetric matrix
raises (LinearSolver.cpp:76,177,280), a singular coarsest GAMG matrix raises (GAMG.cpp:336),
non-convergence only clears `converged`.
"""
from __future__ import annotations

import atexit
import os
import ctypes as C
import weakref
from dataclasses import dataclass

import numpy as np

from . import _ffi
from ._ffi import VlmError, check, load

__all__ = ["SolverControls", "SolverPerformance", "Context", "Mesh", "solve_ldu", "amul", "VlmError", "load"]


@dataclass
class SolverControls:
    """The solver dictionary (LinearSolver.h:15-23) plus additive device keys."""
    solver: str = "PCG"
    preconditioner: str = "diagonal"
    tolerance: float = 1e-8
    relTol: float = 0.0
    maxIter: int = 1000
    minIter: int = 0
    nSweeps: int = 1
    smoother: str = ""          # GAMG smoother: "" / "mcgs-jacobi" | "mcgs" | "jacobi"
    precision: str = ""         # "" / "fp64" | "mixed"
    reproducible: bool = False  # CFD_REPRODUCIBLE semantics
    mergeLevels: int = 0
    innerRelTol: float = 0.0

    def to_c(self) -> _ffi.SolverCtrl:
        c = _ffi.SolverCtrl()
        c.solver = self.solver.encode()
        c.preconditioner = self.preconditioner.encode()
        c.tolerance = self.tolerance
        c.relTol = self.relTol
        c.maxIter = self.maxIter
        c.minIter = self.minIter
        c.nSweeps = self.nSweeps
        c.smoother = self.smoother.encode()
        c.precision = self.precision.encode()
        c.reproducible = 1 if self.reproducible else 0
        c.mergeLevels = self.mergeLevels
        c.innerRelTol = self.innerRelTol
        return c


@dataclass
class SolverPerformance:
    solver: str = ""
    field: str = ""
    initialResidual: float = 0.0
    finalResidual: float = 0.0
    residualSum: float = 0.0
    normFactor: float = 0.0
    iterations: int = 0
    converged: bool = False
    outerIterations: int = 0
    status: int = 0

    @classmethod
    def from_c(cls, p: _ffi.SolverPerf) -> "SolverPerformance":
        return cls(solver=p.solver.decode(), initialResidual=p.initialResidual, finalResidual=p.finalResidual,
                   residualSum=p.residualSum, normFactor=p.normFactor, iterations=p.iterations,
                   converged=bool(p.converged), outerIterations=p.outerIterations, status=p.status)


def _ptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Context:
    """One CUDA device + stream (vlm_ctx)."""

    def __init__(self, device: int = 0):
        L = load()
        h = C.c_void_p()
        check(L.vlm_ctx_create(device, C.byref(h)))
        self._h = h
        _live.add(self)

    @property
    def handle(self):
        return self._h

    def stream(self) -> int:
        return load().vlm_ctx_stream(self._h) or 0

    def device_name(self) -> str:
        buf = C.create_string_buffer(256)
        check(load().vlm_ctx_device_name(self._h, buf, 256), self._h)
        return buf.value.decode()

    def close(self):
        if getattr(self, "_h", None):
            load().vlm_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = None
_live = weakref.WeakSet()  # meshes/contexts still holding native handles


@atexit.register
def _release_all():
    # release meshes before contexts while the interpreter (and the CUDA runtime) are intact
    objs = list(_live)
    for kind in ("Server", "Flow", "Mesh"):  # servers and flows before meshes, meshes before contexts
        for o in objs:
            if type(o).__name__ == kind:
                o.close()
    for o in objs:
        o.close()


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class Mesh:
    """Mesh arrays registered on the device (vlm_mesh_register): addressing, the GAMG
    agglomeration weights and (optionally) the geometry the assembly kernels read."""

    def __init__(self, n_cells, owner, neighbour, magSf, ndc, n_faces=None, ctx: Context | None = None,
                 merge_levels: int = 2, geometry: dict | None = None, agglomeration: str = "host"):
        """agglomeration: "host" (the reference's sequential pairwise pass) or "device" (the parallel
        matching of vlm_mesh_register_ex with VLM_MESH_DEVICE_AGGLOMERATION)."""
        self.ctx = ctx or default_context()
        self.n_systems = 1
        self.owner = np.ascontiguousarray(owner, np.int32)
        self.neighbour = np.ascontiguousarray(neighbour, np.int32)
        self.magSf = _f64(magSf)
        self.ndc = _f64(ndc)
        self.n_cells = int(n_cells)
        self.n_internal_faces = int(self.neighbour.size)
        self.n_faces = int(n_faces if n_faces is not None else self.owner.size)
        self.geometry = geometry or {}
        d = _ffi.MeshDesc()
        d.n_cells = self.n_cells
        d.n_internal_faces = self.n_internal_faces
        d.n_faces = self.n_faces
        d.owner = self.owner.ctypes.data
        d.neighbour = self.neighbour.ctypes.data
        d.magSf = self.magSf.ctypes.data
        d.ndc = self.ndc.ctypes.data
        self._keep = []
        for name in ("V", "Sf", "d", "w", "corrVecs", "C", "Cf", "skewVecs"):
            if name in self.geometry:
                arr = _f64(self.geometry[name])
                self._keep.append(arr)
                setattr(d, name, arr.ctypes.data)
        if "patch_start" in self.geometry:
            ps = np.ascontiguousarray(self.geometry["patch_start"], np.int32)
            pz = np.ascontiguousarray(self.geometry["patch_size"], np.int32)
            self._keep += [ps, pz]
            d.n_patches = ps.size
            d.patch_start = ps.ctypes.data
            d.patch_size = pz.ctypes.data
        d.two_d = int(self.geometry.get("two_d", 0))
        d.empty_dir = int(self.geometry.get("empty_dir", -1))
        if agglomeration not in ("host", "device"):
            raise ValueError(f"agglomeration must be 'host' or 'device', not {agglomeration!r}")
        h = C.c_void_p()
        flags = 1 if agglomeration == "device" else 0
        check(load().vlm_mesh_register_ex(self.ctx.handle, C.byref(d), merge_levels, flags, C.byref(h)),
              self.ctx.handle)
        self._h = h
        _live.add(self)
        self._apply_tuning()

    def _apply_tuning(self):
        """The tuner's launch configuration for this device and mesh size (voluma_b200/tuning/);
        VLM_TUNE=0 keeps the built-in defaults."""
        if os.environ.get("VLM_TUNE", "1") == "0":
            return
        from . import tune
        tune.apply(self)

    @classmethod
    def batch(cls, meshes: list, ctx: Context | None = None, merge_levels: int = 2) -> "Mesh":
        """Registers several meshes (dicts with the cfd::Mesh array names) as one device batch.
        Arrays passed to the batch concatenate the systems: cells and internal faces in system
        order; assembly face arrays hold all internal faces, then all boundary faces."""
        self = cls.__new__(cls)
        self.ctx = ctx or default_context()
        self.n_systems = len(meshes)
        self._keep = []
        descs = (_ffi.MeshDesc * len(meshes))()
        for d, m in zip(descs, meshes):
            own = np.ascontiguousarray(m["owner"], np.int32)
            nei = np.ascontiguousarray(m["neighbour"], np.int32)
            arrs = [own, nei, _f64(m["magSf"]), _f64(m["ndc"])]
            d.n_cells, d.n_internal_faces, d.n_faces = int(m["n_cells"]), nei.size, own.size
            d.owner, d.neighbour, d.magSf, d.ndc = (a.ctypes.data for a in arrs)
            for name in ("V", "Sf", "d", "w", "corrVecs", "C", "Cf", "skewVecs"):
                if name in m:
                    a = _f64(m[name])
                    arrs.append(a)
                    setattr(d, name, a.ctypes.data)
            if "patch_start" in m:
                ps = np.ascontiguousarray(m["patch_start"], np.int32)
                pz = np.ascontiguousarray(m["patch_size"], np.int32)
                arrs += [ps, pz]
                d.n_patches, d.patch_start, d.patch_size = ps.size, ps.ctypes.data, pz.ctypes.data
            d.two_d = int(m.get("two_d", 0))
            d.empty_dir = int(m.get("empty_dir", -1))
            self._keep += arrs
        h = C.c_void_p()
        check(load().vlm_mesh_register_batch(self.ctx.handle, len(meshes), descs, merge_levels, C.byref(h)),
              self.ctx.handle)
        self._h = h
        _live.add(self)
        self._keep = []
        ns, nc, ni, nf = C.c_int32(), C.c_int64(), C.c_int64(), C.c_int64()
        check(load().vlm_mesh_systems(h, C.byref(ns), C.byref(nc), C.byref(ni), C.byref(nf)))
        self.n_cells, self.n_internal_faces, self.n_faces = nc.value, ni.value, nf.value
        self.geometry = {"patch_start": np.concatenate([np.asarray(m.get("patch_start", []), np.int32)
                                                        for m in meshes])}
        self.cell_base = np.cumsum([0] + [int(m["n_cells"]) for m in meshes])
        self.face_base = np.cumsum([0] + [len(m["neighbour"]) for m in meshes])
        self.bface_base = np.cumsum([0] + [len(m["owner"]) - len(m["neighbour"]) for m in meshes])
        self._apply_tuning()
        return self

    @classmethod
    def from_arrays(cls, m: dict, **kw) -> "Mesh":
        """From a dict with the cfd::Mesh array names (n_cells, owner, neighbour, magSf, ndc, ...)."""
        return cls(m["n_cells"], m["owner"], m["neighbour"], m["magSf"], m["ndc"], n_faces=len(m["owner"]),
                   geometry=m, **kw)

    @property
    def handle(self):
        return self._h

    def gamg_levels(self):
        """The device hierarchy's per-level {n, l, u, agg} (natural numbering)."""
        L = load()
        nl = C.c_int32()
        check(L.vlm_gamg_levels(self._h, C.byref(nl)))
        out = []
        for k in range(nl.value):
            s = np.zeros(3, np.int32)
            check(L.vlm_gamg_level(self._h, k, _ptr(s), None, None, None))
            l = np.zeros(s[1], np.int32)
            u = np.zeros(s[1], np.int32)
            agg = np.zeros(s[2], np.int32)
            check(L.vlm_gamg_level(self._h, k, _ptr(s), _ptr(l), _ptr(u), _ptr(agg)))
            out.append(dict(n=int(s[0]), l=l, u=u, agg=agg))
        return out

    def stats(self):
        """(kernel launches executed on this mesh so far, device bytes held)."""
        n, b = C.c_int64(), C.c_int64()
        check(load().vlm_mesh_stats(self._h, C.byref(n), C.byref(b)))
        return n.value, b.value

    def set_tail(self, cluster: int = 0, max_rows: int = 0, full_rows: int = 0):
        """Coarse V-cycle tail launch configuration (vlm_mesh_set_tail): cluster size 1/2/4/8, level
        row limit, whole-V-cycle row limit; 0 keeps a value.  Results are unchanged bit for bit."""
        check(load().vlm_mesh_set_tail(self._h, int(cluster), int(max_rows), int(full_rows)), self.ctx.handle)

    def tail_config(self):
        """(cluster, max_rows, full_rows) of the coarse tail; row limits 0 = scaled defaults."""
        c, a, b = C.c_int32(), C.c_int64(), C.c_int64()
        check(load().vlm_mesh_get_tail(self._h, C.byref(c), C.byref(a), C.byref(b)))
        return c.value, a.value, b.value

    def set_fusion(self, pre_rows: int = -1, restrict_rows: int = -1, post_rows: int = -1):
        """Row limits of the fused Jacobi-level launches (vlm_mesh_set_fusion): both pre-sweeps in one
        pass, residual with restriction, prolongation inside the first post-sweep; negative keeps a
        value, 0 fuses nowhere.  Results are unchanged bit for bit."""
        check(load().vlm_mesh_set_fusion(self._h, int(pre_rows), int(restrict_rows), int(post_rows)), self.ctx.handle)

    def fusion_config(self):
        """(pre_rows, restrict_rows, post_rows) of the fused Jacobi-level launches."""
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        check(load().vlm_mesh_get_fusion(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def stream_config(self):
        """(pencil_rows, stages, ctas) of the plane-streamed level-0 FP64 product
        (vlm_mesh_get_stream); zeros where the four-slot kernel runs instead."""
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        check(load().vlm_mesh_get_stream(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def time_sweeps(self, on: bool = True):
        """Live level-0 sweep timing (vlm_mesh_time_sweeps): solves run eagerly with CUDA events
        around every level-0 sweep."""
        check(load().vlm_mesh_time_sweeps(self._h, int(bool(on))), self.ctx.handle)

    def sweep_time(self):
        """(summed ms, sweeps) of the level-0 sweeps timed since time_sweeps(True)."""
        ms, n = C.c_double(), C.c_int64()
        check(load().vlm_mesh_sweep_time(self._h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def profile_kernel(self, kernel: str, reps: int = 20):
        """(ms per launch, algorithmic bytes per launch) of a level-0 kernel on the last solve's matrix."""
        ms, by = C.c_double(), C.c_double()
        check(load().vlm_profile_kernel(self.ctx.handle, self._h, kernel.encode(), reps, C.byref(ms), C.byref(by)),
              self.ctx.handle)
        return ms.value, by.value

    def colours(self, level):
        n = C.c_int32()
        check(load().vlm_gamg_colours(self._h, level, C.byref(n)))
        return n.value

    def close(self):
        if getattr(self, "_h", None):
            load().vlm_mesh_release(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_BOX_SIDES = ("xMin", "xMax", "yMin", "yMax", "zMin", "zMax")


def box_mesh_device(n, lo=(0, 0, 0), hi=(1, 1, 1), periodic=(False, False, False), two_d=False, beta=(0, 0, 0),
                    points=None, ctx: Context | None = None) -> dict:
    """generateBox + Mesh::build computed on the device (vlm_box_create): the same dict as
    voluma_b200.mesh.box_mesh (the cfd::Mesh array names, patches in side order), bit-identical."""
    ctx = ctx or default_context()
    L = load()
    s = _ffi.BoxSpec()
    for q in range(3):
        s.n[q] = int(n[q])
        s.lo[q] = float(lo[q])
        s.hi[q] = float(hi[q])
        s.periodic[q] = int(bool(periodic[q]))
        s.beta[q] = float(beta[q]) if beta[q] else 0.0
    s.two_d = int(bool(two_d))
    pts = None
    if points is not None:
        pts = _f64(points).reshape(-1)
        if pts.size != 3 * (int(n[0]) + 1) * (int(n[1]) + 1) * (int(n[2]) + 1):
            raise ValueError("points must hold (nx+1)(ny+1)(nz+1) vertices")
        s.points = pts.ctypes.data
    h = C.c_void_p()
    check(L.vlm_box_create(ctx.handle, C.byref(s), C.byref(h)), ctx.handle)
    try:
        d = _ffi.MeshDesc()
        check(L.vlm_box_desc(h, C.byref(d)))
        nC, nI, nF, nP = d.n_cells, d.n_internal_faces, d.n_faces, d.n_patches

        def arr(ptr, n_, dt, shape=None):
            a = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(np.ctypeslib.as_ctypes_type(dt))), (n_,)).copy()
            return a if shape is None else a.reshape(shape)

        sides = np.zeros(max(nP, 1), np.int32)
        check(L.vlm_box_patch_sides(h, sides.ctypes.data))
        m = dict(n_cells=nC, n_internal_faces=nI, n_faces=nF, owner=arr(d.owner, nF, np.int32),
                 neighbour=arr(d.neighbour, nI, np.int32) if nI else np.zeros(0, np.int32),
                 V=arr(d.V, nC, np.float64), C=arr(d.C, 3 * nC, np.float64, (nC, 3)),
                 Sf=arr(d.Sf, 3 * nF, np.float64, (nF, 3)), magSf=arr(d.magSf, nF, np.float64),
                 Cf=arr(d.Cf, 3 * nF, np.float64, (nF, 3)), d=arr(d.d, 3 * nF, np.float64, (nF, 3)),
                 w=arr(d.w, nF, np.float64), ndc=arr(d.ndc, nF, np.float64),
                 corrVecs=arr(d.corrVecs, 3 * nF, np.float64, (nF, 3)),
                 skewVecs=arr(d.skewVecs, 3 * nF, np.float64, (nF, 3)),
                 patch_start=arr(d.patch_start, nP, np.int32) if nP else np.zeros(0, np.int32),
                 patch_size=arr(d.patch_size, nP, np.int32) if nP else np.zeros(0, np.int32),
                 patch_names=[_BOX_SIDES[int(q)] for q in sides[:nP]], two_d=bool(d.two_d),
                 empty_dir=int(d.empty_dir), shape=tuple(int(v) for v in n),
                 periodic=tuple(bool(p) for p in periodic))
    finally:
        L.vlm_box_destroy(h)
    sk = m["skewVecs"][:nI]
    dd = m["d"][:nI]
    m["skewed"] = bool(nI and (np.sqrt((sk * sk).sum(1)) / np.sqrt((dd * dd).sum(1))).max() > 1e-8)
    m["deltaCoeffs"] = 1.0 / np.sqrt((m["d"] * m["d"]).sum(1))
    return m


def topology(n_cells, owner, neighbour, magSf, ndc, merge_levels: int = 2):
    """Host-side GAMG hierarchy + colouring exactly as the device uses them (no GPU needed):
    list of dicts n, l, u, weight, agg, faceMap, faceFlip, colour, ncolours."""
    L = load()
    own = np.ascontiguousarray(owner, np.int32)
    nei = np.ascontiguousarray(neighbour, np.int32)
    h = C.c_void_p()
    check(L.vlm_topology_build(int(n_cells), nei.size, _ptr(own), _ptr(nei), _ptr(_f64(magSf)), _ptr(_f64(ndc)),
                               merge_levels, C.byref(h)))
    try:
        nl = C.c_int32()
        check(L.vlm_topology_levels(h, C.byref(nl)))
        out = []
        for k in range(nl.value):
            s = np.zeros(4, np.int32)
            check(L.vlm_topology_level(h, k, _ptr(s), None, None, None, None, None, None, None))
            n, nf, na, nc = (int(v) for v in s)
            d = dict(n=n, l=np.zeros(nf, np.int32), u=np.zeros(nf, np.int32), weight=np.zeros(nf),
                     agg=np.zeros(na, np.int32), faceMap=np.zeros(nf if na else 0, np.int32),
                     faceFlip=np.zeros(nf if na else 0, np.int8), colour=np.zeros(n, np.int32), ncolours=nc)
            check(L.vlm_topology_level(h, k, _ptr(s), _ptr(d["l"]), _ptr(d["u"]), _ptr(d["weight"]), _ptr(d["agg"]),
                                       _ptr(d["faceMap"]), _ptr(d["faceFlip"]), _ptr(d["colour"])))
            out.append(d)
        return out
    finally:
        L.vlm_topology_destroy(h)


def barrier_check(ctas: int, spin_limit: int, absent_cta: int = -1, rounds: int = 4, ctx: "Context | None" = None):
    """Runs the level-scheduled kernels' bounded group barrier on its own (vlm_barrier_check):
    returns (status name, barriers passed per CTA); status "TIMEOUT" when a wait gave up."""
    ctx = ctx or default_context()
    L = load()
    passed = np.zeros(int(ctas), np.int32)
    st = C.c_int32()
    check(L.vlm_barrier_check(ctx.handle, int(ctas), int(spin_limit), int(absent_cta), int(rounds), _ptr(passed),
                              C.byref(st)), ctx.handle)
    return _ffi.STATUS.get(st.value, str(st.value)), passed


def box_shape(n_cells, owner, neighbour, magSf=None, ndc=None):
    """Whether the face arrays are those of a generateBox mesh (no GPU needed): a dict with the
    shape n = (nx, ny, nz), the periodic flags and `layout` (level 0 of its solves runs the
    structured box kernels), or None when the mesh is not a box."""
    L = load()
    own = np.ascontiguousarray(owner, np.int32)
    nei = np.ascontiguousarray(neighbour, np.int32)
    magSf = np.ones(nei.size) if magSf is None else magSf
    ndc = np.ones(nei.size) if ndc is None else ndc
    h = C.c_void_p()
    check(L.vlm_topology_build(int(n_cells), nei.size, _ptr(own), _ptr(nei), _ptr(_f64(magSf)), _ptr(_f64(ndc)),
                               2, C.byref(h)))
    try:
        s = np.zeros(7, np.int32)
        check(L.vlm_topology_box(h, _ptr(s)))
    finally:
        L.vlm_topology_destroy(h)
    if s[0] == 0:
        return None
    return dict(n=tuple(int(v) for v in s[:3]), periodic=tuple(bool(v) for v in s[3:6]), layout=bool(s[6]))


def solve_ldu(mesh: Mesh, diag, upper, lower, b, x, ctrl: SolverControls) -> SolverPerformance:
    """solveLdu (LinearSolver.cpp:135): solves in place into x (float64 numpy array)."""
    if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous):
        raise TypeError("x must be a C-contiguous float64 array (solved in place)")
    diag, upper, b = _f64(diag), _f64(upper), _f64(b)
    lower = None if lower is None else _f64(lower)
    c = ctrl.to_c()
    p = (_ffi.SolverPerf * mesh.n_systems)()
    check(load().vlm_ldu_solve(mesh.ctx.handle, mesh.handle, _ptr(diag), _ptr(upper), _ptr(lower), _ptr(b), _ptr(x),
                               C.byref(c), p), mesh.ctx.handle)
    out = [SolverPerformance.from_c(q) for q in p]
    return out[0] if mesh.n_systems == 1 else out


def solve_ldu_device(mesh: Mesh, diag_ptr, upper_ptr, lower_ptr, b_ptr, x_ptr, ctrl: SolverControls) -> SolverPerformance:
    """Device-pointer variant (integers, e.g. torch tensor data_ptr()) ordered on the mesh context's stream."""
    c = ctrl.to_c()
    p = (_ffi.SolverPerf * mesh.n_systems)()
    check(load().vlm_ldu_solve_device(mesh.ctx.handle, mesh.handle, C.c_void_p(diag_ptr), C.c_void_p(upper_ptr),
                                      C.c_void_p(lower_ptr) if lower_ptr else None, C.c_void_p(b_ptr),
                                      C.c_void_p(x_ptr), C.byref(c), p), mesh.ctx.handle)
    out = [SolverPerformance.from_c(q) for q in p]
    return out[0] if mesh.n_systems == 1 else out


def _bc(mesh: Mesh, bc_type, bc_values):
    nP = len(mesh.geometry.get("patch_start", []))
    t = np.zeros(max(nP, 1), np.int32)
    if bc_type is not None:
        t[:len(bc_type)] = np.asarray(bc_type, np.int32)
    v = None if bc_values is None else _f64(bc_values)
    return t, v


def laplacian(mesh: Mesh, gamma, psi, bc_type=None, bc_values=None, non_orth_corr=True, grad_scheme=0):
    """fvm::laplacian(gamma, psi) (Fvm.h:141-182) of a scalar field: dict of diag, upper, source,
    internalCoeffs, boundarySource, ffc, hasFfc.  bc_type per patch: 0 zeroGradient, 1 fixedValue,
    2 symmetry (a zero gradient), 5 fixedGradient (bc_values are the gradients)."""
    nC, nI, nF = mesh.n_cells, mesh.n_internal_faces, mesh.n_faces
    out = dict(diag=np.zeros(nC), upper=np.zeros(nI), source=np.zeros(nC), internalCoeffs=np.zeros(nF - nI),
               boundarySource=np.zeros(nF - nI), ffc=np.zeros(nF))
    t, v = _bc(mesh, bc_type, bc_values)
    has = C.c_int32()
    check(load().vlm_laplacian(mesh.ctx.handle, mesh.handle, _ptr(_f64(gamma)), _ptr(_f64(psi)), _ptr(t), _ptr(v),
                               int(non_orth_corr), int(grad_scheme), _ptr(out["diag"]), _ptr(out["upper"]),
                               _ptr(out["source"]), _ptr(out["internalCoeffs"]), _ptr(out["boundarySource"]),
                               _ptr(out["ffc"]), C.byref(has)), mesh.ctx.handle)
    out["hasFfc"] = bool(has.value)
    return out


def grad(mesh: Mesh, psi, bc_type=None, bc_values=None, scheme=0):
    """fvc::grad of a scalar (Fvc.h:209-291): (n_cells, 3); scheme 0 Gauss linear, 1 least squares,
    2 GaussSkew (the mesh registered with skewVecs)."""
    g = np.zeros((mesh.n_cells, 3))
    t, v = _bc(mesh, bc_type, bc_values)
    check(load().vlm_grad(mesh.ctx.handle, mesh.handle, _ptr(_f64(psi)), _ptr(t), _ptr(v), int(scheme), _ptr(g)),
          mesh.ctx.handle)
    return g


def div(mesh: Mesh, face_flux):
    """fvc::div (Fvc.h:294-304), per unit volume."""
    out = np.zeros(mesh.n_cells)
    check(load().vlm_div(mesh.ctx.handle, mesh.handle, _ptr(_f64(face_flux)), _ptr(out)), mesh.ctx.handle)
    return out


def pressure_solve(mesh: Mesh, gamma, div_phi, p, ctrl: SolverControls, final_ctrl: SolverControls | None = None,
                   bc_type=None, bc_values=None, ref_cell=0, ref_value=0.0, n_non_orth=0, grad_scheme=1,
                   want_flux=True):
    """The pressure-corrector loop (IncompressibleFlow.cpp:322-341) on the device; p is solved in
    place.  ref_cell: one cell (single mesh) or one per system of a batch (-1 / None: none).
    Returns (performances per pass [per system for a batch], face flux of the last pass or None)."""
    if not (isinstance(p, np.ndarray) and p.dtype == np.float64 and p.flags.c_contiguous):
        raise TypeError("p must be a C-contiguous float64 array (solved in place)")
    t, v = _bc(mesh, bc_type, bc_values)
    ns = mesh.n_systems
    refs = np.full(ns, -1, np.int32)
    if ref_cell is not None:
        refs[:] = np.asarray(ref_cell, np.int32)
    perf = (_ffi.SolverPerf * ((n_non_orth + 1) * ns))()
    flux = np.zeros(mesh.n_faces) if want_flux else None
    c = ctrl.to_c()
    cf = (final_ctrl or ctrl).to_c()
    check(load().vlm_pressure_solve_batch(mesh.ctx.handle, mesh.handle, _ptr(_f64(gamma)), _ptr(_f64(div_phi)),
                                          _ptr(p), _ptr(t), _ptr(v), _ptr(refs), float(ref_value), int(n_non_orth),
                                          int(grad_scheme), C.byref(c), C.byref(cf), perf, _ptr(flux), 0),
          mesh.ctx.handle)
    rows = [[SolverPerformance.from_c(perf[q * ns + s]) for s in range(ns)] for q in range(n_non_orth + 1)]
    return ([r[0] for r in rows] if ns == 1 else rows), flux


def pressure_solve_device(mesh: Mesh, gamma_ptr: int, div_ptr: int, p_ptr: int, ctrl: SolverControls,
                          final_ctrl: SolverControls | None = None, ref_cell=0, n_non_orth=0, grad_scheme=1,
                          flux_ptr: int | None = None):
    """pressure_solve on device pointers (gamma, div_phi, p, flux: device addresses of float64 arrays in
    the batch layout, ordered on the mesh context's stream); zeroGradient on every patch."""
    t, v = _bc(mesh, None, None)
    ns = mesh.n_systems
    refs = np.full(ns, -1, np.int32)
    if ref_cell is not None:
        refs[:] = np.asarray(ref_cell, np.int32)
    perf = (_ffi.SolverPerf * ((n_non_orth + 1) * ns))()
    c = ctrl.to_c()
    cf = (final_ctrl or ctrl).to_c()
    check(load().vlm_pressure_solve_batch(mesh.ctx.handle, mesh.handle, C.c_void_p(gamma_ptr), C.c_void_p(div_ptr),
                                          C.c_void_p(p_ptr), _ptr(t), _ptr(v), _ptr(refs), 0.0, int(n_non_orth),
                                          int(grad_scheme), C.byref(c), C.byref(cf), perf,
                                          None if flux_ptr is None else C.c_void_p(flux_ptr), 1), mesh.ctx.handle)
    return [[SolverPerformance.from_c(perf[q * ns + s]) for s in range(ns)] for q in range(n_non_orth + 1)]


def exact_sum(values, ctx: Context | None = None) -> float:
    """Order-independent exact sum on the device (par::ExactSum semantics, Comm.h:42-93)."""
    ctx = ctx or default_context()
    v = _f64(values)
    out = C.c_double()
    check(load().vlm_exact_sum(ctx.handle, _ptr(v), v.size, C.byref(out)), ctx.handle)
    return out.value


def amul(mesh: Mesh, diag, upper, lower, x):
    """y = A x (LinearSolver.cpp:121-133)."""
    y = np.zeros(mesh.n_cells)
    check(load().vlm_amul(mesh.ctx.handle, mesh.handle, _ptr(_f64(diag)), _ptr(_f64(upper)),
                          None if lower is None else _ptr(_f64(lower)), _ptr(_f64(x)), _ptr(y)), mesh.ctx.handle)
    return y


def precond_apply(mesh: Mesh, diag, upper, lower, r, preconditioner: str = "DILU", smoother: str = ""):
    """w = M^-1 r (Preconditioner ctor + apply, LinearSolver.cpp:56-107): none, diagonal, DIC, DILU, GAMG."""
    w = np.zeros(mesh.n_cells)
    c = SolverControls(preconditioner=preconditioner, smoother=smoother).to_c()
    check(load().vlm_precond_apply(mesh.ctx.handle, mesh.handle, _ptr(_f64(diag)), _ptr(_f64(upper)),
                                   None if lower is None else _ptr(_f64(lower)), _ptr(_f64(r)), _ptr(w), C.byref(c)),
          mesh.ctx.handle)
    return w


def gamg_apply(mesh: Mesh, diag, upper, lower, r, smoother: str = ""):
    """One device V-cycle w = M^-1 r."""
    w = np.zeros(mesh.n_cells)
    c = SolverControls(smoother=smoother).to_c()
    check(load().vlm_gamg_apply(mesh.ctx.handle, mesh.handle, _ptr(_f64(diag)), _ptr(_f64(upper)),
                                None if lower is None else _ptr(_f64(lower)), _ptr(_f64(r)), _ptr(w), C.byref(c)),
          mesh.ctx.handle)
    return w


# ------------------------------------------------------------------ incompressible step
def _flow_ctrl(case: dict) -> _ffi.FlowCtrl:
    c = _ffi.FlowCtrl()
    c.nu = case["nu"]
    c.steady = int(case["steady"])
    c.div_scheme, c.ddt_scheme = case["div_scheme"], case["ddt_scheme"]
    c.n_outer, c.n_corr, c.n_non_orth_corr = case["n_outer"], case["n_corr"], case["n_non_orth_corr"]
    c.momentum_predictor = int(case["momentum_predictor"])
    c.alpha_u, c.alpha_p = case["alpha_u"], case["alpha_p"]
    c.p_ref_cell, c.p_ref_value = case["p_ref_cell"], case["p_ref_value"]
    c.div_coeff = case.get("div_coeff", 1.0)
    c.grad_scheme = int(case.get("grad_scheme", 0))
    c.grad_p_scheme = int(case.get("grad_p_scheme", 0))
    c._keep = []
    # Robin {a, b} per patch (type 8), advective {lInf, fieldInf} per patch (type 9); copied by vlm_flow_create
    for key in ("u_robin", "p_robin", "u_advective"):
        if case.get(key) is not None:
            a = np.ascontiguousarray(case[key], np.float64).reshape(-1)
            c._keep.append(a)
            setattr(c, key, a.ctypes.data)
    repro = bool(case.get("reproducible", False))
    for name, key in (("U", "U"), ("p", "p"), ("p_final", "pFinal")):
        d = case[key]
        sc = SolverControls(d["solver"], d["preconditioner"], d["tolerance"], d["relTol"], d["maxIter"],
                            d.get("minIter", 0), d.get("nSweeps", 1), reproducible=repro,
                            smoother=d.get("smoother", ""), precision=d.get("precision", ""))
        setattr(c, name, sc.to_c())
    return c


class Flow:
    """IncompressibleFlow (solvers/IncompressibleFlow.h) on the device for a registered single-system mesh
    with geometry.  `case`: dict with nu, steady, div_scheme, ddt_scheme, n_outer, n_corr,
    n_non_orth_corr, momentum_predictor, alpha_u, alpha_p, p_ref_cell, p_ref_value, U / p / pFinal solver
    dictionaries, per-patch u_type / u_value / p_type / p_value and optionally reproducible and the
    face-by-face boundary values u_face / p_face (set_boundary_values) (voluma_b200.cases.lid_cavity
    builds one)."""

    def __init__(self, mesh: Mesh, case: dict):
        self.mesh = mesh
        self.n_cells = mesh.n_cells
        self.n_faces = mesh.n_faces
        self._keep = [np.ascontiguousarray(case["u_type"], np.int32), _f64(case["u_value"]),
                      np.ascontiguousarray(case["p_type"], np.int32), _f64(case["p_value"])]
        c = _flow_ctrl(case)
        h = C.c_void_p()
        check(load().vlm_flow_create(mesh.ctx.handle, mesh.handle, C.byref(c), *(a.ctypes.data for a in self._keep),
                                     C.byref(h)), mesh.ctx.handle)
        self._h = h
        _live.add(self)
        if case.get("u_face") is not None or case.get("p_face") is not None:
            self.set_boundary_values(case.get("u_face"), case.get("p_face"))

    def set_state(self, U=None, p=None):
        Ua = None if U is None else _f64(U).reshape(-1)
        pa = None if p is None else _f64(p)
        check(load().vlm_flow_set_state(self._h, None if Ua is None else Ua.ctypes.data,
                                        None if pa is None else pa.ctypes.data), self.mesh.ctx.handle)

    def set_boundary_values(self, u_face=None, p_face=None):
        """Face-by-face values of the fixedValue / inletOutlet U patches (n_boundary x 3) and of the
        fixedValue p patches (n_boundary), boundary faces in mesh order (vlm_flow_set_boundary_values)."""
        ua = None if u_face is None else _f64(u_face).reshape(-1)
        pa = None if p_face is None else _f64(p_face).reshape(-1)
        check(load().vlm_flow_set_boundary_values(self._h, None if ua is None else ua.ctypes.data,
                                                  None if pa is None else pa.ctypes.data), self.mesh.ctx.handle)

    def step(self, dt=1.0) -> dict:
        i = _ffi.StepInfo()
        check(load().vlm_flow_step(self._h, dt, C.byref(i)), self.mesh.ctx.handle)
        return dict(UInitialResidual=i.UInitialResidual, pInitialResidual=i.pInitialResidual,
                    continuityError=i.continuityError, iterations=i.iterations, launches=i.launches)

    def launches(self) -> int:
        return int(load().vlm_flow_launches(self._h))

    def set_model(self, model: dict):
        """Turbulence model and momentum forcing (vlm_flow_model), before the first step.  `model`: les
        ("laminar" or "Smagorinsky"), Cs, van_driest, Aplus, Cdelta, kappa, delta_coeff, nut_max_ratio,
        depth (2D), wall_patch (per patch 0/1), forcing ("none", "constant", "meanVelocity"), force, Ubar,
        relaxation, grad_p; missing keys take the reference's defaults."""
        mdl = _ffi.FlowModel()
        les = model.get("les", "laminar")
        mdl.les = {"laminar": 0, "Smagorinsky": 1}[les] if isinstance(les, str) else int(les)
        mdl.Cs = model.get("Cs", 0.17)
        mdl.van_driest = int(bool(model.get("van_driest", False)))
        mdl.Aplus = model.get("Aplus", 26.0)
        mdl.Cdelta = model.get("Cdelta", 0.158)
        mdl.kappa = model.get("kappa", 0.41)
        mdl.delta_coeff = model.get("delta_coeff", 1.0)
        mdl.nut_max_ratio = model.get("nut_max_ratio", 1e5)
        mdl.depth = model.get("depth", 0.0)
        wp = model.get("wall_patch")
        self._wall = None if wp is None else np.ascontiguousarray(wp, np.int32)
        mdl.wall_patch = None if self._wall is None else self._wall.ctypes.data
        fo = model.get("forcing", "none")
        mdl.forcing = {"none": 0, "constant": 1, "meanVelocity": 2}[fo] if isinstance(fo, str) else int(fo)
        for k, v in enumerate(model.get("force", (0.0, 0.0, 0.0))):
            mdl.force[k] = v
        for k, v in enumerate(model.get("Ubar", (0.0, 0.0, 0.0))):
            mdl.Ubar[k] = v
        mdl.relaxation = model.get("relaxation", 1.0)
        mdl.grad_p = model.get("grad_p", 0.0)
        check(load().vlm_flow_set_model(self._h, C.byref(mdl)), self.mesh.ctx.handle)

    def write_restart(self, directory: str):
        """The flow's state in the reference's restart directory format (restart::write)."""
        check(load().vlm_flow_write_restart(self._h, os.fspath(directory).encode()), self.mesh.ctx.handle)

    def read_restart(self, directory: str) -> bool:
        """Continue from a restart directory (restart::read); False when it has no state.txt.  Set
        the model first."""
        found = C.c_int32()
        check(load().vlm_flow_read_restart(self._h, os.fspath(directory).encode(), C.byref(found)),
              self.mesh.ctx.handle)
        return bool(found.value)

    def model_state(self):
        """(nu_t per cell, mean-velocity driving pressure gradient)."""
        nut = np.zeros(self.n_cells)
        gp = np.zeros(1)
        check(load().vlm_flow_get_model_state(self._h, nut.ctypes.data, gp.ctypes.data), self.mesh.ctx.handle)
        return nut, float(gp[0])

    def run_steady(self, max_iter=5000, residual_tol=1e-6):
        it = C.c_int32()
        i = _ffi.StepInfo()
        check(load().vlm_flow_run_steady(self._h, max_iter, residual_tol, C.byref(it), C.byref(i)),
              self.mesh.ctx.handle)
        return it.value, dict(UInitialResidual=i.UInitialResidual, pInitialResidual=i.pInitialResidual,
                              continuityError=i.continuityError, iterations=i.iterations)

    def state(self):
        U = np.zeros((self.n_cells, 3))
        p = np.zeros(self.n_cells)
        phi = np.zeros(self.n_faces)
        check(load().vlm_flow_get_state(self._h, U.ctypes.data, p.ctypes.data, phi.ctypes.data),
              self.mesh.ctx.handle)
        return U, p, phi

    def close(self):
        if getattr(self, "_h", None):
            load().vlm_flow_destroy(self._h)
            self._h = None


# ------------------------------------------------------------------ serving
class Server:
    """Continuous-batching server of incompressible solves on one device (vlm_server_*): requests are
    admitted in arrival order as slots and HBM budget free up and run concurrently, each on its own
    stream; results come back with their arrival / admission / completion times."""

    def __init__(self, device: int = 0, hbm_budget: int = 64 << 30, max_active: int = 4):
        h = C.c_void_p()
        check(load().vlm_server_create(device, int(hbm_budget), int(max_active), C.byref(h)))
        self._h = h
        self._keep = {}
        _live.add(self)

    def clock(self) -> float:
        return load().vlm_server_clock(self._h)

    def submit(self, mesh: dict, case: dict, arrival: float = 0.0, max_iter: int = 5000, residual_tol: float = 1e-6,
               n_steps: int = 0, dt: float = 1.0, U0=None, p0=None, device_bytes: int = 0,
               agglomeration: str = "host") -> int:
        """mesh: cfd::Mesh arrays with geometry (voluma_b200.mesh.box_mesh); case: Flow case dict;
        agglomeration "device" builds the request mesh's GAMG hierarchy on the device."""
        arrs = {}
        d = _ffi.MeshDesc()
        own = np.ascontiguousarray(mesh["owner"], np.int32)
        nei = np.ascontiguousarray(mesh["neighbour"], np.int32)
        arrs.update(own=own, nei=nei)
        d.n_cells, d.n_internal_faces, d.n_faces = int(mesh["n_cells"]), nei.size, own.size
        d.owner, d.neighbour = own.ctypes.data, nei.ctypes.data
        for name in ("magSf", "ndc", "V", "Sf", "d", "w", "corrVecs", "C", "Cf", "skewVecs"):
            if name in mesh:
                a = _f64(mesh[name])
                arrs[name] = a
                setattr(d, name, a.ctypes.data)
        ps = np.ascontiguousarray(mesh["patch_start"], np.int32)
        pz = np.ascontiguousarray(mesh["patch_size"], np.int32)
        arrs.update(ps=ps, pz=pz)
        d.n_patches, d.patch_start, d.patch_size = ps.size, ps.ctypes.data, pz.ctypes.data
        d.two_d, d.empty_dir = int(mesh.get("two_d", 0)), int(mesh.get("empty_dir", -1))
        ctrl = _flow_ctrl(case)
        bc = [np.ascontiguousarray(case["u_type"], np.int32), _f64(case["u_value"]),
              np.ascontiguousarray(case["p_type"], np.int32), _f64(case["p_value"])]
        r = _ffi.FlowRequest()
        r.mesh_flags = 1 if agglomeration == "device" else 0
        r.mesh, r.ctrl = C.addressof(d), C.addressof(ctrl)
        r.u_type, r.u_value, r.p_type, r.p_value = (a.ctypes.data for a in bc)
        if U0 is not None:
            arrs["U0"] = _f64(U0).reshape(-1)
            r.U0 = arrs["U0"].ctypes.data
        if p0 is not None:
            arrs["p0"] = _f64(p0)
            r.p0 = arrs["p0"].ctypes.data
        r.n_steps, r.dt, r.max_iter, r.residual_tol = int(n_steps), float(dt), int(max_iter), float(residual_tol)
        r.arrival, r.device_bytes = float(arrival), int(device_bytes)
        rid = C.c_int64()
        check(load().vlm_server_submit(self._h, C.byref(r), C.byref(rid)))  # copies everything
        self._keep[rid.value] = (int(mesh["n_cells"]), own.size)
        return rid.value

    def collect(self, timeout: float = 0.0, capacity: int = 256) -> list:
        out = (_ffi.FlowResult * capacity)()
        n = C.c_int32()
        check(load().vlm_server_collect(self._h, out, capacity, C.byref(n), float(timeout)))
        return [dict(id=q.id, status=q.status, iterations=q.iterations, arrival=q.arrival, admitted=q.admitted,
                     finished=q.finished, UInitialResidual=q.UInitialResidual, pInitialResidual=q.pInitialResidual,
                     continuityError=q.continuityError, device_bytes=q.device_bytes, launches=q.launches)
                for q in out[:n.value]]

    def fields(self, rid: int):
        nC, nF = self._keep[rid]
        U, p, phi = np.zeros((nC, 3)), np.zeros(nC), np.zeros(nF)
        check(load().vlm_server_result_fields(self._h, rid, U.ctypes.data, p.ctypes.data, phi.ctypes.data))
        return U, p, phi

    def close(self):
        if getattr(self, "_h", None):
            load().vlm_server_destroy(self._h)
            self._h = None


def request_bytes(n_cells: int, n_faces: int) -> int:
    return int(load().vlm_flow_request_bytes(int(n_cells), int(n_faces)))
