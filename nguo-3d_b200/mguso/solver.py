"""Host-side mirror of the reference's solver API (scene build -> step -> readback).

``ImplicitSolver`` mirrors engine_core::ImplicitSolver (core-engine/crates/engine-core/src/
implicit.rs:372-2191) as built by Scene::build_implicit plus its set_* calls: construct it
from a scene (positions, triangles, masses, shell faces, stitches, colliders, parameters),
call ``step()``, read ``positions``. Every step runs on the GPU through the C ABI.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, ptr

_PARAM_FIELDS = [("dt", C.c_float), ("gravity", C.c_float * 3), ("newton_iters", C.c_uint32),
                 ("stiffness", C.c_float), ("bend_stiffness", C.c_float), ("max_dx", C.c_float),
                 ("target_toi", C.c_float), ("min_newton_steps", C.c_uint32), ("ccd_max_iter", C.c_uint32),
                 ("eiganalysis_eps", C.c_float), ("contact_dhat", C.c_float), ("contact_kappa", C.c_float),
                 ("contact_dynamic", C.c_float), ("shell_mu", C.c_float), ("shell_lambda", C.c_float),
                 ("friction", C.c_float), ("friction_eps", C.c_float), ("barrier_kind", C.c_int),
                 ("contact_rayleigh", C.c_int), ("self_collision", C.c_int), ("cg_tol", C.c_float),
                 ("cg_max_iter", C.c_uint32), ("floor_y", C.c_float), ("newton_tol", C.c_float),
                 ("precond", C.c_int), ("schwarz_domain", C.c_uint32), ("precision", C.c_int),
                 ("pcg_mode", C.c_int), ("factor_storage", C.c_int), ("schwarz_levels", C.c_uint32),
                 ("pcg_variant", C.c_int), ("membrane_warp", C.c_float), ("membrane_weft", C.c_float),
                 ("membrane_shear", C.c_float), ("constraint_tol", C.c_float), ("schwarz_weight", C.c_float),
                 ("strain_limit_ratio", C.c_float), ("strain_limit_k", C.c_float),
                 ("strain_limit_ratio_weft", C.c_float)]


class Params(C.Structure):
    _fields_ = _PARAM_FIELDS


class SceneDesc(C.Structure):
    _fields_ = [("nv", C.c_uint32), ("positions", C.c_void_p), ("velocities", C.c_void_p),
                ("inv_mass", C.c_void_p), ("nt", C.c_uint32), ("tris", C.c_void_p), ("static_mask", C.c_void_p),
                ("nshell", C.c_uint32), ("shell_faces", C.c_void_p), ("nstitch", C.c_uint32),
                ("stitch_idx", C.c_void_p), ("stitch_w", C.c_void_p), ("stitch_kl", C.c_void_p),
                ("ncollider", C.c_uint32), ("colliders", C.c_void_p), ("params", Params),
                ("shell_rest", C.c_void_p), ("shell_stiff", C.c_void_p), ("uvs", C.c_void_p),
                ("nstretch", C.c_uint32), ("stretch_edges", C.c_void_p)]


class StepStats(C.Structure):
    _fields_ = [("newton_iters", C.c_uint32), ("max_cg_iters", C.c_uint32), ("num_contacts", C.c_uint32),
                ("stencils", C.c_uint32), ("ccd_cap_hits", C.c_uint32), ("max_reresid", C.c_double),
                ("t_min", C.c_double), ("penetration_free", C.c_int), ("all_finite", C.c_int), ("status", C.c_int)]


def _sigs(lib):
    vp, i32 = C.c_void_p, C.c_int
    P = C.POINTER
    for name, res, args in [
        ("mguso_scene_create", i32, [vp, P(SceneDesc), P(vp)]),
        ("mguso_scene_destroy", i32, [vp]),
        ("mguso_step", i32, [vp, i32, vp]),
        ("mguso_read_positions", i32, [vp, vp]),
        ("mguso_write_positions", i32, [vp, vp]),
        ("mguso_read_velocities", i32, [vp, vp]),
        ("mguso_write_velocities", i32, [vp, vp]),
        ("mguso_set_kinematic_collider_positions", i32, [vp, vp]),
        ("mguso_set_pins", i32, [vp, C.c_uint32, vp, vp, vp, vp, vp]),
        ("mguso_set_pulls", i32, [vp, C.c_uint32, vp, vp, vp]),
        ("mguso_set_strain_limit_faces", i32, [vp, C.c_uint32, vp, vp, vp, vp]),
        ("mguso_scene_info", i32, [vp, vp]),
        ("mguso_scene_spmv_time", i32, [vp, i32, P(C.c_float), P(C.c_double)]),
        ("mguso_scene_assemble", i32, [vp, vp, vp, vp]),
        ("mguso_scene_assemble_exact", i32, [vp, vp, vp, vp]),
        ("mguso_scene_ccd", i32, [vp, vp, vp, vp, vp]),
        ("mguso_scene_profile", i32, [vp, i32, vp, vp]),
        ("mguso_scene_profile_pcg", i32, [vp, i32, vp, vp]),
        ("mguso_scene_pcg_kernels", i32, [vp, vp]),
        ("mguso_scene_self_intersections", i32, [vp, vp, vp]),
        ("mguso_batch_create", i32, [vp, vp, C.c_uint32, P(vp)]),
        ("mguso_scene_instances", i32, [vp, P(C.c_uint32), vp]),
        ("mguso_scene_system", i32, [vp, vp, vp, vp, vp, vp, vp, vp]),
        ("mguso_scene_stencils", i32, [vp, C.c_uint32, vp, vp, vp, vp]),
        ("mguso_scene_validate", i32, [vp]),
    ]:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def _desc(scene: dict, precision: str):
    """SceneDesc for one scene dict and the arrays it points into (kept alive by the caller)."""
    keep = {k: np.ascontiguousarray(scene[k]) for k in ("positions", "velocities", "inv_mass", "tris", "shell_faces",
                                                       "stitch_idx", "stitch_w", "stitch_kl", "colliders")}
    keep["positions"] = keep["positions"].astype(np.float32, copy=False)
    keep["velocities"] = keep["velocities"].astype(np.float32, copy=False)
    keep["inv_mass"] = keep["inv_mass"].astype(np.float32, copy=False)
    keep["tris"] = keep["tris"].astype(np.uint32, copy=False)
    keep["shell_faces"] = keep["shell_faces"].astype(np.uint32, copy=False)
    keep["stitch_idx"] = keep["stitch_idx"].astype(np.uint32, copy=False)
    keep["stitch_w"] = keep["stitch_w"].astype(np.float32, copy=False)
    keep["stitch_kl"] = keep["stitch_kl"].astype(np.float32, copy=False)
    keep["colliders"] = keep["colliders"].astype(np.float32, copy=False)
    mask = scene.get("static_mask")
    keep["mask"] = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    d = SceneDesc()
    d.nv = keep["positions"].shape[0]
    d.positions = ptr(keep["positions"])
    d.velocities = ptr(keep["velocities"])
    d.inv_mass = ptr(keep["inv_mass"])
    d.nt = keep["tris"].shape[0]
    d.tris = ptr(keep["tris"]) if d.nt else None
    d.static_mask = ptr(keep["mask"]) if keep["mask"] is not None else None
    d.nshell = keep["shell_faces"].shape[0]
    d.shell_faces = ptr(keep["shell_faces"]) if d.nshell else None
    d.nstitch = keep["stitch_idx"].shape[0]
    d.stitch_idx = ptr(keep["stitch_idx"]) if d.nstitch else None
    d.stitch_w = ptr(keep["stitch_w"]) if d.nstitch else None
    d.stitch_kl = ptr(keep["stitch_kl"]) if d.nstitch else None
    d.ncollider = keep["colliders"].shape[0]
    d.colliders = ptr(keep["colliders"]) if d.ncollider else None
    d.params = make_params(scene["params"], precision)
    for name in ("shell_rest", "shell_stiff", "uvs"):
        if scene.get(name) is not None:
            keep[name] = np.ascontiguousarray(scene[name], np.float32)
            setattr(d, name, ptr(keep[name]))
    if scene.get("stretch_edges") is not None:
        keep["stretch_edges"] = np.ascontiguousarray(scene["stretch_edges"], np.uint32).reshape(-1, 2)
        d.nstretch = keep["stretch_edges"].shape[0]
        d.stretch_edges = ptr(keep["stretch_edges"]) if d.nstretch else None
    return d, keep


def validate_scene(scene: dict, precision: str = "mixed") -> None:
    """Checks a scene description on the host, with no device (mguso_scene_validate): the
    index ranges, the stitch rules of ImplicitSolver::set_stitches (implicit.rs:939-966) and
    the parameters. Raises MgusoError (MGUSO_ERR_INVALID_ARG) with the reason, as building
    the scene would."""
    lib = _lib.load()
    _sigs(lib)
    d, keep = _desc(scene, precision)
    check(lib.mguso_scene_validate(C.byref(d)))
    del keep


def make_params(p: dict, precision: str = "mixed") -> Params:
    s = Params()
    for k, v in p.items():
        if k == "gravity":
            s.gravity[:] = list(v)
        elif any(k == f for f, _ in _PARAM_FIELDS):
            setattr(s, k, v)
    s.precision = {"fp32": _lib.PRECISION_FP32, "mixed": _lib.PRECISION_MIXED}[precision]
    return s


class ImplicitSolver:
    """One drape on the GPU (scene from ``mguso.scenes``)."""

    def __init__(self, ctx, scene: dict, precision: str = "mixed"):
        self.ctx = ctx
        self.lib = ctx.lib
        _sigs(self.lib)
        d, keep = _desc(scene, precision)
        self.nv = d.nv
        self._keep = keep
        h = C.c_void_p()
        check(self.lib.mguso_scene_create(ctx.h, C.byref(d), C.byref(h)))
        self.h = h
        ctx.own(self)
        self.ninst = 1
        self.history: list[dict] = []

    def step(self, n: int = 1) -> list:
        """Advances n steps. Returns one stats dict per step (a single scene) or, for a
        batch, one list of per-instance stats dicts per step."""
        out = (StepStats * (n * self.ninst))()
        check(self.lib.mguso_step(self.h, n, out))
        st = [{f: getattr(o, f) for f, _ in StepStats._fields_} for o in out]
        if self.ninst > 1:
            st = [st[i * self.ninst:(i + 1) * self.ninst] for i in range(n)]
        self.history += st
        return st

    @property
    def positions(self) -> np.ndarray:
        out = np.empty((self.nv, 3), np.float32)
        check(self.lib.mguso_read_positions(self.h, ptr(out)))
        return out

    @positions.setter
    def positions(self, p):
        a = np.ascontiguousarray(p, np.float32).reshape(self.nv, 3)
        check(self.lib.mguso_write_positions(self.h, ptr(a)))

    @property
    def velocities(self) -> np.ndarray:
        out = np.empty((self.nv, 3), np.float32)
        check(self.lib.mguso_read_velocities(self.h, ptr(out)))
        return out

    @velocities.setter
    def velocities(self, v):
        a = np.ascontiguousarray(v, np.float32).reshape(self.nv, 3)
        check(self.lib.mguso_write_velocities(self.h, ptr(a)))

    def set_kinematic_collider_positions(self, x) -> None:
        """Move the static mesh collider to ``x`` (rows of the static mask; the others are
        ignored) between steps, with the velocity of that move
        (ImplicitSolver::set_kinematic_collider_positions, implicit.rs:1368-1398). Raises
        MgusoError, changing nothing, without a static collider or with a non-finite row."""
        a = np.ascontiguousarray(x, np.float32).reshape(self.nv, 3)
        check(self.lib.mguso_set_kinematic_collider_positions(self.h, ptr(a)))

    def set_pins(self, pins) -> None:
        """ImplicitSolver::set_pins (implicit.rs:826-838): each pin (index, target xyz, ghat,
        kinematic, stiffness). All or nothing: raises MgusoError, keeping the previous pins,
        for an index out of range or a ghat <= 0; an empty list clears them."""
        n = len(pins)
        idx = np.array([p[0] for p in pins], np.uint32)
        tgt = np.array([p[1] for p in pins], np.float32).reshape(n, 3)
        gh = np.array([p[2] for p in pins], np.float32)
        kin = np.array([1 if p[3] else 0 for p in pins], np.uint8)
        st = np.array([p[4] for p in pins], np.float32)
        check(self.lib.mguso_set_pins(self.h, n, ptr(idx) if n else None, ptr(tgt) if n else None,
                                      ptr(gh) if n else None, ptr(kin) if n else None, ptr(st) if n else None))

    def set_pulls(self, pulls) -> None:
        """ImplicitSolver::set_pulls (implicit.rs:852-864): each pull (index, target xyz,
        weight); all or nothing as set_pins."""
        n = len(pulls)
        idx = np.array([p[0] for p in pulls], np.uint32)
        tgt = np.array([p[1] for p in pulls], np.float32).reshape(n, 3)
        w = np.array([p[2] for p in pulls], np.float32)
        check(self.lib.mguso_set_pulls(self.h, n, ptr(idx) if n else None, ptr(tgt) if n else None,
                                       ptr(w) if n else None))

    def set_strain_limit_faces(self, faces, limits, masses) -> int:
        """ImplicitSolver::set_strain_limit_faces (implicit.rs:1088-1121): the strain-limit
        barrier on each face (u32 (n, 3)) with its limit (allowed principal-stretch excess)
        and mass, rest shape from the current positions; faces with a limit or mass <= 0 and
        degenerate faces are skipped. Returns the number kept. Raises ValueError when the
        arrays' lengths disagree (the reference's Err), MgusoError for an index out of range
        or a face whose vertex pair shares no element."""
        f = np.ascontiguousarray(faces, np.uint32).reshape(-1, 3)
        lim = np.ascontiguousarray(limits, np.float32).reshape(-1)
        m = np.ascontiguousarray(masses, np.float32).reshape(-1)
        if lim.size != f.shape[0] or m.size != f.shape[0]:
            raise ValueError(f"strain-limit arrays must match the face count: {f.shape[0]} faces, "
                             f"{lim.size} limits, {m.size} masses")
        n = f.shape[0]
        kept = C.c_uint32()
        check(self.lib.mguso_set_strain_limit_faces(self.h, n, ptr(f) if n else None, ptr(lim) if n else None,
                                                    ptr(m) if n else None, C.byref(kept)))
        return int(kept.value)

    def info(self) -> dict:
        out = np.zeros(6, np.uint32)
        check(self.lib.mguso_scene_info(self.h, ptr(out)))
        return dict(zip(["hinges", "shells", "edges", "collider_tris", "nnz_system", "nnz_pinned"], out.tolist()))

    def spmv_time(self, reps: int = 50):
        """(microseconds per system SpMV, algorithmic bytes per SpMV) at the last iterate."""
        us, b = C.c_float(), C.c_double()
        check(self.lib.mguso_scene_spmv_time(self.h, reps, C.byref(us), C.byref(b)))
        return us.value, b.value

    def profile(self, reps: int = 100) -> dict:
        """Per-kernel device time (us) and algorithmic bytes of the linear solver at the last
        assembled system: spmv, precond_apply, precond_factor, pcg_update."""
        us = np.zeros(4, np.float32)
        by = np.zeros(4, np.float64)
        check(self.lib.mguso_scene_profile(self.h, reps, ptr(us), ptr(by)))
        names = ["spmv", "precond_apply", "precond_factor", "pcg_update"]
        return {k: (float(u), float(b)) for k, u, b in zip(names, us, by)}

    def profile_pcg(self, iters: int = 64) -> dict:
        """Device time (us per launch, CUDA events around each launch) and algorithmic bytes
        of the two fused PCG kernels inside a solve of the last assembled system:
        {"rows": (us, bytes), "domains": (us, bytes)}."""
        us = np.zeros(2, np.float32)
        by = np.zeros(2, np.float64)
        check(self.lib.mguso_scene_profile_pcg(self.h, iters, ptr(us), ptr(by)))
        return {"rows": (float(us[0]), float(by[0])), "domains": (float(us[1]), float(by[1]))}

    def self_intersections(self, x) -> np.ndarray:
        """Piercing (edge, triangle) pairs per instance at positions ``x`` (the scan behind
        penetration_free, implicit.rs:618-650); the scene's positions are left at ``x``."""
        xx = np.ascontiguousarray(x, np.float32).reshape(self.nv, 3)
        out = np.zeros(getattr(self, "ninst", 1), np.uint32)
        check(self.lib.mguso_scene_self_intersections(self.h, ptr(xx), ptr(out)))
        return out

    def pcg_kernels(self) -> tuple:
        """(rows variant, domain variant) of the fused PCG in use (-1 before the first solve)."""
        out = np.zeros(2, np.int32)
        check(self.lib.mguso_scene_pcg_kernels(self.h, ptr(out)))
        return int(out[0]), int(out[1])

    def pcg_kernel_names(self) -> dict:
        """Kernel names of the fused PCG in use, for the mixed-precision FP16-tile step."""
        rv, dv = self.pcg_kernels()
        rows = "k_fr_rows_sell<double>" if rv == 3 else f"k_fr_rows<double, {({0: 2, 1: 1, 2: 4}).get(rv, 2)}>"
        if dv >= 4:
            dom = f"k_fr_schwarz_tc<double, {4 if dv == 4 else 8}>"
        else:
            dom = "k_fr_schwarz<double, __half>" if dv <= 0 else f"k_fr_schwarz3<double, __half, {(1, 2, 4)[dv - 1]}>"
        return {"rows": rows, "domains": dom}

    def ccd(self, x, dx):
        """Step fraction the CCD filter allows along ``dx`` from ``x`` (one per instance) and
        its ACCD cap hits (implicit.rs:1690-1947); the scene's positions are left at ``x``."""
        xx = np.ascontiguousarray(x, np.float32).reshape(self.nv, 3)
        dd = np.ascontiguousarray(dx, np.float32).reshape(self.nv, 3)
        k = getattr(self, "ninst", 1)
        t = np.zeros(k, np.float32)
        caps = np.zeros(k, np.uint32)
        check(self.lib.mguso_scene_ccd(self.h, ptr(xx), ptr(dd), ptr(t), ptr(caps)))
        return t, caps

    def assemble(self, x, x_tilde=None, exact: bool = False) -> dict:
        """One Newton-system assembly at positions ``x`` (inertia target ``x_tilde``, ``x``
        when None), downloaded as the fixed-pattern blocks ``ps`` and the contact-only
        blocks ``c`` (each ``(row_ptr, col, val[nnz, 3, 3])``) plus ``rhs``; the scene's
        positions are left at ``x``. ``exact``: the adjoint's exact Hessian instead of the
        step's projected one (mguso_scene_assemble_exact)."""
        xx = np.ascontiguousarray(x, np.float32)
        xt = None if x_tilde is None else np.ascontiguousarray(x_tilde, np.float32)
        n3 = np.zeros(3, np.uint32)
        fn = self.lib.mguso_scene_assemble_exact if exact else self.lib.mguso_scene_assemble
        check(fn(self.h, ptr(xx), ptr(xt) if xt is not None else None, ptr(n3)))
        nps, nc, nst = (int(v) for v in n3)
        ps_rp = np.empty(self.nv + 1, np.uint32)
        ps_col = np.empty(nps, np.uint32)
        ps_val = np.empty((nps, 3, 3), np.float32)
        c_rp = np.empty(self.nv + 1, np.uint32)
        c_col = np.empty(max(nc, 1), np.uint32)
        c_val = np.empty((max(nc, 1), 3, 3), np.float32)
        rhs = np.empty(3 * self.nv, np.float32)
        check(self.lib.mguso_scene_system(self.h, ptr(ps_rp), ptr(ps_col), ptr(ps_val), ptr(c_rp), ptr(c_col),
                                          ptr(c_val), ptr(rhs)))
        return {"ps": (ps_rp, ps_col, ps_val), "c": (c_rp, c_col[:nc], c_val[:nc]), "rhs": rhs, "stencils": nst}

    def stencils(self):
        """Contact stencils of the last ``assemble``: (idx[n, 4], kind[n], gap[n])."""
        n = C.c_uint32()
        check(self.lib.mguso_scene_stencils(self.h, 0, None, None, None, C.byref(n)))
        idx = np.empty((max(n.value, 1), 4), np.uint32)
        kind = np.empty(max(n.value, 1), np.uint32)
        d = np.empty(max(n.value, 1), np.float64)
        check(self.lib.mguso_scene_stencils(self.h, n.value, ptr(idx), ptr(kind), ptr(d), C.byref(n)))
        return idx[:n.value], kind[:n.value], d[:n.value]

    def close(self):
        if self.h:
            self.lib.mguso_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ImplicitBatch(ImplicitSolver):
    """Independent drapes stepped together (mguso_batch_create): one scene whose vertices are
    the instances' vertices concatenated; each instance keeps its own Newton loop."""

    def __init__(self, ctx, scenes_: list, precision: str = "mixed"):
        self.ctx = ctx
        self.lib = ctx.lib
        _sigs(self.lib)
        pairs = [_desc(sc, precision) for sc in scenes_]
        arr = (SceneDesc * len(pairs))(*[d for d, _ in pairs])
        self._keep = (pairs, arr)
        h = C.c_void_p()
        check(self.lib.mguso_batch_create(ctx.h, arr, len(pairs), C.byref(h)))
        self.h = h
        ctx.own(self)
        n = C.c_uint32()
        offs = np.zeros(len(pairs) + 1, np.uint32)
        check(self.lib.mguso_scene_instances(h, C.byref(n), ptr(offs)))
        self.ninst = n.value
        self.offsets = offs
        self.nv = int(offs[-1])
        self.history = []

    def instance_positions(self, k: int) -> np.ndarray:
        return self.positions[self.offsets[k]:self.offsets[k + 1]]
