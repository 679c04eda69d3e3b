"""ctypes wrapper of the CPU oracle (liboracle.so). TEST INFRASTRUCTURE ONLY.

Only tests/, the smoke check and the benchmark's CPU-baseline leg import this module; it
is the checker, never the product.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def build() -> None:
    subprocess.check_call(["make", "-s", "-C", HERE])


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    lib = C.CDLL(LIB)
    vp, u32, i32, f32, f64, u64 = C.c_void_p, C.c_uint32, C.c_int, C.c_float, C.c_double, C.c_uint64
    P = C.POINTER
    sigs = {
        "oracle_csr_from_triplets": (vp, [u32, vp, vp, vp, u64]),
        "oracle_csr_from_sink": (vp, [u32, vp, vp, vp, u64, vp, u32]),
        "oracle_csr_nnz": (u64, [vp]),
        "oracle_csr_copy": (None, [vp, vp, vp, vp]),
        "oracle_csr_free": (None, [vp]),
        "oracle_spmv": (None, [u32, vp, vp, vp, vp, vp]),
        "oracle_cg": (i32, [u32, vp, vp, vp, vp, f32, u32, i32, u32, vp, P(u32), P(f64)]),
        "oracle_linear_solve": (i32, [u32, vp, vp, vp, vp, f32, u32, i32, u32, vp, P(u32), P(f64)]),
        "oracle_schwarz_domains": (u32, [u32, vp, vp, u32, vp]),
        "oracle_schwarz_apply": (None, [u32, vp, vp, vp, u32, vp, vp]),
        "oracle_linear_solve_ml": (i32, [u32, vp, vp, vp, vp, f32, u32, u32, f64, vp, P(u32), P(f64)]),
        "oracle_schwarz_ml_apply": (None, [u32, vp, vp, vp, u32, f64, vp, vp]),
        "oracle_schwarz_ml_plan": (u32, [u32, vp, vp, vp, u32, vp, vp, P(u64), vp, vp, vp]),
        "oracle_morton": (None, [vp, vp, u64, i32, vp]),
        "oracle_centroid_bounds": (None, [vp, vp, u64, vp, vp]),
        "oracle_sort_pairs": (None, [vp, vp, u64]),
        "oracle_karras": (None, [vp, u64, i32, vp, vp]),
        "oracle_refit": (None, [vp, vp, vp, u64, vp]),
        "oracle_lbvh": (u64, [vp, u64, vp, u64, i32, f32, vp, vp, vp, vp, vp, vp, u64]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def csr_from_triplets(n, rows, cols, vals, sink=False, pinned=None):
    """CsrMatrix::from_triplets (csr.rs:37-91), or the TripletSink + finish path."""
    lib = load()
    r = np.ascontiguousarray(rows, np.uint32)
    c = np.ascontiguousarray(cols, np.uint32)
    v = np.ascontiguousarray(vals, np.float32)
    if sink:
        pin = None if pinned is None else np.ascontiguousarray(pinned, np.uint8)
        h = lib.oracle_csr_from_sink(n, _p(r), _p(c), _p(v), r.size, _p(pin), 0 if pin is None else pin.size)
    else:
        h = lib.oracle_csr_from_triplets(n, _p(r), _p(c), _p(v), r.size)
    nnz = lib.oracle_csr_nnz(h)
    rp = np.empty(n + 1, np.uint32)
    ci = np.empty(nnz, np.uint32)
    vv = np.empty(nnz, np.float32)
    lib.oracle_csr_copy(h, _p(rp), _p(ci), _p(vv))
    lib.oracle_csr_free(h)
    return rp, ci, vv


def spmv(n, rp, ci, vv, x):
    lib = load()
    y = np.empty(n, np.float32)
    xx = np.ascontiguousarray(x, np.float32)
    lib.oracle_spmv(n, _p(rp), _p(ci), _p(vv), _p(xx), _p(y))
    return y


def cg(n, rp, ci, vv, b, tol, max_iter, kind="block", domain=32):
    """cg_cpu_precond (linsolve.rs:272-346); kind diagonal | block | schwarz."""
    lib = load()
    k = {"diagonal": 0, "block": 1, "schwarz": 2}[kind]
    x = np.empty(n, np.float32)
    it, res = C.c_uint32(), C.c_double()
    bb = np.ascontiguousarray(b, np.float32)
    lib.oracle_cg(n, _p(rp), _p(ci), _p(vv), _p(bb), tol, max_iter, k, domain, _p(x), C.byref(it), C.byref(res))
    return x, it.value, res.value


def linear_solve(n, rp, ci, vv, b, tol, max_iter, kind="schwarz", domain=32):
    """CgCpu (kind block) / SchwarzCpu(domain) LinearSolver::solve + last_stats."""
    lib = load()
    k = {"block": 1, "schwarz": 2}[kind]
    x = np.empty(n, np.float32)
    it, res = C.c_uint32(), C.c_double()
    bb = np.ascontiguousarray(b, np.float32)
    lib.oracle_linear_solve(n, _p(rp), _p(ci), _p(vv), _p(bb), tol, max_iter, k, domain, _p(x), C.byref(it),
                            C.byref(res))
    return x, it.value, res.value


def linear_solve_ml(n, rp, ci, vv, b, tol, max_iter, domain=16, weight=0.7):
    """SchwarzMlCpu(domain, weight) LinearSolver::solve + last_stats (linsolve.rs:779-836)."""
    lib = load()
    x = np.empty(n, np.float32)
    it, res = C.c_uint32(), C.c_double()
    bb = np.ascontiguousarray(b, np.float32)
    lib.oracle_linear_solve_ml(n, _p(rp), _p(ci), _p(vv), _p(bb), C.c_float(tol), max_iter, domain,
                               C.c_double(weight), _p(x), C.byref(it), C.byref(res))
    return x, it.value, res.value


def schwarz_ml_apply(n, rp, ci, vv, domain, weight, r):
    """z = S0 r + w C1^T S1 (C1 r), the two-level Schwarz apply in f64 (linsolve.rs:641-666)."""
    lib = load()
    rr = np.ascontiguousarray(r, np.float64)
    z = np.empty(n, np.float64)
    lib.oracle_schwarz_ml_apply(n, _p(rp), _p(ci), _p(vv), domain, C.c_double(weight), _p(rr), _p(z))
    return z


def schwarz_ml_plan(n, rp, ci, vv, domain):
    """(agg0[nv], coarse_dom[n_coarse], coarse CSR (rp, ci, v)) of the two-level Schwarz."""
    lib = load()
    agg = np.empty(n // 3, np.uint32)
    cdom = np.empty(n // 3, np.uint32)
    nnz = C.c_uint64()
    nc = lib.oracle_schwarz_ml_plan(n, _p(rp), _p(ci), _p(vv), domain, _p(agg), _p(cdom), C.byref(nnz), None, None,
                                    None)
    crp = np.empty(3 * nc + 1, np.uint32)
    cci = np.empty(nnz.value, np.uint32)
    cv = np.empty(nnz.value, np.float32)
    lib.oracle_schwarz_ml_plan(n, _p(rp), _p(ci), _p(vv), domain, _p(agg), _p(cdom), C.byref(nnz), _p(crp), _p(cci),
                               _p(cv))
    return agg, cdom[:nc], (crp, cci, cv)


def schwarz_domains(n, rp, ci, domain):
    lib = load()
    out = np.empty(n // 3, np.uint32)
    nd = lib.oracle_schwarz_domains(n, _p(rp), _p(ci), domain, _p(out))
    return out, nd


def schwarz_apply(n, rp, ci, vv, domain, r):
    lib = load()
    rr = np.ascontiguousarray(r, np.float64)
    z = np.empty(n, np.float64)
    lib.oracle_schwarz_apply(n, _p(rp), _p(ci), _p(vv), domain, _p(rr), _p(z))
    return z


def morton(pos, tris, bits):
    lib = load()
    p = np.ascontiguousarray(pos, np.float32)
    t = np.ascontiguousarray(tris, np.uint32)
    out = np.empty(t.shape[0], np.uint64)
    lib.oracle_morton(_p(p), _p(t), t.shape[0], bits, _p(out))
    return out


def sort_pairs(keys, vals):
    lib = load()
    k = np.ascontiguousarray(keys, np.uint64).copy()
    v = np.ascontiguousarray(vals, np.uint32).copy()
    lib.oracle_sort_pairs(_p(k), _p(v), k.size)
    return k, v


def karras(keys, bits):
    lib = load()
    k = np.ascontiguousarray(keys, np.uint64)
    n = k.size
    left = np.empty(max(n - 1, 0), np.uint32)
    right = np.empty(max(n - 1, 0), np.uint32)
    lib.oracle_karras(_p(k), n, bits, _p(left) if n > 1 else None, _p(right) if n > 1 else None)
    return left, right


def refit(left, right, leaf):
    lib = load()
    n = leaf.shape[0]
    node = np.empty((max(n - 1, 0), 6), np.float32)
    lib.oracle_refit(_p(left), _p(right), _p(np.ascontiguousarray(leaf, np.float32)), n,
                     _p(node) if n > 1 else None)
    return node


def lbvh(pos, tris, bits, dhat, cap=None):
    """Whole CPU LBVH: (keys, perm, left, right, node boxes, sorted (v, tri) pairs)."""
    lib = load()
    p = np.ascontiguousarray(pos, np.float32)
    t = np.ascontiguousarray(tris, np.uint32)
    nv, nt = p.shape[0], t.shape[0]
    keys = np.empty(nt, np.uint64)
    perm = np.empty(nt, np.uint32)
    left = np.empty(max(nt - 1, 1), np.uint32)
    right = np.empty(max(nt - 1, 1), np.uint32)
    node = np.empty((max(nt - 1, 1), 6), np.float32)
    if cap is None:
        cnt = lib.oracle_lbvh(_p(p), nv, _p(t), nt, bits, dhat, None, None, None, None, None, None, 0)
        cap = cnt
    pairs = np.empty((max(cap, 1), 2), np.uint32)
    cnt = lib.oracle_lbvh(_p(p), nv, _p(t), nt, bits, dhat, _p(keys), _p(perm), _p(left), _p(right), _p(node),
                          _p(pairs), cap)
    return keys, perm, left[:max(nt - 1, 0)], right[:max(nt - 1, 0)], node[:max(nt - 1, 0)], pairs[:min(cnt, cap)]


# ---- implicit step ---------------------------------------------------------------------
class OracleParams(C.Structure):
    _fields_ = [("dt", C.c_float), ("gravity", C.c_float * 3), ("newton_iters", C.c_uint32),
                ("stiffness", C.c_float), ("bend_stiffness", C.c_float), ("max_dx", C.c_float),
                ("target_toi", C.c_float), ("min_newton_steps", C.c_uint32), ("ccd_max_iter", C.c_uint32),
                ("eiganalysis_eps", C.c_float), ("contact_dhat", C.c_float), ("contact_kappa", C.c_float),
                ("contact_dynamic", C.c_float), ("shell_mu", C.c_float), ("shell_lambda", C.c_float),
                ("friction", C.c_float), ("friction_eps", C.c_float), ("barrier_kind", C.c_int),
                ("contact_rayleigh", C.c_int), ("self_collision", C.c_int), ("cg_tol", C.c_float),
                ("cg_max_iter", C.c_uint32), ("floor_y", C.c_float), ("newton_tol", C.c_float),
                ("precond", C.c_int), ("schwarz_domain", C.c_uint32)]


class OracleStats(C.Structure):
    _fields_ = [("newton_iters", C.c_uint32), ("max_cg_iters", C.c_uint32), ("num_contacts", C.c_uint32),
                ("stencils", C.c_uint32), ("ccd_cap_hits", C.c_uint32), ("max_reresid", C.c_double),
                ("t_min", C.c_double), ("penetration_free", C.c_int), ("all_finite", C.c_int)]


def _step_sigs(lib):
    vp, u32, i32, f32 = C.c_void_p, C.c_uint32, C.c_int, C.c_float
    P = C.POINTER
    sigs = {
        "oracle_solver_new": (vp, [i32, u32, vp, vp, vp, u32, vp, vp, u32, vp, u32, vp, vp, vp, u32, vp,
                                   P(OracleParams)]),
        "oracle_solver_free": (None, [vp]),
        "oracle_solver_step": (i32, [vp, i32, i32, vp]),
        "oracle_solver_state": (None, [vp, vp, vp]),
        "oracle_solver_set_state": (None, [vp, vp, vp]),
        "oracle_solver_set_kinematic": (i32, [vp, vp]),
        "oracle_solver_counts": (None, [vp, vp]),
        "oracle_solver_stencils": (u32, [vp, vp, vp, u32]),
        "oracle_solver_assemble": (vp, [vp, vp, vp, vp]),
        "oracle_solver_ccd": (f32, [vp, vp]),
        "oracle_point_tri": (f32, [vp, vp, vp]),
        "oracle_seg_seg": (f32, [vp, vp, vp]),
        "oracle_accd": (f32, [vp, vp, f32, f32, f32, u32, i32]),
        "oracle_barrier": (i32, [i32, C.c_double, C.c_double, C.c_double, i32, vp]),
        "oracle_rayleigh": (f32, [i32, vp, vp, vp, vp, f32]),
        "oracle_friction": (i32, [vp, vp, vp, f32, f32, vp, vp]),
        "oracle_shell": (i32, [i32, vp, vp, C.c_double, C.c_double, C.c_double, vp, vp, vp]),
        "oracle_hinge": (C.c_double, [i32, vp, vp, vp]),
        "oracle_stitch": (None, [vp, vp, C.c_double, C.c_double, vp, vp]),
        "oracle_solver_set_shells": (None, [vp, C.c_uint32, vp, vp, vp, vp]),
        "oracle_solver_scale_stitches": (None, [vp, vp]),
        "oracle_solver_collider_sides": (i32, [vp, vp]),
        "oracle_solver_self_intersect": (i32, [vp, vp]),
        "oracle_solver_set_shell_stiffness": (i32, [vp, u32, vp]),
        "oracle_solver_set_membrane": (i32, [vp, C.c_double, C.c_double, C.c_double, u32, vp]),
        "oracle_membrane_element": (i32, [vp, vp, f32, f32, f32, vp, vp, vp, vp]),
        "oracle_membrane_materials": (None, [vp, vp, vp, i32, vp, vp]),
        "oracle_solver_hinges": (u32, [vp, vp, vp, u32]),
        "oracle_solver_set_pins": (i32, [vp, u32, vp, vp, vp, vp, vp]),
        "oracle_solver_set_pulls": (i32, [vp, u32, vp, vp, vp]),
        "oracle_solver_set_strain_limit_faces": (i32, [vp, u32, vp, vp, vp, u32, u32]),
        "oracle_solver_set_limits": (None, [vp, C.c_double, C.c_double, C.c_double, C.c_double, u32, vp]),
        "oracle_solver_set_stretch_edges": (None, [vp, u32, vp]),
        "oracle_solver_set_friction": (None, [vp, C.c_double, i32]),
        "oracle_strain_limit_face": (i32, [i32, i32, vp, vp, C.c_double, C.c_double, C.c_double, C.c_double, i32,
                                           vp, vp, vp]),
        "oracle_edge_strain": (f32, [vp, vp, f32, f32, f32, vp, vp]),
        "oracle_vt_pairs": (C.c_uint64, [u32, vp, u32, vp, f32, i32, vp, vp, C.c_uint64]),
        "oracle_ee_pairs": (C.c_uint64, [u32, vp, u32, vp, f32, vp, vp, C.c_uint64]),
        "oracle_unique_edges": (u32, [u32, vp, vp]),
        "oracle_grid_cell": (f32, [f32, f32]),
        "oracle_et_pairs": (C.c_uint64, [u32, vp, u32, vp, u32, vp, f32, vp, C.c_uint64]),
        "oracle_sym_eig2": (None, [vp, vp, vp]),
        "oracle_asm_blocks": (None, [u32, u32, vp, u32, vp, vp, vp]),
        "oracle_svd3x2": (None, [vp, vp, vp, vp]),
        "oracle_stvk_density": (f32, [vp, f32, f32, vp, vp]),
        "oracle_et_any": (i32, [u32, vp, u32, vp, u32, vp, f32, vp, i32, vp, C.c_uint64, vp]),
        "oracle_edge_triangle_intersect": (i32, [vp]),
        "oracle_closest_point": (None, [vp, vp, vp]),
        "oracle_ee_witness": (None, [vp, vp]),
        "oracle_signed_point_tri": (f32, [vp, vp, vp]),
        "oracle_collider_distance": (f32, [vp, vp, vp]),
        "oracle_vertex_contact": (None, [vp, u32, vp, f32, f32, f32, f32, vp, vp]),
        "oracle_dynamic_stiffness": (f32, [f32, f32, f32, f32, f32]),
        "oracle_stencil_friction": (i32, [vp, vp, f32, f32, f32, vp, vp]),
        "oracle_adjoint_system": (i32, [vp, u32, u32, vp, vp, vp, vp, vp, vp, vp, vp, C.c_double, vp, vp]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def params_struct(p: dict) -> OracleParams:
    s = OracleParams()
    for k, v in p.items():
        if k == "gravity":
            s.gravity[:] = list(v)
        elif hasattr(s, k):
            setattr(s, k, v)
    return s


class OracleSolver:
    """The reference's ImplicitSolver restated on the CPU (float) or as the FP64 oracle."""

    def __init__(self, scene: dict, precision: str = "f32"):
        lib = load()
        _step_sigs(lib)
        self.lib = lib
        sc = scene
        self.keep = [np.ascontiguousarray(sc[k]) for k in ("positions", "velocities", "inv_mass", "tris",
                                                          "shell_faces", "stitch_idx", "stitch_w", "stitch_kl",
                                                          "colliders")]
        pos, vel, im, tris, sf, si, sw, skl, cols = self.keep
        mask = sc.get("static_mask")
        self.mask = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        self.params = params_struct(sc["params"])
        self.nv = pos.shape[0]
        self.h = lib.oracle_solver_new(0 if precision == "f32" else 1, self.nv, _p(pos), _p(vel), _p(im),
                                       tris.shape[0], _p(tris), _p(self.mask), sf.shape[0], _p(sf), si.shape[0],
                                       _p(si), _p(sw), _p(skl), cols.shape[0], _p(cols), C.byref(self.params))

    def step(self, n: int = 1, check_intersection: bool = True):
        out = (OracleStats * n)()
        self.lib.oracle_solver_step(self.h, n, 1 if check_intersection else 0, out)
        return [{f: getattr(o, f) for f, _ in OracleStats._fields_} for o in out]

    def positions(self) -> np.ndarray:
        p = np.empty((self.nv, 3), np.float64)
        self.lib.oracle_solver_state(self.h, _p(p), None)
        return p

    def velocities(self) -> np.ndarray:
        v = np.empty((self.nv, 3), np.float64)
        self.lib.oracle_solver_state(self.h, None, _p(v))
        return v

    def set_kinematic_collider_positions(self, x) -> bool:
        """Move the static collider to x (its rows; implicit.rs:1368-1398)."""
        p = np.ascontiguousarray(x, np.float64)
        if p.size != 3 * self.nv:
            return False  # a wrong-length array is refused, as the reference's setter does
        return bool(self.lib.oracle_solver_set_kinematic(self.h, _p(p)))

    def set_state(self, pos, vel):
        """Overwrite positions and/or velocities (f64 (nv, 3)); None leaves that one as is."""
        p = None if pos is None else np.ascontiguousarray(pos, np.float64).reshape(self.nv, 3)
        v = None if vel is None else np.ascontiguousarray(vel, np.float64).reshape(self.nv, 3)
        self.lib.oracle_solver_set_state(self.h, _p(p), _p(v))

    def counts(self):
        out = np.zeros(4, np.uint32)
        self.lib.oracle_solver_counts(self.h, _p(out))
        return dict(zip(["hinges", "shells", "edges", "collider_tris"], out.tolist()))

    def stencils(self, cap=1 << 20):
        idx = np.empty((cap, 4), np.uint32)
        d = np.empty(cap, np.float32)
        n = self.lib.oracle_solver_stencils(self.h, _p(idx), _p(d), cap)
        return idx[:min(n, cap)], d[:min(n, cap)]

    def assemble(self, x=None, x_tilde=None):
        n = 3 * self.nv
        rhs = np.empty(n, np.float32)
        xx = None if x is None else np.ascontiguousarray(x, np.float32)
        xt = None if x_tilde is None else np.ascontiguousarray(x_tilde, np.float32)
        h = self.lib.oracle_solver_assemble(self.h, _p(xx), _p(xt), _p(rhs))
        nnz = self.lib.oracle_csr_nnz(h)
        rp = np.empty(n + 1, np.uint32)
        ci = np.empty(nnz, np.uint32)
        vv = np.empty(nnz, np.float32)
        self.lib.oracle_csr_copy(h, _p(rp), _p(ci), _p(vv))
        self.lib.oracle_csr_free(h)
        return (rp, ci, vv), rhs

    def ccd(self, dx):
        d = np.ascontiguousarray(dx, np.float32)
        return float(self.lib.oracle_solver_ccd(self.h, _p(d)))

    def set_shells(self, faces, rest, mu, lam):
        """Replace the shells with explicit rest data (inverse rest shape column-major and
        area per face) and per-face (mu, lambda)."""
        f = np.ascontiguousarray(faces, np.uint32)
        r = np.ascontiguousarray(rest, np.float64)
        m = np.ascontiguousarray(mu, np.float64)
        l_ = np.ascontiguousarray(lam, np.float64)
        self.lib.oracle_solver_set_shells(self.h, f.shape[0], _p(f), _p(r), _p(m), _p(l_))

    def set_membrane(self, warp=0.0, weft=0.0, shear=0.0, per_element=None) -> bool:
        """Baraff-Witkin membrane stiffnesses (ImplicitParams::membrane_*), or per element
        (n, 3) for the membrane built from every triangle; False on a count mismatch."""
        k = None if per_element is None else np.ascontiguousarray(per_element, np.float64).reshape(-1, 3)
        return bool(self.lib.oracle_solver_set_membrane(self.h, warp, weft, shear, 0 if k is None else k.shape[0],
                                                        _p(k)))

    def set_shell_stiffness(self, mu_lam) -> bool:
        """Per-face (mu, lambda) for the shells in order; False when the count differs."""
        a = np.ascontiguousarray(mu_lam, np.float64).reshape(-1, 2)
        return bool(self.lib.oracle_solver_set_shell_stiffness(self.h, a.shape[0], _p(a)))

    def hinges(self):
        """(vertices (n, 4) u32, rest angles (n,) f64) of build_hinges."""
        n = self.lib.oracle_solver_hinges(self.h, None, None, 0)
        idx = np.zeros((max(n, 1), 4), np.uint32)
        rest = np.zeros(max(n, 1), np.float64)
        self.lib.oracle_solver_hinges(self.h, _p(idx), _p(rest), n)
        return idx[:n], rest[:n]

    def self_intersects(self, pos) -> bool:
        """positions_self_intersect (implicit.rs:618-650) at pos."""
        p = np.ascontiguousarray(pos, np.float32).reshape(self.nv, 3)
        return bool(self.lib.oracle_solver_self_intersect(self.h, _p(p)))

    def collider_sides(self):
        """Per-vertex side of the static collider at the current positions (+1 outside, -1
        inside; implicit.rs:1431-1480), or None without a static collider."""
        out = np.ones(self.nv, np.float32)
        return out if self.lib.oracle_solver_collider_sides(self.h, _p(out)) else None

    def set_pins(self, pins) -> bool:
        """Pins (implicit.rs:826-838), each (index, target xyz, ghat, kinematic, stiffness);
        all or nothing: False, with the previous pins kept, when one is out of range or has
        ghat <= 0."""
        n = len(pins)
        idx = np.array([p[0] for p in pins], np.uint32)
        tgt = np.array([p[1] for p in pins], np.float64).reshape(n, 3)
        gh = np.array([p[2] for p in pins], np.float64)
        kin = np.array([1 if p[3] else 0 for p in pins], np.int32)
        st = np.array([p[4] for p in pins], np.float64)
        return bool(self.lib.oracle_solver_set_pins(self.h, n, _p(idx), _p(tgt), _p(gh), _p(kin), _p(st)))

    def set_pulls(self, pulls) -> bool:
        """Pulls (implicit.rs:852-864), each (index, target xyz, weight)."""
        n = len(pulls)
        idx = np.array([p[0] for p in pulls], np.uint32)
        tgt = np.array([p[1] for p in pulls], np.float64).reshape(n, 3)
        w = np.array([p[2] for p in pulls], np.float64)
        return bool(self.lib.oracle_solver_set_pulls(self.h, n, _p(idx), _p(tgt), _p(w)))

    def set_strain_limit_faces(self, faces, limits, masses) -> int:
        """Strain-limit barrier faces (implicit.rs:1088-1121), rest shape from the current
        positions; returns the number kept. Raises ValueError when the lengths disagree."""
        f = np.ascontiguousarray(faces, np.uint32).reshape(-1, 3)
        lim = np.ascontiguousarray(limits, np.float64).reshape(-1)
        m = np.ascontiguousarray(masses, np.float64).reshape(-1)
        k = self.lib.oracle_solver_set_strain_limit_faces(self.h, f.shape[0], _p(f), _p(lim), _p(m), lim.size, m.size)
        if k < 0:
            raise ValueError(f"strain-limit arrays must match the face count: {f.shape[0]} faces, "
                             f"{lim.size} limits, {m.size} masses")
        return int(k)

    def set_limits(self, constraint_tol=1e-2, strain_limit_ratio=0.0, strain_limit_k=0.0,
                   strain_limit_ratio_weft=0.0, uvs=None):
        """Pin gap floor, per-edge strain limit and per-vertex UVs (the ImplicitParams fields
        of the same names; uvs None clears them)."""
        uv = None if uvs is None else np.ascontiguousarray(uvs, np.float64).reshape(-1, 2)
        self.lib.oracle_solver_set_limits(self.h, constraint_tol, strain_limit_ratio, strain_limit_k,
                                          strain_limit_ratio_weft, 0 if uv is None else uv.shape[0], _p(uv))

    def set_collider_friction(self, collider_friction=float("inf"), mode="min"):
        """The collider's coefficient (inf: unset) and the mode it combines with the cloth's
        under (ImplicitParams::collider_friction, friction_mode)."""
        self.lib.oracle_solver_set_friction(self.h, collider_friction, {"min": 0, "max": 1, "mean": 2}[mode])

    def set_stretch_edges(self, edges):
        """Replace the stretch edges (rest lengths from the current positions)."""
        e = np.ascontiguousarray(edges, np.uint32).reshape(-1, 2)
        self.lib.oracle_solver_set_stretch_edges(self.h, e.shape[0], _p(e))

    def scale_stitches(self, factor):
        f = np.ascontiguousarray(factor, np.float64)
        self.lib.oracle_solver_scale_stitches(self.h, _p(f))

    def close(self):
        if self.h:
            self.lib.oracle_solver_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _lib_elem():
    lib = load()
    _step_sigs(lib)
    return lib


def point_tri(p4):
    lib = _lib_elem()
    p = np.ascontiguousarray(p4, np.float32).reshape(12)
    g = np.empty(12, np.float32)
    w = np.empty(3, np.float32)
    d = lib.oracle_point_tri(_p(p), _p(g), _p(w))
    return d, g.reshape(4, 3), w


def seg_seg(p4):
    lib = _lib_elem()
    p = np.ascontiguousarray(p4, np.float32).reshape(12)
    g = np.empty(12, np.float32)
    plain = C.c_float()
    pl = np.empty(1, np.float32)
    d = lib.oracle_seg_seg(_p(p), _p(g), _p(pl))
    return d, g.reshape(4, 3), float(pl[0])


def accd(x4, dx4, offset=0.0, max_t=1.25, reduction=0.01, max_iter=256, kind="pt"):
    lib = _lib_elem()
    x = np.ascontiguousarray(x4, np.float32).reshape(12)
    d = np.ascontiguousarray(dx4, np.float32).reshape(12)
    return lib.oracle_accd(_p(x), _p(d), offset, max_t, reduction, max_iter, 0 if kind == "pt" else 1)


def barrier(d, dhat, kappa, kind="log", f64=False):
    lib = _lib_elem()
    out = np.zeros(3, np.float64)
    on = lib.oracle_barrier(0 if kind == "log" else 1, d, dhat, kappa, 1 if f64 else 0, _p(out))
    return (tuple(out.tolist()) if on else None)


def friction(force_contact, dx, normal, mu, eps):
    """contact.rs friction: (gradient 3, Hessian 3x3), zeros when it does not apply."""
    lib = _lib_elem()
    f = np.ascontiguousarray(force_contact, np.float32)
    d = np.ascontiguousarray(dx, np.float32)
    n = np.ascontiguousarray(normal, np.float32)
    g = np.zeros(3, np.float32)
    h = np.zeros(9, np.float32)
    lib.oracle_friction(_p(f), _p(d), _p(n), mu, eps, _p(g), _p(h))
    return g, h.reshape(3, 3)


def rayleigh(elastic, mass, weights, e, offset=0.0):
    lib = _lib_elem()
    n = len(mass)
    el = np.ascontiguousarray(elastic, np.float32).reshape(n * n * 9)
    m = np.ascontiguousarray(mass, np.float32)
    w = np.ascontiguousarray(weights, np.float32)
    ee = np.ascontiguousarray(e, np.float32)
    return lib.oracle_rayleigh(n, _p(el), _p(m), _p(w), _p(ee), offset)


def shell(rest, p, mu, lam, eps=1e-6, f64=True):
    lib = _lib_elem()
    r = np.ascontiguousarray(rest, np.float64).reshape(9)
    q = np.ascontiguousarray(p, np.float64).reshape(9)
    e = np.zeros(1, np.float64)
    g = np.zeros(9, np.float64)
    h = np.zeros(81, np.float64)
    ok = lib.oracle_shell(1 if f64 else 0, _p(r), _p(q), mu, lam, eps, _p(e), _p(g), _p(h))
    return (float(e[0]), g.reshape(3, 3), h.reshape(9, 9)) if ok else None


def hinge(p4, f64=True):
    lib = _lib_elem()
    q = np.ascontiguousarray(p4, np.float64).reshape(12)
    g = np.zeros(12, np.float64)
    gf = np.zeros(12, np.float64)
    th = lib.oracle_hinge(1 if f64 else 0, _p(q), _p(g), _p(gf))
    return th, g.reshape(4, 3), gf.reshape(4, 3)


def stitch(x6, w6, l0, lcap):
    lib = _lib_elem()
    x = np.ascontiguousarray(x6, np.float64).reshape(18)
    w = np.ascontiguousarray(w6, np.float64)
    g = np.zeros(18, np.float64)
    h = np.zeros(324, np.float64)
    lib.oracle_stitch(_p(x), _p(w), l0, lcap, _p(g), _p(h))
    return g.reshape(6, 3), h.reshape(18, 18)


def strain_limit_face(rest, p, limit, kind="cubic", mass=0.0, elastic_k=0.0, eps=1e-6, dynamic=False, f64=False):
    """Strain-limit barrier of one face (shell_model.rs:438-640): (energy, gradient 3x3,
    Hessian 9x9, active); None for a degenerate rest face."""
    lib = _lib_elem()
    r = np.ascontiguousarray(rest, np.float64).reshape(9)
    q = np.ascontiguousarray(p, np.float64).reshape(9)
    e = np.zeros(1, np.float64)
    g = np.zeros(9, np.float64)
    h = np.zeros(81, np.float64)
    on = lib.oracle_strain_limit_face(1 if f64 else 0, 0 if kind == "log" else 1, _p(r), _p(q), limit, mass,
                                      elastic_k, eps, 1 if dynamic else 0, _p(e), _p(g), _p(h))
    if on < 0:
        return None
    return float(e[0]), g.reshape(3, 3), h.reshape(9, 9), bool(on)


def edge_strain(xi, xj, rest, ratio, k):
    """One-sided edge strain limit (strain_limit.rs:31-63) in f32: (energy, grad_i, h_ii)."""
    lib = _lib_elem()
    a = np.ascontiguousarray(xi, np.float32)
    b = np.ascontiguousarray(xj, np.float32)
    g = np.zeros(3, np.float32)
    h = np.zeros(9, np.float32)
    e = lib.oracle_edge_strain(_p(a), _p(b), rest, ratio, k, _p(g), _p(h))
    return float(e), g, h.reshape(3, 3)


def _pairs(fn, *args):
    n = fn(*args, None, 0)
    out = np.empty((max(n, 1), 2), np.uint32)
    fn(*args, _p(out), n)
    return [tuple(r) for r in out[:n].tolist()]


def vt_pairs(pos, tris, search, exclude_one_ring=True, movable=None):
    """vertex_triangle_pairs (broadphase.rs:250-264): sorted unique (vertex, triangle)."""
    lib = _lib_elem()
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(tris, np.uint32).reshape(-1, 3)
    m = None if movable is None or len(movable) == 0 else np.ascontiguousarray(movable, np.uint8)
    return _pairs(lib.oracle_vt_pairs, p.shape[0], _p(p), t.shape[0], _p(t), search, 1 if exclude_one_ring else 0,
                  _p(m))


def ee_pairs(pos, edges, search, movable=None):
    """edge_edge_pairs (broadphase.rs:356-367): sorted unique (ei, ej), ei < ej."""
    lib = _lib_elem()
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    e = np.ascontiguousarray(edges, np.uint32).reshape(-1, 2)
    m = None if movable is None or len(movable) == 0 else np.ascontiguousarray(movable, np.uint8)
    return _pairs(lib.oracle_ee_pairs, p.shape[0], _p(p), e.shape[0], _p(e), search, _p(m))


def asm_blocks(nv, slot_pairs, triplets):
    """The assembler's elastic-block gather: triplets (row, col, value) pushed in order with
    the vertex pairs slot_pairs requested; returns one row-major 3x3 block per slot."""
    keys = np.ascontiguousarray(slot_pairs, np.uint32).reshape(-1, 2)
    rc = np.ascontiguousarray([(r, c) for r, c, _ in triplets], np.uint32).reshape(-1, 2)
    v = np.ascontiguousarray([t[2] for t in triplets], np.float32)
    out = np.zeros((len(keys), 3, 3), np.float32)
    _lib_elem().oracle_asm_blocks(nv, len(keys), _p(keys), len(v), _p(rc), _p(v), _p(out))
    return out


def sym_eig2(p, q, r):
    """sym_eig2 (shell_model.rs:60-78) of [[p, q], [q, r]] in f32: (eigenvalues descending,
    eigenvectors as the columns of a 2x2)."""
    a = np.array([p, q, r], np.float32)
    lam = np.zeros(2, np.float32)
    v = np.zeros(4, np.float32)
    _lib_elem().oracle_sym_eig2(_p(a), _p(lam), _p(v))
    return lam, v.reshape(2, 2).T


def svd3x2(f):
    """svd3x2 (shell_model.rs:84-106) of a 3x2 F in f32: (U 3x2, sigma descending, V 2x2)."""
    fc = np.ascontiguousarray(np.asarray(f, np.float32).T)
    u = np.zeros(6, np.float32)
    s = np.zeros(2, np.float32)
    v = np.zeros(4, np.float32)
    _lib_elem().oracle_svd3x2(_p(fc), _p(u), _p(s), _p(v))
    return u.reshape(2, 3).T, s, v.reshape(2, 2).T


def stvk_density(sigma, mu, lam):
    """The StVK shell density over principal stretches (shell_model.rs:131-176) in f32:
    (psi, gradient 2, Hessian 2x2)."""
    s = np.ascontiguousarray(sigma, np.float32)
    g = np.zeros(2, np.float32)
    h = np.zeros(4, np.float32)
    e = _lib_elem().oracle_stvk_density(_p(s), mu, lam, _p(g), _p(h))
    return float(e), g, h.reshape(2, 2)


def et_pairs(pos, edges, tris, search):
    """edge_triangle_pairs (broadphase.rs:523-585): sorted unique (edge, triangle) candidates."""
    lib = _lib_elem()
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    e = np.ascontiguousarray(edges, np.uint32).reshape(-1, 2)
    t = np.ascontiguousarray(tris, np.uint32).reshape(-1, 3)
    return _pairs(lib.oracle_et_pairs, p.shape[0], _p(p), e.shape[0], _p(e), t.shape[0], _p(t), search)


ET_NEVER, ET_FIRST, ET_PIERCE = 0, 1, 2


def et_any(pos, edges, tris, search, movable=None, mode=ET_NEVER):
    """any_edge_triangle_pair (broadphase.rs:587-751) with the predicate `mode`: ET_NEVER (never
    matches; the candidates offered are returned, repeats included), ET_FIRST (matches the first
    candidate) or ET_PIERCE (edge_triangle_intersect). Returns (matched, offered): offered is
    the list of (edge, triangle) pairs for ET_NEVER, else the number of candidates seen."""
    lib = _lib_elem()
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    e = np.ascontiguousarray(edges, np.uint32).reshape(-1, 2)
    t = np.ascontiguousarray(tris, np.uint32).reshape(-1, 3)
    m = None if movable is None or len(movable) == 0 else np.ascontiguousarray(movable, np.uint8)
    n = np.zeros(1, np.uint64)
    args = (p.shape[0], _p(p), e.shape[0], _p(e), t.shape[0], _p(t), search, _p(m), mode)
    found = lib.oracle_et_any(*args, None, 0, _p(n))
    if mode != ET_NEVER:
        return bool(found), int(n[0])
    out = np.empty((max(int(n[0]), 1), 2), np.uint32)
    found = lib.oracle_et_any(*args, _p(out), int(n[0]), _p(n))
    return bool(found), [tuple(r) for r in out[:int(n[0])].tolist()]


def unique_edges(tris):
    """unique_edges (broadphase.rs:332-343): sorted (min, max) vertex pairs."""
    lib = _lib_elem()
    t = np.ascontiguousarray(tris, np.uint32).reshape(-1, 3)
    out = np.empty((3 * max(t.shape[0], 1), 2), np.uint32)
    n = lib.oracle_unique_edges(t.shape[0], _p(t), _p(out))
    return out[:n].copy()


def grid_cell(search, extent):
    return _lib_elem().oracle_grid_cell(search, extent)


def edge_triangle_intersect(p0, p1, a, b, c):
    return bool(_lib_elem().oracle_edge_triangle_intersect(_p(np.ascontiguousarray([p0, p1, a, b, c], np.float32))))


def closest_point(p, a, b, c):
    """closest_point_on_triangle_bary (contact.rs:84-124): (q, weights)."""
    lib = _lib_elem()
    x = np.ascontiguousarray([p, a, b, c], np.float32)
    q = np.zeros(3, np.float32)
    w = np.zeros(3, np.float32)
    lib.oracle_closest_point(_p(x), _p(q), _p(w))
    return q, w


def ee_witness(p4):
    """edge_edge_witness (contact.rs:238-311): weights (a0, a1, b0, b1)."""
    lib = _lib_elem()
    x = np.ascontiguousarray(p4, np.float32).reshape(12)
    w = np.zeros(4, np.float32)
    lib.oracle_ee_witness(_p(x), _p(w))
    return w


def signed_point_tri(p, a, b, c):
    """The signed point-triangle gap of a one-triangle collider: (gap, gradient 4x3, inside)."""
    lib = _lib_elem()
    x = np.ascontiguousarray([p, a, b, c], np.float32)
    g = np.zeros(12, np.float32)
    inside = np.zeros(1, np.int32)
    d = lib.oracle_signed_point_tri(_p(x), _p(g), _p(inside))
    return d, g.reshape(4, 3), bool(inside[0])


def collider_distance(col8, x):
    lib = _lib_elem()
    c = np.ascontiguousarray(col8, np.float32)
    xx = np.ascontiguousarray(x, np.float32)
    n = np.zeros(3, np.float32)
    d = lib.oracle_collider_distance(_p(c), _p(xx), _p(n))
    return d, n


def vertex_contact(x, colliders, dhat, kappa, coupling, mass):
    """vertex_contact (contact.rs:1029-1050): (gradient, Hessian 3x3)."""
    lib = _lib_elem()
    xx = np.ascontiguousarray(x, np.float32)
    cs = np.ascontiguousarray(colliders, np.float32).reshape(-1, 8)
    g = np.zeros(3, np.float32)
    h = np.zeros(9, np.float32)
    lib.oracle_vertex_contact(_p(xx), cs.shape[0], _p(cs), dhat, kappa, coupling, mass, _p(g), _p(h))
    return g, h.reshape(3, 3)


def dynamic_stiffness(base, coupling, mass, gap, dhat):
    return _lib_elem().oracle_dynamic_stiffness(base, coupling, mass, gap, dhat)


def stencil_friction(g4, dx4, barrier_grad, mu, eps):
    """stencil_friction (contact.rs:659-705): (gradient 4x3, Hessian 12x12), zeros when off."""
    lib = _lib_elem()
    g = np.ascontiguousarray(g4, np.float32).reshape(12)
    d = np.ascontiguousarray(dx4, np.float32).reshape(12)
    fg = np.zeros(12, np.float32)
    fh = np.zeros(144, np.float32)
    lib.oracle_stencil_friction(_p(g), _p(d), barrier_grad, mu, eps, _p(fg), _p(fh))
    return fg.reshape(4, 3), fh.reshape(12, 12)


def membrane_element(rest, p, kw=1.0, kf=1.0, ks=1.0):
    """Baraff-Witkin element (membrane.rs:225-270) in f32: (conditions, gradient 3x3,
    Hessian 9x9, (wu, wv)), or None for a degenerate rest triangle."""
    lib = _lib_elem()
    r = np.ascontiguousarray(rest, np.float32).reshape(9)
    q = np.ascontiguousarray(p, np.float32).reshape(9)
    c, g, h, w = np.zeros(3, np.float32), np.zeros(9, np.float32), np.zeros(81, np.float32), np.zeros(6, np.float32)
    if not lib.oracle_membrane_element(_p(r), _p(q), kw, kf, ks, _p(c), _p(g), _p(h), _p(w)):
        return None
    return c, g.reshape(3, 3), h.reshape(9, 9), (w[:3].copy(), w[3:].copy())


def membrane_materials(w, wu, wv, clamp=True):
    """(stretch material of w 3x3, shear blocks [uu, uv, vu, vv] 4x3x3) (membrane.rs:100-205)."""
    lib = _lib_elem()
    a, b, c = (np.ascontiguousarray(v, np.float32) for v in (w, wu, wv))
    m9, m36 = np.zeros(9, np.float32), np.zeros(36, np.float32)
    lib.oracle_membrane_materials(_p(a), _p(b), _p(c), 1 if clamp else 0, _p(m9), _p(m36))
    return m9.reshape(3, 3), m36.reshape(4, 3, 3)


def adjoint_system(o: "OracleSolver", scene: dict, theta, xn, vn, xn1, npanel=2, nseam=2, eps=3e-9):
    """One step's adjoint system in FP64 (oracle_adjoint_system): H = dG/dx (n3 x n3) and
    dG/dtheta ((3 npanel + nseam) x n3) of the step's equilibrium residual at x_{n+1}, with
    the contact set and the stiffnesses' elastic parts of x_{n+1} held fixed; the stencil count.
    eps is the central-difference step of H in metres: at 1e-7 the seam's contact stencils
    (edges 1 mm apart, nearly parallel) put differences across region switches of the gap
    into H; from 1e-8 down H is symmetric to 1e-4 and stops changing (3e-9 and 1e-9 agree to
    1e-4 of its entries of ~1e3)."""
    n3 = 3 * o.nv
    npar = 3 * npanel + nseam
    uv = np.ascontiguousarray(scene["shell_uv"], np.float32)
    panel = np.ascontiguousarray(scene["shell_panel"], np.uint8)
    seam = np.ascontiguousarray(scene["stitch_seam"], np.uint8)
    k0 = np.ascontiguousarray(np.asarray(scene["stitch_kl"], np.float64)[:, 0])
    th = np.ascontiguousarray(theta, np.float64)
    H = np.empty((n3, n3), np.float64)
    dG = np.empty((npar, n3), np.float64)
    a = [np.ascontiguousarray(v, np.float64).reshape(-1) for v in (xn, vn, xn1)]
    nst = o.lib.oracle_adjoint_system(o.h, npanel, nseam, _p(uv), _p(panel), _p(seam), _p(k0), _p(th), _p(a[0]),
                                      _p(a[1]), _p(a[2]), C.c_double(eps), _p(H), _p(dG))
    if nst < 0:
        raise ValueError("the adjoint system needs an FP64 oracle solver")
    return H, dG, nst


def fp64_adjoint(scene: dict, theta, xs, vs, dl_dx, npanel=2, nseam=2, eps=3e-9):
    """dL/dtheta of an N-step drape in FP64 on the CPU, along the given trajectory
    (xs, vs: (N + 1, nv, 3), the states the GPU forward pass went through): backwards through
    every step, w = H^-1 (a_x + a_v / h) by a dense LU of the free block of the
    symmetrised H, dL/dtheta -= w . dG/dtheta, a_x <- M/h^2 w - a_v / h, a_v <- M/h w (pinned
    rows 0). The same recursion the GPU adjoint runs, with every derivative in FP64."""
    o = OracleSolver(scene, "f64")
    im = np.asarray(scene["inv_mass"], np.float64)
    free3 = np.repeat(im > 0, 3)
    m3 = np.where(free3, 1.0 / np.where(im > 0, im, 1.0).repeat(3), 0.0)
    h = float(scene["params"]["dt"])
    ax = np.asarray(dl_dx, np.float64).reshape(-1).copy()
    ax[~free3] = 0.0
    av = np.zeros_like(ax)
    grad = np.zeros(3 * npanel + nseam)
    nstencils = []
    f = np.flatnonzero(free3)
    for n in range(len(xs) - 2, -1, -1):
        H, dG, nst = adjoint_system(o, scene, theta, xs[n], vs[n], xs[n + 1], npanel, nseam, eps)
        nstencils.append(nst)
        Hf = H[np.ix_(f, f)]
        Hf = 0.5 * (Hf + Hf.T)
        b = ax + av / h
        w = np.zeros_like(ax)
        w[f] = np.linalg.solve(Hf, b[f])
        grad -= dG @ w
        ax = m3 / (h * h) * w - av / h
        av = m3 / h * w
    o.close()
    return grad, nstencils[::-1]
