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
