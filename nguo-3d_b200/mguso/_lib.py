"""ctypes binding of libmguso_cuda.so (the C ABI in include/mguso_cuda.h).

The library is built in-tree (``nguo-3d_b200/lib``). Loading fails loudly when it is
missing: there is no CPU fallback for anything in this package.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
REPO = os.path.dirname(PKG)
LIB_PATH = os.path.join(PKG, "lib", "libmguso_cuda.so")
HEADER_PATH = os.path.join(REPO, "include", "mguso_cuda.h")

OK = 0
ERR_NAMES = {
    1: "INVALID_ARG", 2: "OOM", 3: "NONFINITE", 4: "PCG_CAP", 5: "CCD_CAP",
    6: "PAIR_OVERFLOW", 7: "BVH_STACK", 8: "CUDA", 9: "TIMEOUT", 10: "UNSUPPORTED",
}
PRECOND_BLOCK_JACOBI = 1
PRECOND_SCHWARZ = 2
PRECISION_FP32 = 0
PRECISION_MIXED = 1

_lib = None


class MgusoError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"mguso error {code} ({ERR_NAMES.get(code, '?')}): {msg}")
        self.code = code


class CsrDesc(C.Structure):
    _fields_ = [("n", C.c_uint32), ("row_ptr", C.c_void_p), ("col_idx", C.c_void_p), ("values", C.c_void_p)]


class LinStats(C.Structure):
    _fields_ = [("iters", C.c_uint32), ("residual", C.c_double), ("status", C.c_int)]


def header_symbols() -> list[str]:
    """Every function the public header declares."""
    src = open(HEADER_PATH).read()
    return sorted(set(re.findall(r"^\s*(?:int|size_t|void\*|void)\s+(mguso_\w+)\s*\(", src, re.M)))


def load() -> C.CDLL:
    """Loads the library (once). Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `make -C nguo-3d_b200` "
            "(there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    vp, u32, i32, f32, f64, u64 = C.c_void_p, C.c_uint32, C.c_int, C.c_float, C.c_double, C.c_uint64
    P = C.POINTER
    sigs = {
        "mguso_version": (i32, []),
        "mguso_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
        "mguso_ctx_create": (i32, [i32, P(vp)]),
        "mguso_ctx_destroy": (i32, [vp]),
        "mguso_ctx_stream": (vp, [vp]),
        "mguso_linear_solver_create": (i32, [vp, i32, u32, i32, P(vp)]),
        "mguso_linear_solver_create_ml": (i32, [vp, u32, C.c_float, i32, P(vp)]),
        "mguso_linear_solver_destroy": (i32, [vp]),
        "mguso_linear_solve": (i32, [vp, P(CsrDesc), vp, f32, u32, vp, P(LinStats)]),
        "mguso_bsr_create_from_csr": (i32, [vp, P(CsrDesc), P(vp)]),
        "mguso_bsr_create": (i32, [vp, u32, vp, vp, vp, P(vp)]),
        "mguso_bsr_destroy": (i32, [vp]),
        "mguso_bsr_info": (i32, [vp, P(u32), P(u32)]),
        "mguso_bsr_spmv": (i32, [vp, vp, vp, vp]),
        "mguso_bsr_spmv_host": (i32, [vp, vp, vp]),
        "mguso_bsr_set_kernel": (i32, [vp, i32, P(i32)]),
        "mguso_bsr_autotune": (i32, [vp, P(f32)]),
        "mguso_bsr_kernel": (i32, [vp, P(C.c_int), P(C.c_int), P(C.c_int)]),
        "mguso_schwarz_create": (i32, [vp, u32, P(vp)]),
        "mguso_schwarz_create_ml": (i32, [vp, u32, C.c_float, P(vp)]),
        "mguso_schwarz_coarse_domains": (i32, [vp, vp]),
        "mguso_schwarz_destroy": (i32, [vp]),
        "mguso_schwarz_info": (i32, [vp, P(u32), P(u64)]),
        "mguso_schwarz_factor": (i32, [vp, vp]),
        "mguso_schwarz_apply": (i32, [vp, vp, vp, vp]),
        "mguso_schwarz_domains": (i32, [vp, vp]),
        "mguso_lbvh_create": (i32, [vp, P(vp)]),
        "mguso_lbvh_destroy": (i32, [vp]),
        "mguso_lbvh_build": (i32, [vp, vp, u32, vp, u32, i32, vp]),
        "mguso_lbvh_query_points": (i32, [vp, vp, u32, f32, vp, u64, vp, vp]),
        "mguso_lbvh_download": (i32, [vp, vp, vp, vp, vp, vp]),
        "mguso_lbvh_status": (i32, [vp]),
        "mguso_lbvh_stage_times": (i32, [vp, i32, vp]),
        "mguso_lbvh_build_query": (i32, [vp, vp, u32, vp, u32, i32, f32, vp, vp, vp, u64, P(u64)]),
        "mguso_radix_sort_pairs": (i32, [vp, vp, vp, u32, i32, vp]),
        "mguso_radix_sort_status": (i32, [vp]),
        "mguso_radix_sort_pairs_noalloc": (i32, [vp, vp, u32, i32, vp]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    lib = load()
    buf = C.create_string_buffer(4096)
    lib.mguso_last_error(buf, 4096)
    return buf.value.decode(errors="replace")


def check(code: int) -> None:
    if code != OK:
        raise MgusoError(code, last_error())


def ptr(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"], "arrays passed through the C ABI must be contiguous"
    return a.ctypes.data


def csr_desc(n: int, row_ptr: np.ndarray, col_idx: np.ndarray, values: np.ndarray):
    """A CsrDesc over numpy arrays (kept alive by the returned tuple)."""
    rp = np.ascontiguousarray(row_ptr, dtype=np.uint32)
    ci = np.ascontiguousarray(col_idx, dtype=np.uint32)
    vv = np.ascontiguousarray(values, dtype=np.float32)
    d = CsrDesc(n, rp.ctypes.data, ci.ctypes.data if ci.size else None, vv.ctypes.data if vv.size else None)
    return d, (rp, ci, vv)
