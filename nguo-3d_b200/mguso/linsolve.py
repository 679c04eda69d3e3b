"""Host-side mirror of the reference's linear-solver seam.

Mirrors ``engine_core::LinearSolver`` (core-engine/crates/engine-core/src/linsolve.rs:21-28):
``solve(a, b, tol, max_iter) -> x`` plus ``last_stats()``, with the solve running on the
GPU through the C ABI. ``CsrMatrix`` mirrors ``engine_core::CsrMatrix`` (csr.rs:9-14).
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check, ptr


@dataclass
class CsrMatrix:
    """Square scalar CSR, ``n`` rows (3 per vertex), columns sorted per row."""

    n: int
    row_ptr: np.ndarray
    col_idx: np.ndarray
    values: np.ndarray

    def nnz(self) -> int:
        return int(self.values.size)


@dataclass
class LinearStats:
    """``engine_core::LinearStats`` (linsolve.rs:12-18)."""

    iters: int = 0
    residual: float = 0.0
    status: int = 0


class Context:
    """One GPU (``GpuContext::new``, engine-gpu/src/lib.rs:91-126)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        check(self.lib.mguso_ctx_create(device, C.byref(h)))
        self.h = h
        self.device = device
        self._deps = weakref.WeakSet()

    @property
    def stream(self) -> int:
        return self.lib.mguso_ctx_stream(self.h)

    def own(self, obj) -> None:
        """Registers an object built on this context, to be closed before the context is
        (the C objects use the context's stream, so they must not outlive it)."""
        self._deps.add(obj)

    def close(self):
        if self.h:
            for d in list(self._deps):
                try:
                    d.close()
                except Exception:
                    pass
            self.lib.mguso_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CudaLinearSolver:
    """A ``LinearSolver`` whose solve is the device PCG.

    ``precond`` is ``"schwarz"`` (SchwarzCpu(domain), linsolve.rs:463-520), ``"schwarz-ml"``
    (SchwarzMlCpu(domain, weight), the two-level Galerkin form, linsolve.rs:779-836) or
    ``"block"`` (CgCpu's block Jacobi, linsolve.rs:413-442). ``precision`` is ``"mixed"`` (FP64
    dot products and norms) or ``"fp32"``.
    """

    def __init__(self, ctx: Context, precond: str = "schwarz", domain: int = 32, precision: str = "mixed",
                 weight: float = 0.7):
        self.ctx = ctx
        self.lib = ctx.lib
        pr = {"mixed": _lib.PRECISION_MIXED, "fp32": _lib.PRECISION_FP32}[precision]
        h = C.c_void_p()
        if precond == "schwarz-ml":
            check(self.lib.mguso_linear_solver_create_ml(ctx.h, domain, C.c_float(weight), pr, C.byref(h)))
        else:
            pc = {"schwarz": _lib.PRECOND_SCHWARZ, "block": _lib.PRECOND_BLOCK_JACOBI}[precond]
            check(self.lib.mguso_linear_solver_create(ctx.h, pc, domain, pr, C.byref(h)))
        self.h = h
        ctx.own(self)
        self._stats = LinearStats()

    def solve(self, a: CsrMatrix, b: np.ndarray, tol: float, max_iter: int) -> np.ndarray:
        assert b.shape == (a.n,)
        desc, keep = _lib.csr_desc(a.n, a.row_ptr, a.col_idx, a.values)
        bb = np.ascontiguousarray(b, dtype=np.float32)
        x = np.zeros(a.n, dtype=np.float32)
        st = _lib.LinStats()
        check(self.lib.mguso_linear_solve(self.h, C.byref(desc), ptr(bb), C.c_float(tol), max_iter, ptr(x),
                                          C.byref(st)))
        self._stats = LinearStats(int(st.iters), float(st.residual), int(st.status))
        del keep
        return x

    def last_stats(self) -> LinearStats:
        return self._stats

    def close(self):
        if self.h:
            self.lib.mguso_linear_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Bsr:
    """A device-resident 3x3 BSR operator."""

    def __init__(self, ctx: Context, nb: int, row_ptr: np.ndarray, col: np.ndarray, val: np.ndarray):
        self.ctx = ctx
        self.lib = ctx.lib
        rp = np.ascontiguousarray(row_ptr, dtype=np.uint32)
        cl = np.ascontiguousarray(col, dtype=np.uint32)
        vl = np.ascontiguousarray(val, dtype=np.float32).reshape(-1)
        assert rp.size == nb + 1 and vl.size == 9 * cl.size
        h = C.c_void_p()
        check(self.lib.mguso_bsr_create(ctx.h, nb, ptr(rp), ptr(cl) if cl.size else None,
                                        ptr(vl) if vl.size else None, C.byref(h)))
        self.h = h
        ctx.own(self)
        self.nb = nb
        self.nnzb = int(cl.size)

    @classmethod
    def from_csr(cls, ctx: Context, a: CsrMatrix) -> "Bsr":
        self = cls.__new__(cls)
        self.ctx = ctx
        self.lib = ctx.lib
        desc, keep = _lib.csr_desc(a.n, a.row_ptr, a.col_idx, a.values)
        h = C.c_void_p()
        check(self.lib.mguso_bsr_create_from_csr(ctx.h, C.byref(desc), C.byref(h)))
        self.h = h
        ctx.own(self)
        nb, nnzb = C.c_uint32(), C.c_uint32()
        check(self.lib.mguso_bsr_info(h, C.byref(nb), C.byref(nnzb)))
        self.nb, self.nnzb = nb.value, nnzb.value
        return self

    def spmv(self, x_dev: int, y_dev: int, stream: int = 0) -> None:
        """y = A x on device pointers."""
        check(self.lib.mguso_bsr_spmv(self.h, x_dev, y_dev, stream))

    def spmv_host(self, x: np.ndarray) -> np.ndarray:
        xx = np.ascontiguousarray(x, dtype=np.float32)
        y = np.empty(3 * self.nb, dtype=np.float32)
        check(self.lib.mguso_bsr_spmv_host(self.h, ptr(xx), ptr(y)))
        return y

    def set_kernel(self, variant: int) -> int:
        act = C.c_int()
        check(self.lib.mguso_bsr_set_kernel(self.h, variant, C.byref(act)))
        return act.value

    def kernel(self) -> dict:
        """The SpMV variant in use: {"variant": name, "tile_rows": r, "stages": s}."""
        v, r, st = C.c_int(), C.c_int(), C.c_int()
        check(self.lib.mguso_bsr_kernel(self.h, C.byref(v), C.byref(r), C.byref(st)))
        name = {0: "auto", 1: "tma", 2: "direct", 3: "sliced_ell"}.get(v.value, str(v.value))
        return {"variant": name, "tile_rows": r.value, "stages": st.value}

    def autotune(self) -> float:
        us = C.c_float()
        check(self.lib.mguso_bsr_autotune(self.h, C.byref(us)))
        return us.value

    def close(self):
        if self.h:
            self.lib.mguso_bsr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Schwarz:
    """Additive Schwarz over a device BSR: one level (linsolve.rs:126-258), or with
    ``levels=2`` the two-level Galerkin form z = S0 r + weight C1^T S1 (C1 r)
    (MultilevelSchwarz, linsolve.rs:534-666)."""

    def __init__(self, a: Bsr, domain: int = 32, levels: int = 1, weight: float = 0.7):
        self.a = a
        self.lib = a.lib
        self.levels = levels
        h = C.c_void_p()
        if levels == 2:
            check(self.lib.mguso_schwarz_create_ml(a.h, domain, C.c_float(weight), C.byref(h)))
        else:
            check(self.lib.mguso_schwarz_create(a.h, domain, C.byref(h)))
        self.h = h
        a.ctx.own(self)
        nd, fb = C.c_uint32(), C.c_uint64()
        check(self.lib.mguso_schwarz_info(h, C.byref(nd), C.byref(fb)))
        self.ndomains, self.factor_bytes = nd.value, fb.value

    def factor(self, stream: int = 0) -> None:
        check(self.lib.mguso_schwarz_factor(self.h, stream))

    def apply(self, r_dev: int, z_dev: int, stream: int = 0) -> None:
        check(self.lib.mguso_schwarz_apply(self.h, r_dev, z_dev, stream))

    def domains(self) -> np.ndarray:
        out = np.empty(self.a.nb, dtype=np.uint32)
        check(self.lib.mguso_schwarz_domains(self.h, ptr(out)))
        return out

    def coarse_domains(self) -> np.ndarray:
        """Coarse domain of every coarse node (= level-0 domain); two levels only."""
        out = np.empty(self.ndomains, dtype=np.uint32)
        check(self.lib.mguso_schwarz_coarse_domains(self.h, ptr(out)))
        return out

    def close(self):
        if self.h:
            self.lib.mguso_schwarz_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
