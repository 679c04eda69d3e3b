"""Adjoint of an N-step drape through the C ABI (mguso_adjoint_*): forward(theta) -> x_N and
backward(dL/dx_N) -> dL/dtheta, the contract of a torch.autograd.Function.

theta = [stiff_0 .. stiff_{P-1}, warp_0, weft_0, .., warp_{P-1}, weft_{P-1}, seam_0 .. seam_{S-1}]
(P panels, S seams): per-panel membrane stiffness factors, per-panel rest-length scales along
the warp (pattern v) and the weft (pattern u), per-seam stitch stiffness factors. The scene
needs the sewing-pattern fields of `scenes.sheath_on_torso` (shell_uv, shell_panel,
stitch_seam)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, ptr
from .solver import StepStats, _desc, _sigs


class AdjointSpec(C.Structure):
    _fields_ = [("npanel", C.c_uint32), ("nseam", C.c_uint32), ("shell_uv", C.c_void_p),
                ("shell_panel", C.c_void_p), ("stitch_seam", C.c_void_p)]


def _adj_sigs(lib):
    vp, i32 = C.c_void_p, C.c_int
    for name, res, args in [
        ("mguso_adjoint_create", i32, [vp, vp, vp, C.POINTER(vp)]),
        ("mguso_adjoint_destroy", i32, [vp]),
        ("mguso_adjoint_forward", i32, [vp, vp, C.c_uint32, C.c_uint32, vp, vp]),
        ("mguso_adjoint_backward", i32, [vp, vp, vp]),
        ("mguso_adjoint_states", i32, [vp, vp, vp]),
    ]:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def pattern_rest(uv: np.ndarray, panel: np.ndarray, theta: np.ndarray, npanel: int, dtype=np.float64):
    """Per shell face: inverse rest shape (column-major 2x2) and area from its pattern
    triangle scaled by (weft, warp) along (u, v), and its stiffness factor."""
    th = np.asarray(theta, dtype)
    su = th[npanel + 2 * panel + 1]
    sv = th[npanel + 2 * panel]
    uv = np.asarray(uv, dtype)
    xx = su * (uv[:, 1, 0] - uv[:, 0, 0])
    xy = sv * (uv[:, 1, 1] - uv[:, 0, 1])
    yx = su * (uv[:, 2, 0] - uv[:, 0, 0])
    yy = sv * (uv[:, 2, 1] - uv[:, 0, 1])
    det = xx * yy - yx * xy
    rest = np.stack([yy / det, -xy / det, -yx / det, xx / det, 0.5 * np.abs(det)], 1)
    return rest, th[panel]


class AdjointDrape:
    """Forward/backward pair of an N-step drape on the GPU."""

    def __init__(self, ctx, scene: dict, precision: str = "mixed", npanel: int = 2, nseam: int = 2):
        self.ctx = ctx
        self.lib = ctx.lib
        _sigs(self.lib)
        _adj_sigs(self.lib)
        d, keep = _desc(scene, precision)
        self.uv = np.ascontiguousarray(scene["shell_uv"], np.float32).reshape(-1, 3, 2)
        self.panel = np.ascontiguousarray(scene["shell_panel"], np.uint8)
        self.seam = np.ascontiguousarray(scene["stitch_seam"], np.uint8)
        spec = AdjointSpec(npanel, nseam, ptr(self.uv), ptr(self.panel), ptr(self.seam))
        self._keep = (d, keep, spec)
        self.npanel, self.nseam = npanel, nseam
        self.nv = d.nv
        h = C.c_void_p()
        check(self.lib.mguso_adjoint_create(ctx.h, C.byref(d), C.byref(spec), C.byref(h)))
        self.h = h
        ctx.own(self)

    @property
    def nparams(self) -> int:
        return 3 * self.npanel + self.nseam

    def forward(self, theta, nsteps: int, checkpoint_every: int = 6):
        th = np.ascontiguousarray(theta, np.float64)
        assert th.shape == (self.nparams,)
        x = np.empty((self.nv, 3), np.float32)
        st = (StepStats * nsteps)()
        check(self.lib.mguso_adjoint_forward(self.h, ptr(th), nsteps, checkpoint_every, ptr(x), st))
        self.stats = [{f: getattr(o, f) for f, _ in StepStats._fields_} for o in st]
        return x

    def backward(self, dl_dx) -> np.ndarray:
        g = np.ascontiguousarray(dl_dx, np.float32).reshape(-1)
        out = np.empty(self.nparams, np.float64)
        check(self.lib.mguso_adjoint_backward(self.h, ptr(g), ptr(out)))
        return out

    def states(self):
        """(x, v) of the last forward pass, each (nsteps + 1, nv, 3), recomputed from its
        checkpoints as the backward pass recomputes them."""
        n = len(self.stats)
        x = np.empty((n + 1, self.nv, 3), np.float32)
        v = np.empty((n + 1, self.nv, 3), np.float32)
        check(self.lib.mguso_adjoint_states(self.h, ptr(x), ptr(v)))
        return x, v

    def close(self):
        if self.h:
            self.lib.mguso_adjoint_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autograd_function(drape: AdjointDrape, nsteps: int, checkpoint_every: int = 6):
    """A torch.autograd.Function applying the drape: theta (float64 tensor) -> x_N."""
    import torch

    class _Drape(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta):
            x = drape.forward(theta.detach().cpu().numpy(), nsteps, checkpoint_every)
            return torch.from_numpy(x.astype(np.float64))

        @staticmethod
        def backward(ctx, grad_x):
            g = drape.backward(grad_x.detach().cpu().numpy().astype(np.float32))
            return torch.from_numpy(g)

    return _Drape.apply
