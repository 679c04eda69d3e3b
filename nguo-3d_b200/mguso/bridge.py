"""The garment app's in-process drape loop on the GPU step: the host-side counterpart of the
bridge's ``InProcessTransport::solve`` (ui/crates/nguo-engine-bridge/src/inproc.rs:72-200),
which builds the implicit solver, sews the submitted stitches, steps and streams frames to a
sink. Here the step is ``ImplicitSolver`` (the whole step on the GPU) instead of the
reference's ``CgCpu``-backed CPU step; the loop's contract is the same:

- a scene whose vertices are all static is rejected (nothing to drape);
- stitches get the reference driver's constants: stiffness 1 (raw, no normalisation),
  ``l0 = max(contact gap, 1e-4)`` and ``l_cap = 10 l0`` (``STITCH_LENGTH_FACTOR``);
- a frame is published every ``frame_stride`` steps and always after the last step;
- the sink can cancel between steps (``is_cancelled``) or at a frame (``push`` returns
  False), which raises ``Cancelled``;
- a non-finite position raises ``Diverged`` with the step and the vertex.
"""
from __future__ import annotations

import time
from typing import Callable, Optional

import numpy as np

STITCH_LENGTH_FACTOR = 10.0
STITCH_STIFFNESS = 1.0


class BridgeError(RuntimeError):
    """A drape the loop could not run or finish."""


class Unsupported(BridgeError):
    pass


class Cancelled(BridgeError):
    pass


class Diverged(BridgeError):
    def __init__(self, step: int, vertex: int):
        super().__init__(f"the drape diverged at step {step} (vertex {vertex} is not finite)")
        self.step, self.vertex = step, vertex


class FrameSink:
    """Receives frames; a subclass overrides ``push`` (return False to cancel) and
    ``is_cancelled``."""

    def push(self, index: int, positions: np.ndarray) -> bool:
        return True

    def is_cancelled(self) -> bool:
        return False


def sew(scene: dict, stitches) -> dict:
    """The scene with ``stitches`` attached: each an (index[6], weight[6]) pair (source
    barycentric, target barycentric; each side's weights sum to 1), at the bridge's
    stiffness and rest/cap lengths."""
    idx = np.asarray([s[0] for s in stitches], np.uint32).reshape(-1, 6)
    w = np.asarray([s[1] for s in stitches], np.float32).reshape(-1, 6)
    nv = np.asarray(scene["positions"]).shape[0]
    if idx.size and int(idx.max()) >= nv:
        raise Unsupported(f"a stitch references vertex {int(idx.max())} of {nv}")
    for side in (w[:, :3], w[:, 3:]):
        if side.size and np.abs(side.sum(1) - 1.0).max() > 1e-3:
            raise Unsupported("a stitch side's weights do not sum to 1")
    l0 = max(float(scene["params"].get("contact_dhat", 1e-3)), 1e-4)
    kl = np.tile(np.array([[STITCH_STIFFNESS, l0, STITCH_LENGTH_FACTOR * l0]], np.float32), (idx.shape[0], 1))
    out = dict(scene)
    out["stitch_idx"], out["stitch_w"], out["stitch_kl"] = idx, w, kl
    return out


def drape(ctx, scene: dict, steps: int, stitches=(), frame_stride: int = 1, sink: Optional[FrameSink] = None,
          precision: str = "mixed", solver_factory: Optional[Callable] = None) -> dict:
    """Drape ``scene`` for ``steps`` implicit steps, sewing ``stitches`` and streaming frames to
    ``sink``; returns the run report (steps, frames, vertex counts, median and total seconds).
    ``solver_factory(ctx, scene, precision)`` builds the stepper (``ImplicitSolver`` by
    default)."""
    started = time.perf_counter()
    sink = sink or FrameSink()
    stride = max(int(frame_stride), 1)
    steps = max(int(steps), 1)
    im = np.asarray(scene["inv_mass"])
    dynamic = int((im > 0).sum())
    if dynamic == 0:
        raise Unsupported("every vertex in the scene is static, so there is nothing to drape")
    if len(stitches):
        scene = sew(scene, stitches)
    if solver_factory is None:
        from .solver import ImplicitSolver as solver_factory  # noqa: N813
    solver = solver_factory(ctx, scene, precision)
    step_s, emitted = [], 0
    try:
        for step in range(steps):
            if sink.is_cancelled():
                raise Cancelled("cancelled")
            t = time.perf_counter()
            solver.step(1)
            step_s.append(time.perf_counter() - t)
            pos = np.asarray(solver.positions)
            bad = np.flatnonzero(~np.isfinite(pos).all(1))
            if bad.size:
                raise Diverged(step, int(bad[0]))
            if step % stride != 0 and step + 1 != steps:
                continue
            if sink.push(emitted, pos.copy()) is False:
                raise Cancelled("cancelled")
            emitted += 1
    finally:
        close = getattr(solver, "close", None)
        if close:
            close()
    return {"backend": "in-process/implicit/cuda", "steps": steps, "frames_emitted": emitted,
            "verts": int(im.shape[0]), "dynamic_verts": dynamic, "tris": int(np.asarray(scene["tris"]).shape[0]),
            "stitches": len(stitches), "median_step_s": float(np.median(step_s)),
            "total_s": time.perf_counter() - started}
