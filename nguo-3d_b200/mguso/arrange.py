"""3-D arrangement of flat pattern pieces before the drape (ui/crates/nguo-sewing/src/
arrange.rs): where each triangulated piece starts in world space.

The placement must be isometric, because the step takes every rest shape from the positions
it is given (a placement that stretches a panel bakes the stretch in as the fabric's rest
state). ``Archetype.TUBE`` therefore wraps each panel onto a vertical cylinder (developable:
arc length equals pattern width) of radius ``max(body + gap, sum of widths / 2 pi)``, the
leftover arc shared between the seams so they start slightly open; ``Archetype.FLAT`` stands
the panels up side by side in a plane in front of the body. An authored placement
(position in mm, rotation quaternion) always wins over the preset. Pattern +y is downward, so
every placement maps it to world -Y, which mirrors the plane: ``flips_winding`` says the
triangles must be re-wound.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

DEFAULT_GAP_M = 0.02


class Archetype:
    TUBE = "tube"
    FLAT = "flat"


@dataclass(frozen=True)
class ArrangeOptions:
    archetype: str = Archetype.TUBE
    center_xz: Tuple[float, float] = (0.0, 0.0)
    body_radius_m: float = 0.15  # a measured girth / 2 pi where the garment sits
    gap_m: float = DEFAULT_GAP_M
    top_y_m: float = 1.3          # world Y of the garment's top edge


def _f32(x) -> np.float32:
    return np.float32(x)


def rotate(q, v) -> np.ndarray:
    """q v q* for a unit quaternion (x, y, z, w), in f32 (arrange.rs:186-200)."""
    x, y, z, w = (_f32(c) for c in q)
    v0, v1, v2 = (_f32(c) for c in v)
    two = _f32(2.0)
    t = (two * (y * v2 - z * v1), two * (z * v0 - x * v2), two * (x * v1 - y * v0))
    return np.array([v0 + w * t[0] + (y * t[2] - z * t[1]), v1 + w * t[1] + (z * t[0] - x * t[2]),
                     v2 + w * t[2] + (x * t[1] - y * t[0])], np.float32)


@dataclass(frozen=True)
class Wrap:
    """A piece wrapped on a vertical cylinder; origin_mm is its pattern top-left corner."""
    center_xz: Tuple[float, float]
    radius_m: float
    theta0: float   # angle of the piece's left edge: 0 faces +Z, increasing toward +X
    top_y_m: float
    origin_mm: Tuple[float, float]

    def apply(self, p_mm) -> np.ndarray:
        """World metres (f32) of pattern points (..., 2) in piece millimetres (arrange.rs:144-163)."""
        p = np.asarray(p_mm, np.float64)
        along = (p[..., 0] - self.origin_mm[0]) * 1e-3
        down = (p[..., 1] - self.origin_mm[1]) * 1e-3
        r = _f32(self.radius_m)
        theta = float(_f32(self.theta0)) + along / float(max(r, _f32(1e-6)))
        return np.stack([_f32(self.center_xz[0]) + r * np.sin(theta).astype(np.float32),
                         _f32(self.top_y_m) - down.astype(np.float32),
                         _f32(self.center_xz[1]) + r * np.cos(theta).astype(np.float32)], -1).astype(np.float32)

    def flips_winding(self) -> bool:
        return True


@dataclass(frozen=True)
class Rigid:
    """The flat plane rotated by a quaternion (x, y, z, w) and translated (an authored
    placement)."""
    quat: Tuple[float, float, float, float]
    offset_m: Tuple[float, float, float]
    origin_mm: Tuple[float, float]

    def apply(self, p_mm) -> np.ndarray:
        p = np.asarray(p_mm, np.float64)
        flat = p.reshape(-1, 2)
        out = np.empty((len(flat), 3), np.float32)
        for i, (x, y) in enumerate(flat):
            local = (np.float32((x - self.origin_mm[0]) * 1e-3), np.float32(-(y - self.origin_mm[1]) * 1e-3), 0.0)
            out[i] = rotate(self.quat, local) + np.asarray(self.offset_m, np.float32)
        return out.reshape(p.shape[:-1] + (3,))

    def flips_winding(self) -> bool:
        return True


@dataclass(frozen=True)
class PieceExtent:
    """A piece as the arranger sees it: pattern bounding box (x0, y0, x1, y1) in mm, an
    optional authored placement ((x, y, z) mm, quaternion) and the arc length of its support
    edge (the girth it contributes where it hangs), if annotated."""
    piece: int
    bounds_mm: Tuple[float, float, float, float]
    manual: Optional[Tuple[Tuple[float, float, float], Tuple[float, float, float, float]]] = None
    support_arc_mm: Optional[float] = None

    def width_mm(self) -> float:
        return self.bounds_mm[2] - self.bounds_mm[0]

    def arc_mm(self) -> float:
        """The arc the piece occupies round the body: its support edge if annotated, else its
        bounding-box width (arrange.rs:238-240)."""
        return self.support_arc_mm if self.support_arc_mm is not None else self.width_mm()

    def origin_mm(self) -> Tuple[float, float]:
        return (self.bounds_mm[0], self.bounds_mm[1])


@dataclass
class Arrangement:
    placements: list
    radius_m: Optional[float]  # None for the flat archetype
    circumference_m: float     # total arc wrapped where the garment hangs
    slack_m: float             # arc left over and shared between the seams


def _manual(p: PieceExtent):
    if p.manual is None:
        return None
    pos, quat = p.manual
    return Rigid(tuple(float(_f32(c)) for c in quat), tuple(float(_f32(c * 1e-3)) for c in pos), p.origin_mm())


def arrange(pieces: Sequence[PieceExtent], opts: ArrangeOptions = ArrangeOptions()) -> Arrangement:
    """Place every piece, in the order given (use ``seam_order`` for one that walks the seam
    graph) (arrange.rs:320-402)."""
    if opts.archetype == Archetype.FLAT:
        total = float(_f32(sum(p.width_mm() for p in pieces) * 1e-3))
        x, out = 0.0, []
        for p in pieces:
            out.append(_manual(p) or Rigid((0.0, 0.0, 0.0, 1.0),
                                           (opts.center_xz[0] - 0.5 * total + x, opts.top_y_m,
                                            opts.center_xz[1] + opts.body_radius_m + opts.gap_m), p.origin_mm()))
            x += float(_f32(p.width_mm() * 1e-3))
        return Arrangement(out, None, total, 0.0)
    tau = _f32(2.0 * math.pi)
    total = _f32(sum(p.arc_mm() for p in pieces) * 1e-3)
    closing = total / tau
    radius = max(_f32(opts.body_radius_m) + _f32(opts.gap_m), closing, _f32(1e-3))
    slack = max(tau * radius - total, _f32(0.0))
    per_seam = slack / _f32(len(pieces)) if pieces else _f32(0.0)
    first = _f32(pieces[0].arc_mm() * 1e-3) if pieces else _f32(0.0)
    theta = -_f32(0.5) * (first + per_seam) / radius
    out = []
    for p in pieces:
        out.append(_manual(p) or Wrap(tuple(opts.center_xz), float(radius),
                                      float(theta + _f32(0.5) * per_seam / radius), opts.top_y_m, p.origin_mm()))
        theta = theta + (_f32(p.arc_mm() * 1e-3) + per_seam) / radius
    return Arrangement(out, float(radius), float(total), float(slack))


def seam_order(pieces: Sequence[int], seams: Sequence[Tuple[int, int]]) -> List[int]:
    """Pieces ordered so that pieces sewn to each other are adjacent: a greedy chain walk over
    the seam graph from the lowest id, restarting at the next unvisited piece
    (arrange.rs:421-452). ``seams`` are (piece, piece) pairs."""
    present = set(pieces)

    def neighbours(p):
        return sorted({b if a == p else a for a, b in seams if p in (a, b) and a != b} - {p})

    out: List[int] = []
    for start in sorted(pieces):
        if start in out:
            continue
        cur = start
        while True:
            out.append(cur)
            nxt = next((q for q in neighbours(cur) if q not in out and q in present), None)
            if nxt is None:
                break
            cur = nxt
    return out
