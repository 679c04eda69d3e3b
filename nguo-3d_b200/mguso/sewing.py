"""Seam correspondence: which points of one seam side sew to which points of the other,
as the stitches the step takes (ui/crates/nguo-sewing/src/correspond.rs).

A side is an ordered chain of pattern edges, each resolved to the mesh vertices lying on it
(here: the vertex ids along a straight edge and their pattern-space positions), plus the
normalised sub-span that sews. Resolved, a side is a monotone list of (vertex, u) with u the
normalised arc length over the sewn span, so pairing two sides is a merge over the same
0..1 parameter; unequal lengths pair proportionally (ease, or gathering). Stitches go from
the denser side's vertices to interpolated points of the other side (a vertex sewn to a
point ``w`` of the way along a mesh edge), so the seam is not quantised to the coarser mesh.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Sequence, Tuple

import numpy as np

EASE_LIMIT = 1.25      # the widest length ratio a plain seam absorbs as ease
MIN_SPAN_MM = 10.0e-3  # a sewn span shorter than this is a point, not a span


class SeamError(ValueError):
    """A seam side that cannot be resolved."""


class BrokenChain(SeamError):
    def __init__(self, edge: int):
        super().__init__(f"seam side is discontinuous at edge {edge}: it does not start where the previous "
                         f"edge ended (its reversed flag is likely wrong)")
        self.edge = edge


class DegenerateSpan(SeamError):
    pass


@dataclass
class EdgeChain:
    """One pattern edge resolved onto the mesh: vertex ids from the edge's start to its end
    and their pattern-space positions (millimetres)."""
    vertices: Sequence[int]
    points_mm: np.ndarray

    def length_mm(self) -> float:
        p = np.asarray(self.points_mm, np.float64)
        return float(np.linalg.norm(np.diff(p, axis=0), axis=1).sum())


@dataclass
class SideSamples:
    """Mesh vertices along a side's sewn span, ascending in normalised arc length u."""
    vertices: List[Tuple[int, float]]
    len_mm: float


@dataclass
class Correspondence:
    stitches: List[Tuple[List[int], List[float]]] = field(default_factory=list)
    len_a_mm: float = 0.0
    len_b_mm: float = 0.0

    def ease(self) -> float:
        """len(b) / len(a): above 1, side b is gathered into side a."""
        return self.len_b_mm / self.len_a_mm if self.len_a_mm > 0 else float("inf")

    def ease_fraction(self) -> float:
        return self.ease() - 1.0

    def arrays(self):
        """(index u32 (S, 6), weight f32 (S, 6)) in the scene description's stitch layout."""
        idx = np.array([s[0] for s in self.stitches], np.uint32).reshape(-1, 6)
        w = np.array([s[1] for s in self.stitches], np.float32).reshape(-1, 6)
        return idx, w


def vertex_to_edge(v: int, i0: int, i1: int, w: float):
    """A single vertex sewn to the point ``w`` of the way from ``i0`` to ``i1``."""
    return [v, v, v, i0, i1, i1], [1.0, 0.0, 0.0, 1.0 - w, w, 0.0]


def _span(span):
    a, b = (min(max(float(s), 0.0), 1.0) for s in span)
    return min(a, b), max(a, b)


def side_samples(edges: Sequence[Tuple[EdgeChain, bool]], span=(0.0, 1.0)) -> SideSamples:
    """Resolve a side (edge chains, each with its reversed flag) onto its mesh vertices with
    normalised arc-length positions over the sewn ``span`` (correspond.rs:188-265). The
    vertex where two edges meet appears once; a chain that does not continue where the
    previous edge ended raises ``BrokenChain``; a span of no length raises
    ``DegenerateSpan``."""
    if not edges:
        raise SeamError("a seam side must name at least one edge")
    walked, along, prev_end = 0.0, [], None
    for k, (chain, reversed_) in enumerate(edges):
        ids = list(chain.vertices)
        p = np.asarray(chain.points_mm, np.float64)
        if len(ids) < 2 or p.shape[0] != len(ids):
            raise SeamError(f"edge {k} resolves to {len(ids)} vertices with {p.shape[0]} positions")
        start, end = (ids[-1], ids[0]) if reversed_ else (ids[0], ids[-1])
        if prev_end is not None and prev_end != start:
            raise BrokenChain(k)
        prev_end = end
        s = np.concatenate([[0.0], np.cumsum(np.linalg.norm(np.diff(p, axis=0), axis=1))])
        length = float(s[-1])
        pts = list(zip(ids, s.tolist()))
        if reversed_:
            pts = [(i, length - t) for i, t in reversed(pts)]
        for i, t in pts:
            if along and along[-1][0] == i:
                continue  # the shared joint arrives twice at the same arc position
            along.append((i, walked + t))
        walked += length
    lo, hi = _span(span)
    a, b = lo * walked, hi * walked
    length = b - a
    if not length > MIN_SPAN_MM:
        raise DegenerateSpan(f"the side sews a span of {length:.6f} mm, which is not a span")
    eps = 1e-9 * max(walked, 1.0)
    verts = [(i, min(max((t - a) / length, 0.0), 1.0)) for i, t in along if a - eps <= t <= b + eps]
    return SideSamples(verts, length)


def interpolate(samples: Sequence[Tuple[int, float]], u: float):
    """The point ``u`` of the way along ``samples`` as (i0, i1, w), p = (1-w) p_i0 + w p_i1
    (correspond.rs:347-366)."""
    if not samples:
        return 0, 0, 0.0
    if len(samples) == 1:
        return samples[0][0], samples[0][0], 0.0
    k = next((j for j, (_, s) in enumerate(samples) if s >= u), len(samples) - 1)
    k = max(k, 1)
    (i0, u0), (i1, u1) = samples[k - 1], samples[k]
    w = min(max((u - u0) / (u1 - u0), 0.0), 1.0) if u1 > u0 else 0.0
    return i0, i1, float(np.float32(w))


def correspond(a: SideSamples, b: SideSamples, flip: bool = False) -> Correspondence:
    """Pair two resolved sides: one stitch per vertex of the denser side onto the
    parameter-matched point of the other; ``flip`` reverses side b (correspond.rs:270-302)."""
    out = Correspondence(len_a_mm=a.len_mm, len_b_mm=b.len_mm)
    if len(a.vertices) >= len(b.vertices):
        for v, u in a.vertices:
            out.stitches.append(vertex_to_edge(v, *interpolate(b.vertices, 1.0 - u if flip else u)))
    else:
        for v, u in b.vertices:
            out.stitches.append(vertex_to_edge(v, *interpolate(a.vertices, 1.0 - u if flip else u)))
    return out


def pairing_distance_m(a: SideSamples, b: SideSamples, positions, flip: bool = False) -> float:
    """Total 3-D distance the pairing of a's vertices to b has to close (metres): a twisted
    seam shows as a flipped pairing far shorter than the straight one (correspond.rs:306-332)."""
    p = np.asarray(positions, np.float64)
    total = 0.0
    for v, u in a.vertices:
        i0, i1, w = interpolate(b.vertices, 1.0 - u if flip else u)
        if max(v, i0, i1) >= p.shape[0]:
            continue
        total += float(np.linalg.norm(p[v] - (p[i0] + (p[i1] - p[i0]) * w)))
    return total


def sew(a: SideSamples, b: SideSamples, positions) -> Tuple[Correspondence, bool]:
    """Correspond two sides straight, or reversed when the reversed pairing closes with less
    than half the travel of the straight one (garment.rs:349-353); returns the correspondence
    and whether side b was flipped."""
    flip = pairing_distance_m(a, b, positions, True) < 0.5 * pairing_distance_m(a, b, positions, False)
    return correspond(a, b, flip), flip
