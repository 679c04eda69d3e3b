"""Pattern piece -> simulation mesh: the host-side counterpart of nguo-triangulate
(ui/crates/nguo-triangulate/src/lib.rs), which turns a drafted piece into the triangles the
drape steps, together with the pattern-space <-> mesh-vertex map that seam correspondence
(``sewing``) and UVs need.

The interface follows the reference: ``triangulate(network, notches, options)`` takes a
``Network`` in millimetres (vertices, and edges that are straight or cubic Bezier, each
tagged Seam / Fold / Cut / Grain / Internal / DartLeg) and returns a ``SimMesh`` in metres
with ``pattern_mm``, per-vertex ``sources`` and one ``EdgeChain`` of (vertex, curve
parameter t) per pattern edge; every failure is a typed ``TriangulateError``.

The pipeline:

1. Flatten and subdivide. A cubic edge is split adaptively (de Casteljau) until its control
   polygon lies within ``curve_tolerance_mm`` of each chord; notches add their parameters;
   every link is then split evenly in t so none is longer than ``target_edge_mm``. Each
   sample keeps its exact t.
2. Snap-round every sample to a ``weld_mm`` grid and deduplicate (lib.rs:630-668).
3. Triangulate: the constrained Delaunay triangulation of the samples with every pattern
   link as an edge (the Delaunay triangulation, each missing link inserted by edge flips,
   Lawson flips around it). A link that runs exactly through another sample is split there,
   at its parameter midpoint on the curve, so a split point is still exactly on its edge
   with an exact t and the chains stay facts. Pattern links that cross away from a shared
   vertex are refused (``CrossingConstraint``).
4. Refine (``refine=True``): a hexagonal lattice at ``target_edge_mm`` spacing seeds the
   fabric away from the pattern links, then triangles over the area bound (the equilateral
   triangle of side ``target_edge_mm``, lib.rs:681) or under ``min_angle_deg`` get their
   circumcentre inserted, or, when that would encroach on a pattern link, the apex of the
   equilateral triangle on that link, until none is left, the insertion cap
   ``max_steiner`` is reached (``refinement_complete`` False) or no candidate helps.
   Pattern links are never split by refinement (the reference's ``keep_constraint_edges``),
   so an acute input corner keeps its angle.
5. Classify faces by the parity of outline crossings from the convex hull (a 0-1 BFS over
   the dual graph, lib.rs:865-915: holes fall out of the parity), then keep the largest
   fabric component across dart legs (lib.rs:925-965: dart wedges and closed-dart lenses are
   sewn out).
6. Emit fabric faces counter-clockwise, millimetres to metres exactly once
   (``MM_TO_M``), and check every invariant of ``SimMesh.check`` before returning.
"""
from __future__ import annotations

import math
from collections import deque
from dataclasses import dataclass, field, replace
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

MM_TO_M = 1e-3
MAX_INPUT_POINTS = 2_000_000

SEAM, FOLD, CUT, GRAIN, INTERNAL, DART_LEG = "seam", "fold", "cut", "grain", "internal", "dart_leg"
BOUNDARY = (SEAM, FOLD, CUT)
_SEMANTICS = (SEAM, FOLD, CUT, GRAIN, INTERNAL, DART_LEG)

# what crossing a mesh edge means to classification, in priority order (lib.rs:435-462)
FREE, K_INTERNAL, K_DART, K_OUTLINE = 0, 1, 2, 3


def _kind(semantic: str) -> Optional[int]:
    if semantic in BOUNDARY:
        return K_OUTLINE
    return {DART_LEG: K_DART, INTERNAL: K_INTERNAL}.get(semantic)


# ---- errors ------------------------------------------------------------------------------

class TriangulateError(ValueError):
    """Every failure of ``triangulate`` is one of these (lib.rs:151-192)."""


class NoRegion(TriangulateError):
    def __init__(self):
        super().__init__("the piece has no fabric region: its outline (Seam/Fold/Cut edges) does not enclose an "
                         "area — check for a gap in the outline or an unwelded corner")


class Degenerate(TriangulateError):
    def __init__(self, distinct: int, weld_mm: float):
        super().__init__(f"only {distinct} distinct point(s) survived snap-rounding to {weld_mm} mm; the piece is "
                         f"degenerate or weld_mm is too coarse")
        self.distinct, self.weld_mm = distinct, weld_mm


class NotchOutOfRange(TriangulateError):
    def __init__(self, edge: int, t: float):
        super().__init__(f"notch parameter {t} on edge {edge} is outside [0, 1]")
        self.edge, self.t = edge, t


class CrossingConstraint(TriangulateError):
    def __init__(self, edge: int):
        super().__init__(f"edge {edge} crosses another pattern edge away from a shared vertex; split both edges at "
                         f"the crossing (Network.split_edge) and weld them first")
        self.edge = edge


class NonFinite(TriangulateError):
    def __init__(self):
        super().__init__("the pattern contains a non-finite coordinate")


class BadOption(TriangulateError):
    def __init__(self, name: str, value: float):
        super().__init__(f"option {name} is out of range: {value}")
        self.name, self.value = name, value


class TooDense(TriangulateError):
    def __init__(self, limit: int, target_edge_mm: float, span_mm: float):
        super().__init__(f"the piece needs more than {limit} boundary points at a {target_edge_mm} mm target edge; "
                         f"raise target_edge_mm, or check the piece is really {span_mm} mm across (the document "
                         f"unit is millimetres)")
        self.limit, self.target_edge_mm, self.span_mm = limit, target_edge_mm, span_mm


class Invalid(TriangulateError):
    def __init__(self, msg: str):
        super().__init__(f"internal error: the triangulation violated its own invariants: {msg}")


# ---- the pattern network -----------------------------------------------------------------

@dataclass
class Edge:
    start: int
    end: int
    semantic: str
    c1: Optional[Tuple[float, float]] = None  # cubic Bezier interior control points, or None for a line
    c2: Optional[Tuple[float, float]] = None


@dataclass
class Network:
    """A piece's vector network in millimetres (nguo-pattern's VectorNetwork): vertices and
    straight or cubic edges addressed by id; a removed edge keeps its id slot empty."""
    vertices: List[Tuple[float, float]] = field(default_factory=list)
    edges: List[Optional[Edge]] = field(default_factory=list)

    def add_vertex(self, x: float, y: float) -> int:
        self.vertices.append((float(x), float(y)))
        return len(self.vertices) - 1

    def add_edge(self, a: int, b: int, semantic: str = CUT, c1=None, c2=None) -> int:
        if semantic not in _SEMANTICS:
            raise ValueError(f"unknown edge semantic {semantic!r}")
        if not (0 <= a < len(self.vertices) and 0 <= b < len(self.vertices)) or a == b:
            raise ValueError(f"edge ({a}, {b}) needs two distinct existing vertices")
        self.edges.append(Edge(a, b, semantic, None if c1 is None else tuple(map(float, c1)),
                               None if c2 is None else tuple(map(float, c2))))
        return len(self.edges) - 1

    def remove_edge(self, e: int) -> None:
        if self.edges[e] is None:
            raise ValueError(f"edge {e} was already removed")
        self.edges[e] = None

    def control_points(self, e: int) -> np.ndarray:
        ed = self.edges[e]
        a, b = np.array(self.vertices[ed.start]), np.array(self.vertices[ed.end])
        if ed.c1 is None:
            return np.stack([a, b])
        return np.stack([a, np.array(ed.c1), np.array(ed.c2), b])

    def eval(self, e: int, t) -> np.ndarray:
        """Points of edge e at parameters t (line: lerp; cubic: Bernstein form)."""
        cp = self.control_points(e)
        t = np.asarray(t, np.float64)[..., None]
        if len(cp) == 2:
            return cp[0] + (cp[1] - cp[0]) * t
        s = 1.0 - t
        return s ** 3 * cp[0] + 3 * s * s * t * cp[1] + 3 * s * t * t * cp[2] + t ** 3 * cp[3]

    def arc_length(self, e: int) -> float:
        cp = self.control_points(e)
        if len(cp) == 2:
            return float(np.linalg.norm(cp[1] - cp[0]))
        p = self.eval(e, np.linspace(0.0, 1.0, 257))
        return float(np.linalg.norm(np.diff(p, axis=0), axis=1).sum())

    def split_edge(self, e: int, t: float) -> int:
        """Split edge e at parameter t (de Casteljau for a cubic): e keeps its id and now ends at
        the new vertex; the second half is appended. Returns the new vertex."""
        ed = self.edges[e]
        cp = self.control_points(e)
        p = self.eval(e, t)
        v = self.add_vertex(*p)
        if len(cp) == 2:
            self.edges[e] = Edge(ed.start, v, ed.semantic)
            self.edges.append(Edge(v, ed.end, ed.semantic))
        else:
            p01, p12, p23 = cp[0] + (cp[1] - cp[0]) * t, cp[1] + (cp[2] - cp[1]) * t, cp[2] + (cp[3] - cp[2]) * t
            p012, p123 = p01 + (p12 - p01) * t, p12 + (p23 - p12) * t
            self.edges[e] = Edge(ed.start, v, ed.semantic, tuple(p01), tuple(p012))
            self.edges.append(Edge(v, ed.end, ed.semantic, tuple(p123), tuple(p23)))
        return v

    def bounds(self):
        if not self.vertices:
            return (0.0, 0.0, 0.0, 0.0)
        a = np.asarray(self.vertices)
        return (*a.min(0), *a.max(0))


# ---- options and the mesh ------------------------------------------------------------------

@dataclass(frozen=True)
class Options:
    """Quality and resolution knobs (lib.rs:73-148): defaults for a garment panel."""
    curve_tolerance_mm: float = 0.5
    target_edge_mm: float = 10.0
    weld_mm: float = 1e-3
    min_angle_deg: float = 30.0
    min_area_mm2: Optional[float] = None
    max_steiner: int = 50_000
    refine: bool = True

    def with_target_edge_mm(self, mm: float) -> "Options":
        return replace(self, target_edge_mm=float(mm))

    def without_refinement(self) -> "Options":
        return replace(self, refine=False)

    def validate(self) -> None:
        for name, value, upper in (("curve_tolerance_mm", self.curve_tolerance_mm, math.inf),
                                   ("target_edge_mm", self.target_edge_mm, math.inf),
                                   ("weld_mm", self.weld_mm, self.target_edge_mm)):
            if not (math.isfinite(value) and 0.0 < value <= upper):
                raise BadOption(name, value)
        if not (math.isfinite(self.min_angle_deg) and 0.0 <= self.min_angle_deg < 60.0):
            raise BadOption("min_angle_deg", self.min_angle_deg)


@dataclass
class EdgeChain:
    """The mesh vertices on one pattern edge, ascending in the edge's parameter t; t = 0 and
    t = 1 are always present, so consecutive edges of a seam side share end vertices."""
    edge: int
    semantic: str
    points: List[Tuple[int, float]]


# vertex sources: ("vertex", id) a network vertex, ("edge", id) inserted on an edge,
# ("interior", -1) added by refinement
@dataclass
class SimMesh:
    positions: np.ndarray    # f32 (n, 3), metres, z = 0
    indices: np.ndarray      # u32 (m, 3), counter-clockwise in pattern space
    pattern_mm: np.ndarray   # f64 (n, 2)
    sources: List[Tuple[str, int]]
    chains: List[EdgeChain]
    refinement_complete: bool = True
    degenerate_dropped: int = 0

    def uvs(self) -> np.ndarray:
        x0, y0, x1, y1 = self.pattern_bounds()
        w, h = max(x1 - x0, np.finfo(float).tiny), max(y1 - y0, np.finfo(float).tiny)
        return np.stack([(self.pattern_mm[:, 0] - x0) / w, (self.pattern_mm[:, 1] - y0) / h], 1).astype(np.float32)

    def pattern_bounds(self):
        return (*self.pattern_mm.min(0), *self.pattern_mm.max(0))

    def vertex_count(self) -> int:
        return len(self.positions)

    def triangle_count(self) -> int:
        return len(self.indices)

    def chain(self, edge: int) -> Optional[EdgeChain]:
        return next((c for c in self.chains if c.edge == edge), None)

    def outline_vertices(self) -> List[int]:
        return sorted({i for c in self.chains if c.semantic in BOUNDARY for i, _ in c.points})

    def signed_areas_mm2(self) -> np.ndarray:
        p = self.pattern_mm[self.indices.astype(np.int64)]
        return 0.5 * ((p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1])
                      - (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 1, 1] - p[:, 0, 1]))

    def area_mm2(self) -> float:
        return float(self.signed_areas_mm2().sum())

    def min_angles_deg(self) -> np.ndarray:
        p = self.pattern_mm[self.indices.astype(np.int64)]
        out = np.full(len(p), 180.0)
        for k in range(3):
            o, a, b = p[:, k], p[:, (k + 1) % 3], p[:, (k + 2) % 3]
            u, v = a - o, b - o
            cross = u[:, 0] * v[:, 1] - u[:, 1] * v[:, 0]
            dot = (u * v).sum(1)
            out = np.minimum(out, np.degrees(np.arctan2(np.abs(cross), dot)))
        return out

    def min_angle_deg(self) -> float:
        a = self.min_angles_deg()
        return float(a.min()) if a.size else 180.0

    def angle_quantile_deg(self, q: float) -> float:
        a = np.sort(self.min_angles_deg())
        if not a.size:
            return 0.0
        return float(a[min(int(round(min(max(q, 0.0), 1.0) * (len(a) - 1))), len(a) - 1)])

    def max_area_mm2(self) -> float:
        a = self.signed_areas_mm2()
        return float(max(a.max(), 0.0)) if a.size else 0.0

    def check(self) -> Optional[str]:
        """None when every invariant holds, else what broke (lib.rs:371-432)."""
        n = len(self.positions)
        if n != len(self.pattern_mm) or n != len(self.sources):
            return (f"vertex arrays disagree: {n} positions, {len(self.pattern_mm)} pattern_mm, "
                    f"{len(self.sources)} sources")
        if not len(self.indices):
            return "no triangles"
        if not (np.isfinite(self.positions).all() and np.isfinite(self.pattern_mm).all()):
            return "a vertex is not finite"
        if (self.positions[:, 2] != 0).any():
            i = int(np.flatnonzero(self.positions[:, 2] != 0)[0])
            return f"vertex {i} left the pattern plane: z = {self.positions[i, 2]}"
        want = (self.pattern_mm * MM_TO_M).astype(np.float32)
        bad = np.flatnonzero((self.positions[:, :2] != want).any(1))
        if bad.size:
            i = int(bad[0])
            return (f"vertex {i}: {self.positions[i, :2].tolist()} m but pattern is {self.pattern_mm[i].tolist()} mm; "
                    f"a second unit conversion has crept in")
        idx = self.indices.astype(np.int64)
        if (idx >= n).any():
            return "a triangle indexes a missing vertex"
        if ((idx[:, 0] == idx[:, 1]) | (idx[:, 1] == idx[:, 2]) | (idx[:, 0] == idx[:, 2])).any():
            return "a triangle repeats a vertex"
        a = self.signed_areas_mm2()
        if (a <= 0).any():
            i = int(np.flatnonzero(a <= 0)[0])
            return f"triangle {i} is flipped or degenerate: area {a[i]} mm²"
        for c in self.chains:
            if len(c.points) < 2:
                return f"chain for edge {c.edge} has {len(c.points)} point(s)"
            ts = [t for _, t in c.points]
            if any(t1 <= t0 for t0, t1 in zip(ts, ts[1:])):
                return f"chain for edge {c.edge} is not ascending in t"
            if any(i >= n for i, _ in c.points):
                return f"chain for edge {c.edge} indexes a missing vertex"
        if any(c0.edge >= c1.edge for c0, c1 in zip(self.chains, self.chains[1:])):
            return "chains are not sorted by edge id"
        return None


# ---- internals -----------------------------------------------------------------------------

def _flatten_ts(cp: np.ndarray, tol: float) -> List[float]:
    """Parameters of an adaptive flattening of a cubic: an interval is split at its middle
    until both interior control points of its sub-curve lie within tol of its chord."""
    out = [0.0]
    stack = [(0.0, 1.0, cp, 0)]
    while stack:
        t0, t1, q, depth = stack.pop()
        a, b = q[0], q[3]
        ab = b - a
        lab = np.linalg.norm(ab)
        if lab > 0:
            d = np.abs(ab[0] * (q[1:3, 1] - a[1]) - ab[1] * (q[1:3, 0] - a[0])) / lab
        else:
            d = np.linalg.norm(q[1:3] - a, axis=1)
        if d.max() <= tol or depth >= 24:
            out.append(t1)
            continue
        p01, p12, p23 = 0.5 * (q[0] + q[1]), 0.5 * (q[1] + q[2]), 0.5 * (q[2] + q[3])
        p012, p123 = 0.5 * (p01 + p12), 0.5 * (p12 + p23)
        m = 0.5 * (p012 + p123)
        tm = 0.5 * (t0 + t1)
        # right half first on the stack so the left half is emitted first
        stack.append((tm, t1, np.stack([m, p123, p23, q[3]]), depth + 1))
        stack.append((t0, tm, np.stack([q[0], p01, p012, m]), depth + 1))
    return out


def _samples(net: Network, e: int, notches: Sequence[float], opts: Options) -> List[Tuple[float, np.ndarray]]:
    """Flatten + subdivide one edge into (t, point), t ascending with 0 and 1 (lib.rs:474-537)."""
    cp = net.control_points(e)
    if not np.isfinite(cp).all():
        raise NonFinite()
    ts = [0.0, 1.0]
    if len(cp) == 4:
        ts += _flatten_ts(cp, opts.curve_tolerance_mm)
    for t in notches:
        if not (math.isfinite(t) and 0.0 <= t <= 1.0):
            raise NotchOutOfRange(e, t)
        ts.append(float(t))
    ts = sorted(set(min(max(t, 0.0), 1.0) for t in ts))
    out = []
    for t0, t1 in zip(ts, ts[1:]):
        p0, p1 = net.eval(e, t0), net.eval(e, t1)
        out.append((t0, p0))
        extra = int(min(math.ceil(float(np.linalg.norm(p1 - p0)) / opts.target_edge_mm), MAX_INPUT_POINTS))
        for k in range(1, max(extra, 1)):
            t = t0 + (t1 - t0) * (k / extra)
            out.append((t, net.eval(e, t)))
    out.append((1.0, net.eval(e, 1.0)))
    if any(not np.isfinite(p).all() for _, p in out):
        raise NonFinite()
    return out


def _round_half_away(v: float) -> int:
    """Nearest integer, ties away from zero (the snap-rounding key, lib.rs:541-543)."""
    return int(math.copysign(math.floor(abs(v) + 0.5), v))


def _segments_cross(p, q, r, s) -> np.ndarray:
    """Proper crossings of segments p_i q_i and r_j s_j (broadcast): strictly opposite sides
    both ways (touching at an endpoint or collinear overlap is not a crossing)."""
    def orient(a, b, c):
        return (b[..., 0] - a[..., 0]) * (c[..., 1] - a[..., 1]) - (b[..., 1] - a[..., 1]) * (c[..., 0] - a[..., 0])
    d1, d2 = orient(p, q, r), orient(p, q, s)
    d3, d4 = orient(r, s, p), orient(r, s, q)
    return (d1 * d2 < 0) & (d3 * d4 < 0)


def _delaunay(pts: np.ndarray):
    from scipy.spatial import Delaunay
    from scipy.spatial import QhullError

    try:
        return Delaunay(pts)
    except (QhullError, ValueError):
        return None


def _circumcentres(p: np.ndarray) -> np.ndarray:
    a, b, c = p[:, 0], p[:, 1], p[:, 2]
    ba, ca = b - a, c - a
    d = 2.0 * (ba[:, 0] * ca[:, 1] - ba[:, 1] * ca[:, 0])
    b2, c2 = (ba * ba).sum(1), (ca * ca).sum(1)
    with np.errstate(divide="ignore", invalid="ignore"):
        ux = (ca[:, 1] * b2 - ba[:, 1] * c2) / d
        uy = (ba[:, 0] * c2 - ca[:, 0] * b2) / d
    return a + np.stack([ux, uy], 1)


class _Mesher:
    def __init__(self, pts: List[np.ndarray], chains: list, opts: Options):
        self.pts = [np.asarray(p, np.float64) for p in pts]
        self.chains = chains  # [edge, semantic, kind, [(vertex, t)]]
        self.opts = opts

    def links(self):
        for ci, (_, _, kind, pts) in enumerate(self.chains):
            for k in range(len(pts) - 1):
                yield ci, k, pts[k][0], pts[k + 1][0], kind

    def link_array(self):
        ls = list(self.links())
        if not ls:
            return np.zeros((0, 2), np.int64), np.zeros(0, np.int64), np.zeros(0, np.int64)
        return (np.array([(a, b) for _, _, a, b, _ in ls], np.int64), np.array([k for *_, k in ls], np.int64),
                np.array([c for c, *_ in ls], np.int64))

    def check_crossings(self, net_edges: List[int]):
        ab, _, ci = self.link_array()
        if len(ab) < 2:
            return
        P = np.asarray(self.pts)
        p, q = P[ab[:, 0]], P[ab[:, 1]]
        for i0 in range(0, len(ab), 512):
            sl = slice(i0, i0 + 512)
            share = ((ab[sl, None, 0] == ab[None, :, 0]) | (ab[sl, None, 0] == ab[None, :, 1])
                     | (ab[sl, None, 1] == ab[None, :, 0]) | (ab[sl, None, 1] == ab[None, :, 1]))
            x = _segments_cross(p[sl, None], q[sl, None], p[None], q[None]) & ~share
            if x.any():
                i = int(np.argwhere(x)[0][0]) + i0
                raise CrossingConstraint(net_edges[int(ci[i])])

    def triangulate(self):
        P = np.asarray(self.pts)
        return _delaunay(P), P

    def recover(self, net, net_edges: List[int], rounds: int = 30):
        """The constrained Delaunay triangulation of the points with every pattern link as an
        edge: the Delaunay triangulation, then each missing link inserted by edge flips
        (Sloan's algorithm) and the Delaunay property restored around it by Lawson flips. A
        link that runs exactly through another point is split there instead, at its
        parameter midpoint on the curve, and the triangulation is rebuilt."""
        for _ in range(rounds):
            tri, P = self.triangulate()
            if tri is None:
                return None
            cdt = _Cdt(P, tri.simplices, tri.neighbors)
            ab, _, _ = self.link_array()
            links = [(ci, k) for ci, k, *_ in self.links()]
            constraints = {(min(a, b), max(a, b)) for a, b in ab.tolist()}
            failed = [i for i, (a, b) in enumerate(ab.tolist()) if not cdt.insert(a, b, constraints)]
            if not failed:
                return cdt
            for i in sorted(failed, reverse=True):
                ci, k = links[i]
                e, _, _, pts = self.chains[ci]
                (_, t0), (_, t1) = pts[k], pts[k + 1]
                tm = 0.5 * (t0 + t1)
                self.pts.append(net.eval(net_edges[ci], tm))
                pts.insert(k + 1, (len(self.pts) - 1, tm))
        raise Invalid("pattern edges could not be recovered as mesh edges")


def _orient(a, b, c) -> float:
    return (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0])


def _incircle(a, b, c, d) -> float:
    """> 0 when d lies inside the circumcircle of the counter-clockwise triangle abc."""
    adx, ady, bdx, bdy, cdx, cdy = a[0] - d[0], a[1] - d[1], b[0] - d[0], b[1] - d[1], c[0] - d[0], c[1] - d[1]
    return ((adx * adx + ady * ady) * (bdx * cdy - cdx * bdy) - (bdx * bdx + bdy * bdy) * (adx * cdy - cdx * ady)
            + (cdx * cdx + cdy * cdy) * (adx * bdy - bdx * ady))


class _Cdt:
    """A mutable triangulation (counter-clockwise triangles, neighbour opposite each vertex)
    that takes constraint edges by flips."""

    def __init__(self, P: np.ndarray, simplices: np.ndarray, neighbors: np.ndarray):
        self.P = P
        self.T = [list(map(int, t)) for t in simplices]
        self.N = [list(map(int, n)) for n in neighbors]
        for f, t in enumerate(self.T):
            if _orient(P[t[0]], P[t[1]], P[t[2]]) < 0:
                t[1], t[2] = t[2], t[1]
                self.N[f][1], self.N[f][2] = self.N[f][2], self.N[f][1]
        self._S = self._Nb = None
        self.V: Dict[int, set] = {}
        for f, t in enumerate(self.T):
            for v in t:
                self.V.setdefault(v, set()).add(f)

    # -- queries (arrays cached until the next flip)
    @property
    def simplices(self) -> np.ndarray:
        if self._S is None:
            self._S = np.asarray(self.T, np.int64).reshape(-1, 3)
        return self._S

    @property
    def neighbors(self) -> np.ndarray:
        if self._Nb is None:
            self._Nb = np.asarray(self.N, np.int64).reshape(-1, 3)
        return self._Nb

    @property
    def vertex_neighbor_vertices(self):
        t = self.simplices
        e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]], t[:, [1, 0]], t[:, [2, 1]], t[:, [0, 2]]])
        e = np.unique(e, axis=0)
        ind = np.searchsorted(e[:, 0], np.arange(len(self.P) + 1))
        return ind, e[:, 1]

    def find_simplex(self, q: np.ndarray) -> np.ndarray:
        """The face containing each query point (-1 when none of the nearest faces does)."""
        from scipy.spatial import cKDTree

        t = self.simplices
        tp = self.P[t]
        out = np.full(len(q), -1, np.int64)
        if not len(t) or not len(q):
            return out
        k = min(12, len(t))
        _, cand = cKDTree(tp.mean(1)).query(q, k=k)
        cand = cand.reshape(len(q), k)
        for j in range(k):
            f = cand[:, j]
            a, b, c = tp[f, 0], tp[f, 1], tp[f, 2]
            inside = ((_orient_v(a, b, q) >= 0) & (_orient_v(b, c, q) >= 0) & (_orient_v(c, a, q) >= 0))
            take = inside & (out < 0)
            out[take] = f[take]
        return out

    def _face_with_edge(self, a: int, b: int) -> Optional[Tuple[int, int]]:
        """(face, index of its vertex opposite the directed edge a->b) or None."""
        for f in self.V.get(a, ()):
            t = self.T[f]
            i = t.index(a)
            if t[(i + 1) % 3] == b:
                return f, (i + 2) % 3
        return None

    def has_edge(self, a: int, b: int) -> bool:
        return self._face_with_edge(a, b) is not None or self._face_with_edge(b, a) is not None

    # -- flips
    def _flip(self, f: int, i: int) -> Tuple[int, int]:
        """Flip the edge of face f opposite its vertex i; returns the new diagonal (p, s)."""
        T, N = self.T, self.N
        self._S = self._Nb = None
        p, q, r = T[f][i], T[f][(i + 1) % 3], T[f][(i + 2) % 3]
        g = N[f][i]
        j = [k for k in range(3) if T[g][k] not in (q, r)][0]
        s = T[g][j]
        # neighbours: A across r-p (opposite q in f), B across p-q (opposite r in f),
        # C across q-s (opposite r in g), D across s-r (opposite q in g)
        A, B = N[f][(i + 1) % 3], N[f][(i + 2) % 3]
        gq, gr = T[g].index(q), T[g].index(r)
        C, D = N[g][gr], N[g][gq]
        for v in (r,):
            self.V[v].discard(f)
        for v in (q,):
            self.V[v].discard(g)
        T[f], N[f] = [p, q, s], [C, g, B]
        T[g], N[g] = [p, s, r], [D, A, f]
        self.V[s].add(f)
        self.V[p].add(g)
        if A >= 0:
            N[A][N[A].index(f)] = g
        if C >= 0:
            N[C][N[C].index(g)] = f
        return p, s

    def _legalise(self, edges, constraints) -> None:
        """Lawson flips of the given edges (and those they expose) that are not constraints."""
        stack = list(edges)
        guard = 0
        while stack and guard < 200000:
            guard += 1
            a, b = stack.pop()
            if (min(a, b), max(a, b)) in constraints:
                continue
            fe = self._face_with_edge(a, b)
            if fe is None:
                continue
            f, i = fe
            g = self.N[f][i]
            if g < 0:
                continue
            t = self.T[f]
            s = [v for v in self.T[g] if v not in (a, b)][0]
            P = self.P
            if _incircle(P[t[0]], P[t[1]], P[t[2]], P[s]) > 0:
                p = t[i]
                # the quad is convex when s is inside the circumcircle of a Delaunay-adjacent pair
                if _orient(P[p], P[a], P[s]) * _orient(P[p], P[b], P[s]) < 0:
                    self._flip(f, i)
                    stack += [(p, a), (a, s), (s, b), (b, p)]

    def insert(self, a: int, b: int, constraints: set) -> bool:
        """Make a-b an edge; False when the segment runs through another vertex."""
        if self.has_edge(a, b):
            return True
        P = self.P
        pa, pb = P[a], P[b]
        crossing = self._crossed_edges(a, b)
        if crossing is None:
            return False
        queue = deque(crossing)
        new_edges = []
        guard = 0
        while queue:
            guard += 1
            if guard > 100000:
                return False
            u, v = queue.popleft()
            fe = self._face_with_edge(u, v) or self._face_with_edge(v, u)
            if fe is None:
                return False
            f, i = fe
            g = self.N[f][i]
            if g < 0:
                return False
            p = self.T[f][i]
            s = [w for w in self.T[g] if w not in (u, v)][0]
            # convex quad p, u, s, v: the diagonals cross properly
            if not _segments_cross(P[p], P[s], P[u], P[v]):
                queue.append((u, v))
                if len(queue) > 1 and guard > 50 * (len(crossing) + 1) ** 2:
                    return False
                continue
            x, y = self._flip(f, i)
            if {x, y} == {a, b}:
                continue
            if _segments_cross(P[x], P[y], pa, pb):
                queue.append((x, y))
            else:
                new_edges.append((x, y))
        self._legalise(new_edges, constraints | {(min(a, b), max(a, b))})
        return self.has_edge(a, b)

    def _crossed_edges(self, a: int, b: int):
        """Edges crossed by the open segment a-b, walking from a; None when the segment meets
        another vertex."""
        P = self.P
        pa, pb = P[a], P[b]
        start = None
        for f in self.V.get(a, ()):
            t = self.T[f]
            i = t.index(a)
            u, v = t[(i + 1) % 3], t[(i + 2) % 3]
            ou, ov = _orient(pa, pb, P[u]), _orient(pa, pb, P[v])
            if (ou == 0 and _between(pa, pb, P[u])) or (ov == 0 and _between(pa, pb, P[v])):
                return None
            if ou < 0 < ov:  # b lies strictly inside the wedge u-a-v, beyond edge u-v
                start = (f, u, v)
                break
        if start is None:
            return None
        out = []
        f, u, v = start
        for _ in range(len(self.T) + 1):
            out.append((u, v))
            fe = self._face_with_edge(v, u)
            if fe is None:
                return None
            g, k = fe
            w = self.T[g][k]
            if w == b:
                return out
            ow = _orient(pa, pb, P[w])
            if ow == 0:
                return None
            if ow < 0:
                u = w
            else:
                v = w
        return None


def _orient_v(a, b, c):
    return (b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (b[:, 1] - a[:, 1]) * (c[:, 0] - a[:, 0])


def _between(a, b, c) -> bool:
    """c (collinear with a-b) lies strictly between a and b."""
    d = b - a
    t = float(np.dot(c - a, d)) / max(float(np.dot(d, d)), 1e-300)
    return 0.0 < t < 1.0


def _classify(simplices: np.ndarray, neighbors: np.ndarray, edge_kind: Dict[Tuple[int, int], int],
              areas: np.ndarray) -> np.ndarray:
    """Fabric faces: odd outline-crossing depth from the hull (0-1 BFS), then the largest
    component by area across everything but dart legs (lib.rs:865-965)."""
    nf = len(simplices)
    t = simplices.astype(np.int64)
    n = int(t.max()) + 1 if nf else 1
    across = np.full((nf, 3), FREE, np.int64)
    if edge_kind:
        keys = np.array([a * n + b for a, b in edge_kind], np.int64)
        kinds = np.array(list(edge_kind.values()), np.int64)
        order = np.argsort(keys)
        keys, kinds = keys[order], kinds[order]
        for k in range(3):
            a, b = t[:, (k + 1) % 3], t[:, (k + 2) % 3]
            fk = np.minimum(a, b) * n + np.maximum(a, b)
            pos = np.minimum(np.searchsorted(keys, fk), len(keys) - 1)
            hit = keys[pos] == fk
            across[hit, k] = kinds[pos[hit]]
    depth = np.full(nf, np.iinfo(np.int64).max)
    q = deque()
    for f in range(nf):
        hull = [int(across[f, k] == K_OUTLINE) for k in range(3) if neighbors[f, k] < 0]
        if hull:
            d = min(hull)
            if depth[f] > d:
                depth[f] = d
                (q.appendleft if d == 0 else q.append)(f)
    while q:
        f = q.popleft()
        d = depth[f]
        for k in range(3):
            g = int(neighbors[f, k])
            if g < 0:
                continue
            w = int(across[f, k] == K_OUTLINE)
            if depth[g] > d + w:
                depth[g] = d + w
                (q.appendleft if w == 0 else q.append)(g)
    inside = depth % 2 == 1
    comp = np.full(nf, -1)
    best, best_area, cid = -1, -1.0, 0
    for s in range(nf):
        if not inside[s] or comp[s] >= 0:
            continue
        comp[s] = cid
        stack, area = [s], 0.0
        while stack:
            f = stack.pop()
            area += areas[f]
            for k in range(3):
                g = int(neighbors[f, k])
                if g >= 0 and inside[g] and comp[g] < 0 and across[f, k] != K_DART:
                    comp[g] = cid
                    stack.append(g)
        if area > best_area:
            best, best_area = cid, area
        cid += 1
    return comp == best if best >= 0 else np.zeros(nf, bool)


def _tri_quality(P: np.ndarray, simp: np.ndarray):
    p = P[simp]
    e = np.stack([p[:, 1] - p[:, 0], p[:, 2] - p[:, 1], p[:, 0] - p[:, 2]], 1)
    area = 0.5 * np.abs(e[:, 0, 0] * (-e[:, 2, 1]) - e[:, 0, 1] * (-e[:, 2, 0]))
    l2 = (e * e).sum(2)
    # smallest angle from the law of sines: sin(min) = 2 A / (longest other two)
    lmax = np.sqrt(l2)
    s = np.sort(lmax, 1)
    with np.errstate(divide="ignore", invalid="ignore"):
        sin_min = np.clip(2.0 * area / (s[:, 1] * s[:, 2]), 0.0, 1.0)
    return area, np.degrees(np.arcsin(sin_min))


def triangulate(net: Network, notches: Sequence[Tuple[int, float]] = (), opts: Options = Options()) -> SimMesh:
    """Triangulate one pattern piece (lib.rs:596-790). ``notches`` are (edge, t) pairs, each
    becoming a mesh vertex exactly on that edge."""
    opts.validate()
    by_edge: Dict[int, List[float]] = {}
    for e, t in notches:
        by_edge.setdefault(int(e), []).append(float(t))
    live = [(i, e) for i, e in enumerate(net.edges) if e is not None and _kind(e.semantic) is not None]
    boundary_mm = sum(net.arc_length(i) for i, _ in live)
    if boundary_mm / opts.target_edge_mm > MAX_INPUT_POINTS:
        x0, y0, x1, y1 = net.bounds()
        raise TooDense(MAX_INPUT_POINTS, opts.target_edge_mm, max(x1 - x0, y1 - y0))

    # 1 & 2: flatten, snap-round, dedup
    pts, sources, index, chains, net_edges = [], [], {}, [], []
    w = opts.weld_mm
    for eid, e in live:
        points = []
        for t, p in _samples(net, eid, by_edge.get(eid, ()), opts):
            k = (_round_half_away(p[0] / w), _round_half_away(p[1] / w))
            src = ("vertex", e.start) if t == 0.0 else (("vertex", e.end) if t == 1.0 else ("edge", eid))
            if k not in index:
                index[k] = len(pts)
                pts.append(np.array([k[0] * w, k[1] * w]))
                sources.append(src)
            slot = index[k]
            if src[0] == "vertex":
                sources[slot] = src
            if not points or points[-1][0] != slot:
                points.append((slot, t))
        if len(points) >= 2:
            chains.append([eid, e.semantic, _kind(e.semantic), points])
            net_edges.append(eid)
    if len(pts) < 3:
        raise Degenerate(len(pts), opts.weld_mm)
    if len(pts) > MAX_INPUT_POINTS:
        x0, y0, x1, y1 = net.bounds()
        raise TooDense(MAX_INPUT_POINTS, opts.target_edge_mm, max(x1 - x0, y1 - y0))

    # 3: Delaunay with every pattern link recovered
    m = _Mesher(pts, chains, opts)
    m.check_crossings(net_edges)
    tri = m.recover(net, net_edges)
    if tri is None:
        raise NoRegion()

    def kinds():
        k = {}
        for _, _, a, b, kind in m.links():
            key = (min(a, b), max(a, b))
            k[key] = max(k.get(key, FREE), kind)
        return k

    def fabric(tri):
        P = np.asarray(m.pts)
        area, _ = _tri_quality(P, tri.simplices)
        return _classify(tri.simplices, tri.neighbors, kinds(), area)

    keep = fabric(tri)
    complete = True
    if opts.refine and keep.any():
        tri, keep, complete = _refine(m, net, net_edges, tri, keep, fabric, opts)

    # 6: emit
    P = np.asarray(m.pts)
    on_edge = {v: eid for eid, _, _, points in m.chains for v, _ in points}
    remap: Dict[int, int] = {}
    out_mm, out_src, faces, dropped = [], [], [], 0
    for f in np.flatnonzero(keep):
        t = [int(v) for v in tri.simplices[f]]
        a, b, c = P[t[0]], P[t[1]], P[t[2]]
        cr = (b[0] - a[0]) * (c[1] - a[1]) - (c[0] - a[0]) * (b[1] - a[1])
        if cr == 0:
            dropped += 1
            continue
        if cr < 0:
            t = [t[0], t[2], t[1]]
        row = []
        for v in t:
            if v not in remap:
                remap[v] = len(out_mm)
                out_mm.append(P[v])
                out_src.append(sources[v] if v < len(sources) else
                               (("edge", on_edge[v]) if v in on_edge else ("interior", -1)))
            row.append(remap[v])
        faces.append(row)
    if not faces:
        raise NoRegion()
    mm = np.asarray(out_mm, np.float64)
    mesh = SimMesh(positions=np.concatenate([(mm * MM_TO_M).astype(np.float32), np.zeros((len(mm), 1), np.float32)], 1),
                   indices=np.asarray(faces, np.uint32), pattern_mm=mm, sources=out_src, chains=[],
                   refinement_complete=complete, degenerate_dropped=dropped)
    for eid, sem, _, points in sorted(m.chains, key=lambda c: c[0]):
        kept = [(remap[v], t) for v, t in points if v in remap]
        if len(kept) >= 2:
            mesh.chains.append(EdgeChain(eid, sem, kept))
    err = mesh.check()
    if err:
        raise Invalid(err)
    return mesh


def _smooth(m, net, net_edges, tri, keep, fabric, lo: int, hi: int, near_link, link_geometry, in_fabric,
            clearance: float, rounds: int = 4):
    """Laplacian smoothing of the points lo..hi-1 (each moved to the mean of its Delaunay
    neighbours), a move kept only if it stays in the fabric and clear of the pattern links."""
    for _ in range(rounds):
        P = np.asarray(m.pts)
        ind, nb = tri.vertex_neighbor_vertices
        cnt = np.diff(ind)
        sums = np.zeros_like(P)
        np.add.at(sums, np.repeat(np.arange(len(P)), cnt), P[nb])
        new = P.copy()
        has = cnt > 0
        new[has] = sums[has] / cnt[has, None]
        moved = np.arange(lo, hi)
        if not len(moved):
            break
        la, lb = link_geometry()
        ok = in_fabric(tri, keep, new[moved]) & ~near_link(new[moved], la, lb, clearance)
        for v, good in zip(moved, ok):
            if good:
                m.pts[v] = new[v]
        tri = m.recover(net, net_edges)
        keep = fabric(tri)
    return tri, keep


def _refine(m: _Mesher, net: Network, net_edges, tri, keep, fabric, opts: Options):
    """Lattice seeding, then circumcentre / link-apex insertion for bad fabric triangles
    (area over the equilateral bound or smallest angle under min_angle_deg)."""
    from scipy.spatial import cKDTree

    h = opts.target_edge_mm
    max_area = math.sqrt(3.0) / 4.0 * h * h
    added = 0

    def link_geometry():
        ab, _, _ = m.link_array()
        P = np.asarray(m.pts)
        return P[ab[:, 0]], P[ab[:, 1]]

    def near_link(c: np.ndarray, la, lb, clearance: float) -> np.ndarray:
        """Candidates within clearance of any link (segment distance), or encroaching one
        (inside its diametral circle)."""
        bad = np.zeros(len(c), bool)
        if not len(la) or not len(c):
            return bad
        mid, half = 0.5 * (la + lb), 0.5 * np.linalg.norm(lb - la, axis=1)
        tree = cKDTree(mid)
        reach = half.max() + clearance

        def test(ci, js):
            a, b = la[js], lb[js]
            ab = b - a
            x = c[ci][:, None, :] if np.ndim(ci) else c[ci][None, :]
            t = np.clip(((x - a) * ab).sum(-1) / np.maximum((ab * ab).sum(-1), 1e-300), 0.0, 1.0)
            d = np.linalg.norm(a + ab * t[..., None] - x, axis=-1)
            enc = np.linalg.norm(x - mid[js], axis=-1) < half[js]
            return ((d < clearance) | enc).any(-1)

        k = min(16, len(mid))
        dist, js = tree.query(c, k=k)
        js = js.reshape(len(c), k)
        bad = test(np.arange(len(c)), js)
        # where more than k links lie within reach, check them all
        crowded = np.flatnonzero(dist.reshape(len(c), k)[:, -1] <= reach) if k < len(mid) else []
        for i in crowded:
            jj = np.asarray(tree.query_ball_point(c[i], reach))
            bad[i] = bool(test(i, jj)) if len(jj) else False
        return bad

    def in_fabric(tri, keep, c):
        f = tri.find_simplex(c)
        return (f >= 0) & keep[np.maximum(f, 0)]

    # lattice seeds over the fabric, half an edge clear of every pattern link
    P = np.asarray(m.pts)
    lo, hi = P.min(0), P.max(0)
    dy = h * math.sqrt(3.0) / 2.0
    seeds = []
    for r, y in enumerate(np.arange(lo[1] + dy, hi[1], dy)):
        xs = np.arange(lo[0] + (0.5 * h if r % 2 else h), hi[0], h)
        seeds.append(np.stack([xs, np.full(len(xs), y)], 1))
    seeds = np.concatenate(seeds) if seeds else np.zeros((0, 2))
    if len(seeds):
        rng = np.random.default_rng(0)
        seeds = seeds + rng.uniform(-0.1 * h, 0.1 * h, seeds.shape)
        la, lb = link_geometry()
        ok = in_fabric(tri, keep, seeds) & ~near_link(seeds, la, lb, 0.5 * h)
        seeds = seeds[ok][: opts.max_steiner]
        first = len(m.pts)
        m.pts.extend(list(seeds))
        added += len(seeds)
        tri = m.recover(net, net_edges)
        keep = fabric(tri)
        tri, keep = _smooth(m, net, net_edges, tri, keep, fabric, first, len(m.pts), near_link, link_geometry,
                            in_fabric, 0.5 * h)

    complete = True
    for _ in range(60):
        P = np.asarray(m.pts)
        area, angle = _tri_quality(P, tri.simplices)
        bad = keep & ((area > max_area) | (angle < opts.min_angle_deg))
        if opts.min_area_mm2 is not None:
            bad &= area > opts.min_area_mm2
        if not bad.any():
            break
        fb = np.flatnonzero(bad)
        fb = fb[np.argsort(angle[fb])]  # worst first
        tp = P[tri.simplices[fb]]
        cand = _circumcentres(tp)
        radius = np.linalg.norm(cand - tp[:, 0], axis=1)
        la, lb = link_geometry()
        enc = near_link(cand, la, lb, 0.0) | ~np.isfinite(cand).all(1) | ~in_fabric(tri, keep, cand)
        # an encroaching circumcentre gives way to the apex of the equilateral triangle on
        # the nearest link, on the triangle's side
        if enc.any():
            tree = cKDTree(0.5 * (la + lb))
            cen = tp[enc].mean(1)
            _, j = tree.query(cen)
            a, b = la[j], lb[j]
            nrm = np.stack([-(b - a)[:, 1], (b - a)[:, 0]], 1)
            side = np.sign(((cen - a) * nrm).sum(1))[:, None]
            cand[enc] = 0.5 * (a + b) + nrm * side * (math.sqrt(3.0) / 2.0)
            radius[enc] = np.linalg.norm(b - a, axis=1)
        good = in_fabric(tri, keep, cand) & ~near_link(cand, la, lb, 0.0)
        cand, radius = cand[good], radius[good]
        if not len(cand):
            break
        # a new point keeps 0.6 of its own radius (the circumradius, or the link length for an
        # apex) from every point, old or new, so one round does not cluster
        d, _ = cKDTree(P).query(cand)
        ok = d >= 0.6 * radius
        cand, radius = cand[ok], radius[ok]
        chosen, taken = [], np.zeros(len(cand), bool)
        near = cKDTree(cand).query_ball_point(cand, 0.6 * radius) if len(cand) else []
        for i in range(len(cand)):
            if taken[i]:
                continue
            chosen.append(i)
            taken[near[i]] = True
        if not chosen:
            break
        room = opts.max_steiner - added
        if room <= 0:
            complete = False
            break
        new = cand[chosen][:room]
        m.pts.extend(list(new))
        added += len(new)
        tri = m.recover(net, net_edges)
        keep = fabric(tri)
    else:
        complete = False
    return tri, keep, complete
