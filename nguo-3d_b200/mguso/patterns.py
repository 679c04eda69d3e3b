"""Pattern panels to simulation meshes and sewn garments: the input side of the drape that
the garment app's pipeline (ui/crates/nguo-triangulate, ui/crates/nguo-sewing) produces.

``mesh_panel`` triangulates a simple polygon panel (straight edges, millimetres, either
winding) at a target edge length: every outline edge is subdivided evenly, the interior is
filled with a jittered triangular lattice, and the Delaunay triangulation of all points is
kept inside the outline. The outline edges must come out as triangle edges (always so for
convex panels; a concave panel whose boundary is not recovered at that resolution is an
error, never a mesh that cuts its corner). Each outline edge gets its chain of mesh vertices
(``sewing.EdgeChain``), which is what seam correspondence consumes.

``Garment`` places panels in 3-D (metres), sews seams between panel edges through
``sewing.correspond`` and emits one scene description with StVK membranes resting at the
pattern shape.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Sequence, Tuple

import numpy as np

from . import sewing


class PatternError(ValueError):
    pass


@dataclass
class PanelMesh:
    """A triangulated panel: pattern-space vertices (mm), counter-clockwise triangles and
    one vertex chain per outline edge (edge k runs from outline point k to k+1)."""
    points_mm: np.ndarray
    tris: np.ndarray
    chains: List[sewing.EdgeChain]

    def area_mm2(self) -> float:
        p = self.points_mm[self.tris]
        u, v = p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]
        return float(0.5 * np.abs(u[:, 0] * v[:, 1] - u[:, 1] * v[:, 0]).sum())


def _signed_area(poly: np.ndarray) -> float:
    x, y = poly[:, 0], poly[:, 1]
    return 0.5 * float(np.dot(x, np.roll(y, -1)) - np.dot(y, np.roll(x, -1)))


def _inside(poly: np.ndarray, pts: np.ndarray) -> np.ndarray:
    """Even-odd point-in-polygon test."""
    x, y = pts[:, 0:1], pts[:, 1:2]
    xa, ya = poly[:, 0], poly[:, 1]
    xb, yb = np.roll(xa, -1), np.roll(ya, -1)
    cond = (ya > y) != (yb > y)
    with np.errstate(divide="ignore", invalid="ignore"):
        xc = xa + (y - ya) * (xb - xa) / (yb - ya)
    return (cond & (x < xc)).sum(1) % 2 == 1


def _seg_dist(poly: np.ndarray, pts: np.ndarray) -> np.ndarray:
    """Distance of each point to the outline."""
    a = poly[None, :, :]
    b = np.roll(poly, -1, axis=0)[None, :, :]
    p = pts[:, None, :]
    ab = b - a
    t = np.clip(((p - a) * ab).sum(-1) / np.maximum((ab * ab).sum(-1), 1e-300), 0.0, 1.0)
    q = a + ab * t[..., None]
    return np.linalg.norm(p - q, axis=-1).min(1)


def mesh_panel(outline_mm: Sequence[Sequence[float]], target_edge_mm: float, seed: int = 0) -> PanelMesh:
    """Triangulate the panel bounded by ``outline_mm`` (a simple polygon, either winding) at
    about ``target_edge_mm``."""
    from scipy.spatial import Delaunay

    poly = np.asarray(outline_mm, np.float64).reshape(-1, 2)
    if poly.shape[0] < 3 or not target_edge_mm > 0:
        raise PatternError("a panel needs at least 3 outline points and a positive target edge")
    if abs(_signed_area(poly)) < 1e-9:
        raise PatternError("the outline encloses no area")
    h = float(target_edge_mm)
    rng = np.random.default_rng(seed)
    n_out = poly.shape[0]
    pts, chain_ids = [], []
    for k in range(n_out):
        a, b = poly[k], poly[(k + 1) % n_out]
        n = max(1, math.ceil(np.linalg.norm(b - a) / h - 1e-9))
        ids = []
        for i in range(n):
            ids.append(len(pts))
            pts.append(a + (b - a) * (i / n))
        chain_ids.append(ids)
    nb = len(pts)
    for k in range(n_out):
        chain_ids[k].append(chain_ids[(k + 1) % n_out][0])
    # interior: a triangular lattice, jittered, kept half an edge clear of the outline
    lo, hi = poly.min(0), poly.max(0)
    dy = h * math.sqrt(3) / 2
    ys = np.arange(lo[1] + dy, hi[1], dy)
    cand = []
    for r, y in enumerate(ys):
        xs = np.arange(lo[0] + h * (0.5 if r % 2 else 1.0), hi[0], h)
        cand += [(x, y) for x in xs]
    cand = np.asarray(cand, np.float64).reshape(-1, 2)
    if cand.size:
        cand = cand + rng.uniform(-0.15 * h, 0.15 * h, cand.shape)
        keep = _inside(poly, cand) & (_seg_dist(poly, cand) > 0.5 * h)
        cand = cand[keep]
    allp = np.concatenate([np.asarray(pts), cand]) if cand.size else np.asarray(pts)
    tri = Delaunay(allp).simplices.astype(np.int64)
    cen = allp[tri].mean(1)
    tri = tri[_inside(poly, cen)]
    a, b, c = allp[tri[:, 0]], allp[tri[:, 1]], allp[tri[:, 2]]
    cross = (b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (b[:, 1] - a[:, 1]) * (c[:, 0] - a[:, 0])
    tri = tri[np.abs(cross) > 1e-12 * h * h]
    cross = cross[np.abs(cross) > 1e-12 * h * h]
    tri[cross < 0] = tri[cross < 0][:, [0, 2, 1]]
    # every outline segment must be a triangle edge (the outline was recovered)
    edges = set()
    for t in tri:
        for i in range(3):
            u, v = int(t[i]), int(t[(i + 1) % 3])
            edges.add((min(u, v), max(u, v)))
    for k, ids in enumerate(chain_ids):
        for u, v in zip(ids, ids[1:]):
            if (min(u, v), max(u, v)) not in edges:
                raise PatternError(f"outline edge {k} was not recovered by the triangulation at "
                                   f"{h} mm; refine the target edge")
    used = np.zeros(len(allp), bool)
    used[tri.ravel()] = True
    if not used[:nb].all():
        raise PatternError("an outline point is not part of the mesh")
    remap = -np.ones(len(allp), np.int64)
    remap[used] = np.arange(used.sum())
    pts_out = allp[used]
    tri = remap[tri]
    chains = [sewing.EdgeChain([int(remap[i]) for i in ids], pts_out[[remap[i] for i in ids]]) for ids in chain_ids]
    return PanelMesh(pts_out, tri.astype(np.uint32), chains)


def panel_from_triangulation(mesh, edges: Sequence[int]) -> PanelMesh:
    """A piece meshed by ``triangulate.triangulate`` as a PanelMesh: the chains of the pattern
    edges ``edges`` (ids, in the order the panel's seams will name them: panel edge k is
    pattern edge edges[k]) become the panel's chains, each from its edge's start to its end."""
    chains = []
    for e in edges:
        c = mesh.chain(e)
        if c is None:
            raise PatternError(f"pattern edge {e} has no chain in the mesh (a grain marker, or outside the fabric)")
        vs = [v for v, _ in c.points]
        chains.append(sewing.EdgeChain(vs, mesh.pattern_mm[vs]))
    return PanelMesh(np.asarray(mesh.pattern_mm, np.float64), mesh.indices.astype(np.uint32), chains)


@dataclass
class _Placed:
    mesh: PanelMesh
    origin_m: np.ndarray
    axes: np.ndarray  # 3x2: pattern x and y axes in world space
    base: int
    placement: object = None  # an arrange.Wrap / arrange.Rigid instead of origin and axes


@dataclass
class Garment:
    """Panels placed in 3-D and sewn along seams; ``scene()`` gives the description."""
    panels: List[_Placed] = field(default_factory=list)
    seams: List[Tuple[int, list, int, list, bool]] = field(default_factory=list)

    def add_panel(self, mesh: PanelMesh, origin_m=(0.0, 0.0, 0.0), x_axis=(1.0, 0.0, 0.0),
                  y_axis=(0.0, 1.0, 0.0)) -> int:
        """Place a panel: pattern (x, y) mm map to origin + (x/1000) x_axis + (y/1000) y_axis."""
        axes = np.stack([np.asarray(x_axis, np.float64), np.asarray(y_axis, np.float64)], 1)
        base = sum(p.mesh.points_mm.shape[0] for p in self.panels)
        self.panels.append(_Placed(mesh, np.asarray(origin_m, np.float64), axes, base))
        return len(self.panels) - 1

    def add_arranged_panel(self, mesh: PanelMesh, placement) -> int:
        """Place a panel by an ``arrange`` placement (a cylinder wrap or a rigid transform of
        the pattern plane); its triangles are re-wound when the placement mirrors the plane."""
        base = sum(p.mesh.points_mm.shape[0] for p in self.panels)
        self.panels.append(_Placed(mesh, np.zeros(3), np.zeros((3, 2)), base, placement))
        return len(self.panels) - 1

    def sew(self, panel_a: int, edges_a, panel_b: int, edges_b, flip=None):
        """Sew panel_a's edge chain (a list of (edge, reversed)) to panel_b's; ``flip`` None
        picks the direction that closes with less travel in the current placement."""
        self.seams.append((panel_a, list(edges_a), panel_b, list(edges_b), flip))

    def positions(self) -> np.ndarray:
        out = []
        for p in self.panels:
            if p.placement is not None:
                out.append(np.asarray(p.placement.apply(p.mesh.points_mm), np.float64))
            else:
                out.append(p.origin_m[None, :] + (p.mesh.points_mm * 1e-3) @ p.axes.T)
        return np.concatenate(out).astype(np.float32)

    def _side(self, pi, edges):
        p = self.panels[pi]
        chains = [(sewing.EdgeChain([v + p.base for v in p.mesh.chains[e].vertices], p.mesh.chains[e].points_mm), r)
                  for e, r in edges]
        return sewing.side_samples(chains)

    def stitches(self):
        """(index u32 (S, 6), weight f32 (S, 6), per-seam (ease, flipped))."""
        pos = self.positions()
        idx, w, info = [], [], []
        for pa, ea, pb, eb, flip in self.seams:
            a, b = self._side(pa, ea), self._side(pb, eb)
            if flip is None:
                c, fl = sewing.sew(a, b, pos)
            else:
                c, fl = sewing.correspond(a, b, flip), flip
            i, ww = c.arrays()
            idx.append(i)
            w.append(ww)
            info.append((c.ease(), fl))
        if not idx:
            return np.zeros((0, 6), np.uint32), np.zeros((0, 6), np.float32), info
        return np.concatenate(idx), np.concatenate(w), info

    def scene(self, density=0.2, young=1e5, poisson=0.3, thickness=5e-4, stitch_k=1.0, stitch_l0=1e-3,
              stitch_cap=1e-2, **params) -> dict:
        """The garment as a scene description: StVK membranes resting at the pattern shape,
        uniform lumped mass, stitches of stiffness ``stitch_k`` (l0, cap as given)."""
        from . import scenes

        pos = self.positions()
        tris = np.concatenate([(p.mesh.tris[:, [0, 2, 1]] if p.placement is not None and p.placement.flips_winding()
                                else p.mesh.tris).astype(np.int64) + p.base for p in self.panels]).astype(np.uint32)
        idx, w, _ = self.stitches()
        mu, lam = scenes.lame_from_young_poisson(young * thickness, poisson)
        m = scenes.uniform_mass(pos, tris, density)
        # rest shapes from the pattern (rigid placements and cylinder wraps are isometric, so they agree)
        rest = np.concatenate([p.mesh.points_mm * 1e-3 for p in self.panels])
        kl = np.tile(np.float32([[stitch_k, stitch_l0, stitch_cap]]), (idx.shape[0], 1))
        return {"positions": pos, "velocities": np.zeros_like(pos), "inv_mass": np.full(len(pos), 1.0 / m, np.float32),
                "tris": tris, "shell_faces": tris.copy(), "static_mask": None, "stitch_idx": idx, "stitch_w": w,
                "stitch_kl": kl, "colliders": np.zeros((0, 8), np.float32), "pattern_mm": rest * 1e3,
                "params": scenes.default_params(shell_mu=mu, shell_lambda=lam, **params)}
