"""A garment document sewn into one simulation scene (ui/crates/nguo-sewing/src/garment.rs):
validate, triangulate every piece (notches become mesh vertices on their edges), arrange the
pieces in seam order, concatenate them placed (re-wound where a placement mirrors the
pattern plane), then resolve every seam onto the meshes and pair it, straight or reversed,
whichever the arrangement actually brings together (a reversed pairing is reported as a
flipped seam). ``SewnGarment.scene`` turns the result into the step's scene description.

``sample_bodice_block`` is the reference's sample document (sample.rs:52-179): two
560 x 560 mm panels, waist and hem cut, sides sewn front-right to back-left and front-left
to back-right round the body, each hanging by its waist.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import arrange as A
from . import sewing
from . import triangulate as T
from .seams import Document, Seam, SeamSide, is_sewable, validate, Diagnostic, WARNING


class SewError(RuntimeError):
    """A document that cannot become a garment (garment.rs:49-70)."""


class NotSewable(SewError):
    def __init__(self, diagnostics):
        first = next((d.message() for d in diagnostics if d.severity == "error"), "no error reported")
        super().__init__(f"the garment cannot be sewn as authored: {first}")
        self.diagnostics = diagnostics


class Empty(SewError):
    def __init__(self):
        super().__init__("the document has no pieces to sew")


@dataclass(frozen=True)
class SewOptions:
    """30 mm target edges (garment.rs:34-46) and the arranger's defaults."""
    triangulate: T.Options = T.Options(target_edge_mm=30.0)
    arrange: A.ArrangeOptions = A.ArrangeOptions()


@dataclass
class PieceMesh:
    piece: int
    name: str
    mesh: T.SimMesh
    placement: object
    vertex_offset: int


@dataclass
class SewnSeam:
    seam: int
    stitches: int
    ease: float
    flipped: bool
    open_m: float


@dataclass
class SewnGarment:
    positions: np.ndarray   # f32 (n, 3) world metres
    tris: np.ndarray        # u32 (m, 3)
    uvs: np.ndarray         # f32 (n, 2)
    stitch_idx: np.ndarray  # u32 (s, 6)
    stitch_w: np.ndarray    # f32 (s, 6)
    pieces: List[PieceMesh]
    seams: List[SewnSeam]
    diagnostics: List[Diagnostic]
    arrangement: A.Arrangement
    timings_ms: dict = field(default_factory=dict)

    def vertex_count(self) -> int:
        return len(self.positions)

    def triangle_count(self) -> int:
        return len(self.tris)

    def max_seam_gap_m(self) -> float:
        if not len(self.stitch_idx):
            return 0.0
        p = self.positions.astype(np.float64)
        a = (p[self.stitch_idx[:, :3]] * self.stitch_w[:, :3, None]).sum(1)
        b = (p[self.stitch_idx[:, 3:]] * self.stitch_w[:, 3:, None]).sum(1)
        return float(np.linalg.norm(a - b, axis=1).max())

    def check(self) -> Optional[str]:
        """None, or what is wrong (garment.rs:188-232)."""
        n = len(self.positions)
        if not n or not len(self.tris):
            return "the garment has no geometry"
        if len(self.uvs) != n:
            return f"{len(self.uvs)} uvs for {n} vertices"
        if not np.isfinite(self.positions).all():
            return "a vertex is not finite"
        if (self.tris >= n).any():
            return f"a triangle indexes past {n} vertices"
        if len(self.stitch_idx) and (self.stitch_idx >= n).any():
            return f"a stitch indexes past {n} vertices"
        return None

    def stitch_pairs(self) -> list:
        """The stitches as the bridge's drape loop takes them: (index[6], weight[6]) each."""
        return [(i.tolist(), w.tolist()) for i, w in zip(self.stitch_idx, self.stitch_w)]

    def scene(self, density=0.2, young=1e5, poisson=0.3, thickness=5e-4, stitch_k=1.0, stitch_l0=1e-3,
              stitch_cap=1e-2, **params) -> dict:
        """The garment as a scene description for ImplicitSolver / the oracle: StVK membranes
        resting at the placed (isometric) shape, uniform lumped mass, the seams' stitches."""
        from . import scenes

        mu, lam = scenes.lame_from_young_poisson(young * thickness, poisson)
        m = scenes.uniform_mass(self.positions, self.tris, density)
        kl = np.tile(np.float32([[stitch_k, stitch_l0, stitch_cap]]), (len(self.stitch_idx), 1))
        return {"positions": self.positions.copy(), "velocities": np.zeros_like(self.positions),
                "inv_mass": np.full(len(self.positions), 1.0 / m, np.float32), "tris": self.tris.copy(),
                "shell_faces": self.tris.copy(), "static_mask": None, "stitch_idx": self.stitch_idx.copy(),
                "stitch_w": self.stitch_w.copy(), "stitch_kl": kl, "colliders": np.zeros((0, 8), np.float32),
                "params": scenes.default_params(shell_mu=mu, shell_lambda=lam, **params)}


def _side_samples(doc: Document, pm: PieceMesh, side: SeamSide) -> sewing.SideSamples:
    chains = []
    for e, rev in side.edges:
        c = pm.mesh.chain(e)
        if c is None:
            raise SewError(f"edge {e} of piece {side.piece} has no vertices in its mesh")
        vs = [v + pm.vertex_offset for v, _ in c.points]
        chains.append((sewing.EdgeChain(vs, pm.mesh.pattern_mm[[v for v, _ in c.points]]), rev))
    return sewing.side_samples(chains, side.span)


def build(doc: Document, opts: SewOptions = SewOptions()) -> SewnGarment:
    """Sew ``doc`` into one garment (garment.rs:234-400)."""
    timings = {}
    t = time.perf_counter()
    diagnostics = validate(doc)
    timings["validate"] = (time.perf_counter() - t) * 1e3
    if not is_sewable(diagnostics):
        raise NotSewable(diagnostics)
    order = A.seam_order(list(doc.pieces), [(s.a.piece, s.b.piece) for s in doc.seams.values()])
    if not order:
        raise Empty()

    t = time.perf_counter()
    meshes = []
    for pid in order:
        f = doc.features.get(pid, {})
        meshes.append((pid, T.triangulate(doc.pieces[pid], f.get("notches", ()), opts.triangulate)))
    timings["triangulate"] = (time.perf_counter() - t) * 1e3

    t = time.perf_counter()
    extents = []
    for pid, mesh in meshes:
        f = doc.features.get(pid, {})
        extents.append(A.PieceExtent(pid, tuple(mesh.pattern_bounds()), f.get("placement"), support_arc_mm(doc, pid)))
    arrangement = A.arrange(extents, opts.arrange)
    timings["arrange"] = (time.perf_counter() - t) * 1e3

    positions, tris, uvs, pieces = [], [], [], []
    base = 0
    for (pid, mesh), placement in zip(meshes, arrangement.placements):
        positions.append(placement.apply(mesh.pattern_mm))
        uvs.append(mesh.uvs())
        tt = mesh.indices.astype(np.int64)
        tris.append((tt[:, [0, 2, 1]] if placement.flips_winding() else tt) + base)
        pieces.append(PieceMesh(pid, doc.features.get(pid, {}).get("name", f"piece {pid}"), mesh, placement, base))
        base += mesh.vertex_count()
    positions = np.concatenate(positions).astype(np.float32)

    t = time.perf_counter()
    idx, w, sewn = [], [], []
    for sid in sorted(doc.seams):
        seam = doc.seams[sid]
        pa = next((p for p in pieces if p.piece == seam.a.piece), None)
        pb = next((p for p in pieces if p.piece == seam.b.piece), None)
        if pa is None or pb is None:
            continue
        a, b = _side_samples(doc, pa, seam.a), _side_samples(doc, pb, seam.b)
        straight = sewing.pairing_distance_m(a, b, positions, False)
        flipped = sewing.pairing_distance_m(a, b, positions, True)
        flip = flipped < 0.5 * straight  # garment.rs:349-353
        if flip:
            diagnostics.append(Diagnostic(WARNING, "flipped", seam=sid))
        c = sewing.correspond(a, b, flip)
        ci, cw = c.arrays()
        idx.append(ci)
        w.append(cw)
        sewn.append(SewnSeam(sid, len(c.stitches), c.ease(), flip, flipped if flip else straight))
    timings["sew"] = (time.perf_counter() - t) * 1e3
    g = SewnGarment(positions, np.concatenate(tris).astype(np.uint32), np.concatenate(uvs).astype(np.float32),
                    np.concatenate(idx) if idx else np.zeros((0, 6), np.uint32),
                    np.concatenate(w) if w else np.zeros((0, 6), np.float32), pieces, sewn, diagnostics,
                    arrangement, timings)
    err = g.check()
    if err:
        raise SewError(f"internal error: the garment violated its own invariants: {err}")
    return g


@dataclass
class Hang:
    """Where a garment hangs, read off the document before any mesh exists (arrange.rs:253-294):
    the first piece's support landmark and the tallest piece's height in pattern mm."""
    landmark: Optional[str] = None
    drop_mm: float = 0.0


def hang(doc: Document) -> Hang:
    out = Hang()
    for pid in sorted(doc.pieces):
        net = doc.pieces[pid]
        if net.vertices:
            x0, y0, x1, y1 = net.bounds()
            out.drop_mm = max(out.drop_mm, y1 - y0)
        if out.landmark is None:
            out.landmark = doc.features.get(pid, {}).get("landmark")
    return out


def support_arc_mm(doc: Document, pid: int) -> Optional[float]:
    """Arc length of the piece's support edge in pattern mm (arrange.rs:296-303)."""
    e = doc.features.get(pid, {}).get("support_edge")
    return None if e is None else doc.pieces[pid].arc_length(e)


PANEL_W_MM = PANEL_H_MM = 560.0
SUPPORT_LANDMARK = "hip"
PANEL_GAP_MM = 80.0
E_WAIST, E_RIGHT, E_HEM, E_LEFT = 0, 1, 2, 3


def _rect_panel(x: float, w: float, h: float):
    n = T.Network()
    v = [n.add_vertex(px, py) for px, py in [(x, 0.0), (x + w, 0.0), (x + w, h), (x, h)]]
    sem = [T.CUT, T.SEAM, T.CUT, T.SEAM]
    return n, [n.add_edge(v[i], v[(i + 1) % 4], sem[i]) for i in range(4)]


def sample_bodice_block() -> Document:
    """Two panels sewn into a tube round the body, both sides authored top-down
    (sample.rs:72-126, 134-179)."""
    doc = Document()
    added = []
    for name, x in (("Front bodice", 0.0), ("Back bodice", PANEL_W_MM + PANEL_GAP_MM)):
        net, e = _rect_panel(x, PANEL_W_MM, PANEL_H_MM)
        added.append((doc.add_piece(net, name=name, support_edge=e[E_WAIST], landmark=SUPPORT_LANDMARK), e))
    (front, fe), (back, be) = added
    doc.add_seam(Seam(SeamSide(front, [(fe[E_RIGHT], False)]), SeamSide(back, [(be[E_LEFT], True)])))
    doc.add_seam(Seam(SeamSide(front, [(fe[E_LEFT], True)]), SeamSide(back, [(be[E_RIGHT], False)])))
    return doc
