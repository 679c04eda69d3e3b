"""Garment documents and seam validation as a maintained constraint (ui/crates/nguo-sewing/
src/validate.rs, with the document model of ui/crates/nguo-doc/src/model.rs): a pure function
of the document, cheap enough to run on every edit, that reports unsewn seam edges,
references that do not resolve, seam sides with no single direction, and the length
difference each seam absorbs as ease (an error past ``sewing.EASE_LIMIT``, a warning when it
drifts from the ease the seam declares). Pattern geometry only: no mesh, no solver.

A ``Document`` holds pieces (a ``triangulate.Network`` each, by id) and seams (two
``SeamSide``: a piece, a chain of (edge, reversed) and a normalised span, plus the declared
``ease_ratio`` = len(b) / len(a)).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

from .sewing import EASE_LIMIT
from .triangulate import SEAM, Network

DECLARED_EASE_TOLERANCE = 0.01  # validate.rs:21

ERROR, WARNING, INFO = "error", "warning", "info"


@dataclass
class SeamSide:
    piece: int
    edges: List[Tuple[int, bool]]
    span: Tuple[float, float] = (0.0, 1.0)


@dataclass
class Seam:
    a: SeamSide
    b: SeamSide
    ease_ratio: float = 1.0

    def references_edge(self, piece: int, edge: int) -> bool:
        return any(s.piece == piece and any(e == edge for e, _ in s.edges) for s in (self.a, self.b))


@dataclass
class Document:
    """Pieces (networks by id) and seams by id. ``features`` per piece may hold ``notches``
    ([(edge, t)], registration marks that become mesh vertices), ``placement`` (an authored
    ((x, y, z) mm, quaternion)), ``support_edge`` (the edge the piece hangs by), ``landmark`` (the
    body landmark it hangs from) and ``name``."""
    pieces: Dict[int, Network] = field(default_factory=dict)
    seams: Dict[int, Seam] = field(default_factory=dict)
    features: Dict[int, dict] = field(default_factory=dict)

    def add_piece(self, net: Network, **features) -> int:
        i = max(self.pieces, default=-1) + 1
        self.pieces[i] = net
        self.features[i] = dict(features)
        return i

    def add_seam(self, seam: Seam) -> int:
        i = max(self.seams, default=-1) + 1
        self.seams[i] = seam
        return i


@dataclass
class Diagnostic:
    severity: str
    kind: str        # unsewn, dangling_piece, dangling_edge, bad_direction, flipped, ease,
    #                  ease_too_large, ease_not_as_declared, unmeasurable
    seam: Optional[int] = None
    piece: Optional[int] = None
    edge: Optional[int] = None
    ratio: Optional[float] = None
    declared: Optional[float] = None

    def message(self) -> str:
        """The user-facing sentence, naming what to do (validate.rs:76-124)."""
        if self.kind == "unsewn":
            return (f"edge {self.edge} is marked as a seam edge but is not sewn to anything — sew it, or set it "
                    f"to Cut or Fold if it is a finished edge")
        if self.kind == "dangling_piece":
            return (f"the seam references piece {self.piece}, which is not in the document — delete the seam or "
                    f"undo the piece deletion")
        if self.kind == "dangling_edge":
            return (f"the seam references edge {self.edge} of piece {self.piece}, which no longer exists — "
                    f"re-sew that side")
        if self.kind == "bad_direction":
            return (f"the seam's side on piece {self.piece} runs in two directions at once: its edges do not "
                    f"join end to start — flip the mis-ordered edge")
        if self.kind == "flipped":
            return ("the seam's two sides run in opposite directions, so it was sewn reversed to close it — check "
                    "which way round the pieces go if the drape looks twisted")
        if self.kind == "ease":
            return f"the two sides differ by {(self.ratio - 1.0) * 100:+.1f} % of their length; the seam absorbs it as ease"
        if self.kind == "ease_too_large":
            return (f"the two sides differ by {(self.ratio - 1.0) * 100:+.1f} % of their length, past the "
                    f"{(EASE_LIMIT - 1.0) * 100:.0f} % a plain seam absorbs — shorten the longer side, or split the "
                    f"seam so the extra length is gathered where you want it")
        if self.kind == "ease_not_as_declared":
            return (f"the seam is set up for {(self.declared - 1.0) * 100:+.1f} % ease but the pieces now differ by "
                    f"{(self.ratio - 1.0) * 100:+.1f} % — update the seam's ease or the piece geometry")
        return "the seam cannot be measured"


def check_chain(net: Network, side: SeamSide) -> bool:
    """The side's edges join end to start under their reversed flags (correspond.rs:162-187)."""
    prev = None
    for e, rev in side.edges:
        ed = net.edges[e]
        start, end = (ed.end, ed.start) if rev else (ed.start, ed.end)
        if prev is not None and prev != start:
            return False
        prev = end
    return True


def side_length_mm(net: Network, side: SeamSide) -> Optional[float]:
    """Arc length of the side's sewn span in pattern mm (correspond.rs:144-158); None for an
    empty side."""
    if not side.edges:
        return None
    total = sum(net.arc_length(e) for e, _ in side.edges)
    a, b = (min(max(float(s), 0.0), 1.0) for s in side.span)
    return total * (max(a, b) - min(a, b))


def _measure(doc: Document, sid: int, side: SeamSide, out: List[Diagnostic]) -> Optional[float]:
    net = doc.pieces.get(side.piece)
    if net is None:
        out.append(Diagnostic(ERROR, "dangling_piece", seam=sid, piece=side.piece))
        return None
    for e, _ in side.edges:
        if not (0 <= e < len(net.edges)) or net.edges[e] is None:
            out.append(Diagnostic(ERROR, "dangling_edge", seam=sid, piece=side.piece, edge=e))
            return None
    if not check_chain(net, side):
        out.append(Diagnostic(ERROR, "bad_direction", seam=sid, piece=side.piece))
        return None
    length = side_length_mm(net, side)
    if length is None:
        out.append(Diagnostic(ERROR, "unmeasurable", seam=sid, piece=side.piece))
    return length


def validate(doc: Document) -> List[Diagnostic]:
    """Every diagnostic the document earns, pieces then seams, both by id (validate.rs:163-244)."""
    out: List[Diagnostic] = []
    for pid in sorted(doc.pieces):
        for eid, ed in enumerate(doc.pieces[pid].edges):
            if ed is None or ed.semantic != SEAM:
                continue
            if not any(s.references_edge(pid, eid) for s in doc.seams.values()):
                out.append(Diagnostic(WARNING, "unsewn", piece=pid, edge=eid))
    for sid in sorted(doc.seams):
        seam = doc.seams[sid]
        la = _measure(doc, sid, seam.a, out)
        lb = _measure(doc, sid, seam.b, out)
        if la is None or lb is None:
            continue
        measured = lb / la
        too_large = max(measured, 1.0 / measured) > EASE_LIMIT
        out.append(Diagnostic(ERROR if too_large else INFO, "ease_too_large" if too_large else "ease", seam=sid,
                              ratio=measured))
        if abs(measured - seam.ease_ratio) > DECLARED_EASE_TOLERANCE:
            out.append(Diagnostic(WARNING, "ease_not_as_declared", seam=sid, ratio=measured,
                                  declared=seam.ease_ratio))
    return out


def is_sewable(diagnostics: List[Diagnostic]) -> bool:
    return not any(d.severity == ERROR for d in diagnostics)


def counts(diagnostics: List[Diagnostic]) -> Tuple[int, int, int]:
    """(errors, warnings, infos)."""
    return (sum(d.severity == ERROR for d in diagnostics), sum(d.severity == WARNING for d in diagnostics),
            sum(d.severity == INFO for d in diagnostics))
