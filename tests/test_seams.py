"""Seam validation of a garment document (mguso.seams) against the reference validator's
tests (ui/crates/nguo-sewing/src/validate.rs:296-565)."""
import time

from mguso import seams as S
from mguso import triangulate as T


def doc_with(h_b):
    """Two 100 mm wide rectangles of Seam edges, 200 and h_b tall (validate.rs:302-327)."""
    doc, pieces, edges = S.Document(), [], []
    for h in (200.0, h_b):
        n = T.Network()
        v = [n.add_vertex(x, y) for x, y in [(0, 0), (100, 0), (100, h), (0, h)]]
        e = [n.add_edge(v[k], v[(k + 1) % 4], T.SEAM) for k in range(4)]
        pieces.append(doc.add_piece(n))
        edges.append(e)
    return doc, pieces, edges


def side_seam(p, e, **kw):
    return S.Seam(S.SeamSide(p[0], [(e[0][1], False)]), S.SeamSide(p[1], [(e[1][3], True)]), **kw)


def test_every_unsewn_seam_edge_is_flagged_and_sewing_one_clears_it():  # validate.rs:339-371
    doc, p, e = doc_with(200.0)
    before = S.validate(doc)
    assert sum(d.kind == "unsewn" for d in before) == 8 and S.is_sewable(before)
    doc.add_seam(side_seam(p, e))
    after = S.validate(doc)
    assert sum(d.kind == "unsewn" for d in after) == 6
    assert any(d.kind == "ease" for d in after) and S.is_sewable(after)


def test_equal_sides_report_zero_ease_and_no_warning():  # validate.rs:373-397
    doc, p, e = doc_with(200.0)
    s = doc.add_seam(side_seam(p, e))
    d = S.validate(doc)
    ease = next(x for x in d if x.seam == s and x.kind == "ease")
    assert ease.severity == S.INFO and abs(ease.ratio - 1.0) < 1e-9
    assert not any(x.kind == "ease_not_as_declared" for x in d)


def test_a_length_mismatch_is_ease_below_the_limit_and_an_error_above_it():  # validate.rs:399-448
    doc, p, e = doc_with(220.0)
    doc.add_seam(side_seam(p, e))
    d = S.validate(doc)
    assert abs(next(x.ratio for x in d if x.kind == "ease") - 1.1) < 1e-9 and S.is_sewable(d)
    doc, p, e = doc_with(400.0)
    doc.add_seam(side_seam(p, e))
    d = S.validate(doc)
    err = next(x for x in d if x.kind == "ease_too_large")
    assert err.severity == S.ERROR and not S.is_sewable(d)
    assert "gathered" in err.message()


def test_the_ease_limit_applies_in_both_directions():  # validate.rs:450-461
    doc, p, e = doc_with(100.0)
    doc.add_seam(side_seam(p, e))
    assert not S.is_sewable(S.validate(doc))


def test_a_side_whose_edges_do_not_join_is_a_direction_error():  # validate.rs:463-481
    doc, p, e = doc_with(200.0)
    doc.add_seam(S.Seam(S.SeamSide(p[0], [(e[0][0], False), (e[0][1], True)]), S.SeamSide(p[1], [(e[1][3], True)])))
    d = S.validate(doc)
    bad = next(x for x in d if x.kind == "bad_direction")
    assert bad.severity == S.ERROR and not S.is_sewable(d)


def test_a_seam_referencing_a_deleted_piece_is_an_error_not_a_panic():  # validate.rs:483-528
    doc, p, e = doc_with(200.0)
    doc.add_seam(side_seam(p, e))
    del doc.pieces[p[1]]  # as a document loaded from a file without integrity checks
    d = S.validate(doc)
    assert any(x.kind == "dangling_piece" for x in d) and not S.is_sewable(d)


def test_a_seam_referencing_a_removed_edge_is_an_error():
    doc, p, e = doc_with(200.0)
    doc.add_seam(side_seam(p, e))
    doc.pieces[p[1]].remove_edge(e[1][3])
    d = S.validate(doc)
    assert any(x.kind == "dangling_edge" and x.edge == e[1][3] for x in d) and not S.is_sewable(d)


def test_a_declared_ease_that_no_longer_matches_the_geometry_is_warned_about():  # validate.rs:530-544
    doc, p, e = doc_with(200.0)
    doc.add_seam(side_seam(p, e, ease_ratio=1.05))
    assert any(x.kind == "ease_not_as_declared" for x in S.validate(doc))


def test_validation_is_cheap_enough_to_run_on_every_revision():  # validate.rs:546-565
    doc, p, e = doc_with(200.0)
    for a, b in zip(e[0], e[1]):
        doc.add_seam(S.Seam(S.SeamSide(p[0], [(a, False)]), S.SeamSide(p[1], [(b, True)])))
    t, total = time.perf_counter(), 0
    for _ in range(200):
        total += len(S.validate(doc))
    per_call_us = (time.perf_counter() - t) / 200 * 1e6
    assert total > 0
    assert per_call_us < 1000.0, per_call_us  # the reference's per-keystroke bound
    assert S.counts(S.validate(doc))[1] == 0  # every seam edge is sewn
