"""A garment document sewn into one scene (mguso.garment) against the reference's sewing
pipeline tests (ui/crates/nguo-sewing/tests/end_to_end.rs, src/sample.rs:314-378), and the
sewn sample draped by the oracle's step with its seams holding."""
import numpy as np

import oracle_py as O
from mguso import arrange as A
from mguso import garment as G
from mguso import seams as S


def garment(**kw):
    return G.build(G.sample_bodice_block(), G.SewOptions(**kw) if kw else G.SewOptions())


def tri_areas(g):
    p = g.positions.astype(np.float64)
    t = g.tris.astype(np.int64)
    return 0.5 * np.linalg.norm(np.cross(p[t[:, 1]] - p[t[:, 0]], p[t[:, 2]] - p[t[:, 0]]), axis=1)


def test_the_sample_is_two_sewn_panels_with_nothing_to_report():  # sample.rs:314-333
    doc = G.sample_bodice_block()
    assert len(doc.pieces) == 2 and len(doc.seams) == 2
    d = S.validate(doc)
    assert S.is_sewable(d) and all(x.severity == S.INFO for x in d)


def test_the_sample_garment_is_a_valid_simulation_mesh():  # end_to_end.rs:22-77
    g = garment()
    assert g.check() is None
    assert len(g.pieces) == 2 and len(g.seams) == 2
    assert g.vertex_count() > 200 and g.triangle_count() > 300
    assert len(g.uvs) == g.vertex_count()
    for pm in g.pieces:
        assert pm.mesh.min_angle_deg() > 5.0
    a = tri_areas(g)
    assert a.min() > 1e-9
    flat = 2.0 * G.PANEL_W_MM * G.PANEL_H_MM * 1e-6
    assert abs(a.sum() / flat - 1.0) < 0.01  # the wrap is isometric


def test_every_seam_is_resolved_paired_and_within_the_arrangers_slack():  # end_to_end.rs:78-132
    g = garment()
    slack = g.arrangement.slack_m
    for s in g.seams:
        assert s.stitches >= 10 and not s.flipped and abs(s.ease - 1.0) < 1e-6
    assert len(g.stitch_idx) == sum(s.stitches for s in g.seams)
    assert g.max_seam_gap_m() <= max(slack, 1e-3) + 1e-3
    offsets = [pm.vertex_offset for pm in g.pieces]

    def piece_of(v):
        return max(i for i, o in enumerate(offsets) if v >= o)

    for row in g.stitch_idx:
        assert piece_of(row[0]) != piece_of(row[3])


def test_no_panel_starts_inside_the_body_cylinder():  # end_to_end.rs:134-160
    o = A.ArrangeOptions(body_radius_m=0.16, center_xz=(0.0, 0.0))
    g = garment(arrange=o)
    closest = float(np.hypot(g.positions[:, 0], g.positions[:, 2]).min())
    assert closest >= o.body_radius_m + o.gap_m - 1e-6


def test_the_same_document_produces_a_bit_identical_garment():  # end_to_end.rs:162-185
    a, b = garment(), garment()
    assert np.array_equal(a.positions, b.positions) and np.array_equal(a.tris, b.tris)
    assert np.array_equal(a.uvs, b.uvs)
    assert np.array_equal(a.stitch_idx, b.stitch_idx) and np.array_equal(a.stitch_w, b.stitch_w)


def test_the_sample_sews_and_arranges_into_a_closed_tube():  # sample.rs:336-378
    g = garment()
    assert len(g.seams) == 2 and all(s.stitches > 4 and not s.flipped for s in g.seams)
    ext = g.positions.max(0) - g.positions.min(0)
    assert ext[0] > 0.15 and ext[2] > 0.15
    assert abs(ext[1] - G.PANEL_H_MM * 1e-3) < 1e-3
    assert g.max_seam_gap_m() < max(g.arrangement.slack_m, 1e-3) + 1e-3


def test_an_unsewn_document_still_builds_and_says_it_has_no_seams():  # end_to_end.rs:339-356
    doc = G.sample_bodice_block()
    doc.seams.clear()
    g = G.build(doc)
    assert not len(g.stitch_idx) and not g.seams
    assert g.check() is None and g.max_seam_gap_m() == 0.0


def test_the_flat_archetype_stands_the_panels_up_side_by_side():  # end_to_end.rs:358-381
    g = garment(arrange=A.ArrangeOptions(archetype=A.Archetype.FLAT))
    assert g.arrangement.radius_m is None and g.arrangement.slack_m == 0.0
    lo, hi = g.positions.min(0), g.positions.max(0)
    assert abs(hi[2] - lo[2]) < 1e-6 and lo[2] > 0.0
    assert abs(hi[0] - lo[0] - 2.0 * G.PANEL_W_MM * 1e-3) < 1e-3


def test_an_unsewable_document_is_refused_with_its_first_error():
    doc = G.sample_bodice_block()
    doc.seams[0].a.edges = [(0, False), (1, True)]  # a side that does not join end to start
    try:
        G.build(doc)
    except G.NotSewable as e:
        assert "flip the mis-ordered edge" in str(e)
    else:
        raise AssertionError("built an unsewable document")


def test_the_sewn_sample_holds_its_seams_in_the_step():
    g = garment(triangulate=G.T.Options(target_edge_mm=80.0))
    sc = g.scene(gravity=(0.0, 0.0, 0.0), self_collision=0, bend_stiffness=0.0)
    idx, w = sc["stitch_idx"], sc["stitch_w"]

    def gap(x):
        a = (x[idx[:, :3]] * w[:, :3, None]).sum(1)
        b = (x[idx[:, 3:]] * w[:, 3:, None]).sum(1)
        return np.linalg.norm(a - b, axis=1).max()

    o = O.OracleSolver(sc)
    o.step(10, check_intersection=False)
    x = o.positions()
    assert np.all(np.isfinite(x)) and gap(x) < 5e-3  # the closed tube stays closed


def test_the_sample_hangs_from_the_girth_it_was_sized_for():  # sample.rs:379-395
    doc = G.sample_bodice_block()
    h = G.hang(doc)
    assert h.landmark == G.SUPPORT_LANDMARK and abs(h.drop_mm - G.PANEL_H_MM) < 1e-9
    arcs = [G.support_arc_mm(doc, p) for p in sorted(doc.pieces)]
    assert arcs == [G.PANEL_W_MM, G.PANEL_W_MM]
    assert 0.025 < sum(arcs) / 1087.3 - 1.0 < 0.035  # 3 % ease over the hip girth it was sized for


def test_hang_reads_the_support_annotation_and_the_garment_drop():  # arrange.rs:694-734
    assert G.hang(S.Document()) == G.Hang()
    n = G.T.Network()
    v = [n.add_vertex(x, y) for x, y in [(0, 0), (400, 0), (400, 700), (0, 700)]]
    e = [n.add_edge(v[k], v[(k + 1) % 4], G.T.CUT) for k in range(4)]
    doc = S.Document()
    pid = doc.add_piece(n, support_edge=e[0], landmark="waist")
    assert G.support_arc_mm(doc, pid) == 400.0
    h = G.hang(doc)
    assert h.landmark == "waist" and abs(h.drop_mm - 700.0) < 1e-9
