"""3-D arrangement of pattern pieces (mguso.arrange) against the reference arranger's tests
(ui/crates/nguo-sewing/src/arrange.rs:454-750), and an arranged two-panel tube closing its
seams in the oracle's step."""
import math

import numpy as np

import oracle_py as O
from mguso import arrange as A
from mguso import patterns
from mguso import triangulate as T


def extent(i, w, h, **kw):
    return A.PieceExtent(i, (0.0, 0.0, w, h), **kw)


def opts():
    return A.ArrangeOptions(A.Archetype.TUBE, (0.0, 0.0), 0.15, 0.02, 1.2)


def test_wrapping_a_panel_preserves_its_width_as_arc_length():  # arrange.rs:482-505
    p = A.arrange([extent(0, 500.0, 600.0)], opts()).placements[0]
    xs = np.linspace(0.0, 500.0, 201)
    q = p.apply(np.stack([xs, np.zeros_like(xs)], 1)).astype(np.float64)
    assert abs(np.linalg.norm(np.diff(q, axis=0), axis=1).sum() - 0.5) < 1e-4


def test_pattern_y_is_down_so_the_hem_ends_up_below_the_top_edge():  # arrange.rs:507-516
    p = A.arrange([extent(0, 500.0, 600.0)], opts()).placements[0]
    assert abs(p.apply([250.0, 0.0])[1] - 1.2) < 1e-6
    assert abs(p.apply([250.0, 600.0])[1] - 0.6) < 1e-6


def test_adjacent_panels_meet_at_their_shared_edge_within_the_slack():  # arrange.rs:518-543
    a = A.arrange([extent(0, 500.0, 600.0), extent(1, 500.0, 600.0)], opts())
    assert abs(a.radius_m - 0.17) < 1e-6 and a.slack_m > 0.0
    gap = float(np.linalg.norm(a.placements[0].apply([500.0, 0.0]).astype(np.float64)
                               - a.placements[1].apply([0.0, 0.0])))
    assert 0.0 < gap <= a.slack_m / 2.0 + 1e-6


def test_no_panel_starts_inside_the_body_cylinder():  # arrange.rs:545-563
    o = opts()
    a = A.arrange([extent(0, 400.0, 600.0), extent(1, 400.0, 600.0)], o)
    for p in a.placements:
        for x in (0.0, 100.0, 200.0, 300.0, 400.0):
            for y in (0.0, 300.0, 600.0):
                w = p.apply([x, y])
                assert math.hypot(w[0] - o.center_xz[0], w[2] - o.center_xz[1]) >= o.body_radius_m + o.gap_m - 1e-5


def test_a_garment_wider_than_the_body_sets_its_own_radius():  # arrange.rs:565-578
    a = A.arrange([extent(0, 1000.0, 600.0), extent(1, 1000.0, 600.0)], opts())
    assert abs(a.radius_m - 2.0 / (2 * math.pi)) < 1e-6
    assert abs(a.slack_m) < 1e-6


def test_an_authored_placement_overrides_the_preset():  # arrange.rs:580-590
    e = extent(0, 500.0, 600.0, manual=((1000.0, 2000.0, 3000.0), (0.0, 0.0, 0.0, 1.0)))
    assert A.arrange([e], opts()).placements[0].apply([0.0, 0.0]).tolist() == [1.0, 2.0, 3.0]


def test_a_quarter_turn_about_y_sends_pattern_x_to_minus_z():  # arrange.rs:592-605
    s = float(np.sin(np.float32(math.pi / 4)))
    e = extent(0, 1000.0, 100.0, manual=((0.0, 0.0, 0.0), (0.0, s, 0.0, s)))
    p = A.arrange([e], opts()).placements[0].apply([1000.0, 0.0])
    assert abs(p[0]) < 1e-6 and abs(p[2] + 1.0) < 1e-6


def test_seam_order_walks_the_seam_graph():  # arrange.rs:607-651
    assert A.seam_order([0, 1, 2], [(0, 2), (2, 1)]) == [0, 2, 1]


def test_a_flared_panel_is_sized_by_its_support_edge_and_not_its_hem():  # arrange.rs:653-690
    hem = A.arrange([extent(0, 700.0, 600.0), extent(1, 700.0, 600.0)], opts())
    assert abs(hem.radius_m - 1.4 / (2 * math.pi)) < 1e-6
    waist = A.arrange([extent(i, 700.0, 600.0, support_arc_mm=300.0) for i in range(2)], opts())
    assert abs(waist.radius_m - 0.17) < 1e-6 and abs(waist.circumference_m - 0.6) < 1e-6
    gap = float(np.linalg.norm(waist.placements[0].apply([300.0, 0.0]).astype(np.float64)
                               - waist.placements[1].apply([0.0, 0.0])))
    assert gap <= waist.slack_m / 2.0 + 1e-6


def test_seam_order_covers_every_piece_even_with_no_seams():  # arrange.rs:736-750
    assert A.seam_order([0, 1, 2], []) == [0, 1, 2]


def test_the_flat_archetype_stands_the_panels_up_side_by_side():  # nguo-sewing tests/end_to_end.rs:359-381
    o = A.ArrangeOptions(A.Archetype.FLAT, (0.0, 0.0), 0.15, 0.02, 1.2)
    a = A.arrange([extent(0, 300.0, 400.0), extent(1, 300.0, 400.0)], o)
    assert a.radius_m is None and abs(a.circumference_m - 0.6) < 1e-6
    left, right = a.placements[0].apply([300.0, 0.0]), a.placements[1].apply([0.0, 0.0])
    assert np.allclose(left, right, atol=1e-6)  # edge to edge in one plane
    assert np.allclose(a.placements[0].apply([0.0, 400.0])[[1, 2]], [0.8, 0.17], atol=1e-6)


def test_an_arranged_tube_closes_its_side_seams_in_the_step():
    def piece(target):
        n = T.Network()
        v = [n.add_vertex(x, y) for x, y in [(0, 0), (500, 0), (500, 300), (0, 300)]]
        e = [n.add_edge(v[i], v[(i + 1) % 4], T.SEAM) for i in range(4)]
        return patterns.panel_from_triangulation(T.triangulate(n, (), T.Options().with_target_edge_mm(target)), e)

    front, back = piece(60.0), piece(80.0)
    a = A.arrange([extent(0, 500.0, 300.0), extent(1, 500.0, 300.0)], opts())
    g = patterns.Garment()
    f = g.add_arranged_panel(front, a.placements[0])
    b = g.add_arranged_panel(back, a.placements[1])
    g.sew(f, [(1, False)], b, [(3, False)])  # front right to back left
    g.sew(b, [(1, False)], f, [(3, False)])  # back right to front left, round the body
    sc = g.scene(gravity=(0.0, 0.0, 0.0), self_collision=0, bend_stiffness=0.0)
    p = sc["positions"]
    t = sc["tris"].astype(np.int64)
    # re-wound: every face normal points away from the cylinder axis
    nrm = np.cross(p[t[:, 1]] - p[t[:, 0]], p[t[:, 2]] - p[t[:, 0]])
    out = p[t].mean(1) * np.array([1, 0, 1])
    assert ((nrm * out).sum(1) > 0).all()
    idx, w = sc["stitch_idx"], sc["stitch_w"]

    def gap(x):
        tt = x[idx[:, 3]] * (1 - w[:, 4:5]) + x[idx[:, 4]] * w[:, 4:5]
        return np.linalg.norm(x[idx[:, 0]] - tt, axis=1).max()

    assert gap(p.astype(np.float64)) <= a.slack_m / 2.0 + 1e-4  # seams start open by the slack
    o = O.OracleSolver(sc)
    o.step(30, check_intersection=False)
    x = o.positions().astype(np.float64)
    assert np.all(np.isfinite(x)) and gap(x) < 0.3 * gap(p.astype(np.float64))
