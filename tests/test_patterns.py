"""Pattern panels to meshes and sewn garments (mguso.patterns): meshing invariants, seams
corresponded across panels of different resolution, and a sewn tube closing in the oracle's
step."""
import numpy as np
import pytest

import oracle_py as O
from mguso import patterns


def _cross2(u, v):
    return u[..., 0] * v[..., 1] - u[..., 1] * v[..., 0]


def _edge_lengths(m):
    t = m.tris
    e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
    return np.linalg.norm(m.points_mm[e[:, 0]] - m.points_mm[e[:, 1]], axis=1)


@pytest.mark.parametrize("clockwise", [False, True])
def test_a_rectangle_meshes_to_its_area_with_chains_along_its_edges(clockwise):
    outline = [(0, 0), (300, 0), (300, 500), (0, 500)]
    if clockwise:
        outline = outline[::-1]
    m = patterns.mesh_panel(outline, 25.0, seed=1)
    assert abs(m.area_mm2() - 300 * 500) < 1e-6 * 300 * 500
    p = m.points_mm[m.tris]
    assert (_cross2(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]) > 0).all()  # counter-clockwise
    assert 0.6 * 25 < _edge_lengths(m).mean() < 1.4 * 25
    poly = np.asarray(outline, float)
    for k, c in enumerate(m.chains):
        a, b = poly[k], poly[(k + 1) % 4]
        assert np.allclose(c.points_mm[0], a) and np.allclose(c.points_mm[-1], b)
        d = c.points_mm - a
        assert np.allclose(_cross2(d, b - a), 0, atol=1e-9)  # on the edge
        s = d @ (b - a)
        assert np.all(np.diff(s) > 0)  # in order
    assert m.chains[0].vertices[-1] == m.chains[1].vertices[0]  # corners shared


def test_a_concave_panel_keeps_its_notch():
    outline = [(0, 0), (200, 0), (200, 100), (100, 100), (100, 200), (0, 200)]
    m = patterns.mesh_panel(outline, 10.0, seed=2)
    assert abs(m.area_mm2() - (200 * 200 - 100 * 100)) < 1e-6 * 3e4
    cen = m.points_mm[m.tris].mean(1)
    assert not ((cen[:, 0] > 100) & (cen[:, 1] > 100)).any()


def test_degenerate_panels_are_refused():
    with pytest.raises(patterns.PatternError):
        patterns.mesh_panel([(0, 0), (1, 0), (2, 0)], 1.0)
    with pytest.raises(patterns.PatternError):
        patterns.mesh_panel([(0, 0), (1, 0), (1, 1)], 0.0)


def _tube(front_edge, back_edge):
    g = patterns.Garment()
    w, h = 300.0, 400.0
    front = patterns.mesh_panel([(0, 0), (w, 0), (w, h), (0, h)], front_edge, seed=3)
    back = patterns.mesh_panel([(0, 0), (w, 0), (w, h), (0, h)], back_edge, seed=4)
    f = g.add_panel(front, origin_m=(0.0, 0.0, 0.02))
    b = g.add_panel(back, origin_m=(0.3, 0.0, -0.02), x_axis=(-1.0, 0.0, 0.0))
    # side seams: front right (edge 1) with back left (edge 3), front left (3) with back right (1)
    g.sew(f, [(1, False)], b, [(3, False)])
    g.sew(f, [(3, False)], b, [(1, False)])
    return g, front, back


def test_seams_between_panels_of_different_resolution_pair_every_dense_vertex():
    g, front, back = _tube(20.0, 35.0)
    idx, w, info = g.stitches()
    n_front_side = len(front.chains[1].vertices)
    assert idx.shape[0] == 2 * n_front_side  # one stitch per vertex of the denser side, both seams
    assert all(abs(e - 1.0) < 1e-9 for e, _ in info)
    assert all(fl for _, fl in info)  # the back panel runs the other way: both seams flip
    pos = g.positions()
    src = pos[idx[:, 0]]
    tgt = pos[idx[:, 3]] * (1 - w[:, 4:5]) + pos[idx[:, 4]] * w[:, 4:5]
    assert np.allclose(np.linalg.norm(src - tgt, axis=1), 0.04, atol=1e-6)  # straight across the gap


def test_a_sewn_tube_closes_its_seams_in_the_step():
    g, _, _ = _tube(50.0, 70.0)
    sc = g.scene(gravity=(0.0, 0.0, 0.0), self_collision=0, bend_stiffness=0.0)
    idx, w = sc["stitch_idx"], sc["stitch_w"]

    def gap(x):
        t = x[idx[:, 3]] * (1 - w[:, 4:5]) + x[idx[:, 4]] * w[:, 4:5]
        return np.linalg.norm(x[idx[:, 0]] - t, axis=1).max()

    o = O.OracleSolver(sc)
    o.step(40, check_intersection=False)
    x = o.positions().astype(np.float64)
    assert np.all(np.isfinite(x))
    assert gap(x) < 0.2 * gap(sc["positions"].astype(np.float64))


def _curved_panel(size, bulge, target):
    """A square piece whose right side bulges out as a cubic, meshed by mguso.triangulate."""
    from mguso import triangulate as T

    n = T.Network()
    v = [n.add_vertex(x, y) for x, y in [(0, 0), (size, 0), (size, size), (0, size)]]
    e = [n.add_edge(v[0], v[1], T.CUT),
         n.add_edge(v[1], v[2], T.SEAM, c1=(size + bulge, size / 3), c2=(size + bulge, 2 * size / 3)),
         n.add_edge(v[2], v[3], T.CUT),
         n.add_edge(v[3], v[0], T.SEAM)]
    m = T.triangulate(n, (), T.Options().with_target_edge_mm(target))
    return patterns.panel_from_triangulation(m, e)


def test_triangulated_panels_with_a_curved_seam_sew_and_close():
    g = patterns.Garment()
    front, back = _curved_panel(300.0, 40.0, 40.0), _curved_panel(300.0, 40.0, 55.0)
    f = g.add_panel(front, origin_m=(0.0, 0.0, 0.02))
    b = g.add_panel(back, origin_m=(0.3, 0.0, -0.02), x_axis=(-1.0, 0.0, 0.0))
    g.sew(f, [(1, False)], b, [(1, False)])  # the two bulging sides face each other
    idx, w, info = g.stitches()
    assert idx.shape[0] == len(front.chains[1].vertices)  # the denser side sews every vertex
    assert abs(info[0][0] - 1.0) < 1e-3  # equal arc lengths: no ease
    sc = g.scene(gravity=(0.0, 0.0, 0.0), self_collision=0, bend_stiffness=0.0)

    def gap(x):
        t = x[idx[:, 3]] * (1 - w[:, 4:5]) + x[idx[:, 4]] * w[:, 4:5]
        return np.linalg.norm(x[idx[:, 0]] - t, axis=1).max()

    o = O.OracleSolver(sc)
    o.step(40, check_intersection=False)
    x = o.positions().astype(np.float64)
    assert np.all(np.isfinite(x))
    assert gap(x) < 0.2 * gap(sc["positions"].astype(np.float64))
