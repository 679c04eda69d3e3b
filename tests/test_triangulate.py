"""Pattern piece -> simulation mesh (mguso.triangulate) against the reference triangulator's
own tests (ui/crates/nguo-triangulate/src/lib.rs:984-1572): validity, units, UVs, internal
lines, notches, welding, grain markers, curves, refinement bounds, holes, darts, typed errors,
the validator and determinism."""
import math

import numpy as np
import pytest

from mguso import triangulate as T


def square(size):
    n = T.Network()
    v = [n.add_vertex(x, y) for x, y in [(0, 0), (size, 0), (size, size), (0, size)]]
    e = [n.add_edge(v[i], v[(i + 1) % 4], T.CUT) for i in range(4)]
    return n, v, e


def mesh_edges(m):
    t = m.indices.astype(np.int64)
    e = np.sort(np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]]), 1)
    return {tuple(r) for r in e.tolist()}


def test_a_square_triangulates_to_a_valid_mesh():  # lib.rs:984-996
    m = T.triangulate(square(100.0)[0])
    assert m.check() is None
    assert abs(m.area_mm2() - 10_000.0) < 1e-6
    assert m.refinement_complete and m.degenerate_dropped == 0


def test_the_square_has_the_euler_characteristic_of_a_disc():  # lib.rs:998-1009
    m = T.triangulate(square(100.0)[0])
    assert m.vertex_count() - len(mesh_edges(m)) + m.triangle_count() == 1


def test_millimetres_become_metres_exactly_once():  # lib.rs:1011-1021
    m = T.triangulate(square(1000.0)[0])
    assert m.check() is None
    assert m.pattern_bounds() == (0.0, 0.0, 1000.0, 1000.0)
    assert (m.positions[:, 0].max(), m.positions[:, 1].max()) == (1.0, 1.0)


def test_pattern_coordinates_are_the_uvs():  # lib.rs:1023-1033
    m = T.triangulate(square(250.0)[0])
    uv = m.uvs()
    assert len(uv) == m.vertex_count()
    assert np.abs(uv - m.pattern_mm / 250.0).max() < 1e-6


def test_an_internal_line_survives_as_mesh_edges():  # lib.rs:1035-1069
    n, _, e = square(100.0)
    right = n.split_edge(e[1], 0.5)
    left = n.split_edge(e[3], 0.5)
    line = n.add_edge(left, right, T.INTERNAL)
    m = T.triangulate(n)
    assert m.check() is None
    c = m.chain(line)
    assert c.semantic == T.INTERNAL and len(c.points) == 11
    edges = mesh_edges(m)
    for (x, _), (y, _) in zip(c.points, c.points[1:]):
        assert (min(x, y), max(x, y)) in edges
    assert abs(m.area_mm2() - 10_000.0) < 1e-6


def test_a_notch_becomes_a_mesh_vertex_on_its_edge():  # lib.rs:1071-1085
    n, _, e = square(100.0)
    m = T.triangulate(n, [(e[0], 0.37)])
    assert m.check() is None
    idx, t = next((i, t) for i, t in m.chain(e[0]).points if abs(t - 0.37) < 1e-12)
    assert t == 0.37
    assert m.pattern_mm[idx].tolist() == [37.0, 0.0]
    assert m.sources[idx] == ("edge", e[0])


def test_a_notch_outside_the_unit_interval_is_an_error():  # lib.rs:1087-1094
    n, _, e = square(100.0)
    with pytest.raises(T.NotchOutOfRange) as x:
        T.triangulate(n, [(e[0], 1.5)])
    assert (x.value.edge, x.value.t) == (e[0], 1.5)


def test_an_open_outline_is_reported_not_panicked():  # lib.rs:1096-1104
    n, _, e = square(100.0)
    n.remove_edge(e[2])
    with pytest.raises(T.NoRegion):
        T.triangulate(n)


def test_near_duplicate_input_is_welded_not_fatal():  # lib.rs:1106-1118
    n, _, _ = square(100.0)
    ghost = n.add_vertex(1e-7, 1e-7)
    apex = n.add_vertex(50.0, 50.0)
    n.add_edge(ghost, apex, T.INTERNAL)
    m = T.triangulate(n)
    assert m.check() is None
    assert abs(m.area_mm2() - 10_000.0) < 1e-3


def test_a_grain_marker_contributes_nothing():  # lib.rs:1120-1135
    n, _, _ = square(100.0)
    a, b = n.add_vertex(-500.0, -500.0), n.add_vertex(-400.0, -500.0)
    g = n.add_edge(a, b, T.GRAIN)
    m = T.triangulate(n)
    assert m.check() is None and m.chain(g) is None
    assert abs(m.area_mm2() - 10_000.0) < 1e-6
    assert m.pattern_bounds()[0] >= 0.0


def test_a_curved_edge_is_flattened_within_tolerance():  # lib.rs:1137-1174
    n = T.Network()
    v = [n.add_vertex(x, y) for x, y in [(0, 0), (100, 0), (100, 100), (0, 100)]]
    curved = n.add_edge(v[0], v[1], T.CUT, c1=(30.0, -40.0), c2=(70.0, -40.0))
    for i in range(1, 4):
        n.add_edge(v[i], v[(i + 1) % 4], T.CUT)
    m = T.triangulate(n)
    assert m.check() is None
    c = m.chain(curved)
    dense = n.eval(curved, np.linspace(0, 1, 20001))
    for (i, _), (j, _) in zip(c.points, c.points[1:]):
        mid = 0.5 * (m.pattern_mm[i] + m.pattern_mm[j])
        assert np.linalg.norm(dense - mid, axis=1).min() < 0.6
    assert m.pattern_bounds()[1] < -25.0
    # every chain point lies on the curve at its own parameter
    for i, t in c.points:
        assert np.linalg.norm(m.pattern_mm[i] - n.eval(curved, t)) < 2e-3


def test_refinement_bounds_the_triangle_area():  # lib.rs:1176-1209
    n, _, _ = square(200.0)
    opts = T.Options().with_target_edge_mm(50.0)
    cap = math.sqrt(3.0) / 4.0 * 50.0 * 50.0
    raw = T.triangulate(n, (), opts.without_refinement())
    refined = T.triangulate(n, (), opts)
    assert raw.max_area_mm2() > cap * 4.0
    assert refined.max_area_mm2() <= cap * 1.5
    assert refined.triangle_count() > raw.triangle_count() * 2
    assert abs(refined.area_mm2() - raw.area_mm2()) < 1e-6


def test_refinement_holds_the_angle_bound_away_from_acute_input_corners():  # lib.rs:1211-1224
    n, _, _ = square(200.0)
    refined = T.triangulate(n, (), T.Options().with_target_edge_mm(20.0))
    assert refined.min_angle_deg() > 25.0


def test_a_panel_thinner_than_the_target_edge_is_still_valid_just_skinny():  # lib.rs:1226-1264
    n = T.Network()
    v = [n.add_vertex(x, y) for x, y in [(0, 0), (400, 0), (400, 12), (0, 12)]]
    for i in range(4):
        n.add_edge(v[i], v[(i + 1) % 4], T.CUT)
    coarse = T.triangulate(n, (), T.Options().with_target_edge_mm(200.0))
    assert coarse.check() is None and abs(coarse.area_mm2() - 4_800.0) < 1e-6
    fine = T.triangulate(n, (), T.Options().with_target_edge_mm(6.0))
    assert fine.check() is None and abs(fine.area_mm2() - 4_800.0) < 1e-6
    assert fine.min_angle_deg() > coarse.min_angle_deg() + 10.0


def test_a_hole_is_excluded():  # lib.rs:1266-1285
    n, _, _ = square(200.0)
    h = [n.add_vertex(x, y) for x, y in [(80, 80), (120, 80), (120, 120), (80, 120)]]
    for i in range(4):
        n.add_edge(h[i], h[(i + 1) % 4], T.CUT)
    m = T.triangulate(n)
    assert m.check() is None
    assert abs(m.area_mm2() - (40_000.0 - 1_600.0)) < 1e-6


def test_a_dart_removes_its_wedge():  # lib.rs:1287-1349
    n = T.Network()
    c = [n.add_vertex(x, y) for x, y in [(0, 0), (80, 0), (120, 0), (200, 0), (200, 200), (0, 200)]]
    for i in range(6):
        n.add_edge(c[i], c[(i + 1) % 6], T.CUT)
    apex = n.add_vertex(100.0, 120.0)
    leg_a = n.add_edge(c[1], apex, T.DART_LEG)
    leg_b = n.add_edge(apex, c[2], T.DART_LEG)
    m = T.triangulate(n)
    assert m.check() is None
    assert abs(m.area_mm2() - (40_000.0 - 2_400.0)) < 1e-6
    ca, cb = m.chain(leg_a), m.chain(leg_b)
    assert ca.semantic == T.DART_LEG
    assert ca.points[-1][0] == cb.points[0][0]
    assert m.sources[ca.points[-1][0]] == ("vertex", apex)
    cen = m.pattern_mm[m.indices.astype(np.int64)].mean(1)
    in_wedge = (cen[:, 1] < 120.0) & (np.abs(cen[:, 0] - 100.0) < 20.0 * (1.0 - cen[:, 1] / 120.0))
    assert not in_wedge.any()


def test_a_closed_dart_removes_its_lens():  # lib.rs:1351-1372
    n, _, _ = square(200.0)
    lo, hi = n.add_vertex(100, 60), n.add_vertex(100, 140)
    left, right = n.add_vertex(85, 100), n.add_vertex(115, 100)
    for a, b in [(lo, left), (left, hi), (hi, right), (right, lo)]:
        n.add_edge(a, b, T.DART_LEG)
    m = T.triangulate(n)
    assert m.check() is None
    assert abs(m.area_mm2() - (40_000.0 - 1_200.0)) < 1e-6


def test_crossing_pattern_edges_are_refused_with_a_fixable_error():  # lib.rs:1374-1390
    n, _, _ = square(100.0)
    a, b = n.add_vertex(20, 20), n.add_vertex(80, 80)
    c, d = n.add_vertex(20, 80), n.add_vertex(80, 20)
    n.add_edge(a, b, T.INTERNAL)
    n.add_edge(c, d, T.INTERNAL)
    with pytest.raises(T.CrossingConstraint):
        T.triangulate(n)


def test_bad_options_are_rejected_before_any_work():  # lib.rs:1392-1421
    n, _, _ = square(100.0)
    for bad in (T.Options(target_edge_mm=0.0), T.Options(weld_mm=1e6), T.Options(curve_tolerance_mm=math.nan),
                T.Options(min_angle_deg=90.0)):
        with pytest.raises(T.BadOption):
            T.triangulate(n, (), bad)


def test_resolution_is_one_knob():  # lib.rs:1423-1446
    n, _, _ = square(200.0)
    coarse = T.triangulate(n, (), T.Options().with_target_edge_mm(50.0))
    fine = T.triangulate(n, (), T.Options().with_target_edge_mm(10.0))
    assert fine.triangle_count() > coarse.triangle_count() * 10
    assert abs(fine.area_mm2() - coarse.area_mm2()) < 1e-6


def test_a_collinear_network_is_a_typed_error():  # lib.rs:1448-1465
    n = T.Network()
    v = [n.add_vertex(x, 0.0) for x in (0.0, 50.0, 100.0)]
    for i in range(2):
        n.add_edge(v[i], v[i + 1], T.CUT)
    with pytest.raises(T.NoRegion):
        T.triangulate(n)


def test_an_empty_network_is_a_typed_error():  # lib.rs:1467-1477
    with pytest.raises(T.Degenerate) as x:
        T.triangulate(T.Network())
    assert (x.value.distinct, x.value.weld_mm) == (0, 1e-3)


def test_outline_vertices_are_the_boundary_ring():  # lib.rs:1479-1493
    m = T.triangulate(square(100.0)[0])
    ring = m.outline_vertices()
    assert len(ring) == 40
    for i in ring:
        x, y = m.pattern_mm[i]
        assert x == 0.0 or y == 0.0 or x == 100.0 or y == 100.0


def test_an_absurd_resolution_is_refused_before_any_work():  # lib.rs:1495-1514
    n, _, _ = square(100.0)
    with pytest.raises(T.TooDense) as x:
        T.triangulate(n, (), T.Options(weld_mm=1e-9, target_edge_mm=1e-5))
    assert "millimetres" in str(x.value)


def test_the_mesh_validator_has_teeth():  # lib.rs:1516-1564
    import copy

    good = T.triangulate(square(100.0)[0])
    assert good.check() is None
    flipped = copy.deepcopy(good)
    flipped.indices[0, [0, 1]] = flipped.indices[0, [1, 0]]
    assert "flipped or degenerate" in flipped.check()
    collapsed = copy.deepcopy(good)
    collapsed.indices[0, 1] = collapsed.indices[0, 0]
    assert "repeats a vertex" in collapsed.check()
    twice = copy.deepcopy(good)
    twice.positions[:, :2] *= np.float32(1e-3)
    assert "second unit conversion" in twice.check()
    lifted = copy.deepcopy(good)
    lifted.positions[0, 2] = 0.1
    assert "pattern plane" in lifted.check()
    unsorted = copy.deepcopy(good)
    unsorted.chains[0], unsorted.chains[1] = unsorted.chains[1], unsorted.chains[0]
    assert "not sorted" in unsorted.check()
    backwards = copy.deepcopy(good)
    backwards.chains[0].points.reverse()
    assert "ascending in t" in backwards.check()


def test_the_same_input_triangulates_identically():  # lib.rs:1566-1572
    n, _, e = square(180.0)
    a, b = T.triangulate(n, [(e[0], 0.25)]), T.triangulate(n, [(e[0], 0.25)])
    assert np.array_equal(a.positions, b.positions) and np.array_equal(a.indices, b.indices)
    assert a.sources == b.sources and a.chains == b.chains


def area_tolerance(poly, weld_mm=1e-3):
    """Snap-rounding moves each boundary point by at most weld_mm (tests/mesh.rs:376-385)."""
    return weld_mm * float(np.linalg.norm(np.roll(poly, -1, 0) - poly, axis=1).sum()) + 1e-9


def star_polygon(seed, k):
    rng = np.random.default_rng(seed)
    ang = np.sort(rng.uniform(0, 2 * np.pi, k))
    r = rng.uniform(40.0, 120.0, k)
    return np.stack([r * np.cos(ang), r * np.sin(ang)], 1)


@pytest.mark.parametrize("seed", range(6))
def test_no_flipped_or_degenerate_triangles_on_star_polygons(seed):  # tests/mesh.rs:398-420
    poly = star_polygon(seed, 5 + seed)
    n = T.Network()
    v = [n.add_vertex(*p) for p in poly]
    for i in range(len(v)):
        n.add_edge(v[i], v[(i + 1) % len(v)], T.CUT)
    m = T.triangulate(n, (), T.Options().with_target_edge_mm(15.0))
    assert m.check() is None
    x, y = poly[:, 0], poly[:, 1]
    area = 0.5 * abs(np.dot(x, np.roll(y, -1)) - np.dot(y, np.roll(x, -1)))
    assert abs(m.area_mm2() - area) < area_tolerance(poly)
    assert m.degenerate_dropped == 0


@pytest.mark.parametrize("seed", range(4))
def test_notches_add_vertices_without_changing_the_area(seed):  # tests/mesh.rs:503-522
    poly = star_polygon(10 + seed, 6)
    n = T.Network()
    v = [n.add_vertex(*p) for p in poly]
    e = [n.add_edge(v[i], v[(i + 1) % 6], T.CUT) for i in range(6)]
    plain = T.triangulate(n, (), T.Options().with_target_edge_mm(20.0))
    ts = np.random.default_rng(seed).uniform(0.05, 0.95, 3)
    notched = T.triangulate(n, [(e[k], float(t)) for k, t in enumerate(ts)], T.Options().with_target_edge_mm(20.0))
    assert notched.check() is None
    assert abs(notched.area_mm2() - plain.area_mm2()) < area_tolerance(poly)
    for k, t in enumerate(ts):
        assert any(tt == float(t) for _, tt in notched.chain(e[k]).points)


def bodice():
    """The reference's half bodice front (tests/mesh.rs:33-111): straight waist in three pieces
    around a dart, cubic side seam, armhole and neckline, a centre-front fold, a grain marker
    and four notches."""
    n = T.Network()
    cf_waist, dart_l, dart_r, side_waist = (n.add_vertex(x, 0.0) for x in (0.0, 45.0, 65.0, 110.0))
    underarm, shoulder_out = n.add_vertex(118.0, 180.0), n.add_vertex(78.0, 330.0)
    shoulder_in, cf_neck = n.add_vertex(28.0, 356.0), n.add_vertex(0.0, 300.0)
    waist_a = n.add_edge(cf_waist, dart_l, T.SEAM)
    n.add_edge(dart_l, dart_r, T.SEAM)
    waist_c = n.add_edge(dart_r, side_waist, T.SEAM)
    side = n.add_edge(side_waist, underarm, T.SEAM, c1=(106.0, 60.0), c2=(108.0, 120.0))
    armhole = n.add_edge(underarm, shoulder_out, T.SEAM, c1=(128.0, 250.0), c2=(108.0, 320.0))
    n.add_edge(shoulder_out, shoulder_in, T.SEAM)
    n.add_edge(shoulder_in, cf_neck, T.SEAM, c1=(14.0, 348.0), c2=(0.0, 330.0))
    n.add_edge(cf_neck, cf_waist, T.FOLD)
    apex = n.add_vertex(55.0, 150.0)
    n.add_edge(dart_l, apex, T.DART_LEG)
    n.add_edge(apex, dart_r, T.DART_LEG)
    g0, g1 = n.add_vertex(60.0, 40.0), n.add_vertex(60.0, 260.0)
    n.add_edge(g0, g1, T.GRAIN)
    return n, [(armhole, 0.5), (side, 0.5), (waist_a, 0.5), (waist_c, 0.25)]


def test_the_bodice_triangulates_and_maps_back_to_the_pattern():  # tests/mesh.rs:213-280
    import copy

    net, notches = bodice()
    m = T.triangulate(net, notches)
    assert m.check() is None
    for e, t in notches:
        i = next(i for i, ct in m.chain(e).points if abs(ct - t) < 1e-12)
        assert np.linalg.norm(m.pattern_mm[i] - net.eval(e, t)) < 1e-3
    no_dart = copy.deepcopy(net)
    for ed in no_dart.edges:
        if ed is not None and ed.semantic == T.DART_LEG:
            ed.semantic = T.INTERNAL
    whole = T.triangulate(no_dart, notches)
    assert abs((whole.area_mm2() - m.area_mm2()) - 1_500.0) < 1e-3  # the 20 x 150 / 2 wedge
    assert all(c.semantic != T.GRAIN for c in m.chains)
    assert len(m.outline_vertices()) > 80
    assert m.angle_quantile_deg(0.01) > 20.0
    assert (m.min_angles_deg() < 15.0).sum() < 0.02 * m.triangle_count()


def golden_panel():
    """tests/mesh.rs:144-201: a 200 x 300 panel with a waist dart, a pocket line T-junction to
    T-junction, a triangular cut-out and three notches."""
    n = T.Network()
    o = [n.add_vertex(x, y) for x, y in [(0, 0), (70, 0), (110, 0), (200, 0), (200, 300), (0, 300)]]
    e = [n.add_edge(o[i], o[(i + 1) % 6], T.SEAM) for i in range(6)]
    apex = n.add_vertex(90.0, 160.0)
    n.add_edge(o[1], apex, T.DART_LEG)
    n.add_edge(apex, o[2], T.DART_LEG)
    n.add_edge(n.add_vertex(40.0, 220.0), n.add_vertex(160.0, 220.0), T.INTERNAL)
    h = [n.add_vertex(x, y) for x, y in [(150, 60), (180, 60), (180, 100)]]
    for i in range(3):
        n.add_edge(h[i], h[(i + 1) % 3], T.CUT)
    return n, [(e[0], 0.5), (e[3], 0.25), (e[3], 0.75)]


def test_the_panel_mesh_has_the_golden_panels_shape():  # tests/mesh.rs:286-307
    net, notches = golden_panel()
    m = T.triangulate(net, notches, T.Options().with_target_edge_mm(40.0))
    assert m.check() is None
    assert 80 < m.triangle_count() < 400
    assert abs(m.area_mm2() - (60_000.0 - 3_200.0 - 600.0)) < 1e-6


def ref_star(seed):
    """tests/mesh.rs:350-368: 3..39 vertices at jittered even angles, radii 5..400 mm."""
    rng = np.random.default_rng(seed)
    k = int(rng.integers(3, 40))
    step = 2 * np.pi / k
    ang = (np.arange(k) + rng.uniform(-0.2, 0.2, k)) * step
    r = rng.uniform(5.0, 400.0, k)
    return np.stack([r * np.cos(ang), r * np.sin(ang)], 1)


def _star_net(poly):
    n = T.Network()
    v = [n.add_vertex(*p) for p in poly]
    for i in range(len(v)):
        n.add_edge(v[i], v[(i + 1) % len(v)], T.CUT)
    return n


@pytest.mark.parametrize("seed", range(8))
def test_duplicate_vertices_produce_an_identical_mesh(seed):  # tests/mesh.rs:438-466
    poly = ref_star(100 + seed)

    def build(duplicate):
        net = _star_net(poly)
        hub = net.add_vertex(0.0, 0.0)
        for c in range(len(poly)):
            start = net.add_vertex(*net.vertices[c]) if duplicate else c
            net.add_edge(start, hub, T.INTERNAL)
        return net

    opts = T.Options().with_target_edge_mm(25.0)
    want, got = T.triangulate(build(False), (), opts), T.triangulate(build(True), (), opts)
    assert got.check() is None
    assert np.array_equal(got.pattern_mm, want.pattern_mm) and np.array_equal(got.indices, want.indices)
    assert got.chains == want.chains


@pytest.mark.parametrize("seed", range(8))
def test_nothing_degenerate_ever_panics_or_lies(seed):  # tests/mesh.rs:476-499
    rng = np.random.default_rng(200 + seed)
    poly = ref_star(200 + seed)
    jitter, t = float(rng.uniform(0.0, 1e-3)), float(rng.uniform(0.0, 1.0))
    net = _star_net(poly)
    hub = net.add_vertex(0.0, 0.0)
    for p in poly:
        ghost = net.add_vertex(p[0] + jitter, p[1] - jitter)
        net.add_edge(ghost, hub, T.DART_LEG)
    notches = [(e, tt) for e in range(len(net.edges)) for tt in (t, 1.0 - t)]
    try:
        m = T.triangulate(net, notches, T.Options().with_target_edge_mm(15.0))
    except T.TriangulateError as err:
        assert str(err)
    else:
        assert m.check() is None
