"""Contact primitives of the CPU oracle against the reference's contact.rs tests that the
other oracle test files do not cover: degenerate triangles, the edge-edge witness policy,
witness vs clamped segment distance, the signed point-triangle gap, analytic colliders,
dynamic and Rayleigh stiffness, and stencil friction."""
import numpy as np
import oracle_py as O

f32 = np.float32
X, Y, Z0 = np.array([1, 0, 0], f32), np.array([0, 1, 0], f32), np.zeros(3, f32)


def test_degenerate_triangles_never_produce_nan():  # contact.rs:1305-1353
    o = np.array([1.0e4, 0, 0], f32)
    cases = [(Z0, Z0, X), (Z0, X, Z0), (Z0, X, X), (Z0, Z0, Z0), (Z0, X, 2 * X), (o, o, o + X), (o, o + X, o),
             (o, o + X, o + X)]
    offsets = [(0.5, 1, 0), (-0.5, 1, 0), (1.5, 1, 0), (0.5, -1, 0.25), (3, 0, 0), (0, 0, 0)]
    for a, b, c in cases:
        mid = (a + b + c) / f32(3)
        for d in offsets:
            p = mid + np.array(d, f32)
            q, w = O.closest_point(p, a, b, c)
            assert np.all(np.isfinite(q)) and np.all(np.isfinite(w)), (a, b, c, p)
            assert abs(float(w.sum()) - 1.0) < 1e-5
            assert np.linalg.norm(w[0] * a + w[1] * b + w[2] * c - q) < 1e-3


def test_parallel_segments_follow_the_reference_weight_policy():  # contact.rs:1407-1445
    pts = np.array([[0, 0, 0], [1, 0, 0], [0, 0.4, 0], [1, 0.4, 0]], f32)
    w = O.ee_witness(pts)
    assert w[0] == 1.0 and w[1] == 0.0
    d, g, _ = O.seg_seg(pts)
    assert abs(d - 0.4) < 1e-6
    assert abs(np.linalg.norm(g[0]) - 1.0) < 1e-5 and np.linalg.norm(g[1]) < 1e-6
    assert np.linalg.norm(g.sum(0)) < 1e-5
    assert 0.0 <= w[2] <= 1.0 and 0.0 <= w[3] <= 1.0


def _f(k, o, a, b):
    return f32(np.fmod(f32(k) * f32(a) + f32(o) * f32(b), f32(2.0)) - f32(1.0))


def test_witness_distance_agrees_with_the_clamped_segment_distance():  # contact.rs:1455-1533
    checked = 0
    for i in range(12):
        for j in range(12):
            f = lambda k, o: _f(k, o, 0.37, 0.11)  # noqa: E731
            p1 = np.array([f(i, 0), f(j, 1), f(i, 2)], f32)
            q1 = p1 + np.array([f(j, 3), f(i, 4), f(j, 5)], f32)
            p2 = np.array([f(i, 6), f(j, 7), f(i, 8)], f32)
            q2 = p2 + np.array([f(j, 9), f(i, 10), f(j, 11)], f32)
            got, _, want = O.seg_seg(np.array([p1, q1, p2, q2]))
            assert abs(got - want) <= 1e-5 * max(want, 1.0), (p1, q1, p2, q2)
            checked += 1
    cases = [
        [Z0, X, (0, 0.4, 0), (1, 0.4, 0)],
        [Z0, X, (2, 0.7, 0), (3, 0.7, 0)],
        [Z0, X, (2, 0, 0), (3, 0, 0)],
        [Z0, Z0, (1, 1, 0), X],
        [Z0, Z0, Y, Y],
    ]
    for c in cases:
        got, g, want = O.seg_seg(np.array(c, f32))
        assert abs(got - want) <= 1e-5 * max(want, 1.0), c
        assert np.all(np.isfinite(g))
        assert np.linalg.norm(g.sum(0)) < 1e-4
        checked += 1
    assert checked > 140


def test_edge_edge_witness_weights_are_convex_on_each_edge():  # contact.rs:1535-1560
    for i in range(10):
        f = lambda k, o: _f(k, o, 0.53, 0.17)  # noqa: E731
        p1 = np.array([f(i, 0), f(i, 1), f(i, 2)], f32)
        q1 = p1 + np.array([f(i, 3), f(i, 4), f(i, 5)], f32)
        p2 = np.array([f(i, 6), f(i, 7), f(i, 8)], f32)
        q2 = p2 + np.array([f(i, 9), f(i, 10), f(i, 11)], f32)
        w = O.ee_witness(np.array([p1, q1, p2, q2]))
        assert abs(w[0] + w[1] - 1.0) < 1e-5 and abs(w[2] + w[3] - 1.0) < 1e-5
        assert np.all((w >= -1e-6) & (w <= 1.0 + 1e-6))


def test_rayleigh_stiffness_grows_with_material_stiffness():  # contact.rs:1752-1782
    e = np.array([0, 0.03, 0], f32)
    mass, weights = [0.5, 0.5], [-1.0, 1.0]
    inertia_only = O.rayleigh(np.zeros((4, 9), f32), mass, weights, e)
    prev = inertia_only
    for k_el in (10.0, 100.0, 1000.0):
        el = np.zeros((4, 9), f32)
        for ii in range(2):
            el[ii * 2 + ii, [0, 4, 8]] = k_el
        k = O.rayleigh(el, mass, weights, e)
        assert k > prev
        expect = k_el + inertia_only
        assert abs(k - expect) < 1e-2 * expect
        prev = k


def test_signed_point_triangle_negates_gap_and_gradient_behind_the_triangle():  # contact.rs:1860-1933
    a, b, c = np.array([-1, 0, -1], f32), np.array([0, 0, 1], f32), np.array([1, 0, -1], f32)
    assert np.cross(b - a, c - a)[1] > 0
    for p in ([0, 0.3, 0], [0.05, 0.001, 0.1], [3, 0.2, 0]):
        p = np.array(p, f32)
        du, gu, _ = O.point_tri(np.array([p, a, b, c]))
        ds, gs, inside = O.signed_point_tri(p, a, b, c)
        assert not inside
        assert du == ds and np.array_equal(gu, gs)
        q = np.array([p[0], -p[1], p[2]], f32)
        dm, gm, inside = O.signed_point_tri(q, a, b, c)
        assert inside
        assert abs(dm + du) < 1e-6
        assert gm[0, 1] > 0 and gu[0, 1] > 0
    # a collapsed triangle has no side: the gap stays positive
    dz, _, inside = O.signed_point_tri(np.array([0, -1, 0], f32), a, a, a)
    assert not inside and dz > 0


def test_halfspace_distance_and_push():  # contact.rs:2045-2057
    floor = [0, 0, 0, 0, 0, 1, 0, 0]
    d, n = O.collider_distance(floor, [3.0, 0.05, -2.0])
    assert d == f32(0.05) and np.array_equal(n, Y)
    g, _ = O.vertex_contact([0, 0.02, 0], [floor], 0.1, 10.0, 0.0, 1.0)
    assert g[1] < 0


def test_dynamic_stiffness_scales_with_inertia():  # contact.rs:2084-2097
    base, dhat = 100.0, 0.02
    assert O.dynamic_stiffness(base, 0.0, 1.0, 0.01, dhat) == base
    assert O.dynamic_stiffness(base, 1.0, 0.0, 0.01, dhat) == base
    far = O.dynamic_stiffness(base, 1.0, 0.02, 0.015, dhat)
    near = O.dynamic_stiffness(base, 1.0, 0.02, 0.005, dhat)
    assert far > base and near > far


def test_sphere_keeps_point_outside():  # contact.rs:2099-2110
    s = [1, 0, 0, 0, 0, 0, 0, 1.0]
    d, n = O.collider_distance(s, [1.05, 0, 0])
    assert abs(d - 0.05) < 1e-6 and np.linalg.norm(n - X) < 1e-6
    g, h = O.vertex_contact([1.02, 0, 0], [s], 0.1, 10.0, 0.0, 1.0)
    assert g[0] < 0 and h[0, 0] >= 0


def test_stencil_friction_uses_proximity_weights_and_is_psd():  # contact.rs:2220-2286
    p = np.array([0.5, 0.2, 0.28867513], f32)
    a, b, c = np.array([0, 0, 0], f32), np.array([1, 0, 0], f32), np.array([0.5, 0, 0.8660254], f32)
    _, g, _ = O.point_tri(np.array([p, a, b, c]))
    n = g[0] / np.linalg.norm(g[0])
    assert abs(float((g @ n).sum())) < 1e-2
    assert abs(float(g[0] @ n) - 1.0) < 1e-2
    dx = np.zeros((4, 3), f32)
    dx[0, 0] = 0.02
    fg, fh = O.stencil_friction(g, dx, -50.0, 0.5, 1e-3)
    assert np.linalg.norm(fg.sum(0)) < 1e-2
    assert abs(float(fg[0] @ n)) < 1e-4
    assert float(fg[0] @ dx[0]) > 0
    assert np.abs(fh - fh.T).max() < 1e-5
    for t in range(8):
        xv = np.array([((t * 7919 + k * 104729) % 200) / 100.0 - 1.0 for k in range(12)], f32)
        assert float(xv @ fh @ xv) >= -1e-4
    z, zh = O.stencil_friction(g, dx, -50.0, 0.0, 1e-3)
    assert not z.any() and not zh.any()
