"""Pins the implicit-step oracle against the reference's own unit tests
(engine-core/src/contact.rs, shell_model.rs, bending.rs, stitch.rs, implicit.rs tests)."""
import numpy as np
import oracle_py as O
import pytest

from mguso import scenes


def fd(pts, f, h=1e-3):
    pts = np.array(pts, np.float64)
    g = np.zeros_like(pts)
    for i in range(pts.shape[0]):
        for c in range(3):
            pp, pm = pts.copy(), pts.copy()
            pp[i, c] += h
            pm[i, c] -= h
            g[i, c] = (f(pp) - f(pm)) / (2 * h)
    return g


def pt_dist(q):
    return O.point_tri(q)[0]


def test_point_triangle_gradient_matches_fd_in_every_branch():  # contact.rs:1238-1268
    a, b, c = (0, 0, 0), (1, 0, 0), (0, 1, 0)
    for p in [(0.25, 0.25, 0.4), (0.5, -0.3, 0.3), (-0.3, 0.5, 0.3), (0.8, 0.8, 0.3), (-0.4, -0.4, 0.2),
              (1.6, -0.4, 0.2), (-0.4, 1.6, 0.2)]:
        pts = [p, a, b, c]
        d, g, _ = O.point_tri(pts)
        assert d > 0.05
        want = fd(pts, pt_dist)
        assert np.abs(g - want).max() < 2e-3
        assert abs(np.linalg.norm(g[0]) - 1.0) < 1e-4


def test_closest_point_weights_are_a_partition_of_unity():  # contact.rs:1271-1303
    rng = np.random.default_rng(1)
    for _ in range(200):
        pts = rng.uniform(-1, 1, (4, 3))
        _, _, w = O.point_tri(pts)
        assert abs(w.sum() - 1.0) < 1e-5 and np.all(w >= -1e-6)


def test_segment_gradient_matches_fd():  # contact.rs:1356-1404
    cases = [[(-1, 0, 0), (1, 0, 0), (0, 0.5, -1), (0, 0.5, 1)],
             [(0, 0, 0), (1, 0, 0), (2, 0.6, -1), (2, 0.6, 1)],
             [(0, 0, 0), (1, 0, 0), (2, 0.7, 0), (3, 0.7, 0)]]
    for pts in cases:
        d, g, plain = O.seg_seg(pts)
        assert d > 0.05 and abs(d - plain) < 1e-5
        want = fd(pts, lambda q: O.seg_seg(q)[2])
        assert np.abs(g - want).max() < 2e-3


def test_distance_known_answers():  # contact.rs:1800-1814, 1935-1969
    a, b, c = (0, 0, 0), (1, 0, 0), (0, 1, 0)
    assert abs(O.point_tri([(0.25, 0.25, 0.7), a, b, c])[0] - 0.7) < 1e-5
    assert abs(O.point_tri([(-1, -1, 0), a, b, c])[0] - np.sqrt(2)) < 1e-5
    assert abs(O.point_tri([(0.5, -0.3, 0), a, b, c])[0] - 0.3) < 1e-5
    assert O.seg_seg([(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0)])[2] < 1e-5


def test_accd_edge_through_edge():  # contact.rs:1971-1996
    x0 = [(-1, 0.5, 0), (1, 0.5, 0), (0, 0, -1), (0, 0, 1)]
    dx = [(0, -2, 0), (0, -2, 0), (0, 0, 0), (0, 0, 0)]
    toi = O.accd(x0, dx, kind="ee")
    assert toi < 1.25
    m = np.array(x0, np.float32)
    m[:2] += np.array(dx[:2], np.float32) * np.float32(toi)
    assert O.seg_seg(m)[2] > 0


def test_accd_point_into_triangle():  # contact.rs:1998-2025
    x0 = [(0.25, 0.25, 1.0), (0, 0, 0), (1, 0, 0), (0, 1, 0)]
    dx = [(0, 0, -2), (0, 0, 0), (0, 0, 0), (0, 0, 0)]
    toi = O.accd(x0, dx)
    assert 0.40 <= toi < 0.55
    moved = np.array(x0, np.float32)
    moved[0] += np.array(dx[0], np.float32) * np.float32(toi)
    assert O.point_tri(moved)[0] > 0


def test_accd_no_relative_motion():  # contact.rs:2027-2043
    x0 = [(0.25, 0.25, 1.0), (0, 0, 0), (1, 0, 0), (0, 1, 0)]
    v = (0, 0, -5)
    assert O.accd(x0, [v] * 4) == np.float32(1.25)


def test_rayleigh_reduces_to_inertial_term():  # contact.rs:1664-1696
    e = np.array([0, 0.03, 0], np.float32)
    g = 0.03
    for n in (2, 3, 4):
        w = np.full(n, 1.0 / (n - 1), np.float32)
        w[0] = -1.0
        k = O.rayleigh(np.zeros((n * n, 9)), np.full(n, 0.7), w, e)
        assert abs(k - 0.7 / g ** 2) < 1e-3 * 0.7 / g ** 2
    w = np.array([-1, 1], np.float32)
    far = O.rayleigh(np.zeros((4, 9)), [0.7, 0.7], w, e)
    near = O.rayleigh(np.zeros((4, 9)), [0.7, 0.7], w, e * 0.5)
    assert abs(near / far - 4.0) < 1e-2


def test_rayleigh_substitutes_static_side_mass():  # contact.rs:1698-1722
    e = np.array([0, 0.04, 0], np.float32)
    w = np.array([-1, 1], np.float32)
    both = O.rayleigh(np.zeros((4, 9)), [0.9, 0.9], w, e)
    one = O.rayleigh(np.zeros((4, 9)), [0.9, 0.0], w, e)
    assert abs(both - one) < 1e-4 * both


def test_log_barrier_is_c2_at_dhat_and_blows_up_near_zero():  # contact.rs:1784-1798
    assert O.barrier(0.1, 0.1, 1.0) is None and O.barrier(0.2, 0.1, 1.0) is None
    e_edge, g_edge, _ = O.barrier(0.0999, 0.1, 1.0)
    assert 0 < e_edge < 1e-3 and abs(g_edge) < 1e-2
    e_near, g_near, _ = O.barrier(1e-4, 0.1, 1.0)
    assert e_near > 100 * e_edge and g_near < 0


def test_cubic_barrier_derivatives_match_fd():  # contact.rs:1591-1630
    for gap in (-0.02, 0.0, 0.03, 0.07):
        e, g, h = O.barrier(gap, 0.1, 2.0, kind="cubic", f64=True)
        hh = 1e-6
        ep = O.barrier(gap + hh, 0.1, 2.0, kind="cubic", f64=True)
        em = O.barrier(gap - hh, 0.1, 2.0, kind="cubic", f64=True)
        assert abs((ep[0] - em[0]) / (2 * hh) - g) < 1e-5 * max(1, abs(g))
        assert abs((ep[1] - em[1]) / (2 * hh) - h) < 1e-4 * max(1, abs(h))
        assert g < 0 and h > 0


def test_stvk_shell_gradient_matches_fd_and_hessian_is_psd():  # shell_model.rs:1077-1250
    rng = np.random.default_rng(3)
    rest = np.array([[0, 0, 0], [1, 0, 0], [0.2, 0.9, 0]], np.float64)
    mu, lam = scenes.lame_from_young_poisson(1e5 * 5e-4, 0.3)
    for _ in range(10):
        p = rest @ np.diag([1.3, 0.8, 1.0]) + rng.normal(0, 0.05, (3, 3))
        e, g, h = O.shell(rest, p, mu, lam)
        want = fd(p, lambda q: O.shell(rest, q, mu, lam)[0], h=1e-6)
        assert np.abs(g - want).max() < 1e-5 * max(1.0, np.abs(want).max())
        assert np.abs(h - h.T).max() < 1e-9 * max(1.0, np.abs(h).max())
        assert np.linalg.eigvalsh(h).min() > -1e-9 * max(1.0, np.abs(h).max())
    # rest state: zero energy and gradient
    e, g, _ = O.shell(rest, rest, mu, lam)
    assert abs(e) < 1e-12 and np.abs(g).max() < 1e-9


def test_hinge_analytic_gradient_matches_fd():  # bending.rs:228-260
    rng = np.random.default_rng(5)
    for _ in range(20):
        p = np.array([[0, 1, 0], [0, 0, 0], [1, 0, 0], [0.5, -1, 0.3]], np.float64) + rng.normal(0, 0.1, (4, 3))
        th, g, gf = O.hinge(p)
        assert np.abs(g - gf).max() < 1e-4 * max(1.0, np.abs(gf).max())
        assert np.abs(g.sum(0)).max() < 1e-9


def test_flat_hinge_reads_zero():  # bending.rs:27-48
    p = np.array([[0, 1, 0], [0, 0, 0], [1, 0, 0], [0.5, -1, 0]], np.float64)
    th, _, _ = O.hinge(p)
    assert abs(th) < 1e-12
    q = np.array([[0, 1, 0], [0, 0, 0], [1, 0, 0], [1, 1, 0]], np.float64)  # folded shut
    assert abs(abs(O.hinge(q)[0]) - np.pi) < 1e-12


def test_stitch_gradient_matches_fd_and_hessian_is_psd():  # stitch.rs:138-230
    rng = np.random.default_rng(7)
    w = np.array([0.2, 0.3, 0.5, 0.6, 0.4, 0.0])
    l0, lcap = 1e-3, 0.05
    for _ in range(10):
        x = rng.normal(0, 0.01, (6, 3))
        x[3:] += 0.02

        def energy(q):
            t = (w[:3, None] * q[:3]).sum(0) - (w[3:, None] * q[3:]).sum(0)
            e = np.linalg.norm(t) - l0
            return 0.5 * e * e / l0

        g, h = O.stitch(x, w, l0, lcap)
        want = fd(x, energy, h=1e-7)
        assert np.abs(g - want).max() < 1e-5 * max(1.0, np.abs(want).max())
        assert np.linalg.eigvalsh(0.5 * (h + h.T)).min() > -1e-9


def small_sheet(n=12, **kw):
    return scenes.sheet_on_sphere(n, side=0.4, **kw)


def test_cloth_drapes_over_sphere_without_penetration():  # implicit.rs:4595-4632
    sc = small_sheet(12, height=0.33)
    s = O.OracleSolver(sc)
    stats = s.step(20)
    p = s.positions()
    assert all(st["all_finite"] and st["penetration_free"] for st in stats)
    r = np.linalg.norm(p, axis=1)
    assert r.min() >= 0.3 - 1e-3 * 1e-3 - 1e-6
    assert p[:, 1].min() < 0.33 - 0.01  # it fell


def test_implicit_is_deterministic():  # implicit.rs:4929-4949
    sc = small_sheet(10)
    a, b = O.OracleSolver(sc), O.OracleSolver(sc)
    a.step(6)
    b.step(6)
    assert np.array_equal(a.positions(), b.positions())


def test_f64_oracle_tracks_f32_oracle():
    sc = small_sheet(10)
    a, b = O.OracleSolver(sc, "f32"), O.OracleSolver(sc, "f64")
    for _ in range(8):
        a.step(1)
        b.step(1)
    pa, pb = a.positions(), b.positions()
    assert np.abs(pa - pb).max() < 1e-3 * np.abs(pb).max()


def test_self_contact_stencils_are_exact_predicate():
    """Stencils = every (v, t) with 1-ring excluded and d < dhat, plus every edge pair with
    no shared vertex and d < dhat (implicit.rs:678-753), independent of the hash grid."""
    rng = np.random.default_rng(2)
    n = 6
    sc = scenes.sheet_on_sphere(n, side=0.05, jitter=0.0, dhat=5e-3)
    # fold a second layer just above the first
    pos = sc["positions"].copy()
    top = pos.copy()
    top[:, 1] += 2e-3
    top += rng.uniform(-5e-4, 5e-4, top.shape).astype(np.float32)
    sc["positions"] = np.concatenate([pos, top]).astype(np.float32)
    sc["velocities"] = np.zeros_like(sc["positions"])
    sc["tris"] = np.concatenate([sc["tris"], sc["tris"] + n * n]).astype(np.uint32)
    sc["shell_faces"] = sc["tris"].copy()
    sc["inv_mass"] = np.concatenate([sc["inv_mass"], sc["inv_mass"]])
    s = O.OracleSolver(sc)
    idx, d = s.stencils()
    P = sc["positions"]
    T = sc["tris"]
    dh = np.float32(5e-3)
    ring = [set() for _ in range(P.shape[0])]
    for t in T:
        for a in t:
            ring[a] |= set(int(x) for x in t)
    want_vt = set()
    for v in range(P.shape[0]):
        for ti, t in enumerate(T):
            if ring[v] & set(int(x) for x in t) or v in t:
                continue
            dd, _, _ = O.point_tri([P[v], P[t[0]], P[t[1]], P[t[2]]])
            if dd < dh:
                want_vt.add((v, int(t[0]), int(t[1]), int(t[2])))
    got = set(map(tuple, idx.tolist()))
    got_vt = {g for g in got if any(g == w for w in want_vt) or (g[0], g[1], g[2], g[3]) in want_vt}
    assert want_vt <= got
    assert len(got) > len(want_vt)  # edge-edge stencils too


def test_stepping_along_the_gradient_changes_the_distance_as_predicted():  # contact.rs:1560-1582
    pts = [(0.25, 0.25, 0.4), (0, 0, 0), (1, 0, 0), (0, 1, 0)]
    d0, g, _ = O.point_tri(pts)
    eps = 1e-3
    moved = [tuple(np.asarray(pts[0]) + eps * g[0])] + pts[1:]
    d1, _, _ = O.point_tri(moved)
    assert abs(d1 - (d0 + eps * float(g[0] @ g[0]))) < 1e-5


def test_cubic_barrier_is_finite_and_repulsive_including_penetration():  # contact.rs:1632-1662
    ghat = 0.1
    assert O.barrier(0.1, ghat, 1.0, kind="cubic") is None
    assert O.barrier(0.5, ghat, 1.0, kind="cubic") is None
    for gap in (0.09, 0.05, 0.01, 0.0, -0.05, -0.5):
        e, g, c = O.barrier(gap, ghat, 1.0, kind="cubic")
        assert e > 0 and np.isfinite(e), gap
        assert g < 0 and np.isfinite(g), gap
        assert c > 0 and np.isfinite(c), gap
    e0, _, c0 = O.barrier(1e-9, ghat, 1.0, kind="cubic")
    assert e0 < 1.0 and c0 <= 4.0 + 1e-5
    assert O.barrier(-0.2, ghat, 1.0, kind="cubic")[1] < O.barrier(0.01, ghat, 1.0, kind="cubic")[1]


def reference_defaults(**kw):
    """ImplicitParams::default() (implicit.rs:176-229) in this library's parameter names."""
    return scenes.default_params(**dict(dict(newton_iters=4, stiffness=1.0e3, bend_stiffness=0.0,
                                             contact_dhat=1.0e-2, contact_kappa=1.0e2, contact_rayleigh=0,
                                             self_collision=0), **kw))


def _two_point_stitch(stiffness):
    pos = np.array([[0, 0, 0], [0.05, 0, 0]], np.float32)
    return dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=np.array([0.0, 1.0], np.float32),
                tris=np.zeros((0, 3), np.uint32), shell_faces=np.zeros((0, 3), np.uint32), static_mask=None,
                stitch_idx=np.array([[0, 0, 0, 1, 1, 1]], np.uint32),
                stitch_w=np.array([[1, 0, 0, 1, 0, 0]], np.float32),
                stitch_kl=np.array([[stiffness, 0.001, 0.01]], np.float32),
                colliders=np.zeros((0, 8), np.float32), params=reference_defaults(gravity=(0.0, 0.0, 0.0)))


def test_a_stitch_closes_the_seam_it_sews():  # implicit.rs:3426-3490
    o = O.OracleSolver(_two_point_stitch(1.0))
    st = o.step(400, check_intersection=False)
    p = o.positions().astype(np.float64)
    assert np.all(np.isfinite(p)) and len(st) == 400
    assert abs(np.linalg.norm(p[1] - p[0]) - 0.001) <= 1e-4 * 0.001
    assert np.linalg.norm(p[0]) < 1e-6
    # zero stiffness sews nothing
    o = O.OracleSolver(_two_point_stitch(0.0))
    o.step(400, check_intersection=False)
    p = o.positions().astype(np.float64)
    assert abs(np.linalg.norm(p[1] - p[0]) - 0.05) < 1e-6


def _two_layers(n, y_upper, mass, **params):
    pos, tris = [], []
    for li, y in ((0, 0.0), (1, y_upper)):
        base = len(pos)
        pos += [(i * 0.1, y, j * 0.1) for j in range(n) for i in range(n)]
        for j in range(n - 1):
            for i in range(n - 1):
                v = base + j * n + i
                r = v + n
                tris += [(v, v + 1, r), (r, v + 1, r + 1)]
    pos = np.array(pos, np.float32)
    im = np.full(len(pos), 1.0 / mass, np.float32)
    im[: n * n] = 0.0  # the lower layer is pinned
    si, sw, skl = scenes._empty_stitches()
    return dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=im, tris=np.array(tris, np.uint32),
                shell_faces=np.zeros((0, 3), np.uint32), static_mask=None, stitch_idx=si, stitch_w=sw,
                stitch_kl=skl, colliders=np.zeros((0, 8), np.float32),
                params=reference_defaults(self_collision=1, **params)), n * n


def test_self_collision_holds_resting_contact():  # implicit.rs:4294-4345
    sc, lower = _two_layers(5, 0.018, 0.02, dt=1.0 / 480.0, stiffness=500.0, gravity=(0.0, -4.0, 0.0),
                            contact_dhat=0.02, contact_kappa=2.0e3)
    o = O.OracleSolver(sc)
    o.step(300)
    p = o.positions()
    assert np.all(np.isfinite(p))
    assert p[lower:, 1].min() > -0.005


def test_self_collision_rayleigh_stiffness_holds_a_heavy_resting_contact():  # implicit.rs:4359-4412
    sc, lower = _two_layers(4, 0.02, 0.1, dt=1.0 / 240.0, stiffness=500.0, gravity=(0.0, -9.8, 0.0),
                            contact_dhat=0.02, contact_kappa=1.0e2)
    o = O.OracleSolver(sc)
    st = o.step(200)
    p = o.positions()
    assert np.all(np.isfinite(p))
    assert all(s["penetration_free"] for s in st)  # no self-intersection develops
    assert p[lower:, 1].min() > -0.01


def _vertex_over_triangle(z):
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0.3, 0.3, z]], np.float32)
    si, sw, skl = scenes._empty_stitches()
    return dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=np.array([0, 0, 0, 1], np.float32),
                tris=np.array([[0, 1, 2]], np.uint32), shell_faces=np.zeros((0, 3), np.uint32), static_mask=None,
                stitch_idx=si, stitch_w=sw, stitch_kl=skl, colliders=np.zeros((0, 8), np.float32),
                params=reference_defaults(self_collision=1, contact_dhat=0.02))


@pytest.mark.parametrize("z, step", [(0.05, -0.2), (4.0, -8.0)])
def test_ccd_clamps_a_step_toward_a_triangle(z, step):  # implicit.rs:4634-4668, 4722-4760
    o = O.OracleSolver(_vertex_over_triangle(z))
    dx = np.zeros((4, 3), np.float32)
    dx[3, 2] = step
    t = o.ccd(dx)
    assert t < 1.0
    assert z + t * step > 0.0


def test_implicit_hanging_cloth_is_stable():  # implicit.rs:4806-4834
    n = 6
    pos = np.array([(i * 0.1, 1.0, j * 0.1) for j in range(n) for i in range(n)], np.float32)
    tris = []
    for j in range(n - 1):
        for i in range(n - 1):
            v = j * n + i
            tris += [(v, v + 1, v + n), (v + n, v + 1, v + n + 1)]
    im = np.full(n * n, 1.0 / 0.05, np.float32)
    im[0] = im[n - 1] = 0.0
    si, sw, skl = scenes._empty_stitches()
    sc = dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=im, tris=np.array(tris, np.uint32),
              shell_faces=np.zeros((0, 3), np.uint32), static_mask=None, stitch_idx=si, stitch_w=sw,
              stitch_kl=skl, colliders=np.zeros((0, 8), np.float32), params=reference_defaults())
    o = O.OracleSolver(sc)
    o.step(120)
    p = o.positions()
    assert np.all(np.isfinite(p))
    assert p[n // 2 * n + n // 2, 1] < 1.0  # it hangs: the middle has fallen


def test_friction_is_tangential_opposes_slip_and_respects_coulomb():  # contact.rs:2112-2172
    n = np.array([0, 1, 0], np.float32)
    f_c = -10.0 * n
    mu, eps = 0.4, 1e-3
    contact = -float(n @ f_c)
    slip = np.array([0.05, 0.02, -0.03], np.float32)
    g, h = O.friction(f_c, slip, n, mu, eps)
    assert abs(float(g @ n)) < 1e-5
    pdx = slip - float(n @ slip) * n
    assert float(g @ pdx) > 0
    assert abs(np.linalg.norm(g) - mu * contact) < 1e-3 * mu * contact
    assert np.abs(h - h.T).max() < 1e-6
    for t in range(8):
        x = np.array([(t * 7919 % 100) / 50 - 1, (t * 104729 % 100) / 50 - 1, (t * 1299709 % 100) / 50 - 1])
        assert x @ h @ x >= -1e-5
    g0, h0 = O.friction(f_c, slip, n, 0.0, eps)
    assert not g0.any() and not h0.any()


def test_friction_regularization_caps_tiny_slip():  # contact.rs:2174-2204
    n = np.array([0, 1, 0], np.float32)
    f_c = -10.0 * n
    mu, eps = 0.5, 1e-3
    bound = mu * -float(n @ f_c)
    prev = 0.0
    for k in range(6):
        s = 1e-6 * 10.0 ** k
        g, _ = O.friction(f_c, np.array([s, 0, 0], np.float32), n, mu, eps)
        m = float(np.linalg.norm(g))
        assert np.isfinite(m) and m <= bound + 1e-4 and m >= prev - 1e-6
        prev = m
        if s < eps:
            assert abs(m - bound * s / eps) < 1e-3 * max(bound, 1.0)


def test_friction_vanishes_without_normal_force():  # contact.rs:2206-2214
    n = np.array([0, 1, 0], np.float32)
    g, h = O.friction(5.0 * n, np.array([0.1, 0, 0], np.float32), n, 0.5, 1e-3)
    assert not g.any() and not h.any()


def test_a_degenerate_stitch_source_reduces_to_a_single_vertex():  # stitch.rs:256-282
    p = np.zeros(3)
    t1, t2 = np.array([0.003, 0.001, 0.0]), np.array([0.013, 0.001, 0.0])
    x = np.array([p, p, p, t1, t2, t2])
    w = np.array([1.0, 0.0, 0.0, 0.75, 0.25, 0.0])
    g, _ = O.stitch(x, w, 0.001, 0.01)
    t = p - (0.75 * t1 + 0.25 * t2)
    l = min(np.linalg.norm(t), 0.01)
    dedt = (l / 0.001 - 1.0) * (t / l)
    n = np.linalg.norm(dedt)
    assert np.linalg.norm(g[0] - dedt) <= 1e-4 * n
    assert np.linalg.norm(g[1]) < 1e-9 and np.linalg.norm(g[2]) < 1e-9
    assert np.linalg.norm(g[3] + 0.75 * dedt) <= 1e-4 * n
    assert np.linalg.norm(g[4] + 0.25 * dedt) <= 1e-4 * n
    assert np.linalg.norm(g[5]) < 1e-9


def test_beyond_the_stitch_cap_the_pull_grows_linearly():  # stitch.rs:284-305
    w = np.array([1.0, 0, 0, 1.0, 0, 0])

    def mag(sep):
        x = np.array([[0, 0, 0]] * 3 + [[sep, 0, 0]] * 3, np.float64)
        return np.linalg.norm(O.stitch(x, w, 0.001, 0.01)[0][0])

    assert abs(mag(0.08) / mag(0.04) - 2.0) < 1e-3


def _flap(fold_deg):
    a = np.radians(fold_deg)
    return np.array([[0.5, -1.0, 0.0], [0, 0, 0], [1, 0, 0], [0.5, np.cos(a), np.sin(a)]])


def test_folding_changes_the_hinge_angle_monotonically():  # bending.rs:267-272
    assert abs(O.hinge(_flap(90.0))[0]) > abs(O.hinge(_flap(45.0))[0])


def test_the_hinge_gradient_reduces_energy_toward_rest():  # bending.rs:274-290
    p = _flap(120.0)
    th0, g, _ = O.hinge(p)
    step = 1e-3 * np.sign(th0)
    th1 = O.hinge(p - g * step * 50.0)[0]
    assert abs(th1) < abs(th0)


def test_kinematic_collider_repose_moves_only_the_collider_and_sets_its_velocity():  # implicit.rs:1368-1398
    sc = scenes.sheath_on_torso(edge=0.05, torso_res=(24, 23), width=0.5, torso_scale=0.9)
    o = O.OracleSolver(sc, "f64")
    o.step(1, check_intersection=False)
    x0, v0 = o.positions().copy(), o.velocities().copy()
    body = np.asarray(sc["static_mask"], bool)
    x = x0.copy()
    x[body, 1] += 0.002
    x[~body] = 123.0  # rows that are not the collider's are ignored
    bad = x.copy()
    bad[np.flatnonzero(body)[0], 0] = np.nan
    assert not o.set_kinematic_collider_positions(bad)
    assert np.array_equal(o.positions(), x0)  # nothing written
    assert o.set_kinematic_collider_positions(x)
    x1, v1 = o.positions(), o.velocities()
    assert np.allclose(x1[body], x0[body] + [0, 0.002, 0]) and np.array_equal(x1[~body], x0[~body])
    assert np.allclose(v1[body], [0, 0.002 / sc["params"]["dt"], 0]) and np.array_equal(v1[~body], v0[~body])
    st = o.step(1)
    assert st[0]["penetration_free"] and np.all(np.isfinite(o.positions()))
    free = dict(sc, static_mask=None)
    assert not O.OracleSolver(free, "f64").set_kinematic_collider_positions(x)


def test_elastic_block_gather_handles_off_diagonals_and_duplicates():  # implicit.rs:6330-6388
    """The assembler's requested blocks (the Rayleigh stiffnesses' gathers): off-diagonal
    blocks at their own local (row, column), duplicates accumulated, unrequested pairs
    ignored."""
    trips = [(1, 2, 5.0), (0, 3, 1.5), (0, 3, 2.5), (5, 1, -7.0), (6, 8, 9.0), (9, 9, 100.0), (3, 6, 100.0)]
    b = O.asm_blocks(4, [(0, 0), (0, 1), (1, 0), (2, 2)], trips)
    assert b.shape == (4, 3, 3)
    assert b[0][1, 2] == 5.0 and np.count_nonzero(b[0]) == 1
    assert b[1][0, 0] == 4.0, "duplicate triplets must accumulate"
    assert b[2][2, 1] == -7.0
    assert not np.array_equal(b[1], b[2]), "(0,1) and (1,0) must be distinct blocks"
    assert b[3][0, 2] == 9.0
    assert np.abs(b).sum() == 5.0 + 4.0 + 7.0 + 9.0, "unrequested pairs must be ignored"


def test_shell_energy_is_rigid_motion_invariant_and_its_hessian_annihilates_translations():
    """shell_model.rs:1112-1147 and 1200-1250 on the StVK model this path runs (the reference
    tests ARAP there): the unit triangle's rest state is stress-free, the deformed energy is unchanged by the tests' rotation and shift, the forces sum to zero, and
    the element Hessian is symmetric, PSD and has the three translations as null modes; a
    degenerate triangle builds no element."""
    rest = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float64)
    mu, lam = 400.0, 250.0
    e, g, _ = O.shell(rest, rest, mu, lam, f64=False)
    assert abs(e) < 1e-5 and np.abs(g).max() < 1e-3
    flat = np.array([[0, 0, 0], [1, 0, 0], [2, 0, 0]], np.float64)
    assert O.shell(flat, flat, mu, lam) is None  # a degenerate rest triangle builds no element
    deformed = np.array([[0.01, -0.02, 0.0], [1.25, 0.05, 0.03], [-0.04, 0.88, -0.02]], np.float64)
    base, g, _ = O.shell(rest, deformed, mu, lam)
    assert base > 1e-3
    assert np.abs(g.sum(axis=0)).max() < 1e-9 * max(1.0, np.abs(g).max())
    a, b, c = 0.8, -1.2, 0.4  # glam's EulerRot::XYZ: R = Rx(a) Ry(b) Rz(c)
    rx = np.array([[1, 0, 0], [0, np.cos(a), -np.sin(a)], [0, np.sin(a), np.cos(a)]])
    ry = np.array([[np.cos(b), 0, np.sin(b)], [0, 1, 0], [-np.sin(b), 0, np.cos(b)]])
    rz = np.array([[np.cos(c), -np.sin(c), 0], [np.sin(c), np.cos(c), 0], [0, 0, 1]])
    moved = deformed @ (rx @ ry @ rz).T + np.array([-3.0, 4.0, 2.0])
    after = O.shell(rest, moved, mu, lam)[0]
    assert abs(after - base) < 1e-3 * max(base, 1.0), (base, after)
    p = np.array([[0, 0, 0], [1.22, 0.05, 0.0], [0.03, 0.9, 0.02]], np.float64)
    _, _, h = O.shell(rest, p, mu, lam)
    scale = max(1.0, np.abs(h).max())
    assert np.abs(h - h.T).max() < 1e-4 * scale
    assert np.linalg.eigvalsh(0.5 * (h + h.T)).min() > -1e-3 * scale
    for axis in range(3):
        t = np.zeros(9)
        t[axis::3] = 1.0
        assert np.abs(h @ t).max() < 1e-3 * scale, axis
