"""Whole-step behaviour of the oracle against the reference's ImplicitSolver tests
(implicit.rs) not covered elsewhere: the non-finite step guard, bending against sag, the
self-intersection predicate, resting on a floor with each barrier and stiffness choice,
a single spring's static equilibrium, friction on an incline and sheet on sheet, and the
Newton loop's target_toi / min_newton_steps / max_dx controls, each at the test's own
parameters over ImplicitParams::default() and stepped with CgCpu (block Jacobi)."""
import numpy as np
import oracle_py as O

from mguso import scenes

f32 = np.float32
FLOOR = np.array([[0, 0, 0, 0, 0, 1, 0, 0]], f32)


def grid(n, y, spacing=0.1, nx=None, alt=False):
    nx = nx or n
    pos = np.array([(i * spacing, y, j * spacing) for j in range(n) for i in range(nx)], f32)
    tris = []
    for j in range(n - 1):
        for i in range(nx - 1):
            v = j * nx + i
            r = v + nx
            tris += [(v, v + 1, r), (v + 1, r + 1, r) if alt else (r, v + 1, r + 1)]
    return pos, np.array(tris, np.uint32).reshape(-1, 3)


def scene(pos, tris, vertex_mass, colliders=None, **kw):
    p = dict(dt=1.0 / 60.0, gravity=(0.0, -9.8, 0.0), newton_iters=4, stiffness=1.0e3, bend_stiffness=0.0,
             contact_dhat=1.0e-2, contact_kappa=1.0e2, contact_rayleigh=0, self_collision=0, barrier_kind=0,
             precond=1)
    p.update(kw)
    si, sw, skl = scenes._empty_stitches()
    return dict(positions=np.asarray(pos, f32), velocities=np.zeros((len(pos), 3), f32),
                inv_mass=np.full(len(pos), 1.0 / vertex_mass, f32), tris=np.asarray(tris, np.uint32).reshape(-1, 3),
                shell_faces=np.zeros((0, 3), np.uint32), static_mask=None, stitch_idx=si, stitch_w=sw,
                stitch_kl=skl, colliders=np.zeros((0, 8), f32) if colliders is None else colliders,
                params=scenes.default_params(**p))


def run(sc, steps, **kw):
    o = O.OracleSolver(sc)
    st = o.step(steps, check_intersection=False)
    return o, st


def test_nan_guard_rejects_bad_step():  # implicit.rs:4129-4148
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]], f32)
    sc = scene(pos, [[0, 1, 2], [2, 1, 3]], 0.05)
    sc["inv_mass"][0] = 0.0
    sc["velocities"][1, 0] = np.nan
    o, _ = run(sc, 1)
    assert np.all(np.isfinite(o.positions())) and np.all(np.isfinite(o.velocities()))


def cantilever_far_edge_sag(bend):  # implicit.rs:4150-4197
    nx, nz = 7, 3
    pos, tris = grid(nz, 1.0, nx=nx)
    sc = scene(pos, tris, 0.02, dt=1.0 / 120.0, stiffness=500.0, bend_stiffness=bend)
    for j in range(nz):
        sc["inv_mass"][[j * nx, j * nx + 1]] = 0.0
    o, _ = run(sc, 300)
    p = o.positions()
    return float(np.mean([1.0 - p[j * nx + nx - 1, 1] for j in range(nz)]))


def test_bending_stiffness_resists_sag():  # implicit.rs:4200-4210
    soft, stiff = cantilever_far_edge_sag(0.0), cantilever_far_edge_sag(2000.0)
    assert np.isfinite(soft) and np.isfinite(stiff)
    assert stiff < soft * 0.85, (soft, stiff)


def test_detects_transverse_self_intersection():  # implicit.rs:4423-4461
    clean = np.array([[-1, -1, 0], [2, -1, 0], [-1, 2, 0], [0.2, 0.2, 0.3], [0.4, 0.2, 0.3], [0.3, 0.4, 0.6]], f32)
    o = O.OracleSolver(scene(clean, [[0, 1, 2], [3, 4, 5]], 1.0, self_collision=1))
    assert not o.self_intersects(clean)
    pierced = clean.copy()
    pierced[4] = [0.4, 0.2, -0.3]
    pierced[5] = [0.3, 0.4, 0.3]
    assert o.self_intersects(pierced)


def test_cloth_rests_on_plane_without_penetration():  # implicit.rs:4557-4592
    pos, tris = grid(6, 0.3)
    o, _ = run(scene(pos, tris, 0.02, FLOOR, dt=1.0 / 120.0, stiffness=500.0, contact_dhat=0.02,
                     contact_kappa=1.0e3), 400)
    p = o.positions()
    assert np.all(np.isfinite(p)) and p[:, 1].min() > -1e-3
    assert max(0.0, float(p[:, 1].max())) < 0.1


def test_single_spring_reaches_static_equilibrium():  # implicit.rs:4775-4804
    pos = np.array([[0, 1, 0], [0, 0, 0]], f32)
    sc = scene(pos, np.zeros((0, 3)), 1.0, dt=1.0 / 120.0, newton_iters=3, stiffness=1000.0)
    sc["inv_mass"][0] = 0.0
    o = O.OracleSolver(sc)
    o.set_stretch_edges([[0, 1]])
    o.step(2000, check_intersection=False)
    p = o.positions()
    assert abs(p[1, 1] - (-(1.0 * 9.8 / 1000.0))) <= 5e-4
    assert p[0, 1] == 1.0


def _floor_drop(y0, steps, **kw):
    pos, tris = grid(5, y0)
    o, _ = run(scene(pos, tris, 0.1, FLOOR, dt=1.0 / 240.0, stiffness=500.0, contact_dhat=0.02, **kw), steps)
    return o.positions()


def test_barrier_wiring_leaves_defaults_bit_identical():  # implicit.rs:4951-5008
    a = _floor_drop(0.35, 60, contact_kappa=1.0e2)
    b = _floor_drop(0.35, 60, contact_kappa=1.0e2, barrier_kind=0, contact_rayleigh=0)
    assert np.array_equal(a, b)


def test_cubic_barrier_runs_and_stays_non_penetrating():  # implicit.rs:5011-5064
    p = _floor_drop(0.3, 400, contact_kappa=1.0e3, barrier_kind=1)
    assert np.isfinite(p[:, 1].min()) and p[:, 1].min() < 0.2 and p[:, 1].min() > -0.01


def test_rayleigh_contact_stiffness_holds_resting_contact():  # implicit.rs:5067-5117
    p = _floor_drop(0.05, 300, contact_kappa=1.0e2, contact_rayleigh=1)
    assert np.isfinite(p[:, 1].min()) and p[:, 1].min() > -0.01


def test_friction_slows_sliding_and_is_off_by_default():  # implicit.rs:5994-6052
    normal = np.array([0.30, 0.954, 0.0], f32)
    normal = normal / f32(np.linalg.norm(normal))

    def slide(mu):
        pos, tris = grid(5, 0.0)
        pos = pos + normal * f32(0.004)
        col = np.array([[0, 0, 0, 0, *normal, 0]], f32)
        o, _ = run(scene(pos, tris, 0.1, col, dt=1.0 / 240.0, stiffness=800.0, contact_dhat=0.01,
                         contact_kappa=1.0e4, friction=mu, friction_eps=1.0e-4), 200)
        p = o.positions()
        assert np.all(np.isfinite(p))
        d = p - pos
        return float(np.mean(np.linalg.norm(d - np.outer(d @ normal, normal), axis=1))), p

    free, pos_free = slide(0.0)
    rough, _ = slide(0.8)
    assert free > 1e-4 and rough < free, (free, rough)
    assert np.array_equal(pos_free, slide(0.0)[1])


def test_self_collision_friction_damps_sheet_on_sheet_sliding():  # implicit.rs:7281-7345
    def slide(mu):
        n = 4
        lo, tl = grid(n, 0.0)
        hi, th = grid(n, 0.03)
        pos = np.concatenate([lo, hi])
        tris = np.concatenate([tl, th + n * n])
        sc = scene(pos, tris, 0.1, dt=1.0 / 240.0, stiffness=600.0, self_collision=1, contact_dhat=0.02,
                   contact_kappa=1.0e3, friction=mu, friction_eps=1.0e-4)
        sc["inv_mass"][: n * n] = 0.0
        sc["velocities"][n * n:, 0] = 0.5
        o, _ = run(sc, 50)
        p = o.positions()
        assert np.all(np.isfinite(p))
        return float(np.mean(np.abs(p[n * n:, 0] - pos[n * n:, 0]))), p

    free, pos_free = slide(0.0)
    rough, _ = slide(0.9)
    assert free > 1e-3 and rough < free, (free, rough)
    assert np.array_equal(pos_free, slide(0.0)[1])


def test_target_toi_terminates_newton_early_and_is_inert_by_default():  # implicit.rs:6206-6260
    def max_iters(target_toi, min_steps, cap):
        pos, tris = grid(4, 0.3)
        o, st = run(scene(pos, tris, 0.1, FLOOR, stiffness=5.0e2, contact_dhat=0.05, contact_kappa=1.0e3,
                          newton_iters=cap, target_toi=target_toi, min_newton_steps=min_steps), 40)
        assert np.all(np.isfinite(o.positions()))
        return max(s["newton_iters"] for s in st)

    assert max_iters(0.0, 0, 8) == 8
    assert max_iters(0.0, 0, 3) == 3
    assert max_iters(0.25, 0, 8) == 2
    assert max_iters(0.25, 3, 8) == 5
    assert max_iters(0.25, 10, 5) == 5


def test_max_dx_rescales_the_search_direction_without_changing_it():  # implicit.rs:6267-6331
    def step(max_dx):
        pos, tris = grid(4, 0.0)
        o, _ = run(scene(pos, tris, 0.1, stiffness=5.0e2, gravity=(0.0, -5000.0, 0.0), newton_iters=1,
                         max_dx=max_dx), 1)
        return (o.positions() - pos).astype(f32)

    free = step(float("inf"))
    free_max = float(np.linalg.norm(free, axis=1).max())
    assert free_max > 0.05
    assert np.array_equal(free, step(float("inf")))
    capped = step(0.25 * free_max)
    assert float(np.linalg.norm(capped, axis=1).max()) < free_max
    fl = np.linalg.norm(free, axis=1)
    moving = fl > 1e-6
    scales = np.linalg.norm(capped, axis=1)[moving] / fl[moving]
    assert scales.size and scales.max() - scales.min() < 1e-3 * max(scales.max(), 1e-6)


def _shell_sheet(y, pinned_row, **kw):
    pos, tris = grid(5, y)
    sc = scene(pos, tris, 0.1, dt=1.0 / 240.0, **kw)
    sc["shell_faces"] = tris.copy()
    if pinned_row:
        sc["inv_mass"][:5] = 0.0
    return sc


def test_shell_faces_with_zero_stiffness_are_bit_identical():  # implicit.rs:5719-5749
    a, _ = run(_shell_sheet(0.3, False, stiffness=500.0), 40)
    sc = _shell_sheet(0.3, False, stiffness=500.0)
    sc["shell_faces"] = np.zeros((0, 3), np.uint32)
    b, _ = run(sc, 40)
    assert a.counts()["shells"] > 0 and b.counts()["shells"] == 0
    assert np.array_equal(a.positions(), b.positions())


def test_shell_only_sheet_is_elastic():  # implicit.rs:5755-5776 (StVK, the model this path runs)
    def sag(mu):
        o, _ = run(_shell_sheet(0.0, True, stiffness=0.0, shell_mu=mu, shell_lambda=0.5 * mu), 200)
        p = o.positions()
        assert np.all(np.isfinite(p))
        return float(p[-1, 1])

    soft, stiff = sag(50.0), sag(5000.0)
    assert soft < -0.001 and stiff > soft, (soft, stiff)


def test_per_face_shell_stiffness_works_without_the_scalars():  # implicit.rs:5783-5820
    mu, lam = 800.0, 400.0
    a, _ = run(_shell_sheet(0.0, True, stiffness=0.0, shell_mu=mu, shell_lambda=lam), 120)
    o = O.OracleSolver(_shell_sheet(0.0, True, stiffness=0.0))
    assert not o.set_shell_stiffness([[mu, lam]] * 3)
    assert o.set_shell_stiffness([[mu, lam]] * o.counts()["shells"])
    o.step(120, check_intersection=False)
    assert np.all(np.isfinite(o.positions()))
    assert o.positions()[-1, 1] == a.positions()[-1, 1]


def test_build_hinges_finds_shared_edge():  # bending.rs:292-306
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]], f32)
    idx, rest = O.OracleSolver(scene(pos, [[0, 1, 2], [2, 1, 3]], 1.0)).hinges()
    assert len(idx) == 1 and abs(rest[0]) < 1e-3
    assert sorted(idx[0][1:3].tolist()) == [1, 2]  # the shared edge is the hinge's axis


def test_the_stitch_energy_is_translation_invariant():  # stitch.rs:239-255 (the cog terms cancel)
    x = np.array([[0, 0, 0], [0.01, 0, 0], [0, 0.01, 0], [0.03, 0.002, 0], [0.04, 0.002, 0], [0.03, 0.012, 0]])
    w = np.array([0.2, 0.3, 0.5, 0.25, 0.25, 0.5])
    g0, h0 = O.stitch(x, w, 0.001, 0.01)
    g1, h1 = O.stitch(x + [1.5, -2.0, 0.25], w, 0.001, 0.01)
    assert np.allclose(g0, g1, rtol=1e-9, atol=1e-12) and np.allclose(h0, h1, rtol=1e-9, atol=1e-9)


def _slide_on_floor(collider_friction, mode):
    pos, tris = grid(4, 0.25)
    o = O.OracleSolver(scene(pos, tris, 0.1, FLOOR, stiffness=5.0e2, gravity=(2.0, -9.8, 0.0), contact_dhat=0.02,
                             contact_kappa=1.0e3, friction=0.9))
    o.set_collider_friction(collider_friction, mode)
    o.step(80, check_intersection=False)
    p = o.positions()
    assert np.all(np.isfinite(p))
    return float((p[:, 0] - pos[:, 0]).astype(f32).mean())


def test_collider_friction_combines_as_min_with_the_vertex_value():  # implicit.rs:6877-6928
    rough, slick = _slide_on_floor(0.9, "min"), _slide_on_floor(0.0, "min")
    assert slick > rough * 1.5 and slick > 1e-3, (slick, rough)
    assert abs(_slide_on_floor(float("inf"), "min") - rough) < 1e-6


def test_unset_collider_friction_is_inert_under_every_friction_mode():  # implicit.rs:6938-6991
    for mode in ("min", "max", "mean"):
        unset, explicit = _slide_on_floor(float("inf"), mode), _slide_on_floor(0.9, mode)
        assert abs(unset - explicit) < 1e-4 and np.isfinite(unset), mode
