"""A kinematic (re-posed) static collider in the oracle, against the reference's tests of
set_kinematic_collider_positions (implicit.rs:8001-8230): a sliding body drags the cloth
resting on it through friction on the body's own move (the fdx_override slip), a rotated
body signs contact by its recomputed pseudonormals, and a rejected move changes nothing."""
import numpy as np
import oracle_py as O

from test_oracle_static_proxy import body_scene, cloth, cube_mesh, params, sphere_mesh

f32 = np.float32


def drag_on_moving_sphere(mu, dx, slide_steps):
    """implicit.rs:8009-8066: settle a 5 x 5 patch on a sphere of radius 0.2 for 300 steps,
    then move the sphere +x by dx per step; returns (cloth centroid travel, body travel,
    deepest cloth point inside the analytic sphere)."""
    r = 0.2
    body = sphere_mesh(np.zeros(3, f32), r, 20, 10)
    sc, nc = body_scene(cloth(5, 0.45, 0.06), body, friction=mu, friction_eps=1.0e-4)
    o = O.OracleSolver(sc)
    o.step(300, check_intersection=False)

    def cx():
        return float(np.float32(o.positions()[:nc, 0].astype(f32).sum()) / f32(nc))

    x0 = cx()
    centre = f32(0.0)
    worst = 0.0
    for _ in range(slide_steps):
        centre = f32(centre + f32(dx))
        target = o.positions()
        target[nc:, 0] = body[0][:, 0] + centre
        assert o.set_kinematic_collider_positions(target)
        o.step(1, check_intersection=False)
        c = np.array([centre, 0, 0])
        worst = max(worst, float((r - np.linalg.norm(o.positions()[:nc] - c, axis=1)).max()))
    return cx() - x0, float(centre), worst


def test_a_sliding_kinematic_collider_drags_the_cloth_it_carries():  # implicit.rs:8081-8105
    dragged, travel, pen = drag_on_moving_sphere(0.35, 0.002, 100)
    free, _, pen0 = drag_on_moving_sphere(0.0, 0.002, 100)
    assert dragged > 0.5 * travel, (dragged, travel)
    assert free < 0.5 * dragged, (free, dragged)
    sag = 0.2 * (1.0 - np.cos(np.pi / 20.0))
    assert pen < sag + 1e-3 and pen0 < sag + 1e-3


def test_a_rotated_kinematic_collider_signs_contact_by_its_new_pseudonormals():  # implicit.rs:8116-8180
    cube, cube_tris = cube_mesh()
    c = np.full(3, 0.5, f32)
    rot = (cube - c) * np.array([-1, -1, 1], f32) + c
    probes = np.array([[1.003, 1.003, 0.5], [-0.003, -0.003, 0.5], [1.003, -0.003, 0.5], [0.5, 0.997, 0.5]], f32)
    np_ = len(probes)
    sc, _ = body_scene((probes, np.array([[0, 1, 2], [0, 2, 3]], np.uint32)), (rot, cube_tris))
    sc["params"] = params(True)
    o = O.OracleSolver(sc)
    target = o.positions()
    target[np_:] = cube
    assert o.set_kinematic_collider_positions(target)
    side = o.collider_sides()
    assert side is not None
    assert all(side[i] == 1.0 for i in range(np_ - 1))
    assert side[np_ - 1] == -1.0


def test_a_rejected_kinematic_move_changes_nothing():  # implicit.rs:8186-8229
    body = sphere_mesh(np.zeros(3, f32), 0.2, 8, 4)
    pos, tris = body
    n = len(pos)
    from test_oracle_static_proxy import _empty

    sc = dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=np.full(n, 1 / 0.02, f32), tris=tris,
              static_mask=None, colliders=np.zeros((0, 8), f32), params=params(False), **_empty())
    o = O.OracleSolver(sc)
    ones = np.tile([1.0, 0, 0], (n, 1))
    assert not o.set_kinematic_collider_positions(ones)  # no static collider declared
    o = O.OracleSolver(dict(sc, static_mask=np.ones(n, np.uint8)))
    assert not o.set_kinematic_collider_positions(ones[:-1])  # wrong length
    assert np.array_equal(o.positions(), pos.astype(np.float64))
    for bad in (np.nan, np.inf):
        x = ones.copy()
        x[n // 2, 1] = bad
        assert not o.set_kinematic_collider_positions(x)
        assert np.array_equal(o.positions(), pos.astype(np.float64))
    assert o.set_kinematic_collider_positions(ones)
    assert np.array_equal(o.positions(), ones)
