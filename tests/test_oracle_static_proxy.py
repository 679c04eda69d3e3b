"""Static mesh colliders in the CPU oracle (the torso's path: signed point-triangle gap from
mesh-wide pseudonormals, winding check, Rayleigh-stiffened stencils against pinned
triangles), pinned by the reference's own static-proxy tests (implicit.rs:7382-7990) at
their own parameters: a 5 x 5 cloth patch dropped for 400 steps at dt = 1/240 on
triangulated planes, cubes and UV spheres whose vertices are all pinned.
"""
import functools

import numpy as np
import oracle_py as O
import pytest

from mguso import scenes

f32 = np.float32
DHAT, KAPPA, STEPS = 0.02, 2.0e3, 400


def params(self_collision, **kw):
    """The tests' params(self_collision) (implicit.rs:7463-7473) over ImplicitParams::default(),
    stepped with CgCpu (block Jacobi)."""
    p = dict(dt=1.0 / 240.0, stiffness=500.0, gravity=(0.0, -9.8, 0.0), contact_dhat=DHAT, contact_kappa=KAPPA,
             self_collision=1 if self_collision else 0, newton_iters=4, bend_stiffness=0.0, contact_rayleigh=0,
             barrier_kind=0, precond=1)
    p.update(kw)
    return scenes.default_params(**p)


def plane_mesh(n, y0, half):
    """implicit.rs:7382-7403: an n x n grid over [-half, half]^2 at height y0, in f32."""
    step = f32(2.0) * f32(half) / f32(n - 1)
    pos = [(f32(-half) + f32(i) * step, f32(y0), f32(-half) + f32(j) * step) for j in range(n) for i in range(n)]
    tris = []
    for j in range(n - 1):
        for i in range(n - 1):
            v = j * n + i
            r = v + n
            tris += [(v, v + 1, r), (r, v + 1, r + 1)]
    return np.array(pos, f32), np.array(tris, np.uint32)


def floor_mesh(n, y0, half):
    """implicit.rs:7411-7425: the plane wound so every normal points +Y."""
    pos, tris = plane_mesh(n, y0, half)
    out = []
    for t in tris:
        a, b, c = pos[t]
        ny = (b - a)[2] * (c - a)[0] - (b - a)[0] * (c - a)[2]
        out.append(t if ny > 0 else t[[0, 2, 1]])
    return pos, np.array(out, np.uint32)


def sphere_mesh(c, r, seg, rings):
    """implicit.rs:7429-7448: a UV sphere (pole rows repeated, as the reference builds it)."""
    pos, tris = [], []
    for ri in range(rings + 1):
        phi = f32(np.pi) * f32(ri) / f32(rings)
        for si in range(seg):
            th = f32(2 * np.pi) * f32(si) / f32(seg)
            d = np.array([np.sin(phi) * np.cos(th), np.cos(phi), np.sin(phi) * np.sin(th)], f32)
            pos.append(np.asarray(c, f32) + f32(r) * d)
    for ri in range(rings):
        for si in range(seg):
            a = ri * seg + si
            b = ri * seg + (si + 1) % seg
            tris += [(a, b, a + seg), (a + seg, b, b + seg)]
    return np.array(pos, f32), np.array(tris, np.uint32)


def cloth(k, y0, extent):
    return plane_mesh(k, y0, extent)


def mean_y(p):
    return float(functools.reduce(lambda s, y: f32(s + y), p[:, 1].astype(f32), f32(0)) / f32(len(p)))


def _empty():
    si, sw, skl = scenes._empty_stitches()
    return dict(shell_faces=np.zeros((0, 3), np.uint32), stitch_idx=si, stitch_w=sw, stitch_kl=skl)


def body_scene(cloth_mesh, body, **kw):
    """Cloth first, then the body with every vertex pinned and marked static
    (drop_on_mesh, implicit.rs:7478-7508)."""
    nc = len(cloth_mesh[0])
    pos = np.concatenate([cloth_mesh[0], body[0]]).astype(f32)
    tris = np.concatenate([cloth_mesh[1].astype(np.int64), body[1].astype(np.int64) + nc]).astype(np.uint32)
    im = np.full(len(pos), 1.0 / 0.02, f32)
    im[nc:] = 0.0
    mask = np.zeros(len(pos), np.uint8)
    mask[nc:] = 1
    return dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=im, tris=tris, static_mask=mask,
                colliders=np.zeros((0, 8), f32), params=params(True, **kw), **_empty()), nc


def drop_on_mesh(cloth_mesh, body):
    sc, nc = body_scene(cloth_mesh, body)
    o = O.OracleSolver(sc)
    o.step(STEPS, check_intersection=False)
    return o.positions()[:nc]


def drop_on_analytic(cloth_mesh, collider):
    """implicit.rs:7511-7519; collider = (kind, point/centre, normal, radius)."""
    pos, tris = cloth_mesh
    kind, a, n, r = collider
    sc = dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=np.full(len(pos), 1.0 / 0.02, f32), tris=tris,
              static_mask=None, colliders=np.array([[kind, *a, *n, r]], f32), params=params(False), **_empty())
    o = O.OracleSolver(sc)
    o.step(STEPS, check_intersection=False)
    return o.positions()


HALF_SPACE = (0, (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 0.0)


def test_a_triangulated_plane_matches_the_analytic_half_space():  # implicit.rs:7543-7545, 7761-7797
    start = 0.25
    patch = cloth(5, start, 0.2)
    mesh = drop_on_mesh(patch, floor_mesh(9, 0.0, 0.6))
    analytic = drop_on_analytic(patch, HALF_SPACE)
    assert np.all(np.isfinite(mesh)) and np.all(np.isfinite(analytic))
    my, ay = mean_y(mesh), mean_y(analytic)
    assert my < 0.5 * start and ay < 0.5 * start
    assert mesh[:, 1].min() > -DHAT and analytic[:, 1].min() > -DHAT
    assert abs(my - ay) < DHAT


def test_a_triangulated_plane_recovers_from_initial_penetration_like_the_analytic_one():  # implicit.rs:7579-7612
    for start in (-0.00001, -0.0001, -0.001):
        mesh = drop_on_mesh(cloth(5, start, 0.2), floor_mesh(9, 0.0, 0.6))
        assert np.all(np.isfinite(mesh))
        my, ny = mean_y(mesh), float(mesh[:, 1].min())
        assert ny > -DHAT and my < DHAT, (start, my, ny)
    free = drop_on_analytic(cloth(5, -0.00001, 0.2), (0, (0.0, -1000.0, 0.0), (0.0, 1.0, 0.0), 0.0))
    assert free[:, 1].min() < -1.0


def cube_mesh():
    """implicit.rs:7614-7648: the unit cube, every face turned to point away from the centre."""
    pos = np.array([[0, 0, 0], [1, 0, 0], [1, 0, 1], [0, 0, 1], [0, 1, 0], [1, 1, 0], [1, 1, 1], [0, 1, 1]], f32)
    tris = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4], [3, 6, 2], [3, 7, 6],
                     [0, 4, 7], [0, 7, 3], [1, 2, 6], [1, 6, 5]], np.uint32)
    ctr = np.full(3, 0.5, f32)
    for t in tris:
        a, b, c = pos[t]
        if np.dot(np.cross(b - a, c - a), (a + b + c) / f32(3) - ctr) < 0:
            t[[1, 2]] = t[[2, 1]]
    return pos, tris


def test_a_vertex_outside_a_closed_collider_gets_no_negative_gap_from_any_facet():  # implicit.rs:7686-7759
    cube_pos, cube_tris = cube_mesh()
    cloth_pos = np.array([[0.5, 1.0001, 0.9991], [0.52, 1.0002, 0.9991], [0.5, 1.0002, 0.9971],
                          [0.5, 0.998, 0.9991]], f32)
    inside_v = 3
    sc, nc = body_scene((cloth_pos, np.array([[0, 1, 2], [0, 2, 3]], np.uint32)), (cube_pos, cube_tris),
                        contact_dhat=0.005)
    o = O.OracleSolver(sc)
    idx, gap = o.stencils()
    body = [(i, g) for i, g in zip(idx, gap) if i[0] < nc and all(int(v) >= nc for v in i[1:])]
    assert sum(1 for i, _ in body if i[0] != inside_v) >= 2
    inside_seen = 0
    for i, g in body:
        if i[0] == inside_v:
            inside_seen += 1
            assert g < 0.0, (i, g)
        else:
            assert g >= 0.0, (i, g)
    assert inside_seen > 0


def _cube(flip):
    lo, hi = -0.5, 0.5
    pos = np.array([(lo, lo, lo), (hi, lo, lo), (hi, lo, hi), (lo, lo, hi), (lo, hi, lo), (hi, hi, lo), (hi, hi, hi),
                    (lo, hi, hi)], f32)
    tris = np.array([[0, 1, 2], [0, 2, 3], [4, 7, 6], [4, 6, 5], [0, 4, 5], [0, 5, 1], [2, 6, 7], [2, 7, 3],
                     [0, 3, 7], [0, 7, 4], [1, 5, 6], [1, 6, 2]], np.uint32)
    vol = sum(float(np.dot(np.cross(pos[t[0]], pos[t[1]]), pos[t[2]])) / 6.0 for t in tris)
    assert vol > 0.9
    if flip:
        tris = tris[:, [0, 2, 1]].copy()
    return pos, tris


def _accepted(body):
    pos, tris = body
    sc = dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=np.zeros(len(pos), f32), tris=tris,
              static_mask=np.ones(len(pos), np.uint8), colliders=np.zeros((0, 8), f32), params=params(True),
              **_empty())
    return O.OracleSolver(sc).counts()["collider_tris"] > 0


def test_an_inward_wound_collider_is_rejected_rather_than_inverting_contact():  # implicit.rs:7805-7881
    assert _accepted(_cube(False))
    assert not _accepted(_cube(True))
    assert _accepted(floor_mesh(3, 0.0, 0.5))


def _point_triangle_distance(p, a, b, c):
    return O.point_tri(np.array([p, a, b, c], f32))[0]


def test_cloth_rests_in_barrier_contact_with_a_curved_static_proxy():  # implicit.rs:7896-7943
    c, r = np.zeros(3, f32), 0.2
    body = sphere_mesh(c, r, 24, 12)
    settled = drop_on_mesh(cloth(5, 0.45, 0.06), body)
    assert np.all(np.isfinite(settled))
    assert mean_y(settled) < 0.35
    nearest = min(min(_point_triangle_distance(p, *body[0][t]) for t in body[1]) for p in settled)
    facet = max(float((body[0][t].max(0) - body[0][t].min(0)).max()) for t in body[1])
    assert nearest <= DHAT + facet
    sag = r * (1.0 - np.cos(np.pi / 24.0))
    assert np.linalg.norm(settled - c, axis=1).min() > r - sag


def test_cloth_on_a_static_body_mesh_is_finite_outside_and_deterministic():  # implicit.rs:7949-7990
    body = sphere_mesh(np.zeros(3, f32), 0.2, 20, 10)
    patch = cloth(5, 0.45, 0.06)
    a, b = drop_on_mesh(patch, body), drop_on_mesh(patch, body)
    assert np.all(np.isfinite(a))
    assert mean_y(a) < 0.35
    sag = 0.2 * (1.0 - np.cos(np.pi / 20.0))
    assert np.linalg.norm(a, axis=1).min() > 0.2 - DHAT - sag
    assert np.array_equal(a, b)
