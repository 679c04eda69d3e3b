"""Friction on the GPU step against the oracle, through the C ABI: lagged smoothed Coulomb
friction on an analytic collider (contact.rs:613-657) and on self-contact stencils
(stencil_friction, contact.rs:659-705), compared step by step from identical states, and a
re-posed static collider dragging the cloth it carries through friction on its own move
(the fdx_override slip, implicit.rs:3063-3078; the reference's test at implicit.rs:8009-8105)."""
import numpy as np
import pytest

import oracle_py as O
from mguso import ImplicitSolver
from test_oracle_solver import grid, scene
from test_oracle_static_proxy import body_scene, cloth, sphere_mesh

pytestmark = pytest.mark.gpu
f32 = np.float32


def _pairwise(ctx, sc, steps, precision="fp32", check=None):
    """GPU and oracle steps from identical states: max relative difference over the step
    displacement and the Newton counts, per step; returns the GPU's last positions."""
    g = ImplicitSolver(ctx, sc, precision)
    o = O.OracleSolver(sc)
    rows = []
    for k in range(steps):
        p0, v0 = o.positions().copy(), o.velocities().copy()
        g.positions, g.velocities = p0.astype(f32), v0.astype(f32)
        sg = g.step(1)[0]
        so = o.step(1, check_intersection=False)[0]
        pg, po = g.positions.astype(np.float64), o.positions()
        rel = np.abs(pg - po).max() / (np.abs(po - p0).max() + 1e-12)
        rows.append((k, rel, sg["newton_iters"], so["newton_iters"], sg["status"]))
        if check:
            check(k, sg, so)
    return rows, o


def _incline(mu):
    normal = np.array([0.30, 0.954, 0.0], f32)
    normal = normal / f32(np.linalg.norm(normal))
    pos, tris = grid(5, 0.0)
    pos = pos + normal * f32(0.004)
    col = np.array([[0, 0, 0, 0, *normal, 0]], f32)
    return scene(pos, tris, 0.1, col, dt=1.0 / 240.0, stiffness=800.0, contact_dhat=0.01, contact_kappa=1.0e4,
                 friction=mu, friction_eps=1.0e-4), normal, pos


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_incline_friction_matches_oracle(ctx, precision):
    """implicit.rs:5994-6052 on the GPU: a 5 x 5 patch sliding down a tilted plane with
    mu = 0.8 and mu = 0, each step against the oracle's from the same state; the rough patch
    slides less."""
    travel = {}
    for mu in (0.8, 0.0):
        sc, normal, pos = _incline(mu)
        rows, o = _pairwise(ctx, sc, 40, precision)
        for k, rel, ng, no, stt in rows:
            assert stt == 0 and abs(ng - no) <= 1, (mu, k, ng, no)
            assert rel < 1e-3, (mu, k, rel)
        g = ImplicitSolver(ctx, sc, precision)
        g.step(200)
        d = g.positions.astype(np.float64) - pos
        travel[mu] = float(np.mean(np.linalg.norm(d - np.outer(d @ normal, normal), axis=1)))
    assert travel[0.0] > 1e-4 and travel[0.8] < travel[0.0], travel


def test_sheet_on_sheet_friction_matches_oracle(ctx):
    """implicit.rs:7281-7345 on the GPU: a sheet sliding over a pinned one with self-contact
    friction (mu = 0.9), each step against the oracle's from the same state."""
    n = 4
    lo, tl = grid(n, 0.0)
    hi, th = grid(n, 0.03)
    pos = np.concatenate([lo, hi])
    tris = np.concatenate([tl, th + n * n])
    sc = scene(pos, tris, 0.1, dt=1.0 / 240.0, stiffness=600.0, self_collision=1, contact_dhat=0.02,
               contact_kappa=1.0e3, friction=0.9, friction_eps=1.0e-4)
    sc["inv_mass"][: n * n] = 0.0
    sc["velocities"][n * n:, 0] = 0.5
    seen = []

    def check(k, sg, so):
        assert sg["stencils"] == so["stencils"], (k, sg["stencils"], so["stencils"])
        seen.append(so["stencils"])

    rows, _ = _pairwise(ctx, sc, 30, "fp32", check)
    assert max(seen) > 0
    for k, rel, ng, no, stt in rows:
        assert stt == 0 and abs(ng - no) <= 1, (k, ng, no)
        assert rel < 1e-3, (k, rel)


def test_kinematic_collider_drags_cloth_through_friction(ctx):
    """A 5 x 5 patch settled on a sphere mesh (radius 0.2) that then slides +x by 2 mm a step
    (implicit.rs:8009-8105): with mu = 0.35 the cloth follows the body through the slip of the
    body's own move, without friction it stays behind; sliding steps from identical states
    agree with the oracle's."""
    r = 0.2
    body = sphere_mesh(np.zeros(3, f32), r, 20, 10)

    def drag(mu, slide_steps, compare):
        sc, nc = body_scene(cloth(5, 0.45, 0.06), body, friction=mu, friction_eps=1.0e-4)
        g = ImplicitSolver(ctx, sc, "fp32")
        g.step(300)
        x0 = float(g.positions[:nc, 0].mean())
        centre = f32(0.0)
        o = O.OracleSolver(sc) if compare else None
        for k in range(slide_steps):
            centre = f32(centre + f32(0.002))
            target = g.positions.copy()
            target[nc:, 0] = body[0][:, 0] + centre
            if compare:
                o.set_state(g.positions.astype(np.float64), g.velocities.astype(np.float64))
                assert o.set_kinematic_collider_positions(target.astype(np.float64))
            g.set_kinematic_collider_positions(target)
            p0 = g.positions.astype(np.float64)
            g.step(1)
            if compare:
                o.step(1, check_intersection=False)
                pg, po = g.positions.astype(np.float64), o.positions()
                rel = np.abs(pg - po).max() / (np.abs(po - p0).max() + 1e-12)
                assert rel < 1e-3, (mu, k, rel)
        return float(g.positions[:nc, 0].mean()) - x0, float(centre)

    dragged, travel = drag(0.35, 100, False)
    free, _ = drag(0.0, 100, False)
    assert dragged > 0.5 * travel, (dragged, travel)
    assert free < 0.5 * dragged, (free, dragged)
    drag(0.35, 3, True)
