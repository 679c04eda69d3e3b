"""Pins (FixPair, implicit.rs:230-262, 826-838, 1755-1789, 2809-2856) and pulls (PullPair,
implicit.rs:264-282, 852-864, 2858-2872) in the CUDA step, through the C ABI: the reference's
own tests of them run on the GPU, and every step is compared with the oracle's step from the
same state (positions within 1e-3 of the step's displacement, Newton counts within +-1)."""
import numpy as np
import pytest

import oracle_py as O
from mguso import ImplicitSolver, MgusoError
from test_oracle_strain_limit import scene, sheet

pytestmark = pytest.mark.gpu


def _pair_step(g, o, pins=None, pulls=None):
    """One step of both solvers from the oracle's state (pins/pulls set on both first)."""
    p0, v0 = o.positions().copy(), o.velocities().copy()
    g.positions, g.velocities = p0.astype(np.float32), v0.astype(np.float32)
    if pins is not None:
        g.set_pins(pins)
        assert o.set_pins(pins)
    if pulls is not None:
        g.set_pulls(pulls)
        assert o.set_pulls(pulls)
    sg = g.step(1)[0]
    so = o.step(1, check_intersection=False)[0]
    pg, po = g.positions.astype(np.float64), o.positions()
    rel = np.abs(pg - po).max() / (np.abs(po - p0).max() + 1e-12)
    assert sg["status"] == 0 and abs(sg["newton_iters"] - so["newton_iters"]) <= 1, (sg, so)
    assert rel < 1e-3, rel
    return pg


@pytest.mark.parametrize("gravity,steps", [(-9.8, 40), (-2000.0, 60)])
def test_a_static_pin_holds_its_vertex_in_its_ghat_ball(ctx, gravity, steps):
    """implicit.rs:6134-6190 and 6684-6725: the pinned corner never leaves its ghat ball (the
    pin's CCD clamp), the rest of the sheet falls; each step matches the oracle's."""
    ghat = 0.01
    pos, tris = sheet(4, 0.0)
    sc = scene(pos, tris, 0.1, stiffness=5.0e2, gravity=(0.0, gravity, 0.0))
    g, o = ImplicitSolver(ctx, sc, "fp32"), O.OracleSolver(sc)
    pins = [(0, pos[0].astype(np.float64), ghat, False, 1.0)]
    worst = 0.0
    for _ in range(steps):
        p = _pair_step(g, o, pins=pins)
        worst = max(worst, float(np.linalg.norm(p[0] - pos[0])))
    assert worst <= ghat * (1 + 1e-4)
    assert float(pos[0, 1] - p[-1, 1]) > 10 * ghat


def test_a_vertex_follows_a_moving_kinematic_pin(ctx):  # implicit.rs:7114-7160
    ghat, per_step, steps = 0.02, np.float32(0.01), 60
    pos, tris = sheet(4, 0.0)
    sc = scene(pos, tris, 0.1, stiffness=5.0e2, gravity=(0.0, 0.0, 0.0))
    g, o = ImplicitSolver(ctx, sc, "mixed"), O.OracleSolver(sc)
    start = pos[0].astype(np.float64)
    for k in range(1, steps + 1):
        target = start + [0, float(per_step * np.float32(k)), 0]
        p = _pair_step(g, o, pins=[(0, target, ghat, True, 1.0)])
    want = start + [0, float(per_step * np.float32(steps)), 0]
    assert np.linalg.norm(p[0] - want) <= 2 * ghat
    assert np.linalg.norm(p[0] - start) > 0.5 * float(per_step) * steps


def test_a_weighted_pull_moves_its_vertex(ctx):  # implicit.rs:6999-7061
    def run(weight):
        pos, tris = sheet(4, 0.0)
        sc = scene(pos, tris, 0.1, stiffness=5.0e2, gravity=(0.0, 0.0, 0.0))
        g, o = ImplicitSolver(ctx, sc, "fp32"), O.OracleSolver(sc)
        pulls = None if weight is None else [(0, pos[0].astype(np.float64) + [0, 0.30, 0], weight)]
        for _ in range(40):
            p = _pair_step(g, o, pulls=pulls)
        return float(p[0, 1] - pos[0, 1])

    assert abs(run(None)) < 1e-6
    soft, firm = run(5.0), run(500.0)
    assert soft > 1e-4 and firm > soft and firm <= 0.30 * 1.10
    # the reference's recorded run: "Measured 0.3073 against a 0.30 target" (implicit.rs:7051-7054)
    assert round(firm, 4) == 0.3073, firm


def test_pins_and_pulls_are_validated_all_or_nothing(ctx):  # implicit.rs:7167-7210, 7065-7107
    pos, tris = sheet(4, 0.0)
    sc = scene(pos, tris, 0.1, stiffness=5.0e2)
    a, b = ImplicitSolver(ctx, sc, "fp32"), ImplicitSolver(ctx, sc, "fp32")
    b.set_pins([])
    b.set_pulls([])
    a.step(10)
    b.step(10)
    assert np.array_equal(a.positions, b.positions)
    n = len(pos)
    for bad in ([(n, (0, 0, 0), 0.01, False, 1.0)], [(0, (0, 0, 0), 0.0, False, 1.0)]):
        with pytest.raises(MgusoError):
            b.set_pins(bad)
    for bad in ([(n, (0, 0, 0), 1.0)], [(0, (0, 0, 0), 0.0)]):
        with pytest.raises(MgusoError):
            b.set_pulls(bad)
    b.step(1)
    a.step(1)
    assert np.array_equal(a.positions, b.positions)  # the rejected calls changed nothing
