"""Strain limiting in the CUDA step, through the C ABI, against the oracle: the per-face
barrier with its dynamic stiffness (set_strain_limit_faces, implicit.rs:1088-1121 and
2743-2807; shell_model.rs:438-640) and its bisection line search (implicit.rs:1709-1753), and
the one-sided edge limit with warp/weft ratios (strain_limit.rs:24-63, implicit.rs:798-817,
2508-2530). The reference's own tests of them run on the GPU; every step is compared with the
oracle's step from the same state."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle_py as O
from mguso import ImplicitSolver, MgusoError
from test_oracle_strain_limit import max_excess, scene, sheet
from test_gpu_step import _bsr_sum

pytestmark = pytest.mark.gpu
f32 = np.float32


def _pair_step(g, o, pins=None, tol=1e-3):
    p0, v0 = o.positions().copy(), o.velocities().copy()
    g.positions, g.velocities = p0.astype(f32), v0.astype(f32)
    if pins is not None:
        g.set_pins(pins)
        assert o.set_pins(pins)
    sg = g.step(1)[0]
    so = o.step(1, check_intersection=False)[0]
    pg, po = g.positions.astype(np.float64), o.positions()
    rel = np.abs(pg - po).max() / (np.abs(po - p0).max() + 1e-12)
    assert sg["status"] == 0 and abs(sg["newton_iters"] - so["newton_iters"]) <= 1, (sg, so)
    assert rel < tol, rel
    return pg


def _pulled_pins(pos, step):
    """The reference's pulled sheet (implicit.rs:6397-6560): the left column of a 4 x 4 sheet
    held by static pins, the right one dragged outward 4 mm per step by kinematic pins."""
    cols = 4
    right = [j * cols + cols - 1 for j in range(cols)]
    left = [j * cols for j in range(cols)]
    push = np.float32(0.004) * np.float32(step)
    pins = [(v, pos[v].astype(np.float64) + [float(push), 0, 0], 0.02, True, 1.0) for v in right]
    pins += [(v, pos[v].astype(np.float64), 0.02, False, 1.0) for v in left]
    return pins


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
@pytest.mark.parametrize("membrane", [5.0, 5.0e3])
def test_pulled_sheet_steps_match_oracle_with_the_barrier(ctx, precision, membrane):
    """implicit.rs:6397-6567 step by step: 40 steps of the pulled sheet with the face barrier
    at a 5 % limit, each GPU step from the oracle's state, and the sheet ends inside 1.02 of
    the limit (the elastic half of the stiffness does not weaken it, at either membrane).

    The tolerance is 2e-2 of the step's displacement, not 1e-3: the barrier's stiffness reaches
    mass / d^2 ~ 4e8 against m / h^2 = 360, and the reference's test parameters stop Newton at
    4 iterations, so a step depends on the linear solver's rounding. Two oracle runs of this
    sequence that differ only in the preconditioner (block Jacobi vs Schwarz) differ by up to
    4e-2 (membrane 5) and 8e-2 (membrane 5e3) of the displacement at the default PCG
    tolerance, and by 3e-3 at a PCG tolerance of 1e-8."""
    limit = 0.05
    pos, tris = sheet(4, 0.0)
    sc = scene(pos, tris, 0.1, stiffness=membrane, gravity=(0.0, 0.0, 0.0), barrier_kind=1)
    g, o = ImplicitSolver(ctx, sc, precision), O.OracleSolver(sc)
    assert g.set_strain_limit_faces(tris, [limit] * len(tris), [1.0] * len(tris)) == len(tris)
    assert o.set_strain_limit_faces(tris, [limit] * len(tris), [1.0] * len(tris)) == len(tris)
    for step in range(1, 41):
        p = _pair_step(g, o, pins=_pulled_pins(pos, step), tol=2e-2)
    assert np.all(np.isfinite(p))
    assert max_excess(pos.astype(np.float64), p, tris) <= limit * 1.02


def test_pulled_sheet_free_run_enforces_the_limit(ctx):
    """implicit.rs:6473-6567 run freely on the GPU: without the barrier the sheet stretches
    far past 5 %; with it the worst face ends within 1.02 of the limit, and the final
    excess agrees with the oracle's own run (the reference records 0.0500 and 0.8181)."""
    limit = 0.05
    out = {}
    for with_barrier in (False, True):
        pos, tris = sheet(4, 0.0)
        sc = scene(pos, tris, 0.1, stiffness=5.0, gravity=(0.0, 0.0, 0.0), barrier_kind=1)
        g = ImplicitSolver(ctx, sc, "fp32")
        if with_barrier:
            assert g.set_strain_limit_faces(tris, [limit] * len(tris), [1.0] * len(tris)) == len(tris)
        for step in range(1, 41):
            g.set_pins(_pulled_pins(pos, step))
            st = g.step(1)[0]
            assert st["status"] == 0
        out[with_barrier] = max_excess(pos.astype(np.float64), g.positions.astype(np.float64), tris)
    assert out[False] > 1.5 * limit and out[True] <= limit * 1.02
    assert round(out[True], 4) == 0.0500, out
    assert abs(out[False] - 0.8181) < 5e-3, out


def test_the_barrier_assembly_matches_oracle(ctx):
    """One Newton system of a sheet stretched 3-4 % with the face barrier on: every matrix
    and right-hand-side entry agrees with the oracle's to a few FP32 ulps of the largest."""
    limit = 0.05
    pos, tris = sheet(5, 0.0)
    sc = scene(pos, tris, 0.1, stiffness=50.0, gravity=(0.0, -9.8, 0.0), barrier_kind=1)
    sc["inv_mass"][0] = 0.0  # one pinned corner: its blocks stay outside the system
    nv = len(pos)
    g, o = ImplicitSolver(ctx, sc, "fp32"), O.OracleSolver(sc)
    assert g.set_strain_limit_faces(tris, [limit] * len(tris), [2.0] * len(tris)) == len(tris)
    assert o.set_strain_limit_faces(tris, [limit] * len(tris), [2.0] * len(tris)) == len(tris)
    rng = np.random.default_rng(3)
    x1 = (pos * np.array([1.035, 1.0, 1.03], f32) + rng.uniform(-2e-4, 2e-4, pos.shape)).astype(f32)
    x1[0] = pos[0]
    xt = pos.copy()
    a = g.assemble(x1, xt)
    (orp, oci, ovv), orhs = o.assemble(x1, xt)
    ao = sp.csr_matrix((ovv.astype(np.float64), oci.astype(np.int64), orp.astype(np.int64)), shape=(3 * nv, 3 * nv))
    ag = _bsr_sum(a, nv)
    # the barrier adds to the diagonal blocks well beyond the elastic terms alone
    assert abs(ao).max() > 10 * 0.1 / (1 / 60.0) ** 2
    ulp = np.spacing(np.float32(abs(ao).max()))
    assert abs(ag - ao).max() <= 16 * ulp, (abs(ag - ao).max(), ulp)
    assert np.abs(a["rhs"] - orhs).max() <= 1e-5 * np.abs(orhs).max()


def test_the_line_search_bisects_onto_the_limit(ctx):
    """implicit.rs:1709-1753: a 10 cm jump of the right column is cut back to the step
    fraction the oracle finds, which lands within 1 % below the limit; a step inside the
    limit is not clamped."""
    pos, tris = sheet(4, 0.0)
    sc = scene(pos, tris, 0.1, stiffness=5.0, gravity=(0.0, 0.0, 0.0), barrier_kind=1)
    g, o = ImplicitSolver(ctx, sc, "fp32"), O.OracleSolver(sc)
    g.set_strain_limit_faces(tris, [0.05] * len(tris), [1.0] * len(tris))
    o.set_strain_limit_faces(tris, [0.05] * len(tris), [1.0] * len(tris))
    dx = np.zeros((len(pos), 3), f32)
    dx[3::4, 0] = 0.1
    t, _ = g.ccd(pos, dx)
    to = o.ccd(dx)
    assert 0.0 < t[0] < 1.0 and abs(float(t[0]) - to) <= 1e-6, (t, to)
    reached = max_excess(pos.astype(np.float64), pos + float(t[0]) * dx, tris)
    assert 0.05 * 0.99 < reached < 0.05
    t2, _ = g.ccd(pos, 0.01 * dx)
    assert t2[0] == 1.0


def test_strain_limit_faces_are_validated(ctx):  # implicit.rs:1088-1121
    pos, tris = sheet(3, 0.0)
    g = ImplicitSolver(ctx, scene(pos, tris, 0.1), "fp32")
    with pytest.raises(ValueError):
        g.set_strain_limit_faces(tris, [0.05] * (len(tris) - 1), [1.0] * len(tris))
    limits = [0.05] * len(tris)
    limits[0] = 0.0  # "no limit on this face"
    masses = [1.0] * len(tris)
    masses[1] = 0.0
    assert g.set_strain_limit_faces(tris, limits, masses) == len(tris) - 2
    with pytest.raises(MgusoError):
        g.set_strain_limit_faces([[0, 1, 99]], [0.05], [1.0])  # out of range
    with pytest.raises(MgusoError):
        g.set_strain_limit_faces([[0, 2, 6]], [0.05], [1.0])  # 0, 2 and 6 share no element
    assert g.set_strain_limit_faces(np.zeros((0, 3), np.uint32), [], []) == 0


def _edge_pair(ratio, weft=0.0, uvs=None):
    """Two edges (0, 1) and (2, 3), their first ends pinned, pulled along +x by a 2 m/s^2
    field (implicit.rs:4837-4925)."""
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]], f32)
    sc = scene(pos, np.zeros((0, 3), np.uint32), 1.0, gravity=(2.0, 0.0, 0.0), newton_iters=8, stiffness=0.0)
    sc["inv_mass"][[0, 2]] = 0.0
    o = O.OracleSolver(sc)
    o.set_stretch_edges([[0, 1], [2, 3]])
    o.set_limits(strain_limit_ratio=ratio, strain_limit_k=5000.0, strain_limit_ratio_weft=weft, uvs=uvs)
    gs = dict(sc, stretch_edges=np.array([[0, 1], [2, 3]], np.uint32),
              params=dict(sc["params"], strain_limit_ratio=ratio, strain_limit_k=5000.0,
                          strain_limit_ratio_weft=weft))
    if uvs is not None:
        gs["uvs"] = np.array(uvs, f32)
    return gs, o


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_anisotropic_edge_limit_matches_oracle(ctx, precision):  # implicit.rs:4837-4885
    gs, o = _edge_pair(1.1, weft=1.5, uvs=[[0, 0], [1, 0], [0, 0], [0, 1]])
    g = ImplicitSolver(ctx, gs, precision)
    for _ in range(300):
        p0, v0 = o.positions().copy(), o.velocities().copy()
        g.positions, g.velocities = p0.astype(f32), v0.astype(f32)
        sg = g.step(1)[0]
        so = o.step(1, check_intersection=False)[0]
        assert sg["status"] == 0 and abs(sg["newton_iters"] - so["newton_iters"]) <= 1
        po = o.positions()
        assert np.abs(g.positions - po).max() <= 1e-3 * (np.abs(po - p0).max() + 1e-6)
    p = g.positions.astype(np.float64)
    warp, weft = np.linalg.norm(p[1] - p[0]), np.linalg.norm(p[3] - p[2])
    assert 1.1 <= warp < 1.25 and 1.5 <= weft < 1.65 and weft > warp + 0.2


def test_edge_limit_caps_stretch_under_load(ctx):  # implicit.rs:4888-4925
    def length(ratio):
        pos = np.array([[0, 0, 0], [1, 0, 0]], f32)
        sc = scene(pos, np.zeros((0, 3), np.uint32), 1.0, gravity=(2.0, 0.0, 0.0), newton_iters=8, stiffness=0.0)
        sc["inv_mass"][0] = 0.0
        sc = dict(sc, stretch_edges=np.array([[0, 1]], np.uint32),
                  params=dict(sc["params"], strain_limit_ratio=ratio, strain_limit_k=5000.0))
        g = ImplicitSolver(ctx, sc, "fp32")
        g.step(300)
        p = g.positions.astype(np.float64)
        return float(np.linalg.norm(p[1] - p[0]))

    assert 1.2 <= length(1.2) < 1.3
    assert length(0.0) > 3.0
