"""GPU implicit step vs the CPU oracle of the reference's step, through the C ABI.

Per-step parity is compared from identical states: both solvers start every compared step
from the same positions and velocities, and the resulting positions must agree within a
relative tolerance of the step's displacement. Newton iteration counts must agree within
+-1 over the run."""
import numpy as np
import pytest

import oracle_py as O
from mguso import ImplicitSolver, scenes

pytestmark = pytest.mark.gpu


def sphere_scene(n=16, height=0.34, **kw):
    return scenes.sheet_on_sphere(n, side=0.5, height=height, **kw)


def newton_bound(sg, so, tol):
    """The position bound of a contact step: tol when the two Newton loops stopped after the
    same number of iterations; 2e-2 when they stopped one iteration apart, since the extra
    iteration moves the iterate by up to the Newton tolerance (1e-3 dt, 1.7e-5 m), which is
    up to 1e-3 of a falling sheet's step and 6e-3 of a resting sheet's."""
    return tol if sg["newton_iters"] == so["newton_iters"] else 2e-2


def run_pair(ctx, sc, steps, precision="mixed"):
    g = ImplicitSolver(ctx, sc, precision)
    o = O.OracleSolver(sc)
    out = []
    for k in range(steps):
        p0 = o.positions().copy()
        v0 = o.velocities().copy()
        g.positions = p0.astype(np.float32)
        g.velocities = v0.astype(np.float32)
        sg = g.step(1)[0]
        so = o.step(1, check_intersection=True)[0]
        pg = g.positions.astype(np.float64)
        po = o.positions()
        disp = np.abs(po - p0).max() + 1e-12
        # penetration_free includes the self-intersection scan on both sides
        assert bool(sg["penetration_free"]) == bool(so["penetration_free"]), (k, sg, so)
        out.append((k, sg, so, np.abs(pg - po).max() / disp))
        print(f"step {k}: newton gpu {sg['newton_iters']} oracle {so['newton_iters']} stencils "
              f"{sg['stencils']}/{so['stencils']} t_min {sg['t_min']:.4f}/{so['t_min']:.4f} rel {out[-1][3]:.3e}")
    return g, o, out


def test_scene_topology_matches_oracle(ctx):
    sc = sphere_scene(12)
    g = ImplicitSolver(ctx, sc)
    o = O.OracleSolver(sc)
    gi, oi = g.info(), o.counts()
    assert gi["hinges"] == oi["hinges"] and gi["shells"] == oi["shells"] and gi["edges"] == oi["edges"]


def test_free_fall_step_matches_oracle(ctx):  # engine-gpu pcg.rs:848-901 (the GPU-solved step vs the CPU one)
    sc = sphere_scene(12, height=0.6)
    g, o, out = run_pair(ctx, sc, 3)
    for k, sg, so, rel in out:
        assert sg["status"] == 0 and sg["all_finite"]
        assert abs(sg["newton_iters"] - so["newton_iters"]) <= 1
        assert rel < 1e-3, (k, rel)


def test_sphere_contact_steps_match_oracle(ctx):
    """Steps through first contact with the sphere (collider barrier + CCD clamp)."""
    sc = sphere_scene(12)
    o = O.OracleSolver(sc)
    o.step(6, check_intersection=False)  # fall until just above the sphere
    sc2 = dict(sc)
    sc2["positions"] = o.positions().astype(np.float32)
    sc2["velocities"] = o.velocities().astype(np.float32)
    g, o2, out = run_pair(ctx, sc2, 8)
    for k, sg, so, rel in out:
        assert sg["status"] == 0 and sg["all_finite"] and sg["penetration_free"]
        assert abs(sg["newton_iters"] - so["newton_iters"]) <= 1, (k, sg["newton_iters"], so["newton_iters"])
        assert rel < newton_bound(sg, so, 1e-3), (k, rel)
    assert any(so["num_contacts"] > 0 for _, _, so, _ in out)


def test_drape_invariants_on_gpu(ctx):
    sc = sphere_scene(16)
    g = ImplicitSolver(ctx, sc, "mixed")
    st = g.step(20)
    p = g.positions
    assert all(s["all_finite"] and s["penetration_free"] and s["status"] == 0 for s in st)
    assert np.linalg.norm(p, axis=1).min() >= 0.3 - 1e-6
    assert p[:, 1].min() < 0.33


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_self_contact_stencils_and_step(ctx, precision):
    """Two stacked sheets 0.6 mm apart: self-contact stencils active from the first
    iteration; the GPU step matches the oracle's from the same state. The first step (11 Newton
    iterations over 1 286 stencils at 0.6 mm, d-hat 1 mm) has measured 1.9e-4 (FP32) and
    3.4e-4 (mixed) of its displacement away from the oracle's, against 1e-5 or less for the
    other steps: its barrier stiffness magnifies the rounding-level differences of the PCG
    solutions (tolerance 1e-4 per Newton iteration) into the iterate, so the bound is 2e-3."""
    rng = np.random.default_rng(4)
    n = 10
    sc = scenes.sheet_on_sphere(n, side=0.05, height=0.5, jitter=0.0, dhat=1e-3)
    pos = sc["positions"]
    top = pos.copy()
    top[:, 1] += 6e-4
    top[:, 0] += 2e-3
    top += rng.uniform(-1e-4, 1e-4, top.shape).astype(np.float32)
    sc["positions"] = np.concatenate([pos, top]).astype(np.float32)
    sc["velocities"] = np.zeros_like(sc["positions"])
    sc["tris"] = np.concatenate([sc["tris"], sc["tris"] + n * n]).astype(np.uint32)
    sc["shell_faces"] = sc["tris"].copy()
    sc["inv_mass"] = np.concatenate([sc["inv_mass"], sc["inv_mass"]])
    sc["colliders"] = np.zeros((0, 8), np.float32)
    g, o, out = run_pair(ctx, sc, 3, precision)
    for k, sg, so, rel in out:
        assert sg["stencils"] == so["stencils"], (k, sg["stencils"], so["stencils"])
        assert abs(sg["newton_iters"] - so["newton_iters"]) <= 1
        assert rel < newton_bound(sg, so, 2e-3), (k, rel)


def coarse_sheath(**kw):
    """The garment configuration at a coarser resolution (30 mm edges, 1 740-triangle torso)."""
    return scenes.sheath_on_torso(edge=0.03, torso_res=(30, 29), **kw)


def _mid_step_state(sc):
    """Positions after the oracle's first Newton iteration of step 0 (seams closing, cloth
    near itself and the torso) and the step's inertia target."""
    sc1 = dict(sc)
    sc1["params"] = dict(sc["params"], newton_iters=1)
    o = O.OracleSolver(sc1)
    o.step(1, check_intersection=False)
    x1 = o.positions().astype(np.float32)
    x0 = sc["positions"].astype(np.float32)
    dt = sc["params"]["dt"]
    grav = np.array(sc["params"]["gravity"], np.float32)
    free = sc["inv_mass"][:, None] > 0
    xt = (x0 + np.where(free, dt * sc["velocities"] + dt * dt * grav[None, :], 0)).astype(np.float32)
    return x1, xt


def _bsr_sum(a, nv):
    import scipy.sparse as sp

    rp, col, val = a["ps"]
    m = sp.bsr_matrix((val.astype(np.float64), col.astype(np.int64), rp.astype(np.int64)), shape=(3 * nv, 3 * nv))
    crp, ccol, cval = a["c"]
    if len(ccol):
        m = m + sp.bsr_matrix((cval.astype(np.float64), ccol.astype(np.int64), crp.astype(np.int64)),
                              shape=(3 * nv, 3 * nv))
    return m.tocsr()


def test_sheath_assembly_matches_oracle_fp32(ctx):
    """One Newton system of the seamed sheath (stitches, StVK shells, hinges, static torso
    collider and self contact): the FP32 stencil set equals the oracle's, and every matrix
    and right-hand-side entry agrees to a few FP32 ulps (the contact sums are added to the
    elastic slot as one term, the reference adds them one by one)."""
    import scipy.sparse as sp

    sc = coarse_sheath()
    nv = sc["positions"].shape[0]
    x1, xt = _mid_step_state(sc)
    g = ImplicitSolver(ctx, sc, "fp32")
    a = g.assemble(x1, xt)
    gi, gk, gd = g.stencils()
    o = O.OracleSolver(sc)
    o.set_state(x1, sc["velocities"])
    oi, od = o.stencils()
    assert a["stencils"] > 100
    assert set(map(tuple, gi.tolist())) == set(map(tuple, oi.tolist()))
    (orp, oci, ovv), orhs = o.assemble(x1, xt)
    ao = sp.csr_matrix((ovv.astype(np.float64), oci.astype(np.int64), orp.astype(np.int64)), shape=(3 * nv, 3 * nv))
    ag = _bsr_sum(a, nv)
    d = abs(ag - ao)
    ulp = np.spacing(np.float32(abs(ao).max()))
    assert d.max() <= 8 * ulp, (d.max(), ulp)
    assert np.abs(a["rhs"] - orhs).max() <= 1e-5 * np.abs(orhs).max()


def test_sheath_steps_match_oracle(ctx):  # engine-gpu pcg.rs:905-965 (Schwarz-solved steps vs the CPU)
    """Seamed sheath steps from identical states: Newton counts within +-1, positions within
    1e-3 of the step's displacement (FP32 and mixed)."""
    sc = coarse_sheath()
    for prec in ("fp32", "mixed"):
        g, o, out = run_pair(ctx, sc, 3, prec)
        for k, sg, so, rel in out:
            assert sg["status"] == 0 and sg["all_finite"] and sg["penetration_free"]
            assert abs(sg["newton_iters"] - so["newton_iters"]) <= 1, (prec, k)
            assert rel < 1e-3, (prec, k, rel)
        assert max(sg["stencils"] for _, sg, _, _ in out) > 100


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
@pytest.mark.parametrize("precond", [2, 1])
def test_persistent_pcg_matches_per_kernel_pcg(ctx, precision, precond):
    """The fused two-kernel PCG (mode 0), the per-kernel PCG (mode 1) and the one-launch
    persistent PCG (mode 2) are the same iteration; they differ only in the order of
    dot-product partial sums, so two drape steps agree to the Newton tolerance and their PCG
    iteration counts stay close."""
    sc = coarse_sheath()
    sc["params"] = dict(sc["params"], precond=precond)
    runs = []
    for mode in (0, 1, 2):
        s2 = dict(sc)
        s2["params"] = dict(sc["params"], pcg_mode=mode)
        g = ImplicitSolver(ctx, s2, precision)
        st = g.step(2)
        runs.append((g.positions.astype(np.float64), st))
    (p1, s1) = runs[1]
    disp = np.abs(p1 - sc["positions"]).max()
    for p0, s0 in (runs[0], runs[2]):
        assert np.abs(p0 - p1).max() <= 1e-3 * disp
        for a, b in zip(s0, s1):
            assert a["status"] == 0 and b["status"] == 0
            assert abs(a["newton_iters"] - b["newton_iters"]) <= 1
            assert abs(a["max_cg_iters"] - b["max_cg_iters"]) <= max(5, b["max_cg_iters"] // 10)


def graded_coarse(n=3):
    widths = (0.50, 0.60, 0.70, 0.55, 0.65, 0.75)[:n]
    scales = (0.9, 1.02, 1.14, 0.96, 1.08, 1.2)[:n]
    return [scenes.sheath_on_torso(edge=0.03, torso_res=(30, 29), width=w, torso_scale=t) for w, t in zip(widths, scales)]


@pytest.mark.parametrize("pcg_mode", [0, 2])
@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_batch_matches_instances_run_alone(ctx, precision, pcg_mode):
    """Three graded sheaths stepped as one batch give each instance the trajectory it has when
    stepped alone: the element, stencil and CCD work is per instance, and only the order of
    the PCG's dot-product partial sums differs."""
    from mguso import ImplicitBatch

    scs = graded_coarse(3)
    for sc in scs:
        sc["params"] = dict(sc["params"], pcg_mode=pcg_mode)
    b = ImplicitBatch(ctx, scs, precision)
    assert b.ninst == 3
    bst = b.step(3)
    for k, sc in enumerate(scs):
        g = ImplicitSolver(ctx, sc, precision)
        gst = g.step(3)
        pa, pb = g.positions.astype(np.float64), b.instance_positions(k).astype(np.float64)
        disp = np.abs(pa - sc["positions"]).max()
        assert np.abs(pa - pb).max() <= 1e-3 * disp, (k, np.abs(pa - pb).max(), disp)
        for i in range(3):
            assert bst[i][k]["status"] == 0 and bst[i][k]["penetration_free"]
            assert abs(bst[i][k]["newton_iters"] - gst[i]["newton_iters"]) <= 1
        g.close()


def test_batch_instance_matches_oracle(ctx):
    """Every instance of a batch against the oracle of that instance alone, step by step from
    identical states (the batch's state set from the oracles' before each step): positions
    within 1e-3 of each instance's step displacement, Newton counts within +-1."""
    from mguso import ImplicitBatch

    scs = graded_coarse(2)
    b = ImplicitBatch(ctx, scs, "mixed")
    os_ = [O.OracleSolver(sc) for sc in scs]
    off = b.offsets
    for i in range(3):
        p0 = [o.positions().copy() for o in os_]
        b.positions = np.concatenate(p0).astype(np.float32)
        b.velocities = np.concatenate([o.velocities() for o in os_]).astype(np.float32)
        st = b.step(1)[0]
        for k, o in enumerate(os_):
            so = o.step(1, check_intersection=False)[0]
            assert st[k]["status"] == 0 and abs(st[k]["newton_iters"] - so["newton_iters"]) <= 1, (i, k)
            pb = b.positions[off[k]:off[k + 1]].astype(np.float64)
            po = o.positions()
            rel = np.abs(pb - po).max() / (np.abs(po - p0[k]).max() + 1e-12)
            print(f"step {i} instance {k}: rel {rel:.3e}")
            assert rel < 1e-3, (i, k, rel)


def test_kinematic_collider_repose_matches_oracle(ctx):
    """The torso moved between steps (0.3 mm sideways, 0.2 mm up) on both solvers: its
    vertices take the new positions, the following steps agree with the oracle's from identical
    states, and a non-finite collider row is refused with nothing written
    (implicit.rs:1368-1398)."""
    from mguso import MgusoError

    sc = coarse_sheath()
    body = np.asarray(sc["static_mask"], bool)
    g = ImplicitSolver(ctx, sc, "mixed")
    o = O.OracleSolver(sc)
    g.step(1)
    o.step(1, check_intersection=False)
    x = o.positions().astype(np.float32)
    x[body] += np.float32([3e-4, 2e-4, 0.0])
    bad = x.copy()
    bad[np.flatnonzero(body)[0], 0] = np.nan
    before = g.positions.copy()
    with pytest.raises(MgusoError):
        g.set_kinematic_collider_positions(bad)
    assert np.array_equal(g.positions, before)
    g.positions = o.positions().astype(np.float32)
    g.velocities = o.velocities().astype(np.float32)
    g.set_kinematic_collider_positions(x)
    assert o.set_kinematic_collider_positions(x.astype(np.float64))
    assert np.array_equal(g.positions[body], x[body])
    assert np.array_equal(g.positions[~body], o.positions()[~body].astype(np.float32))
    for k in range(2):
        p0, v0 = o.positions().copy(), o.velocities().copy()
        g.positions = p0.astype(np.float32)
        g.velocities = v0.astype(np.float32)
        sg = g.step(1)[0]
        so = o.step(1, check_intersection=False)[0]
        pg, po = g.positions.astype(np.float64), o.positions()
        rel = np.abs(pg - po).max() / (np.abs(po - p0).max() + 1e-12)
        assert sg["status"] == 0 and sg["penetration_free"]
        assert abs(sg["newton_iters"] - so["newton_iters"]) <= 1
        assert rel < 1e-3, (k, rel)


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_ccd_step_fraction_matches_oracle(ctx, precision):
    """The CCD filter alone (pruned traversal, widening passes merged after the first) against
    the oracle's ccd_max_step on the coarse sheath, for directions from well inside the first
    pass's radius to several passes beyond it, with collisions and without."""
    sc = coarse_sheath()
    g = ImplicitSolver(ctx, sc, precision)
    o = O.OracleSolver(sc)
    o.step(1, check_intersection=False)
    x = o.positions().astype(np.float32)
    free = np.asarray(sc["inv_mass"]) > 0
    rng = np.random.default_rng(7)
    ts = []
    for mag in (5e-4, 5e-3, 3e-2, 0.2, 0.6):
        dx = np.zeros_like(x)
        dx[free] = rng.normal(0, 0.3 * mag, (free.sum(), 3)) + np.float32([0.0, -mag, 0.0])
        t_gpu, _ = g.ccd(x, dx)
        o.set_state(x.astype(np.float64), None)
        t_o = o.ccd(dx)
        ts.append((mag, float(t_gpu[0]), t_o))
        assert abs(float(t_gpu[0]) - t_o) <= 1e-4 * max(t_o, 1e-3), (mag, t_gpu, t_o)
    print(ts)
    assert min(t for _, _, t in ts) < 1.0  # some direction collides


def _crossing_sheets(cross: bool, n=8):
    """A horizontal sheet and a vertical one whose lower edge dips `cross`-ingly through it
    (2 mm below the horizontal sheet) or stops 2 mm above it."""
    sc = scenes.sheet_on_sphere(n, side=0.1, height=0.5, jitter=0.0, dhat=1e-3)
    pos = sc["positions"].astype(np.float64)
    v = pos.copy()
    # rotate the copy into the vertical x-y plane through the sheet's middle
    c = pos[:, [0, 2]].mean(0)
    v[:, 1] = 0.5 + (pos[:, 2] - c[1]) + 0.05 + (-0.002 if cross else 0.002)
    v[:, 2] = c[1] + 1e-4 * np.sin(7.0 * pos[:, 0])
    sc["positions"] = np.concatenate([pos, v]).astype(np.float32)
    sc["velocities"] = np.zeros_like(sc["positions"])
    sc["tris"] = np.concatenate([sc["tris"], sc["tris"] + n * n]).astype(np.uint32)
    sc["shell_faces"] = sc["tris"].copy()
    sc["inv_mass"] = np.concatenate([sc["inv_mass"], sc["inv_mass"]])
    sc["colliders"] = np.zeros((0, 8), np.float32)
    return sc


@pytest.mark.parametrize("cross", [True, False])
def test_self_intersection_scan_matches_oracle(ctx, cross):
    """has_self_intersection (implicit.rs:618-650) on the GPU (LBVH candidates, exact FP32
    edge-triangle predicate) against the oracle's: two sheets that cross transversally and the
    same sheets apart; then the flag through a step, where penetration_free must agree."""
    sc = _crossing_sheets(cross)
    g = ImplicitSolver(ctx, sc, "fp32")
    o = O.OracleSolver(sc)
    x = sc["positions"]
    cnt = int(g.self_intersections(x)[0])
    assert (cnt > 0) == o.self_intersects(x) == cross, (cnt, cross)
    sg = g.step(1)[0]
    so = o.step(1, check_intersection=True)[0]
    assert bool(sg["penetration_free"]) == bool(so["penetration_free"]) == (not cross)


def test_self_intersection_scan_on_perturbed_drapes(ctx):
    """The scan's verdict equals the oracle's on a crumpled coarse sheath: its state after a
    few steps (no crossing), then the same state with growing random displacements of the
    free vertices (crossings appear)."""
    sc = coarse_sheath()
    g = ImplicitSolver(ctx, sc, "fp32")
    o = O.OracleSolver(sc)
    o.step(2, check_intersection=False)
    x0 = o.positions().astype(np.float32)
    free = np.asarray(sc["inv_mass"]) > 0
    rng = np.random.default_rng(11)
    verdicts = []
    for mag in (0.0, 2e-3, 1e-2, 3e-2):
        x = x0.copy()
        x[free] += rng.normal(0, mag, (free.sum(), 3)).astype(np.float32)
        cnt = int(g.self_intersections(x)[0])
        assert (cnt > 0) == o.self_intersects(x), (mag, cnt)
        verdicts.append(cnt > 0)
    assert verdicts[0] is False and verdicts[-1] is True


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_fused_kernel_variants_agree(ctx, precision):
    """Every variant of the fused PCG kernels the autotuner chooses between (rows kernel with
    2, 1 or 4 lanes per block row, or over the sliced-ELL copy; Schwarz domains with one warp
    each, three warps each at 1, 2 or 4 domains per CTA, or on the tensor cores at 4 or 8
    domains per CTA) runs the same iteration: two batched steps agree with the first
    variant's to the Newton tolerance."""
    from mguso import ImplicitBatch

    scs = graded_coarse(2)
    runs = []
    for v in range(1, 25):
        s2 = [dict(sc, params=dict(sc["params"], pcg_variant=v)) for sc in scs]
        b = ImplicitBatch(ctx, s2, precision)
        st = b.step(2)
        runs.append((v, b.positions.astype(np.float64), st))
        b.close()
    _, p1, s1 = runs[0]
    disp = np.abs(p1 - np.concatenate([sc["positions"] for sc in scs])).max()
    for v, p, st in runs[1:]:
        assert np.abs(p - p1).max() <= 1e-3 * disp, (v, np.abs(p - p1).max() / disp)
        for a, b_ in zip(st, s1):
            for x, y in zip(a, b_):
                assert x["status"] == 0 and abs(x["newton_iters"] - y["newton_iters"]) <= 1, (v, x, y)
