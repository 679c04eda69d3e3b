"""The solver-invariant checker (mguso/metrics.py) against the reference's metrics.rs tests,
and the two implicit.rs runs that exercise it end to end (a good drape passes, a starved
linear solve fails cg_converged), stepped by the oracle."""
import numpy as np
import oracle_py as O

from mguso import scenes
from mguso.metrics import check_invariants


def good_step():
    return dict(max_reresid=1e-4, max_cg_iters=50, newton_iters=4, max_sigma=1.001, num_contacts=3,
                penetration_free=1, all_finite=1)


def test_good_run_passes_all_invariants():  # metrics.rs:193-201
    r = check_invariants([good_step() for _ in range(10)], 1e-3, 10000)
    assert r.all_ok(), r.checks
    assert [c.name for c in r.checks] == ["penetration_free", "all_frames_finite", "strain_limit_respected",
                                          "cg_converged", "cg_iter_under_cap", "zero_steady_state_alloc"]


def test_diverged_run_fails():  # metrics.rs:203-224
    steps = []
    for k in range(10):
        s = good_step()
        if k >= 5:
            s.update(all_finite=0, penetration_free=0, max_reresid=0.9, max_cg_iters=100)
        steps.append(s)
    r = check_invariants(steps, 1e-3, 100)
    assert not r.all_ok()
    for name in ("all_frames_finite", "penetration_free", "cg_converged", "cg_iter_under_cap"):
        assert not r.by_name(name).ok


def test_strain_limit_gate():  # metrics.rs:226-237
    s = good_step()
    s["max_sigma"] = 1.10
    assert not check_invariants([s], 1e-3, 10000, strain_limit=0.05).all_ok()
    s["max_sigma"] = 1.06
    assert check_invariants([s], 1e-3, 10000, strain_limit=0.05).all_ok()


def test_a_batch_run_is_checked_per_instance():
    steps = [[good_step(), good_step()] for _ in range(4)]
    steps[2][1] = dict(good_step(), all_finite=0)
    r = check_invariants(steps, 1e-3, 10000)
    assert not r.by_name("all_frames_finite").ok and r.by_name("cg_converged").ok


def flat_cloth(n, y, spacing, **params):
    """implicit.rs:4214-4229: an n x n sheet, vertex mass 0.02, over ImplicitParams::default()."""
    pos = np.array([(i * spacing, y, j * spacing) for j in range(n) for i in range(n)], np.float32)
    tris = []
    for j in range(n - 1):
        for i in range(n - 1):
            v = j * n + i
            r = v + n
            tris += [(v, v + 1, r), (r, v + 1, r + 1)]
    si, sw, skl = scenes._empty_stitches()
    p = dict(dt=1.0 / 60.0, gravity=(0.0, -9.8, 0.0), newton_iters=4, stiffness=1.0e3, bend_stiffness=0.0,
             contact_dhat=1.0e-2, contact_kappa=1.0e2, contact_rayleigh=0, self_collision=0, barrier_kind=0,
             precond=1)
    p.update(params)
    return dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=np.full(len(pos), 1 / 0.02, np.float32),
                tris=np.array(tris, np.uint32), shell_faces=np.zeros((0, 3), np.uint32), static_mask=None,
                stitch_idx=si, stitch_w=sw, stitch_kl=skl, colliders=np.zeros((0, 8), np.float32),
                params=scenes.default_params(**p))


def test_good_drape_passes_invariants():  # implicit.rs:4231-4262
    sc = flat_cloth(6, 0.3, 0.1, dt=1.0 / 120.0, stiffness=500.0, cg_tol=1e-3, cg_max_iter=2000,
                    contact_dhat=0.02, contact_kappa=1.0e3)
    sc["colliders"] = np.array([[0, 0, 0, 0, 0, 1, 0, 0]], np.float32)
    st = O.OracleSolver(sc).step(120, check_intersection=False)
    assert len(st) == 120
    r = check_invariants(st, 1e-3, 2000)
    assert r.all_ok(), [c for c in r.checks if not c.ok]


def test_diverged_run_fails_invariants():  # implicit.rs:4265-4290
    sc = flat_cloth(8, 1.0, 0.1, stiffness=1.0e5, cg_tol=1e-6, cg_max_iter=1, newton_iters=2)
    sc["inv_mass"][0] = 0.0
    st = O.OracleSolver(sc).step(10, check_intersection=False)
    r = check_invariants(st, 1e-6, 1)
    assert not r.all_ok()
    assert not r.by_name("cg_converged").ok
