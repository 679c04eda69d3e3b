"""The oracle's FP64 adjoint (oracle_py.fp64_adjoint: the step's equilibrium residual
differentiated by central differences in FP64, contact set and the stiffnesses' elastic
parts held at each converged step) against central finite differences of the oracle's own
FP64 drape, on a drape small and smooth enough for the differences to be exact to ~1e-6:
the two-panel sheath at 10 cm edges falling onto its torso for 3 steps with Newton and PCG
run to convergence, 8 pattern parameters, a landmark loss with targets from a +5% run."""
import numpy as np
import pytest

import oracle_py as O
from mguso import scenes
from mguso.adjoint import pattern_rest

N = 3


def _scene():
    sc = scenes.sheath_on_torso(edge=0.1, torso_res=(12, 11), width=0.5, torso_scale=0.9)
    sc["params"] = dict(sc["params"], newton_tol=0.0, newton_iters=60, cg_tol=1e-12, cg_max_iter=20000)
    return sc


def _forward(sc, theta, keep=False):
    o = O.OracleSolver(sc, "f64")
    rest, k = pattern_rest(sc["shell_uv"], sc["shell_panel"], theta, 2)
    p = sc["params"]
    o.set_shells(sc["shell_faces"], rest, p["shell_mu"] * k, p["shell_lambda"] * k)
    o.scale_stitches(np.asarray(theta, np.float64)[6 + sc["stitch_seam"]])
    xs, vs, st = [o.positions()], [o.velocities()], []
    for _ in range(N):
        st += o.step(1, check_intersection=False)
        xs.append(o.positions())
        vs.append(o.velocities())
    o.close()
    return np.array(xs), np.array(vs), st


def test_fp64_adjoint_matches_finite_differences_of_the_oracle_drape():
    sc = _scene()
    theta = np.ones(8)
    xs, vs, st = _forward(sc, theta)
    assert max(s["stencils"] for s in st) > 100  # the drape is in contact
    free = np.flatnonzero(sc["inv_mass"] > 0)
    lm = np.sort(np.random.default_rng(4).choice(free, 40, replace=False))
    target = _forward(sc, theta * 1.05)[0][-1][lm]
    dl = np.zeros_like(xs[-1])
    dl[lm] = 2.0 * (xs[-1][lm] - target)
    g, nst = O.fp64_adjoint(sc, theta, xs, vs, dl)
    assert len(nst) == N and min(nst) > 0
    eps = 1e-5
    fd = np.zeros(8)
    for i in range(8):
        loss = []
        for sgn in (1.0, -1.0):
            th = theta.copy()
            th[i] += sgn * eps
            loss.append(((_forward(sc, th)[0][-1][lm] - target) ** 2).sum())
        fd[i] = (loss[0] - loss[1]) / (2 * eps)
    err = np.abs(g - fd).max() / np.abs(fd).max()
    print("adjoint", g, "\nfd", fd, "\nerr", err)
    assert err <= 1e-4, err


def test_adjoint_system_rejects_a_float_solver():
    sc = _scene()
    o = O.OracleSolver(sc, "f32")
    x = sc["positions"].astype(np.float64)
    with pytest.raises(ValueError):
        O.adjoint_system(o, sc, np.ones(8), x, np.zeros_like(x), x)
