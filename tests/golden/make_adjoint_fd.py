"""Golden finite differences for the adjoint test: central differences of the landmark loss
of the FP64 oracle drape in each of the 8 pattern parameters, one oracle run per perturbed
parameter vector, in a process pool.

  python tests/golden/make_adjoint_fd.py     # writes adjoint_fd_coarse.npz beside this file

The drape is the XS sheath meshed at 5 cm edges (1 060 vertices with its torso) for 24 steps.
The loss is the sum of squared distances of 40 seeded landmark vertices to targets taken from
a forward run at parameters raised by 5%. Differences at eps = 1e-4 (`fd`) and, as a measure
of the differences' own error, at eps = 1e-5 (`fd_fine`)."""
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(HERE, "..", ".."), os.path.join(HERE, "..", "..", "oracle"),
                os.path.join(HERE, "..", "..", "nguo-3d_b200")]

EPS, EPS_FINE, NPARAM = 1e-4, 1e-5, 8
# (steps, checkpoint interval) per scene
HORIZON = {"coarse": (24, 6)}


def adjoint_scene(name: str = "coarse"):
    """The drape the adjoint test differentiates: the XS sheath (0.5 m panels on a torso
    scaled 0.9) meshed at 5 cm edges on a 24x23 torso. Newton runs until its step is below
    1e-7 m, 40 iterations at most (the drape's last five steps cycle at that cap)."""
    from mguso import scenes
    assert name == "coarse"
    sc = scenes.sheath_on_torso(edge=0.05, torso_res=(24, 23), width=0.5, torso_scale=0.9)
    sc["params"] = dict(sc["params"], newton_tol=0.0, newton_iters=40, cg_tol=1e-6)
    free = np.flatnonzero(sc["inv_mass"] > 0)
    landmarks = np.sort(np.random.default_rng(4).choice(free, 40, replace=False))
    return sc, landmarks


def oracle_final(name: str, theta, steps: int = 0):
    """x_N of the FP64 oracle drape at pattern parameters theta (the scene's horizon unless
    `steps` is given)."""
    steps = steps or HORIZON[name][0]
    import oracle_py as O
    from mguso.adjoint import pattern_rest
    sc, _ = adjoint_scene(name)
    o = O.OracleSolver(dict(sc, params=dict(sc["params"], cg_tol=1e-10)), "f64")
    rest, k = pattern_rest(sc["shell_uv"], sc["shell_panel"], theta, 2)
    p = sc["params"]
    o.set_shells(sc["shell_faces"], rest, p["shell_mu"] * k, p["shell_lambda"] * k)
    o.scale_stitches(np.asarray(theta, np.float64)[6 + sc["stitch_seam"]])
    o.step(steps, check_intersection=False)
    x = o.positions().astype(np.float64)
    o.close()
    return x


def _run(args):
    name, theta = args
    return oracle_final(name, np.asarray(theta))


def main(name: str):
    t0 = time.time()
    _, lm = adjoint_scene(name)
    theta = np.ones(NPARAM)
    runs = [theta * 1.05, theta]
    for eps in (EPS, EPS_FINE):
        for i in range(NPARAM):
            for s in (1.0, -1.0):
                th = theta.copy()
                th[i] += s * eps
                runs.append(th)
    with mp.get_context("spawn").Pool(min(os.cpu_count() or 1, len(runs))) as pool:
        xs = pool.map(_run, [(name, r) for r in runs])
    target = xs[0][lm]
    loss = [float(((x[lm] - target) ** 2).sum()) for x in xs[1:]]
    fd = np.array([(loss[1 + 2 * i] - loss[2 + 2 * i]) / (2 * EPS) for i in range(NPARAM)])
    o = 1 + 2 * NPARAM
    fd_fine = np.array([(loss[o + 2 * i] - loss[o + 1 + 2 * i]) / (2 * EPS_FINE) for i in range(NPARAM)])
    out = os.path.join(HERE, f"adjoint_fd_{name}.npz")
    np.savez_compressed(out, theta=theta, landmarks=lm.astype(np.int64), target=target, loss=loss[0], fd=fd, fd_fine=fd_fine,
                        x_final=xs[1].astype(np.float32), steps=HORIZON[name][0], every=HORIZON[name][1], eps=EPS)
    print(name, "fd", fd, "fd_fine", fd_fine, "loss", loss[0], f"{time.time() - t0:.0f} s")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "coarse")
