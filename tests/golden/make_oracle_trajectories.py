"""Golden trajectories of the CPU oracle: the FP32 and FP64 oracle's positions after a few
steps of three small drapes, so that a change to the oracle that moves any of them is seen
(the reference publishes no trajectory for this path, so these pin the restatement against
itself, not against the reference).

  python tests/golden/make_oracle_trajectories.py   # writes oracle_trajectories.npz here

Scenes: a 12 x 12 sheet (0.4 m) falling onto the analytic sphere, 8 steps; two 5 x 5 layers
in resting self contact (the lower pinned), 40 steps at dt = 1/480; the XS sheath meshed at
5 cm edges sewn on its torso (stitches, StVK shells, hinges, signed static-mesh contact),
2 steps."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(HERE, ".."), os.path.join(HERE, "..", "..", "oracle"),
                os.path.join(HERE, "..", "..", "nguo-3d_b200")]

OUT = os.path.join(HERE, "oracle_trajectories.npz")


def two_layers():
    from mguso import scenes

    n, pos, tris = 5, [], []
    for y in (0.0, 0.018):
        base = len(pos)
        pos += [(i * 0.1, y, j * 0.1) for j in range(n) for i in range(n)]
        for j in range(n - 1):
            for i in range(n - 1):
                v = base + j * n + i
                tris += [(v, v + 1, v + n), (v + n, v + 1, v + n + 1)]
    pos = np.array(pos, np.float32)
    im = np.full(len(pos), 1.0 / 0.02, np.float32)
    im[: n * n] = 0.0
    si, sw, skl = scenes._empty_stitches()
    return dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=im, tris=np.array(tris, np.uint32),
                shell_faces=np.zeros((0, 3), np.uint32), static_mask=None, stitch_idx=si, stitch_w=sw,
                stitch_kl=skl, colliders=np.zeros((0, 8), np.float32),
                params=scenes.default_params(dt=1.0 / 480.0, stiffness=500.0, gravity=(0.0, -4.0, 0.0),
                                             contact_dhat=0.02, contact_kappa=2.0e3, newton_iters=4,
                                             bend_stiffness=0.0, contact_rayleigh=0, precond=1))


def cases():
    """(name, scene, steps) of every golden trajectory."""
    from mguso import scenes

    return [("sheet_on_sphere", scenes.sheet_on_sphere(12, side=0.4, height=0.33), 8),
            ("two_layers", two_layers(), 40),
            ("sheath_xs", scenes.sheath_on_torso(edge=0.05, torso_res=(24, 23), width=0.5, torso_scale=0.9), 2)]


def run(scene, steps, precision):
    import oracle_py as O

    o = O.OracleSolver(scene, precision)
    st = o.step(steps, check_intersection=False)
    return o.positions(), np.array([s["newton_iters"] for s in st], np.int32)


def main():
    out = {}
    for name, sc, steps in cases():
        for prec in ("f32", "f64"):
            x, it = run(sc, steps, prec)
            out[f"{name}_{prec}"] = x
            out[f"{name}_{prec}_newton"] = it
            print(name, prec, x.shape, it.tolist())
    np.savez_compressed(OUT, **out)


if __name__ == "__main__":
    main()
