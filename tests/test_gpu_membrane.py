"""The Baraff-Witkin membrane (membrane.rs; assembled as implicit.rs:2532-2596) in the CUDA
step, through the C ABI: the reference's anisotropy test (implicit.rs:4674-4773) on the GPU,
each step of it against the oracle's from the same state, and zero stiffness inert."""
import numpy as np
import pytest

import oracle_py as O
from mguso import ImplicitSolver, scenes

pytestmark = pytest.mark.gpu
f32 = np.float32


def hanging_sheet(warp, weft, shear=200.0):
    n = 6
    pos = np.array([(i * 0.1, j * 0.1, 0.0) for j in range(n) for i in range(n)], f32)
    tris = []
    for j in range(n - 1):
        for i in range(n - 1):
            v = j * n + i
            tris += [(v, v + 1, v + n), (v + n, v + 1, v + n + 1)]
    im = np.full(n * n, 1 / 0.05, f32)
    im[(n - 1) * n:] = 0.0  # the top row
    si, sw, skl = scenes._empty_stitches()
    p = scenes.default_params(dt=1.0 / 120.0, stiffness=0.0, newton_iters=5, bend_stiffness=0.0, contact_dhat=1e-2,
                              contact_rayleigh=0, self_collision=0, precond=1, membrane_warp=warp,
                              membrane_weft=weft, membrane_shear=shear)
    return dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=im, tris=np.array(tris, np.uint32),
                shell_faces=np.zeros((0, 3), np.uint32), static_mask=None, stitch_idx=si, stitch_w=sw, stitch_kl=skl,
                colliders=np.zeros((0, 8), f32), params=p), n


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_membrane_steps_match_oracle(ctx, precision):
    sc, n = hanging_sheet(5000.0, 100.0)
    g = ImplicitSolver(ctx, sc, precision)
    o = O.OracleSolver(sc)
    assert o.set_membrane(5000.0, 100.0, 200.0)
    for k in range(30):
        p0, v0 = o.positions().copy(), o.velocities().copy()
        g.positions, g.velocities = p0.astype(f32), v0.astype(f32)
        sg = g.step(1)[0]
        so = o.step(1, check_intersection=False)[0]
        pg, po = g.positions.astype(np.float64), o.positions()
        rel = np.abs(pg - po).max() / (np.abs(po - p0).max() + 1e-12)
        assert sg["status"] == 0 and abs(sg["newton_iters"] - so["newton_iters"]) <= 1, (k, sg, so)
        assert rel < 1e-3, (k, rel)


def test_membrane_is_anisotropic_on_the_gpu(ctx):  # implicit.rs:4763-4773
    def bottom_y(warp, weft):
        sc, n = hanging_sheet(warp, weft)
        g = ImplicitSolver(ctx, sc, "fp32")
        g.step(300)
        return float(g.positions[:n, 1].astype(f32).mean())

    weft_stiff, warp_stiff = bottom_y(100.0, 5000.0), bottom_y(5000.0, 100.0)
    assert np.isfinite(weft_stiff) and np.isfinite(warp_stiff)
    assert weft_stiff > warp_stiff + 0.02, (weft_stiff, warp_stiff)


def test_zero_membrane_stiffness_is_inert(ctx):
    sc, _ = hanging_sheet(0.0, 0.0, 0.0)
    sc["params"]["stiffness"] = 500.0
    plain = dict(sc, params={k: v for k, v in sc["params"].items() if not k.startswith("membrane")})
    a, b = ImplicitSolver(ctx, sc, "fp32"), ImplicitSolver(ctx, plain, "fp32")
    a.step(5)
    b.step(5)
    assert np.array_equal(a.positions, b.positions)
