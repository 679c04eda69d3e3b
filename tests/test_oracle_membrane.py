"""The Baraff-Witkin membrane in the oracle (membrane.rs restated in
oracle/implicit_oracle.hpp) against the reference's membrane tests (membrane.rs:336-657) and
its anisotropy test through the whole step (implicit.rs:4674-4773)."""
import numpy as np
import oracle_py as O

from mguso import scenes

f32 = np.float32


def tri(*p):
    return np.array(p, f32)


def conds(rest, p):
    return O.membrane_element(rest, p)[0]


def test_analytic_grads_match_fd():  # membrane.rs:338-362 (through the element gradient)
    rest = tri([0.1, -0.2, 0.0], [1.3, 0.1, 0.0], [0.2, 0.9, 0.0])
    p = tri([0.15, -0.18, 0.05], [1.55, 0.22, -0.1], [0.05, 1.15, 0.2])
    kw, kf, ks = 3.0, 2.0, 5.0
    area = 0.5 * np.linalg.norm(np.cross(rest[1] - rest[0], rest[2] - rest[0]))

    def energy(q):
        c = conds(rest, q).astype(np.float64)
        return 0.5 * area * (kw * c[0] ** 2 + kf * c[1] ** 2 + ks * c[2] ** 2)

    _, g, _, _ = O.membrane_element(rest, p, kw, kf, ks)
    h = 1e-3
    fd = np.zeros((3, 3))
    for a in range(3):
        for c in range(3):
            pp, pm = p.copy(), p.copy()
            pp[a, c] += h
            pm[a, c] -= h
            fd[a, c] = (energy(pp) - energy(pm)) / (2 * h)
    assert np.abs(fd - g).max() < 1e-2 * max(np.abs(fd).max(), 1.0)


def test_stretch_eigen_material_eigenvalues():  # membrane.rs:364-389
    m, _ = O.membrane_materials([1.5, 0, 0], [1, 0, 0], [0, 1, 0])
    perp = 1.0 - 1.0 / 1.5
    assert abs(m[0, 0] - 1.0) < 1e-5 and abs(m[1, 1] - perp) < 1e-5 and abs(m[2, 2] - perp) < 1e-5
    assert np.abs(m - m.T).max() < 1e-6 and (np.diag(m) >= -1e-6).all()
    mc, _ = O.membrane_materials([0.6, 0, 0], [1, 0, 0], [0, 1, 0])
    assert abs(mc[0, 0] - 1.0) < 1e-6 and abs(mc[1, 1]) < 1e-6 and abs(mc[2, 2]) < 1e-6


def test_shear_material_unclamped_reconstructs_h6():  # membrane.rs:391-420
    wu, wv = np.array([1.1, 0.3, -0.2], f32), np.array([0.2, 0.9, 0.4], f32)
    f = float(wu @ wv)
    _, m = O.membrane_materials([1, 0, 0], wu, wv, clamp=False)
    eye = np.eye(3) * f
    expect = [np.outer(wv, wv), np.outer(wv, wu) + eye, np.outer(wu, wv) + eye, np.outer(wu, wu)]
    for b in range(4):
        assert np.abs(m[b] - expect[b]).max() < 1e-4


def test_shear_material_clamped_is_psd():  # membrane.rs:479-508
    rng = np.random.default_rng(7)
    for _ in range(32):
        wu, wv = rng.uniform(-1.5, 1.5, 3).astype(f32), rng.uniform(-1.5, 1.5, 3).astype(f32)
        _, m = O.membrane_materials([1, 0, 0], wu, wv, clamp=True)
        h6 = np.block([[m[0], m[1]], [m[2], m[3]]]).astype(np.float64)
        assert np.abs(h6 - h6.T).max() < 1e-4
        assert np.linalg.eigvalsh(0.5 * (h6 + h6.T)).min() > -1e-4 * max(1.0, np.abs(h6).max())


def test_the_element_hessian_matches_the_energy_hessian_in_tension():  # membrane.rs:510-558
    rest = tri([0, 0, 0], [1, 0, 0], [0.2, 0.9, 0])
    p = tri([0, 0, 0], [1.3, 0.0, 0.0], [0.25, 1.2, 0.0])  # both columns stretched, in plane
    _, _, hm, _ = O.membrane_element(rest, p, 2.0, 3.0, 0.0)  # stretch only
    area = 0.5 * np.linalg.norm(np.cross(rest[1] - rest[0], rest[2] - rest[0]))

    def grad(q):
        return O.membrane_element(rest, q, 2.0, 3.0, 0.0)[1].reshape(9).astype(np.float64)

    h = 1e-3
    fd = np.zeros((9, 9))
    for k in range(9):
        qp, qm = p.copy().reshape(9), p.copy().reshape(9)
        qp[k] += h
        qm[k] -= h
        fd[:, k] = (grad(qp.reshape(3, 3)) - grad(qm.reshape(3, 3))) / (2 * h)
    assert area > 0 and np.abs(fd - hm).max() < 2e-2 * np.abs(hm).max()


def test_rest_shape_has_zero_conditions():  # membrane.rs:593-605
    rest = tri([0, 0, 0], [1, 0, 0], [0.3, 0.8, 0])
    assert np.abs(conds(rest, rest)).max() < 1e-4


def test_uniaxial_stretch_excites_only_warp():  # membrane.rs:607-634
    rest = tri([0, 0, 0], [1, 0, 0], [0, 1, 0])
    c = conds(rest, tri([0, 0, 0], [1.2, 0, 0], [0, 1, 0]))
    assert abs(c[0] - 0.2) < 1e-3 and abs(c[1]) < 1e-3 and abs(c[2]) < 1e-3


def test_shear_excites_shear_condition():  # membrane.rs:636-656
    rest = tri([0, 0, 0], [1, 0, 0], [0, 1, 0])
    assert abs(conds(rest, tri([0, 0, 0], [1, 0, 0], [0.3, 1, 0]))[2]) > 0.1


def membrane_bottom_y(warp, weft):  # implicit.rs:4674-4712
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
    sc = dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=im, tris=np.array(tris, np.uint32),
              shell_faces=np.zeros((0, 3), np.uint32), static_mask=None, stitch_idx=si, stitch_w=sw, stitch_kl=skl,
              colliders=np.zeros((0, 8), f32),
              params=scenes.default_params(dt=1.0 / 120.0, stiffness=0.0, newton_iters=5, bend_stiffness=0.0,
                                           contact_dhat=1e-2, contact_rayleigh=0, self_collision=0, precond=1))
    o = O.OracleSolver(sc)
    assert o.set_membrane(warp, weft, 200.0)
    o.step(300, check_intersection=False)
    return float(o.positions()[:n, 1].astype(f32).mean())


def test_membrane_is_anisotropic():  # implicit.rs:4763-4773
    weft_stiff, warp_stiff = membrane_bottom_y(100.0, 5000.0), membrane_bottom_y(5000.0, 100.0)
    assert np.isfinite(weft_stiff) and np.isfinite(warp_stiff)
    assert weft_stiff > warp_stiff + 0.02, (weft_stiff, warp_stiff)


def test_membrane_with_zero_stiffness_is_inert():
    n = 4
    pos = np.array([(i * 0.1, 0.5, j * 0.1) for j in range(n) for i in range(n)], f32)
    tris = np.array([(j * n + i, j * n + i + 1, j * n + i + n) for j in range(n - 1) for i in range(n - 1)] +
                    [(j * n + i + n, j * n + i + 1, j * n + i + n + 1) for j in range(n - 1) for i in range(n - 1)],
                    np.uint32)
    si, sw, skl = scenes._empty_stitches()
    sc = dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=np.full(n * n, 10.0, f32), tris=tris,
              shell_faces=np.zeros((0, 3), np.uint32), static_mask=None, stitch_idx=si, stitch_w=sw, stitch_kl=skl,
              colliders=np.zeros((0, 8), f32), params=scenes.default_params(self_collision=0, stiffness=500.0))
    x, y = O.OracleSolver(sc), O.OracleSolver(sc)
    assert y.set_membrane(0.0, 0.0, 0.0)
    assert not y.set_membrane(1.0, 1.0, 1.0, per_element=np.ones((3, 3)))  # wrong element count
    x.step(5, check_intersection=False)
    y.step(5, check_intersection=False)
    assert np.array_equal(x.positions(), y.positions())
