"""The host's material conversion (mguso.scenes.lame_from_young_poisson) against the
reference's material tests (engine-core/src/material.rs:47-101), and the oracle's shell
primitives (sym_eig2, svd3x2 and the StVK density over principal stretches) against the
reference's shell-model tests (shell_model.rs:856-958), at the reference tests' inputs."""
import math

import numpy as np
import oracle_py as O

from mguso.scenes import lame_from_young_poisson


def test_matches_the_reference_conversion_for_every_gauge_poisson_ratio():  # material.rs:52-78
    mu, lam = lame_from_young_poisson(100.0, 0.35)
    assert abs(mu - 37.03704) < 1e-3 and abs(lam - 86.41975) < 1e-2
    mu, lam = lame_from_young_poisson(100.0, 0.25)
    assert abs(mu - 40.0) < 1e-3 and abs(lam - 40.0) < 1e-3
    mu, lam = lame_from_young_poisson(100.0, 0.49)
    assert abs(mu - 33.55705) < 1e-3 and abs(lam - 1644.295) < 0.1
    assert lam / 0.5 / 100.0 > 30.0


def test_both_parameters_are_linear_in_youngs_modulus():  # material.rs:80-88
    m1, l1 = lame_from_young_poisson(100.0, 0.35)
    m2, l2 = lame_from_young_poisson(400.0, 0.35)
    assert abs(m2 / m1 - 4.0) < 1e-4 and abs(l2 / l1 - 4.0) < 1e-4


def test_degenerate_poisson_ratios_stay_finite():  # material.rs:90-101
    for nu in (-1.0, 0.0, 0.5, 0.75, 1.0, float("nan")):
        mu, lam = lame_from_young_poisson(100.0, nu)
        assert math.isfinite(mu) and math.isfinite(lam), nu
        assert mu > 0.0 and lam >= 0.0, nu
    assert lame_from_young_poisson(0.0, 0.35) == (0.0, 0.0)


def test_sym_eig2_reconstructs():  # shell_model.rs:856-882
    for p, q, r in ((3.0, 1.0, 2.0), (5.0, 0.0, 5.0), (1.0, -2.0, 4.0), (0.0, 0.0, 0.0), (-1.0, 0.5, 2.0)):
        lam, v = O.sym_eig2(p, q, r)
        assert lam[0] >= lam[1] - 1e-6
        back = (v * lam) @ v.T
        assert np.abs(back - np.array([[p, q], [q, r]], np.float32)).max() < 1e-4, (p, q, r)
        assert abs(float(v[:, 0] @ v[:, 1])) < 1e-5
        assert abs(float(np.linalg.norm(v[:, 0])) - 1.0) < 1e-5


def test_svd3x2_reconstructs_with_orthonormal_frames():  # shell_model.rs:884-914
    cols = [((1.0, 0.0, 0.0), (0.0, 1.0, 0.0)), ((1.3, 0.1, 0.05), (-0.2, 0.9, 0.1)),
            ((2.0, 0.0, 0.0), (0.0, 0.5, 0.0)), ((1.0, 0.0, 0.0), (2.0, 0.0, 0.0))]  # the last: rank 1
    for i, (c0, c1) in enumerate(cols):
        f = np.array([c0, c1], np.float32).T
        u, s, v = O.svd3x2(f)
        assert s[0] >= s[1] - 1e-6 and s[1] >= -1e-6, i
        assert abs(float(u[:, 0] @ u[:, 1])) < 1e-4, i
        assert abs(float(np.linalg.norm(u[:, 0])) - 1.0) < 1e-4
        assert abs(float(np.linalg.norm(u[:, 1])) - 1.0) < 1e-4
        back = (u * s) @ v.T
        assert np.linalg.norm(back[:, 0] - f[:, 0]) < 2e-3 and np.linalg.norm(back[:, 1] - f[:, 1]) < 2e-3, i


def test_shell_derivatives_are_self_consistent():  # shell_model.rs:916-958 (the StVK model)
    mu, lam, h = 400.0, 250.0, np.float32(1e-3)
    for base in ((1.25, 0.9), (1.0, 1.0), (0.8, 1.15)):
        b = np.array(base, np.float32)
        _, g, hh = O.stvk_density(b, mu, lam)
        for i in range(2):
            sp, sm = b.copy(), b.copy()
            sp[i] += h
            sm[i] -= h
            fd = (O.stvk_density(sp, mu, lam)[0] - O.stvk_density(sm, mu, lam)[0]) / (2.0 * float(h))
            assert abs(g[i] - fd) < 2e-2 * max(abs(g[i]), 1.0), (base, i, g[i], fd)
        for j in range(2):
            sp, sm = b.copy(), b.copy()
            sp[j] += h
            sm[j] -= h
            gp, gm = O.stvk_density(sp, mu, lam)[1], O.stvk_density(sm, mu, lam)[1]
            for i in range(2):
                fd = (gp[i] - gm[i]) / (2.0 * float(h))
                assert abs(hh[i, j] - fd) < 3e-2 * max(abs(hh[i, j]), 1.0), (base, i, j, hh[i, j], fd)
