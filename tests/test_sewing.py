"""Seam correspondence (mguso.sewing) with the reference's correspondence tests restated
(ui/crates/nguo-sewing/src/correspond.rs:401-618) on rectangles resolved at a target edge
length; and the stitches it makes closing a seam in the oracle's step."""
import math

import numpy as np
import pytest

import oracle_py as O
from mguso import scenes, sewing


def rect(w, h, target):
    """Boundary of a w x h rectangle (mm) sampled at about `target`: the pattern positions of
    its vertices and one EdgeChain per edge (0 bottom, 1 right, 2 top, 3 left)."""
    corners = [(0.0, 0.0), (w, 0.0), (w, h), (0.0, h)]
    pts, starts = [], []
    for k in range(4):
        a, b = np.array(corners[k]), np.array(corners[(k + 1) % 4])
        n = max(1, math.ceil(np.linalg.norm(b - a) / target))
        starts.append(len(pts))
        pts += [tuple(a + (b - a) * i / n) for i in range(n)]
    pts = np.array(pts)
    chains = []
    for k in range(4):
        ids = list(range(starts[k], starts[k + 1] if k < 3 else len(pts))) + [starts[(k + 1) % 4]]
        chains.append(sewing.EdgeChain(ids, pts[ids]))
    return pts, chains


def test_a_full_side_is_sampled_end_to_end_in_normalised_arc_length():  # correspond.rs:416-431
    _, e = rect(100, 200, 20)
    s = sewing.side_samples([(e[1], False)])
    assert abs(s.len_mm - 200) < 1e-6 and len(s.vertices) >= 3
    assert s.vertices[0][1] == 0.0 and s.vertices[-1][1] == 1.0
    assert all(a[1] <= b[1] for a, b in zip(s.vertices, s.vertices[1:]))


def test_a_two_edge_side_is_one_parameter_space_with_no_duplicate_join():  # correspond.rs:435-458
    _, e = rect(100, 200, 25)
    s = sewing.side_samples([(e[0], False), (e[1], False)])
    assert abs(s.len_mm - 300) < 1e-6
    corner = e[0].vertices[-1]
    assert sum(1 for i, _ in s.vertices if i == corner) == 1
    assert abs(dict(s.vertices)[corner] - 1 / 3) < 1e-6


def test_reversing_an_edge_reverses_its_parameter():  # correspond.rs:460-472
    _, e = rect(100, 200, 20)
    fwd = sewing.side_samples([(e[1], False)])
    rev = sewing.side_samples([(e[1], True)])
    assert len(fwd.vertices) == len(rev.vertices)
    for (vf, uf), (vr, ur) in zip(fwd.vertices, reversed(rev.vertices)):
        assert vf == vr and abs(uf - (1 - ur)) < 1e-9


def test_a_partial_span_keeps_only_its_own_vertices_and_renormalises():  # correspond.rs:474-490
    _, e = rect(100, 200, 10)
    s = sewing.side_samples([(e[1], False)], span=(0.5, 1.0))
    assert abs(s.len_mm - 100) < 1e-6
    assert s.vertices[0][1] == 0.0 and s.vertices[-1][1] == 1.0
    assert len(s.vertices) < len(sewing.side_samples([(e[1], False)]).vertices)
    assert sewing.side_samples([(e[1], False)], span=(1.0, 0.5)).len_mm == s.len_mm


def test_a_discontinuous_side_is_an_error_naming_the_edge():  # correspond.rs:492-503
    _, e = rect(100, 200, 25)
    with pytest.raises(sewing.BrokenChain) as err:
        sewing.side_samples([(e[0], False), (e[1], True)])
    assert err.value.edge == 1


def test_a_zero_length_span_is_an_error_not_a_division_by_zero():  # correspond.rs:505-515
    _, e = rect(100, 200, 25)
    with pytest.raises(sewing.DegenerateSpan):
        sewing.side_samples([(e[1], False)], span=(0.4, 0.4))


def test_unequal_resolutions_pair_by_parameter_not_by_vertex_count():  # correspond.rs:520-547
    fine_p, fe = rect(100, 200, 8)
    coarse_p, ce = rect(100, 200, 40)
    a = sewing.side_samples([(fe[1], False)])
    b = sewing.side_samples([(ce[1], False)])
    assert len(a.vertices) > len(b.vertices)
    c = sewing.correspond(a, b)
    assert len(c.stitches) == len(a.vertices) and abs(c.ease() - 1) < 1e-9
    for (v, u), (idx, w) in zip(a.vertices, c.stitches):
        got = coarse_p[idx[3]][1] * (1 - w[4]) + coarse_p[idx[4]][1] * w[4]
        assert abs(fine_p[v][1] - got) < 1e-4  # the weight is f32, as in the stitch
        assert abs(sum(w[:3]) - 1) < 1e-6 and abs(sum(w[3:]) - 1) < 1e-6


def test_unequal_lengths_become_ease_and_pair_proportionally():  # correspond.rs:551-586
    long_p, le = rect(100, 250, 10)
    short_p, se = rect(100, 200, 10)
    a = sewing.side_samples([(se[1], False)])
    b = sewing.side_samples([(le[1], False)])
    c = sewing.correspond(a, b)
    assert abs(c.ease() - 1.25) < 1e-9 and abs(c.ease_fraction() - 0.25) < 1e-9
    assert len(c.stitches) == len(b.vertices)
    v = min(b.vertices, key=lambda x: abs(x[1] - 0.5))[0]
    idx, w = next(s for s in c.stitches if s[0][0] == v)
    target = short_p[idx[3]][1] * (1 - w[4]) + short_p[idx[4]][1] * w[4]
    assert abs(target / 200 - long_p[v][1] / 250) < 1e-6


def test_a_flipped_pairing_measures_shorter_when_the_seam_is_twisted():  # correspond.rs:590-617
    p, e = rect(100, 200, 20)
    a = sewing.side_samples([(e[1], False)])
    b0 = sewing.side_samples([(e[1], False)])
    pos = np.concatenate([np.c_[p * 1e-3, np.zeros(len(p))], np.c_[p[:, 0] * 1e-3, 0.2 - p[:, 1] * 1e-3,
                                                                    np.zeros(len(p))]])
    b = sewing.SideSamples([(i + len(p), u) for i, u in b0.vertices], b0.len_mm)
    straight = sewing.pairing_distance_m(a, b, pos, False)
    flipped = sewing.pairing_distance_m(a, b, pos, True)
    assert flipped < 0.5 * straight
    _, flip = sewing.sew(a, b, pos)
    assert flip


def test_corresponded_stitches_close_a_seam_in_the_step():
    """Two flat strips side by side (2 cm apart), their facing long edges corresponded at
    different resolutions; the oracle's step with those stitches closes the gap."""
    def strip(x0, n_long):
        ys = np.linspace(0.0, 0.2, n_long)
        return [(x0, y, 0.0) for y in ys] + [(x0 + 0.02, y, 0.0) for y in ys]

    na, nb = 9, 6
    pa, pb = np.array(strip(0.0, na)), np.array(strip(0.04, nb))
    pos = np.concatenate([pa, pb]).astype(np.float32)

    def tris(base, n):
        t = []
        for i in range(n - 1):
            t += [(base + i, base + n + i, base + i + 1), (base + i + 1, base + n + i, base + n + i + 1)]
        return t

    all_tris = np.array(tris(0, na) + tris(2 * na, nb), np.uint32)
    right_of_a = sewing.EdgeChain(list(range(na, 2 * na)), pa[na:, :2] * 1e3)
    left_of_b = sewing.EdgeChain([2 * na + i for i in range(nb)], pb[:nb, :2] * 1e3)
    c = sewing.correspond(sewing.side_samples([(right_of_a, False)]), sewing.side_samples([(left_of_b, False)]))
    idx, w = c.arrays()
    assert idx.shape == (na, 6) and abs(c.ease() - 1) < 1e-9
    im = np.full(len(pos), 50.0, np.float32)
    im[0] = 0.0
    sc = dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=im, tris=all_tris,
              shell_faces=np.zeros((0, 3), np.uint32), static_mask=None, stitch_idx=idx, stitch_w=w,
              stitch_kl=np.tile(np.float32([[1.0, 1e-3, 1e-2]]), (len(idx), 1)),
              colliders=np.zeros((0, 8), np.float32),
              params=scenes.default_params(gravity=(0.0, 0.0, 0.0), self_collision=0, stiffness=1e3,
                                           bend_stiffness=0.0))

    def gap(x):
        t = x[idx[:, 3]] * (1 - w[:, 4:5]) + x[idx[:, 4]] * w[:, 4:5]
        return np.linalg.norm(x[idx[:, 0]] - t, axis=1).max()

    o = O.OracleSolver(sc)
    o.step(100, check_intersection=False)
    x = o.positions().astype(np.float64)
    assert gap(pos.astype(np.float64)) > 0.019 and gap(x) < 0.1 * gap(pos.astype(np.float64))
