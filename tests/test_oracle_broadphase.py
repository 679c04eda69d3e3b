"""The oracle's uniform-grid broad phase (broadphase.rs restated in oracle/implicit_oracle.hpp)
against the reference's own broad-phase tests: candidates are a superset of brute force,
the movable filter drops exactly the inert pairs, the edge-edge candidate count of the
reference's fixture is its pinned number (broadphase.rs:994-1002: 268 075 over 5 162 edges),
and the self-intersection predicate's streamed edge-triangle candidates equal the
materialised list, stop at the first match and see cloth-through-body pierces only.
"""
import numpy as np
import oracle_py as O

f32 = np.float32


def _grid(n, spacing, y, base, second_winding):
    pos = [(f32(i) * f32(spacing), f32(y), f32(j) * f32(spacing)) for j in range(n) for i in range(n)]
    tris = []
    for j in range(n - 1):
        for i in range(n - 1):
            v = base + j * n + i
            r = v + n
            tris += [(v, v + 1, r), (v + 1, r + 1, r) if second_winding else (r, v + 1, r + 1)]
    return pos, tris


def two_layers(n, spacing, gap, second_winding=True):
    pos, tris = [], []
    for y in (0.0, gap):
        p, t = _grid(n, spacing, y, len(pos), second_winding)
        pos += p
        tris += t
    return np.array(pos, f32), np.array(tris, np.uint32)


def seg_dist(p, a, b, c, d):
    return O.seg_seg(np.array([p[a], p[b], p[c], p[d]], f32))[2]


def test_hash_is_superset_of_brute_force():  # broadphase.rs:867-911
    pos, tris = two_layers(5, 0.1, 0.03, second_winding=False)
    dhat = 0.05
    pairs = set(O.vt_pairs(pos, tris, dhat))
    # one-ring exclusion: every vertex sharing a triangle with v, and v itself
    ring = [set([v]) for v in range(len(pos))]
    for t in tris:
        for a in t:
            ring[a].update(int(b) for b in t)
    for vi in range(len(pos)):
        for ti, t in enumerate(tris):
            if ring[vi] & set(int(v) for v in t):
                continue
            d = O.point_tri(np.array([pos[vi], *pos[t]], f32))[0]
            if d < dhat:
                assert (vi, ti) in pairs, (vi, ti, d)
    assert pairs


def test_edge_edge_pairs_is_a_superset_of_brute_force():  # broadphase.rs:938-986
    for n, spacing, gap, search in ((12, 0.02, 0.03, 0.10), (12, 0.02, 0.03, 0.02), (18, 0.05, 0.01, 0.02)):
        pos, tris = two_layers(n, spacing, gap)
        edges = O.unique_edges(tris)
        got = set(O.ee_pairs(pos, edges, search))
        # brute force over pairs whose boxes come within search (the distance is checked
        # only there; farther pairs cannot be within search)
        lo = np.minimum(pos[edges[:, 0]], pos[edges[:, 1]])
        hi = np.maximum(pos[edges[:, 0]], pos[edges[:, 1]])
        near = np.all((lo[:, None, :] - search <= hi[None, :, :]) & (lo[None, :, :] - search <= hi[:, None, :]), -1)
        true_close = 0
        for i, j in zip(*np.nonzero(np.triu(near, 1))):
            a, b = edges[i], edges[j]
            if len({int(a[0]), int(a[1]), int(b[0]), int(b[1])}) < 4:
                continue
            if seg_dist(pos, a[0], a[1], b[0], b[1]) <= search:
                true_close += 1
                assert (int(i), int(j)) in got, (n, search, i, j)
        assert true_close > 100


def test_edge_edge_candidate_count_is_the_reference_number():  # broadphase.rs:994-1002
    pos, tris = two_layers(30, 0.02, 0.01)
    edges = O.unique_edges(tris)
    assert len(edges) == 5162
    assert len(O.ee_pairs(pos, edges, 0.02)) == 268075


def two_sheets():
    """broadphase.rs:1131-1161: a static lower sheet and a movable upper one 0.02 above it,
    with one pinned vertex inside the upper sheet."""
    n = 6
    pos, tris, movable = [], [], []
    for y, cloth in ((0.0, False), (0.02, True)):
        p, t = _grid(n, 0.05, y, len(pos), True)
        pos += p
        tris += t
        movable += [cloth] * (n * n)
    movable[n * n + (n // 2) * n + n // 2] = False
    tris = np.array(tris, np.uint32)
    return np.array(pos, f32), tris, O.unique_edges(tris), np.array(movable, np.uint8)


def test_an_all_movable_mask_changes_nothing():  # broadphase.rs:1170-1196
    pos, tris, edges, _ = two_sheets()
    allm = np.ones(len(pos), np.uint8)
    for search in (0.01, 0.05, 0.2):
        off, on = O.vt_pairs(pos, tris, search), O.vt_pairs(pos, tris, search, movable=allm)
        assert off and off == on
        off, on = O.ee_pairs(pos, edges, search), O.ee_pairs(pos, edges, search, movable=allm)
        assert off and off == on


def test_a_static_body_drops_exactly_the_inert_pairs():  # broadphase.rs:1198-1280
    pos, tris, edges, movable = two_sheets()

    def inert(vs):
        return all(not movable[int(v)] for v in vs)

    ee_dropped = ee_cross = 0
    for search in (0.01, 0.05, 0.2):
        off = O.vt_pairs(pos, tris, search)
        on = O.vt_pairs(pos, tris, search, movable=movable)
        want = [(v, t) for v, t in off if not (inert([v]) and inert(tris[t]))]
        dropped = len(off) - len(want)
        cross = sum(1 for v, t in want if bool(movable[v]) != inert(tris[t]))
        assert dropped > 0 and cross > 0
        assert on == want
        on = O.ee_pairs(pos, edges, search, movable=movable)
        seen = set(on)
        assert not any(inert(edges[i]) and inert(edges[j]) for i, j in on)
        for i in range(len(edges)):
            for j in range(i + 1, len(edges)):
                a, b = edges[i], edges[j]
                if len({int(a[0]), int(a[1]), int(b[0]), int(b[1])}) < 4:
                    continue
                if seg_dist(pos, a[0], a[1], b[0], b[1]) > search:
                    continue
                ia, ib = inert(a), inert(b)
                if ia and ib:
                    ee_dropped += 1
                    continue
                ee_cross += int(ia != ib)
                assert (i, j) in seen, (search, i, j)
    assert ee_dropped > 0 and ee_cross > 0


def test_large_elements_with_tiny_search_still_find_every_pair():  # broadphase.rs:1361-1445
    search = f32(1.0e-3)
    pos = []
    for i in range(6):
        x = f32(i) * f32(0.5)
        pos += [(x, 0, 0), (x, 0, 1), (x, 0.4e-3, 0), (x, 0.4e-3, 1)]
    pos = np.array(pos, f32)
    edges = np.array([e for i in range(6) for e in ([4 * i, 4 * i + 1], [4 * i + 2, 4 * i + 3])], np.uint32)
    tris = np.array([[4 * i, 4 * i + 1, 4 * i + 2] for i in range(6)], np.uint32)
    got = set(O.ee_pairs(pos, edges, search))
    brute = 0
    for i in range(len(edges)):
        for j in range(i + 1, len(edges)):
            a, b = edges[i], edges[j]
            if len({int(a[0]), int(a[1]), int(b[0]), int(b[1])}) < 4:
                continue
            alo, ahi = np.minimum(pos[a[0]], pos[a[1]]), np.maximum(pos[a[0]], pos[a[1]])
            blo, bhi = np.minimum(pos[b[0]], pos[b[1]]), np.maximum(pos[b[0]], pos[b[1]])
            if np.all((alo - search <= bhi) & (blo - search <= ahi)):
                brute += 1
                assert (i, j) in got
    assert brute > 0
    vt = set(O.vt_pairs(pos, tris, search, exclude_one_ring=False))
    vt_brute = 0
    for ti, t in enumerate(tris):
        lo, hi = pos[t].min(0), pos[t].max(0)
        for vi, p in enumerate(pos):
            if np.all((p >= lo - search) & (p <= hi + search)):
                vt_brute += 1
                assert (vi, ti) in vt
    assert vt_brute > 0


def test_grid_cell_is_bounded_below_by_both_inputs():  # broadphase.rs:1449-1468
    assert O.grid_cell(1.0e-3, 0.15) == f32(0.15)
    assert O.grid_cell(0.5, 0.15) == f32(0.5)
    assert O.grid_cell(0.0, 0.0) > 0.0


def test_edge_triangle_intersect_cases():  # contact.rs:1816-1853
    a, b, c = (0, 0, 0), (1, 0, 0), (0, 1, 0)
    assert O.edge_triangle_intersect((0.25, 0.25, 1), (0.25, 0.25, -1), a, b, c)
    assert not O.edge_triangle_intersect((0.25, 0.25, 1), (0.25, 0.25, 0.5), a, b, c)  # same side
    assert not O.edge_triangle_intersect((2, 0.25, 1), (2, 0.25, -1), a, b, c)  # outside the triangle
    assert not O.edge_triangle_intersect((-1, 0.25, 0), (2, 0.25, 0), a, b, c)  # coplanar


def stabbed_sheet():
    """broadphase.rs:1011-1033: a 7 x 7 sheet at 0.1 spacing and a vertical edge through it
    near its middle, appended after the sheet's unique edges."""
    p, t = _grid(7, 0.1, 0.0, 0, True)
    base = len(p)
    pos = np.array(p + [(0.32, -0.2, 0.31), (0.32, 0.2, 0.31)], f32)
    tris = np.array(t, np.uint32)
    edges = np.concatenate([O.unique_edges(tris), np.array([[base, base + 1]], np.uint32)])
    return pos, edges, tris


def test_streaming_offers_the_same_candidate_set_as_the_materialised_list():  # broadphase.rs:1036-1066
    pos, edges, tris = stabbed_sheet()
    for search in (0.05, 0.15, 0.4):
        want = O.et_pairs(pos, edges, tris, search)
        found, got = O.et_any(pos, edges, tris, search, mode=O.ET_NEVER)
        assert not found, "a never-matching predicate must exhaust the candidates"
        assert sorted(set(got)) == want, search
        assert want, search


def test_streaming_short_circuits_on_the_first_match():  # broadphase.rs:1068-1086
    pos, edges, tris = stabbed_sheet()
    total = len(O.et_pairs(pos, edges, tris, 0.4))
    found, seen = O.et_any(pos, edges, tris, 0.4, mode=O.ET_FIRST)
    assert found and seen == 1
    assert total > 10


def test_streaming_agrees_on_whether_an_edge_pierces():  # broadphase.rs:1088-1117
    pos, edges, tris = stabbed_sheet()
    assert O.et_any(pos, edges, tris, 0.15, mode=O.ET_PIERCE)[0], "the spike through the sheet must be detected"
    pos[-2, 1] = 0.2
    pos[-1, 1] = 0.6
    assert not O.et_any(pos, edges, tris, 0.15, mode=O.ET_PIERCE)[0], "a spike clear of the sheet must not be"


def test_the_intersection_predicate_sees_cloth_through_body_but_not_body_through_body():  # broadphase.rs:1279-1346
    pos, tris, edges, movable = two_sheets()

    def pierced(pos, edges, movable):
        return O.et_any(pos, edges, tris, 0.05, movable=movable, mode=O.ET_PIERCE)[0]

    assert not pierced(pos, edges, movable), "the undisturbed two-sheet scene must not intersect"
    # a movable spike through the static lower sheet, ending below the movable upper one
    base = len(pos)
    pos = np.concatenate([pos, np.array([(0.12, 0.015, 0.13), (0.12, -0.03, 0.13)], f32)])
    movable = np.concatenate([movable, np.ones(2, np.uint8)])
    edges = np.concatenate([edges, np.array([[base, base + 1]], np.uint32)])
    assert pierced(pos, edges, movable), "a movable edge piercing the static body must be reported"
    # the same spike static: a pierce between immovable primitives only is not reported ...
    movable[base] = movable[base + 1] = 0
    assert not pierced(pos, edges, movable)
    # ... although it is there: unfiltered, it is found
    assert pierced(pos, edges, None)
    # a static edge through the movable upper sheet (the second pass's case)
    base = len(pos)
    pos = np.concatenate([pos, np.array([(0.07, 0.05, 0.08), (0.07, 0.008, 0.08)], f32)])
    movable = np.concatenate([movable, np.zeros(2, np.uint8)])
    edges = np.concatenate([edges, np.array([[base, base + 1]], np.uint32)])
    assert pierced(pos, edges, movable), "a static edge piercing a movable triangle must be reported"


def test_edges_are_unique_and_deterministic():  # geometry.rs:50-63
    tris = np.array([[0, 1, 2], [2, 1, 3]], np.uint32)
    e = O.unique_edges(tris)
    assert len(e) == 5
    assert np.array_equal(e, O.unique_edges(tris))
    assert sum(1 for a, b in e.tolist() if (a, b) == (1, 2)) == 1
    assert e.tolist() == sorted(e.tolist())
