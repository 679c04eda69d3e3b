"""Pins the LBVH oracle against the reference's own tests (engine-gpu/src/karras.rs:313-333,
radix.rs:361-417, morton.rs:273-311, bvh_traverse.rs:287-377) and brute force."""
import numpy as np
import oracle_py as O

from mguso import scenes


def grid_mesh(n, a=73, b=179, m=17, s=0.005):
    """The reference's jittered test grid (morton.rs:234-255 / karras.rs:292-311)."""
    pos = []
    for j in range(n):
        for i in range(n):
            h = np.float32(((i * a + j * b) % m)) * np.float32(s)
            pos.append((np.float32(i) * np.float32(0.1), h, np.float32(j) * np.float32(0.1)))
    tris = []
    for j in range(n - 1):
        for i in range(n - 1):
            v = j * n + i
            r = v + n
            tris.append((v, v + 1, r))
            tris.append((r, v + 1, r + 1))
    return np.array(pos, np.float32), np.array(tris, np.uint32)


def compact_bits(x):
    x &= 0x09249249
    x = (x | (x >> 2)) & 0x030c30c3
    x = (x | (x >> 4)) & 0x0300f00f
    x = (x | (x >> 8)) & 0x030000ff
    x = (x | (x >> 16)) & 0x000003ff
    return x


def inorder_leaves(left, right, n):
    """karras.rs:264-283: left-first leaf order; 0..n for a well-formed tree."""
    if n < 2:
        return list(range(n))
    out, st = [], [(0, False)]
    while st:
        node, leaf = st.pop()
        if leaf:
            out.append(node)
            continue
        r, l = int(right[node]), int(left[node])
        st.append((r & 0x7fffffff, bool(r & 0x80000000)))
        st.append((l & 0x7fffffff, bool(l & 0x80000000)))
    return out


def test_karras_tree_is_well_formed():  # karras.rs:313-333
    cases = [list(range(16)), [i // 3 for i in range(1000)], [5] * 6, [0, 0, 1, 2, 2, 2, 9, 9]]
    for codes in cases:
        for bits in (30, 63):
            left, right = O.karras(np.array(codes, np.uint64), bits)
            assert left.size == len(codes) - 1
            assert inorder_leaves(left, right, len(codes)) == list(range(len(codes)))


def test_morton30_quantises_centroids():
    pos, tris = grid_mesh(20)
    keys = O.morton(pos, tris, 30)
    cent = pos[tris].sum(axis=1, dtype=np.float32) / np.float32(3.0)
    lo, hi = cent.min(0), cent.max(0)
    n = (cent - lo) * (np.float32(1.0) / (hi - lo))
    q = np.clip(np.clip(n, 0, 1) * np.float32(1023.0), 0, 1023).astype(np.uint32)
    dec = np.array([[compact_bits(int(k) >> 2), compact_bits(int(k) >> 1), compact_bits(int(k))] for k in keys])
    assert np.array_equal(dec, q)


def test_morton63_bit_layout():
    pos, tris = grid_mesh(12)
    keys = O.morton(pos, tris, 63)
    cent = pos[tris].sum(axis=1, dtype=np.float32) / np.float32(3.0)
    lo, hi = cent.min(0), cent.max(0)
    n = (cent - lo) * (np.float32(1.0) / (hi - lo))
    q = np.clip(np.clip(n, 0, 1) * np.float32(2097151.0), 0, 2097151).astype(np.uint64)
    for k, (x, y, z) in zip(keys.tolist(), q.tolist()):
        want = 0
        for b in range(21):
            want |= ((x >> b) & 1) << (3 * b + 2) | ((y >> b) & 1) << (3 * b + 1) | ((z >> b) & 1) << (3 * b)
        assert k == want
    assert int(keys.max()) < (1 << 63)


def test_sort_pairs_is_stable():  # radix.rs:382-417
    for n in (1, 3, 257, 1000, 5000):
        keys = np.array([(i * 40503 + 12345) % 500 for i in range(n)], np.uint64)
        k, v = O.sort_pairs(keys, np.arange(n, dtype=np.uint32))
        assert np.all(k[1:] >= k[:-1])
        assert np.array_equal(keys[v], k)
        eq = k[1:] == k[:-1]
        assert np.all(v[1:][eq] > v[:-1][eq])


def test_refit_boxes_are_subtree_unions():
    pos, tris = grid_mesh(9)
    keys, perm, left, right, node, _ = O.lbvh(pos, tris, 30, 0.01)
    leaf = np.stack([pos[tris[perm]].min(1), pos[tris[perm]].max(1)], 1).reshape(-1, 6)

    def subtree(i, is_leaf):
        if is_leaf:
            return [i]
        l, r = int(left[i]), int(right[i])
        return subtree(l & 0x7fffffff, bool(l >> 31)) + subtree(r & 0x7fffffff, bool(r >> 31))

    for i in range(left.size):
        lv = subtree(i, False)
        assert np.array_equal(node[i, :3], leaf[lv, :3].min(0))
        assert np.array_equal(node[i, 3:], leaf[lv, 3:].max(0))


def test_lbvh_pair_set_equals_the_box_predicate():  # bvh_traverse.rs:287-377 + exact set
    pos, tris = scenes.triangle_soup(3000, seed=11, edge=0.02)
    dhat = np.float32(0.01)
    _, _, _, _, _, pairs = O.lbvh(pos, tris, 30, float(dhat))
    lo = pos[tris].min(1)
    hi = pos[tris].max(1)
    qlo = pos - dhat
    qhi = pos + dhat
    want = []
    for v in range(pos.shape[0]):
        ok = np.all(qlo[v] <= hi, axis=1) & np.all(lo <= qhi[v], axis=1)
        want += [(v, t) for t in np.nonzero(ok)[0]]
    got = sorted(map(tuple, pairs.tolist()))
    assert got == sorted(want)
