"""GPU LBVH parity through the C ABI: Morton keys, sort permutation, Karras tree, node boxes
and the candidate pair set must be bit-exact against the CPU oracle."""
import numpy as np
import pytest

import oracle_py as O
from mguso import lbvh, scenes

pytestmark = pytest.mark.gpu


def sorted_pairs(p):
    p = np.asarray(p, np.uint64).reshape(-1, 2)
    key = (p[:, 0] << np.uint64(32)) | p[:, 1]
    return np.sort(key)


def two_layer_mesh(n=40, gap=0.03):
    """bvh_traverse.rs:250-285 style: two stacked jittered grid sheets."""
    xs = np.linspace(0, 1, n, dtype=np.float32)
    X, Z = np.meshgrid(xs, xs)
    rng = np.random.default_rng(5)
    pos = []
    for layer in range(2):
        Y = np.full_like(X, layer * gap) + (rng.random(X.shape, dtype=np.float32) * np.float32(0.002))
        pos.append(np.stack([X, Y, Z], -1).reshape(-1, 3))
    pos = np.concatenate(pos).astype(np.float32)
    t = scenes.grid_tris(n)
    tris = np.concatenate([t, t + n * n]).astype(np.uint32)
    return pos, tris


@pytest.mark.parametrize("bits", [30, 63])
@pytest.mark.parametrize("case", ["two_layer", "soup", "degenerate"])
def test_lbvh_bit_exact(ctx, bits, case):  # engine-gpu morton.rs:272-328 (codes, then the radix sort)
    if case == "two_layer":
        pos, tris = two_layer_mesh()
        dhat = 0.05
    elif case == "soup":
        pos, tris = scenes.triangle_soup(200_000, seed=9)
        dhat = 1e-3
    else:
        # duplicate centroids (all-equal codes) and a single triangle repeated
        pos = np.zeros((30, 3), np.float32)
        pos[:, 0] = np.repeat(np.arange(10, dtype=np.float32) * np.float32(1e-7), 3)
        tris = np.arange(30, dtype=np.uint32).reshape(10, 3)
        dhat = 1e-3
    keys, perm, pairs, cnt = lbvh.build_query(ctx, pos, tris, bits, dhat)
    ok, op, ol, orr, on, opairs = O.lbvh(pos, tris, bits, dhat)
    assert np.array_equal(keys, ok), "Morton keys differ"
    assert np.array_equal(perm, op), "sort permutation differs"
    assert cnt == opairs.shape[0]
    assert np.array_equal(sorted_pairs(pairs), sorted_pairs(opairs)), "pair set differs"


def test_lbvh_tree_and_boxes_bit_exact(ctx):
    import torch
    pos, tris = scenes.triangle_soup(100_000, seed=4)
    b = lbvh.Lbvh(ctx)
    pd, td = torch.from_numpy(pos).cuda(), torch.from_numpy(tris.astype(np.int32)).cuda()
    b.build(pd.data_ptr(), pos.shape[0], td.data_ptr(), tris.shape[0], 63, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    keys, perm, left, right, node = b.download()
    ok, op, ol, orr, on, _ = O.lbvh(pos, tris, 63, 1e-3, cap=1)
    assert np.array_equal(keys, ok) and np.array_equal(perm, op)
    assert np.array_equal(left, ol) and np.array_equal(right, orr)
    assert np.array_equal(node, on)


def test_lbvh_empty_and_single(ctx):
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    keys, perm, pairs, cnt = lbvh.build_query(ctx, pos, np.array([[0, 1, 2]], np.uint32), 30, 0.1)
    assert cnt == 3 and sorted(pairs[:, 0].tolist()) == [0, 1, 2]
    keys, perm, pairs, cnt = lbvh.build_query(ctx, pos, np.zeros((0, 3), np.uint32), 30, 0.1)
    assert cnt == 0


def test_pair_overflow_reports_total(ctx):
    pos, tris = two_layer_mesh(20)
    _, _, _, _, _, opairs = O.lbvh(pos, tris, 30, 0.05)
    keys, perm, pairs, cnt = lbvh.build_query(ctx, pos, tris, 30, 0.05, cap=10)  # retried internally
    assert cnt == opairs.shape[0]


@pytest.mark.parametrize("bits", [32, 64])
def test_onesweep_sort_stable(ctx, bits):
    import torch
    from mguso.lbvh import radix_sort_pairs
    rng = np.random.default_rng(7)
    # sizes in the order of a growing buffer: each larger n reallocates the scratch
    for n in (1, 3, 2047, 2048, 2049, 100_003, 1_054_816, 3_000_000, 1_044_128):
        if bits == 32:
            keys = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
            keys[: n // 3] = keys[: n // 3] % 500  # duplicate-heavy prefix
            kt = torch.from_numpy(keys.view(np.int32)).cuda()
        else:
            keys = rng.integers(0, 1 << 63, n, dtype=np.uint64)
            keys[: n // 3] = keys[: n // 3] % 500
            kt = torch.from_numpy(keys.view(np.int64)).cuda()
        vt = torch.arange(n, dtype=torch.int32, device="cuda")
        radix_sort_pairs(ctx, kt.data_ptr(), vt.data_ptr(), n, bits, torch.cuda.current_stream().cuda_stream)
        lbvh.radix_sort_status(ctx)  # no look-back wait gave up
        gk = kt.cpu().numpy().view(np.uint32 if bits == 32 else np.uint64)
        gv = vt.cpu().numpy().view(np.uint32)
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(gv, order.astype(np.uint32))
        assert np.array_equal(gk, keys[order])


def test_lbvh_full_size_4m(ctx):
    """4 194 304 triangles (uniform in the unit cube, 2 mm edges). Keys, permutation, tree and boxes bit-exact
    against the oracle; the pair count and a hash of the sorted pair set equal too."""
    pos, tris = scenes.triangle_soup(4 << 20, seed=3)
    for bits in (30, 63):
        keys, perm, pairs, cnt = lbvh.build_query(ctx, pos, tris, bits, 1e-3)
        ok, op, _, _, _, opairs = O.lbvh(pos, tris, bits, 1e-3)
        assert np.array_equal(keys, ok) and np.array_equal(perm, op)
        assert cnt == opairs.shape[0]
        assert np.array_equal(sorted_pairs(pairs), sorted_pairs(opairs))
