"""Pins the CPU oracle's CSR and CG against the reference's own unit tests
(engine-core/src/csr.rs:471-588, linsolve.rs:856-1030)."""
import numpy as np
import oracle_py as O


def laplacian_1d(n):
    r, c, v = [], [], []
    for i in range(n):
        r.append(i); c.append(i); v.append(2.0)
        if i > 0:
            r.append(i); c.append(i - 1); v.append(-1.0)
        if i + 1 < n:
            r.append(i); c.append(i + 1); v.append(-1.0)
    return O.csr_from_triplets(n, r, c, v)


def lcg_triplets(n, count, seed=12345):
    s = seed
    out_r, out_c, out_v = [], [], []
    M = (1 << 64) - 1
    for _ in range(count):
        vals = []
        for _k in range(3):
            s = (s * 6364136223846793005 + 1442695040888963407) & M
            vals.append(s >> 33)
        out_r.append(vals[0] % n)
        out_c.append(vals[1] % n)
        out_v.append(np.float32(vals[2] % 1000) * np.float32(1.0e-3))
    return np.array(out_r, np.uint32), np.array(out_c, np.uint32), np.array(out_v, np.float32)


def test_triplets_coalesce_and_sort():  # csr.rs:582-588
    rp, ci, vv = O.csr_from_triplets(2, [0, 0, 0], [1, 1, 0], [1.0, 2.0, 5.0])
    assert rp.tolist() == [0, 2, 2]
    assert ci.tolist() == [0, 1]
    assert vv.tolist() == [5.0, 3.0]


def test_laplacian_spmv_is_correct():  # csr.rs:573-580
    rp, ci, vv = laplacian_1d(5)
    y = O.spmv(5, rp, ci, vv, np.ones(5, np.float32))
    assert y.tolist() == [1.0, 0.0, 0.0, 0.0, 1.0]


def test_sink_matches_from_triplets():  # csr.rs:471-531
    n = 3 * 64
    r, c, v = lcg_triplets(n, 200_000)
    want = O.csr_from_triplets(n, r, c, v)
    got = O.csr_from_triplets(n, r, c, v, sink=True)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    big = [np.tile(a, 12) for a in (r, c, v)]
    got = O.csr_from_triplets(n, *big, sink=True)
    want = O.csr_from_triplets(n, *big)
    assert np.array_equal(got[1], want[1])
    assert np.all(np.abs(got[2] - want[2]) <= 1e-4 * np.maximum(np.abs(want[2]), 1.0))


def test_finish_dirichlet_equals_retaining_triplets():  # csr.rs:536-571
    n = 3 * 8
    pinned = np.array([0, 1, 0, 0, 1, 0, 0, 0], np.uint8)
    r, c, v = [], [], []
    for i in range(n):
        for j in range(n):
            if (i * 7 + j * 3) % 5 != 0:
                r.append(i); c.append(j); v.append(np.float32(0.25) + np.float32(i) * np.float32(0.5)
                                                     - np.float32(j) * np.float32(0.125))
    got = O.csr_from_triplets(n, r, c, v, sink=True, pinned=pinned)
    kept = [(a, b, w) for a, b, w in zip(r, c, v) if not pinned[a // 3] and not pinned[b // 3]]
    for i, p in enumerate(pinned):
        if p:
            for k in range(3):
                kept.append((3 * i + k, 3 * i + k, 1.0))
    want = O.csr_from_triplets(n, *zip(*kept))
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


def test_cpu_cg_solves_laplacian():  # linsolve.rs:856-867
    rp, ci, vv = laplacian_1d(64)
    xs = np.cos(np.arange(64, dtype=np.float32) * np.float32(0.05)).astype(np.float32)
    b = O.spmv(64, rp, ci, vv, xs)
    x, it, _ = O.cg(64, rp, ci, vv, b, 1e-8, 500, "block")  # n % 3 != 0 -> diagonal
    assert np.abs(x - xs).max() < 1e-3


def block_system():
    v = 40
    n = 3 * v
    d = [[6.0, 3.0, 2.0], [3.0, 6.0, 3.0], [2.0, 3.0, 6.0]]
    r, c, val = [], [], []
    for i in range(v):
        for a in range(3):
            for b in range(3):
                r.append(3 * i + a); c.append(3 * i + b); val.append(d[a][b])
        if i + 1 < v:
            for a in range(3):
                r.append(3 * i + a); c.append(3 * (i + 1) + a); val.append(-1.0)
                r.append(3 * (i + 1) + a); c.append(3 * i + a); val.append(-1.0)
    return n, O.csr_from_triplets(n, r, c, val)


def test_block_jacobi_cuts_iterations():  # linsolve.rs:872-909
    n, (rp, ci, vv) = block_system()
    xs = (np.sin(np.arange(n, dtype=np.float32) * np.float32(0.1)) + np.float32(0.5)).astype(np.float32)
    b = O.spmv(n, rp, ci, vv, xs)
    x1, i_scalar, _ = O.cg(n, rp, ci, vv, b, 1e-8, 2000, "diagonal")
    x2, i_block, _ = O.cg(n, rp, ci, vv, b, 1e-8, 2000, "block")
    assert np.abs(x1 - xs).max() < 1e-3 and np.abs(x2 - xs).max() < 1e-3
    assert i_block < i_scalar


def grid_system(gx, gy, diag, neigh4=True):
    nv = gx * gy
    n = 3 * nv
    r, c, v = [], [], []
    idx = lambda i, j: j * gx + i  # noqa: E731
    for j in range(gy):
        for i in range(gx):
            w = idx(i, j)
            if isinstance(diag, list):
                for a in range(3):
                    for b in range(3):
                        r.append(3 * w + a); c.append(3 * w + b); v.append(diag[a][b])
            else:
                for a in range(3):
                    r.append(3 * w + a); c.append(3 * w + a); v.append(diag)
            for di, dj in ((1, 0), (-1, 0), (0, 1), (0, -1)) if not isinstance(diag, list) else \
                    [(-1, 0), (1, 0), (0, -1), (0, 1)]:
                ni, nj = i + di, j + dj
                if 0 <= ni < gx and 0 <= nj < gy:
                    u = idx(ni, nj)
                    for a in range(3):
                        r.append(3 * w + a); c.append(3 * u + a); v.append(-1.0)
    return n, O.csr_from_triplets(n, r, c, v)


def test_schwarz_beats_block_jacobi_on_grid():  # linsolve.rs:914-966
    n, (rp, ci, vv) = grid_system(12, 12, [[6.0, 1.0, 0.5], [1.0, 6.0, 1.0], [0.5, 1.0, 6.0]])
    xs = np.sin(np.arange(n, dtype=np.float32) * np.float32(0.05)).astype(np.float32)
    b = O.spmv(n, rp, ci, vv, xs)
    _, i_block, _ = O.cg(n, rp, ci, vv, b, 1e-8, 3000, "block")
    x, i_sch, _ = O.cg(n, rp, ci, vv, b, 1e-8, 3000, "schwarz", 16)
    assert np.abs(x - xs).max() < 1e-3
    assert i_sch < i_block


def test_stateful_schwarz_matches_and_caches():  # linsolve.rs:1032-1070
    n, (rp, ci, vv) = grid_system(10, 10, 5.0)
    xs = np.cos(np.arange(n, dtype=np.float32) * np.float32(0.07)).astype(np.float32)
    b = O.spmv(n, rp, ci, vv, xs)
    x1, _, _ = O.linear_solve(n, rp, ci, vv, b, 1e-8, 3000, "schwarz", 16)
    x2, _, _ = O.linear_solve(n, rp, ci, vv, b, 1e-8, 3000, "schwarz", 16)
    assert np.array_equal(x1, x2)
    assert np.abs(x1 - xs).max() < 1e-3


def test_schwarz_domains_are_bfs_aggregates():
    # linsolve.rs:152-173: domain 0 is seeded at vertex 0 and grows breadth-first.
    n, (rp, ci, vv) = grid_system(10, 10, 5.0)
    dom, nd = O.schwarz_domains(n, rp, ci, 16)
    counts = np.bincount(dom)
    assert counts.max() <= 16 and counts.sum() == 100 and nd == counts.size
    assert dom[0] == 0 and dom[1] == 0 and dom[10] == 0


def _vector_laplacian(g, diag):
    """Elliptic g x g vector Laplacian: `diag` on every scalar diagonal, -1 to the four grid
    neighbours per component (the reference's multilevel test system)."""
    r, c, v = [], [], []
    idx = lambda i, j: j * g + i  # noqa: E731
    for j in range(g):
        for i in range(g):
            a = idx(i, j)
            for k in range(3):
                r.append(3 * a + k); c.append(3 * a + k); v.append(diag)
            for di, dj in ((1, 0), (-1, 0), (0, 1), (0, -1)):
                ni, nj = i + di, j + dj
                if 0 <= ni < g and 0 <= nj < g:
                    w = idx(ni, nj)
                    for k in range(3):
                        r.append(3 * a + k); c.append(3 * w + k); v.append(-1.0)
    return O.csr_from_triplets(3 * g * g, r, c, v)


def test_multilevel_schwarz_solves_and_cuts_iterations():  # linsolve.rs:970-1027
    g = 32
    n = 3 * g * g
    rp, ci, vv = _vector_laplacian(g, 4.01)
    x_star = np.sin(np.arange(n, dtype=np.float32) * np.float32(0.03)).astype(np.float32)
    b = O.spmv(n, rp, ci, vv, x_star)
    x1, i1, _ = O.linear_solve(n, rp, ci, vv, b, 1e-8, 5000, "schwarz", 8)
    x2, i2, _ = O.linear_solve_ml(n, rp, ci, vv, b, 1e-8, 5000, 8, 0.7)
    assert np.abs(x2 - x_star).max() < 1e-3, "2-level Schwarz must solve"
    assert i2 < i1, (i2, i1)
    # a second solve on the same sparsity is identical
    x3, _, _ = O.linear_solve_ml(n, rp, ci, vv, b, 1e-8, 5000, 8, 0.7)
    assert np.array_equal(x2, x3)


def test_multilevel_apply_is_level0_plus_weighted_coarse_correction():  # linsolve.rs:641-666
    g = 12
    n = 3 * g * g
    rp, ci, vv = _vector_laplacian(g, 4.5)
    r = np.cos(np.arange(n) * 0.37)
    z0 = O.schwarz_apply(n, rp, ci, vv, 8, r)
    agg, cdom, (crp, cci, cv) = O.schwarz_ml_plan(n, rp, ci, vv, 8)
    nc = crp.size // 3
    # Galerkin coarse operator: every fine entry summed into its (coarse row, coarse col)
    dense = np.zeros((n, n))
    for i in range(n):
        dense[i, ci[rp[i]:rp[i + 1]]] = vv[rp[i]:rp[i + 1]]
    C = np.zeros((3 * nc, n))
    for v_ in range(g * g):
        for k in range(3):
            C[3 * agg[v_] + k, 3 * v_ + k] = 1.0
    a1 = C @ dense @ C.T
    cd = np.zeros((3 * nc, 3 * nc))
    for i in range(3 * nc):
        cd[i, cci[crp[i]:crp[i + 1]]] = cv[crp[i]:crp[i + 1]]
    assert np.allclose(cd, a1, rtol=1e-6, atol=1e-5)
    # z = S0 r + w C^T S1 (C r), S1 = one-level Schwarz over the coarse operator
    ec = O.schwarz_apply(3 * nc, crp, cci, cv, 8, C @ r)
    for w in (0.7, 1.0):
        z = O.schwarz_ml_apply(n, rp, ci, vv, 8, w, r)
        assert np.allclose(z, z0 + w * (C.T @ ec), rtol=1e-12, atol=1e-12)
