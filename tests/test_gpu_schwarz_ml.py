"""Two-level Galerkin additive Schwarz on the GPU against the oracle's MultilevelSchwarz /
SchwarzMlCpu (engine-core/src/linsolve.rs:534-836), through the C ABI: the coarse domains,
the apply z = S0 r + w C1^T S1 (C1 r), the PCG solve, and an implicit step preconditioned by
it."""
import numpy as np
import pytest

import oracle_py as O
from mguso import Bsr, CsrMatrix, CudaLinearSolver, ImplicitSolver, Schwarz, scenes

pytestmark = pytest.mark.gpu


def torch_dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def vector_laplacian(g, diag):
    """The reference's multilevel test system: g x g grid, `diag` on the diagonal, -1 to the
    four neighbours per component (linsolve.rs:976-996)."""
    nv = g * g
    rows, cols = [], []
    for j in range(g):
        for i in range(g):
            v = j * g + i
            nb = [v] + [(j + dj) * g + i + di for di, dj in ((1, 0), (-1, 0), (0, 1), (0, -1))
                        if 0 <= i + di < g and 0 <= j + dj < g]
            for w in sorted(nb):
                rows.append(v)
                cols.append(w)
    rp = np.zeros(nv + 1, np.uint32)
    np.add.at(rp, np.array(rows) + 1, 1)
    rp = np.cumsum(rp).astype(np.uint32)
    col = np.array(cols, np.uint32)
    val = np.zeros((col.size, 3, 3), np.float32)
    for k, (v, w) in enumerate(zip(rows, cols)):
        val[k] = np.eye(3, dtype=np.float32) * (np.float32(diag) if v == w else np.float32(-1.0))
    return nv, rp, col, val


def systems():
    nb, rp, col, val = vector_laplacian(32, 4.01)
    yield "laplacian32", 8, (nb, rp, col, val)
    yield "cloth_grid23", 16, scenes.grid_bsr(23, 5)


@pytest.mark.parametrize("name,domain,sysm", list(systems()))
def test_two_level_apply_matches_oracle(ctx, name, domain, sysm):
    import torch

    nb, rp, col, val = sysm
    N, srp, sci, svv = scenes.bsr_to_csr(nb, rp, col, val)
    a = Bsr(ctx, nb, rp, col, val)
    s = Schwarz(a, domain, levels=2, weight=0.7)
    agg, cdom, _ = O.schwarz_ml_plan(N, srp, sci, svv, domain)
    assert np.array_equal(s.domains(), agg)
    assert np.array_equal(s.coarse_domains(), cdom)
    st = torch.cuda.current_stream().cuda_stream
    s.factor(st)
    for seed in (4, 5):
        r = np.random.default_rng(seed).standard_normal(N).astype(np.float32)
        rd, zd = torch_dev(r), torch.zeros(N, device="cuda")
        s.apply(rd.data_ptr(), zd.data_ptr(), st)
        torch.cuda.synchronize()
        z = zd.cpu().numpy()
        want = O.schwarz_ml_apply(N, srp, sci, svv, domain, 0.7, r.astype(np.float64))
        assert np.abs(z - want).max() <= 1e-4 * np.abs(want).max(), (name, np.abs(z - want).max())


@pytest.mark.parametrize("precision", ["mixed", "fp32"])
def test_two_level_pcg_matches_oracle_and_cuts_iterations(ctx, precision):
    """linsolve.rs:970-1027 on the GPU: the 2-level solver solves the 32 x 32 vector
    Laplacian, in fewer iterations than one level with the same domains, with the oracle's
    iteration count and solution."""
    nb, rp, col, val = vector_laplacian(32, 4.01)
    N, srp, sci, svv = scenes.bsr_to_csr(nb, rp, col, val)
    A = CsrMatrix(N, srp, sci, svv)
    x_star = np.sin(np.arange(N, dtype=np.float32) * np.float32(0.03)).astype(np.float32)
    b = O.spmv(N, srp, sci, svv, x_star)
    tol = 1e-8 if precision == "mixed" else 1e-5
    one = CudaLinearSolver(ctx, "schwarz", 8, precision)
    two = CudaLinearSolver(ctx, "schwarz-ml", 8, precision, weight=0.7)
    one.solve(A, b, tol, 5000)
    x2 = two.solve(A, b, tol, 5000)
    i1, i2 = one.last_stats().iters, two.last_stats().iters
    assert np.abs(x2 - x_star).max() < 1e-3
    assert i2 < i1, (i2, i1)
    xo, it_o, _ = O.linear_solve_ml(N, srp, sci, svv, b, tol, 5000, 8, 0.7)
    assert abs(int(i2) - int(it_o)) <= 2, (i2, it_o)
    assert np.abs(x2 - xo).max() <= 1e-4 * np.abs(xo).max()
    assert np.array_equal(x2, two.solve(A, b, tol, 5000))


def test_step_with_two_level_schwarz_matches_oracle(ctx):
    """A seamed sheath (stitches, torso, self contact) stepped with the two-level
    preconditioner against the oracle's step with SchwarzMlCpu, from identical states."""
    sc = scenes.sheath_on_torso(edge=0.03, torso_res=(30, 29))
    sg = dict(sc, params=dict(sc["params"], schwarz_levels=2, schwarz_weight=0.7, schwarz_domain=16))
    so = dict(sc, params=dict(sc["params"], precond=3, schwarz_domain=16))
    g = ImplicitSolver(ctx, sg, "mixed")
    o = O.OracleSolver(so)
    for k in range(3):
        p0, v0 = o.positions().copy(), o.velocities().copy()
        g.positions, g.velocities = p0.astype(np.float32), v0.astype(np.float32)
        st = g.step(1)[0]
        sto = o.step(1, check_intersection=False)[0]
        pg, po = g.positions.astype(np.float64), o.positions()
        rel = np.abs(pg - po).max() / (np.abs(po - p0).max() + 1e-12)
        print(k, st["newton_iters"], sto["newton_iters"], st["max_cg_iters"], sto["max_cg_iters"], rel)
        assert st["status"] == 0 and st["penetration_free"]
        assert abs(st["newton_iters"] - sto["newton_iters"]) <= 1
        # PCG iteration counts differ where contact couples vertices across domains: the
        # reference rebuilds its domains and coarse graph from each system's pattern
        # (contact blocks included), the GPU keeps those of the elastic pattern
        assert rel < 1e-3, (k, rel)
