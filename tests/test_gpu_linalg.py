"""GPU parity of the BSR SpMV, the Schwarz preconditioner and the PCG against the CPU
oracle (a restatement of engine-core/src/{csr,linsolve}.rs), all through the C ABI."""
import numpy as np
import pytest

import oracle_py as O
from mguso import Bsr, CsrMatrix, CudaLinearSolver, Schwarz, scenes

pytestmark = pytest.mark.gpu


def torch_dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def small_grid(n=12, seed=5):
    nb, rp, col, val = scenes.grid_bsr(n, seed)
    N, srp, sci, svv = scenes.bsr_to_csr(nb, rp, col, val)
    return nb, rp, col, val, N, srp, sci, svv


@pytest.mark.parametrize("variant", [1, 2, 3])
def test_spmv_matches_oracle_small(ctx, variant):  # engine-gpu pcg.rs:791-807 (gpu_spmv_matches_cpu)
    nb, rp, col, val, N, srp, sci, svv = small_grid(37)
    a = Bsr(ctx, nb, rp, col, val)
    a.set_kernel(variant)
    x = np.random.default_rng(0).standard_normal(N).astype(np.float32)
    y = a.spmv_host(x)
    want = O.spmv(N, srp, sci, svv, x)
    bound = scenes.bsr_spmv_f64(rp, col, np.abs(val), np.abs(x))
    assert np.all(np.abs(y - want) <= 1e-5 * bound + 1e-30)


def test_spmv_from_reference_csr_equals_bsr(ctx):
    nb, rp, col, val, N, srp, sci, svv = small_grid(9)
    a = Bsr.from_csr(ctx, CsrMatrix(N, srp, sci, svv))
    assert (a.nb, a.nnzb) == (nb, col.size)
    x = np.linspace(-1, 1, N).astype(np.float32)
    want = O.spmv(N, srp, sci, svv, x)
    bound = scenes.bsr_spmv_f64(rp, col, np.abs(val), np.abs(x))
    assert np.all(np.abs(a.spmv_host(x) - want) <= 1e-5 * bound + 1e-30)


def test_spmv_edge_cases(ctx):
    # empty rows, a single dense row, a row longer than any TMA tile
    nb = 3000
    rows = [[0, 1, 2], [], [2], list(range(0, 3000, 1))] + [[i] for i in range(4, nb)]
    rp = np.zeros(nb + 1, np.uint32)
    col = []
    for r, cs in enumerate(rows):
        col += cs
        rp[r + 1] = len(col)
    col = np.array(col, np.uint32)
    val = np.random.default_rng(1).standard_normal((col.size, 3, 3)).astype(np.float32)
    a = Bsr(ctx, nb, rp, col, val)
    x = np.random.default_rng(2).standard_normal(3 * nb).astype(np.float32)
    want = scenes.bsr_spmv_f64(rp, col, val, x)
    bound = scenes.bsr_spmv_f64(rp, col, np.abs(val), np.abs(x))
    for variant in (1, 2, 3):
        a.set_kernel(variant)
        assert np.all(np.abs(a.spmv_host(x) - want) <= 1e-5 * bound + 1e-30)


def test_spmv_full_size_property(ctx):
    """The 1024^2 cloth grid at full size (7 331 842 blocks): GPU y vs float64, and
    linearity A(x1 + x2) = A x1 + A x2 within FP32 rounding."""
    import torch
    nb, rp, col, val = scenes.grid_bsr(1024, seed=2)
    assert col.size == 7331842
    a = Bsr(ctx, nb, rp, col, val)
    a.autotune()
    rng = np.random.default_rng(3)
    x1 = rng.standard_normal(3 * nb).astype(np.float32)
    x2 = rng.standard_normal(3 * nb).astype(np.float32)
    y1 = a.spmv_host(x1)
    y2 = a.spmv_host(x2)
    y12 = a.spmv_host(x1 + x2)
    want = scenes.bsr_spmv_f64(rp, col, val, x1)
    bound = scenes.bsr_spmv_f64(rp, col, np.abs(val), np.abs(x1))
    assert np.all(np.abs(y1 - want) <= 1e-5 * bound)
    b12 = scenes.bsr_spmv_f64(rp, col, np.abs(val), np.abs(x1) + np.abs(x2))
    assert np.all(np.abs(y12 - (y1 + y2)) <= 2e-5 * b12)
    # device-pointer entry point on torch memory and stream
    xd, yd = torch_dev(x1), torch.empty(3 * nb, device="cuda")
    a.spmv(xd.data_ptr(), yd.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(yd.cpu().numpy(), y1)


def test_schwarz_domains_equal_oracle(ctx):
    nb, rp, col, val, N, srp, sci, svv = small_grid(23)
    a = Bsr(ctx, nb, rp, col, val)
    s = Schwarz(a, 32)
    want, nd = O.schwarz_domains(N, srp, sci, 32)
    assert s.ndomains == nd
    assert np.array_equal(s.domains(), want)


def test_schwarz_apply_matches_oracle(ctx):  # engine-gpu schwarz.rs:404-430
    import torch
    nb, rp, col, val, N, srp, sci, svv = small_grid(23)
    a = Bsr(ctx, nb, rp, col, val)
    s = Schwarz(a, 32)
    st = torch.cuda.current_stream().cuda_stream
    s.factor(st)
    r = np.random.default_rng(4).standard_normal(N).astype(np.float32)
    rd, zd = torch_dev(r), torch.zeros(N, device="cuda")
    s.apply(rd.data_ptr(), zd.data_ptr(), st)
    torch.cuda.synchronize()
    z = zd.cpu().numpy()
    want = O.schwarz_apply(N, srp, sci, svv, 32, r.astype(np.float64))
    assert np.abs(z - want).max() <= 1e-4 * np.abs(want).max()


@pytest.mark.parametrize("precond,kind", [("schwarz", "schwarz"), ("block", "block")])
@pytest.mark.parametrize("precision", ["mixed", "fp32"])
def test_pcg_matches_oracle(ctx, precond, kind, precision):  # engine-gpu pcg.rs:809-836, schwarz.rs:434-463
    nb, rp, col, val, N, srp, sci, svv = small_grid(30)
    A = CsrMatrix(N, srp, sci, svv)
    xs = np.sin(np.arange(N, dtype=np.float32) * np.float32(0.05)).astype(np.float32)
    b = O.spmv(N, srp, sci, svv, xs)
    solver = CudaLinearSolver(ctx, precond=precond, domain=32, precision=precision)
    x = solver.solve(A, b, 1e-6, 500)
    st = solver.last_stats()
    xo, it_o, res_o = O.linear_solve(N, srp, sci, svv, b, 1e-6, 500, kind, 32)
    assert st.residual <= 1e-6 or (precision == "fp32" and st.residual < 1e-5)
    assert abs(int(st.iters) - int(it_o)) <= 2
    assert np.abs(x - xo).max() <= 1e-4 * np.abs(xo).max()
    # a second solve on the same pattern reuses the cached layout and gives the same x
    x2 = solver.solve(A, b, 1e-6, 500)
    assert np.array_equal(x, x2)


def test_pcg_reports_cap_and_breakdown(ctx):
    nb, rp, col, val, N, srp, sci, svv = small_grid(16)
    A = CsrMatrix(N, srp, sci, svv)
    b = np.ones(N, np.float32)
    s = CudaLinearSolver(ctx, precond="block")
    s.solve(A, b, 1e-12, 3)
    assert s.last_stats().iters == 3 and s.last_stats().status == 4  # PCG_CAP
    # b = 0: pAp = 0 -> break, x = 0 (engine-gpu pcg.rs:838-846, pcg_zero_rhs_is_zero)
    x = s.solve(A, np.zeros(N, np.float32), 1e-6, 100)
    assert np.all(x == 0) and s.last_stats().iters == 0


def grid_with_isolated(n=17, extra=70, seed=6):
    """A cloth-grid matrix plus `extra` vertices that own only a diagonal block (pinned
    collider vertices look like this), interleaved with the grid's vertices."""
    nb0, rp0, col0, val0 = scenes.grid_bsr(n, seed)
    nb = nb0 + extra
    iso = np.sort(np.random.default_rng(seed).choice(nb, extra, replace=False))
    is_iso = np.zeros(nb, bool)
    is_iso[iso] = True
    new_of_old = np.flatnonzero(~is_iso).astype(np.int64)  # grid vertex g -> new index
    rows, cols, vals = [], [], []
    for g in range(nb0):
        for k in range(rp0[g], rp0[g + 1]):
            rows.append(new_of_old[g])
            cols.append(new_of_old[col0[k]])
            vals.append(val0[k])
    for v in iso:
        rows.append(v)
        cols.append(v)
        vals.append(np.eye(3, dtype=np.float32) * np.float32(2.0 + v % 5))
    order = np.lexsort((np.array(cols), np.array(rows)))
    rows, cols = np.array(rows)[order], np.array(cols)[order]
    vals = np.array(vals, np.float32).reshape(-1, 9)[order]
    rp = np.zeros(nb + 1, np.uint32)
    np.add.at(rp, rows + 1, 1)
    rp = np.cumsum(rp).astype(np.uint32)
    return nb, rp, cols.astype(np.uint32), vals.reshape(-1, 3, 3).astype(np.float32), iso


def test_schwarz_packs_isolated_vertices(ctx):
    """Vertices without off-diagonal blocks are packed D per domain instead of forming one
    domain each; every other vertex keeps the oracle's BFS domain, and the apply still
    matches the oracle's additive Schwarz (the packed blocks do not couple)."""
    import torch
    nb, rp, col, val, iso = grid_with_isolated()
    N, srp, sci, svv = scenes.bsr_to_csr(nb, rp, col, val)
    a = Bsr(ctx, nb, rp, col, val)
    s = Schwarz(a, 32)
    want, nd = O.schwarz_domains(N, srp, sci, 32)
    got = s.domains()
    assert s.ndomains == nd - len(iso) + (len(iso) + 31) // 32
    conn = np.setdiff1d(np.arange(nb), iso)
    # same partition of the connected vertices (domain ids may be renumbered)
    pairs = set(zip(got[conn].tolist(), want[conn].tolist()))
    assert len(pairs) == len(set(got[conn].tolist())) == len(set(want[conn].tolist()))
    assert len(set(got[iso].tolist())) == (len(iso) + 31) // 32
    st = torch.cuda.current_stream().cuda_stream
    s.factor(st)
    r = np.random.default_rng(9).standard_normal(N).astype(np.float32)
    rd, zd = torch_dev(r), torch.zeros(N, device="cuda")
    s.apply(rd.data_ptr(), zd.data_ptr(), st)
    torch.cuda.synchronize()
    z = zd.cpu().numpy()
    ref = O.schwarz_apply(N, srp, sci, svv, 32, r.astype(np.float64))
    assert np.abs(z - ref).max() <= 1e-4 * np.abs(ref).max()
