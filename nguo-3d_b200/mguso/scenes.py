"""Seeded synthetic inputs for the benchmark and parity configurations.

No public dataset is involved: every workload is generated here from a seed with the shapes,
sizes and value distributions of the configurations it stands for.
"""
from __future__ import annotations

import numpy as np


def grid_edges(n: int) -> np.ndarray:
    """Undirected edges of an n x n vertex grid triangulated along one diagonal per quad
    (the stiffness pattern of a cloth grid: 6 neighbours per interior vertex)."""
    idx = np.arange(n * n, dtype=np.int64).reshape(n, n)  # [j, i]
    h = np.stack([idx[:, :-1].ravel(), idx[:, 1:].ravel()], 1)
    v = np.stack([idx[:-1, :].ravel(), idx[1:, :].ravel()], 1)
    d = np.stack([idx[:-1, :-1].ravel(), idx[1:, 1:].ravel()], 1)
    return np.concatenate([h, v, d], 0)


def grid_tris(n: int) -> np.ndarray:
    """Triangles of the n x n grid, split along the (i,j)-(i+1,j+1) diagonal, wound
    consistently."""
    idx = np.arange(n * n, dtype=np.int64).reshape(n, n)
    a = idx[:-1, :-1].ravel()
    b = idx[:-1, 1:].ravel()
    c = idx[1:, 1:].ravel()
    d = idx[1:, :-1].ravel()
    t1 = np.stack([a, b, c], 1)
    t2 = np.stack([a, c, d], 1)
    return np.concatenate([t1, t2], 0).astype(np.uint32)


def grid_bsr(n: int, seed: int = 2):
    """Operator microbenchmark matrix: the block pattern of an n x n cloth grid
    (n^2 vertices, 7 blocks per interior row: the vertex, its 4 axis neighbours and its 2
    neighbours along the quad diagonal), 3x3 blocks with FP32 values drawn N(0,1),
    symmetric (A_ji = A_ij^T) and made strictly diagonally dominant
    (a_rr = |a_rr| + sum_{k != r} |a_rk| + 1), hence SPD.

    Built directly in row order (no global sort): row v's columns are
    v-n-1, v-n, v-1, v, v+1, v+n, v+n+1 where they exist.
    Returns (nb, row_ptr u32[nb+1], col u32[nnzb], val f32[nnzb, 3, 3]).
    """
    rng = np.random.default_rng(seed)
    nb = n * n
    # one block per undirected edge, indexed by its lower vertex: horizontal (v, v+1),
    # vertical (v, v+n), diagonal (v, v+n+1); plus a symmetric diagonal block per vertex
    gh = rng.standard_normal((nb, 3, 3), dtype=np.float32)
    gv = rng.standard_normal((nb, 3, 3), dtype=np.float32)
    gd = rng.standard_normal((nb, 3, 3), dtype=np.float32)
    dg = rng.standard_normal((nb, 3, 3), dtype=np.float32)
    dg = 0.5 * (dg + dg.transpose(0, 2, 1))
    i = np.tile(np.arange(n), n)
    j = np.repeat(np.arange(n), n)
    valid = np.stack([(i > 0) & (j > 0), j > 0, i > 0, np.ones(nb, bool), i < n - 1, j < n - 1,
                      (i < n - 1) & (j < n - 1)], 1)
    offs = np.array([-n - 1, -n, -1, 0, 1, n, n + 1], dtype=np.int64)
    full = np.zeros((nb, 7, 3, 3), dtype=np.float32)
    full[n + 1:, 0] = gd[:-(n + 1)].transpose(0, 2, 1)
    full[n:, 1] = gv[:-n].transpose(0, 2, 1)
    full[1:, 2] = gh[:-1].transpose(0, 2, 1)
    full[:, 3] = dg
    full[:, 4] = gh
    full[:, 5] = gv
    full[:, 6] = gd
    full *= valid[:, :, None, None]
    absrow = np.abs(full).sum(axis=(1, 3), dtype=np.float64)  # (nb, 3) incl. the diagonal entry
    d_vals = np.stack([full[:, 3, k, k] for k in range(3)], 1)
    absrow -= np.abs(d_vals)
    for k in range(3):
        full[:, 3, k, k] = (np.abs(d_vals[:, k]) + absrow[:, k] + 1.0).astype(np.float32)
    cnt = valid.sum(1)
    row_ptr = np.zeros(nb + 1, dtype=np.int64)
    row_ptr[1:] = np.cumsum(cnt)
    vflat = valid.reshape(-1)
    cols = (np.arange(nb, dtype=np.int64)[:, None] + offs[None, :]).reshape(-1)[vflat]
    val = full.reshape(-1, 3, 3)[vflat]
    return nb, row_ptr.astype(np.uint32), cols.astype(np.uint32), np.ascontiguousarray(val)


def bsr_to_csr(nb: int, row_ptr: np.ndarray, col: np.ndarray, val: np.ndarray):
    """Expands a 3x3 BSR into the reference's scalar CSR (n = 3 nb)."""
    row_ptr = row_ptr.astype(np.int64)
    nblk = np.diff(row_ptr)
    n = 3 * nb
    srp = np.zeros(n + 1, dtype=np.int64)
    per_row = np.repeat(3 * nblk, 3)
    srp[1:] = np.cumsum(per_row)
    # scalar row (v, i) lists blocks k in row v, then j in 0..2
    blk_of_row = np.repeat(np.arange(nb), nblk)
    # For each scalar row (v,i): entries ordered by (k, j)
    k_idx = np.arange(col.size)
    # build arrays of shape (nnzb, 3 rows, 3 cols) -> reorder to rows
    cols3 = (3 * col.astype(np.int64))[:, None] + np.arange(3)[None, :]  # (nnzb, 3)
    out_cols = np.empty(9 * col.size, dtype=np.uint32)
    out_vals = np.empty(9 * col.size, dtype=np.float32)
    # position of entry (k, i, j) in the scalar CSR
    base = 9 * row_ptr[blk_of_row]  # start of vertex row block
    local = k_idx - row_ptr[blk_of_row]
    for i in range(3):
        pos = base + 3 * i * nblk[blk_of_row] + 3 * local
        for j in range(3):
            out_cols[pos + j] = cols3[:, j]
            out_vals[pos + j] = val[:, i, j]
    return n, srp.astype(np.uint32), out_cols, out_vals


def bsr_spmv_f64(row_ptr: np.ndarray, col: np.ndarray, val: np.ndarray, x: np.ndarray) -> np.ndarray:
    """y = A x in float64 (the reference value for size-independent SpMV checks)."""
    nb = row_ptr.size - 1
    xb = x.reshape(-1, 3).astype(np.float64)
    rp = row_ptr.astype(np.int64)
    prod = np.einsum("kij,kj->ki", val.astype(np.float64), xb[col.astype(np.int64)])
    y = np.zeros((nb, 3), dtype=np.float64)
    nonempty = rp[1:] > rp[:-1]
    if prod.shape[0]:
        sums = np.add.reduceat(prod, rp[:-1][nonempty], axis=0)
        y[nonempty] = sums
    return y.reshape(-1)


def triangle_soup(nt: int, seed: int = 3, edge: float = 2.0e-3):
    """LBVH microbenchmark input: `nt` triangles with centroids uniform in the unit cube and
    unshared vertices at centroid + offsets uniform in [-edge/2, edge/2]^3 (edge-length
    scale `edge`, 2 mm by default). Returns (positions f32[3nt, 3], tris u32[nt, 3])."""
    rng = np.random.default_rng(seed)
    c = rng.random((nt, 3), dtype=np.float32)
    off = (rng.random((nt, 3, 3), dtype=np.float32) - np.float32(0.5)) * np.float32(edge)
    pos = (c[:, None, :] + off).reshape(-1, 3)
    tris = np.arange(3 * nt, dtype=np.uint32).reshape(nt, 3)
    return np.ascontiguousarray(pos), tris


# ---------------------------------------------------------------------------------------
# Drape scenes (the implicit step's inputs). A scene is a dict of numpy arrays plus
# `params`, the solver knobs named as in the reference's ImplicitParams
# (engine-core/src/implicit.rs:30-229).
# ---------------------------------------------------------------------------------------
def lame_from_young_poisson(young: float, poisson: float):
    """material::lame_from_young_poisson (engine-core/src/material.rs:31-45), in f32: the
    Poisson ratio clamped into [1e-6, 0.5 - 1e-4], a non-finite one replaced by 0.35."""
    p = float(poisson)
    nu = np.float32(min(max(p, 1.0e-6), 0.5 - 1.0e-4)) if np.isfinite(p) else np.float32(0.35)
    y = np.float32(young)
    mu = y / (np.float32(2.0) * (np.float32(1.0) + nu))
    lam = y * nu / ((np.float32(1.0) + nu) * (np.float32(1.0) - np.float32(2.0) * nu))
    return float(mu), float(lam)


def default_params(**kw):
    p = dict(dt=1.0 / 60.0, gravity=(0.0, -9.8, 0.0), newton_iters=32, stiffness=0.0, bend_stiffness=1.0e-5,
             max_dx=float("inf"), target_toi=0.0, min_newton_steps=0, ccd_max_iter=256, eiganalysis_eps=1.0e-6,
             contact_dhat=1.0e-3, contact_kappa=1.0e2, contact_dynamic=0.0, shell_mu=0.0, shell_lambda=0.0,
             friction=0.0, friction_eps=1.0e-3, barrier_kind=0, contact_rayleigh=1, self_collision=1,
             cg_tol=1.0e-4, cg_max_iter=2000, floor_y=float("-inf"), newton_tol=0.0, precond=2,
             schwarz_domain=32)
    p.update(kw)
    return p


def uniform_mass(positions: np.ndarray, tris: np.ndarray, density: float) -> float:
    """Scene::lower's lumped mass: total area * density / vertex count
    (engine-api/src/scene.rs:128-131), floored at 1e-6."""
    p = positions.astype(np.float64)
    t = tris.astype(np.int64)
    area = 0.5 * np.linalg.norm(np.cross(p[t[:, 1]] - p[t[:, 0]], p[t[:, 2]] - p[t[:, 0]]), axis=1).sum()
    return max(float(area * density / max(p.shape[0], 1)), 1.0e-6)


def _empty_stitches():
    return (np.zeros((0, 6), np.uint32), np.zeros((0, 6), np.float32), np.zeros((0, 3), np.float32))


def sheet_on_sphere(n: int = 64, side: float = 1.0, height: float = 0.5, jitter: float = 1.0e-3, seed: int = 0,
                    radius: float = 0.3, young: float = 1.0e5, poisson: float = 0.3, thickness: float = 5.0e-4,
                    bend: float = 1.0e-5, density: float = 0.2, dhat: float = 1.0e-3, dt: float = 1.0 / 60.0,
                    newton_tol_mps: float = 1.0e-3, **kw):
    """Square cloth sheet as an n x n vertex grid (side `side`, horizontal at y = height,
    every vertex jittered by a seeded uniform +-jitter per axis), StVK membrane from
    (E * thickness, nu), hinge bending k_b, uniform lumped mass from the areal density,
    dropped under gravity onto an analytic sphere of `radius` at the origin.
    newton_tol_mps * dt is the added Newton termination on the step taken (metres)."""
    rng = np.random.default_rng(seed)
    s = np.linspace(-0.5 * side, 0.5 * side, n, dtype=np.float64)
    X, Z = np.meshgrid(s, s)  # [j, i]
    pos = np.stack([X, np.full_like(X, height), Z], -1).reshape(-1, 3)
    pos = (pos + rng.uniform(-jitter, jitter, pos.shape)).astype(np.float32)
    tris = grid_tris(n)
    mu, lam = lame_from_young_poisson(young * thickness, poisson)
    m = uniform_mass(pos, tris, density)
    si, sw, skl = _empty_stitches()
    params = default_params(dt=dt, bend_stiffness=bend, contact_dhat=dhat, shell_mu=mu, shell_lambda=lam,
                            newton_tol=newton_tol_mps * dt, **kw)
    return dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=np.full(pos.shape[0], 1.0 / m, np.float32),
                tris=tris, shell_faces=tris.copy(), static_mask=None, stitch_idx=si, stitch_w=sw, stitch_kl=skl,
                colliders=np.array([[1, 0, 0, 0, 0, 0, 0, radius]], np.float32), params=params,
                name=f"{n}x{n} sheet on r={radius} sphere")


def _panel(width: float, height: float, edge: float, rng):
    """Rectangular panel [0, width] x [0, height] triangulated by a seeded Delaunay of a
    jittered lattice (mean edge ~ `edge`), with evenly spaced boundary points so the two
    side seams of two panels sample identical heights. Returns (uv points, triangles,
    left-seam vertex ids bottom->top, right-seam vertex ids bottom->top)."""
    from scipy.spatial import Delaunay

    nx = max(int(round(width / edge)), 2)
    ny = max(int(round(height / edge)), 2)
    xs = np.linspace(0.0, width, nx + 1)
    ys = np.linspace(0.0, height, ny + 1)
    # boundary
    left = np.stack([np.zeros(ny + 1), ys], 1)
    right = np.stack([np.full(ny + 1, width), ys], 1)
    bottom = np.stack([xs[1:-1], np.zeros(nx - 1)], 1)
    top = np.stack([xs[1:-1], np.full(nx - 1, height)], 1)
    # interior: jittered lattice, offset every other row (near-equilateral triangles)
    ix, iy = np.meshgrid(np.arange(1, nx), np.arange(1, ny))
    px = (ix + 0.5 * (iy % 2) - 0.25).astype(np.float64) * (width / nx)
    py = iy.astype(np.float64) * (height / ny)
    jit = rng.uniform(-0.2, 0.2, (2,) + px.shape)
    px = np.clip(px + jit[0] * width / nx, 0.3 * width / nx, width - 0.3 * width / nx)
    py = np.clip(py + jit[1] * height / ny, 0.3 * height / ny, height - 0.3 * height / ny)
    interior = np.stack([px.ravel(), py.ravel()], 1)
    pts = np.concatenate([left, right, bottom, top, interior])
    tri = Delaunay(pts).simplices.astype(np.int64)
    # drop slivers along the convex hull (none expected on a rectangle) and fix winding
    a, b, c = pts[tri[:, 0]], pts[tri[:, 1]], pts[tri[:, 2]]
    cross = (b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (b[:, 1] - a[:, 1]) * (c[:, 0] - a[:, 0])
    tri = tri[np.abs(cross) > 1e-12]
    flip = ((pts[tri[:, 1], 0] - pts[tri[:, 0], 0]) * (pts[tri[:, 2], 1] - pts[tri[:, 0], 1]) -
            (pts[tri[:, 1], 1] - pts[tri[:, 0], 1]) * (pts[tri[:, 2], 0] - pts[tri[:, 0], 0])) < 0
    tri[flip] = tri[flip][:, [0, 2, 1]]
    return pts, tri, np.arange(ny + 1), np.arange(ny + 1, 2 * (ny + 1))


def torso_mesh(seed: int = 0, scale: float = 1.0, n_phi: int = 100, n_y: int = 99):
    """Closed, outward-wound torso: the union of three vertical-axis ellipsoids (chest,
    waist, hip) with semi-axes drawn U[0.12, 0.20] m, meshed as a star-shaped surface
    r(y, phi) = max over ellipsoids of their radial extent, with a pole vertex at each end.
    n_phi * n_y * 2 + 2 * n_phi triangles (20 000 by default)."""
    rng = np.random.default_rng(seed)
    centers = np.array([1.30, 1.05, 0.85]) * scale
    axes = rng.uniform(0.12, 0.20, (3, 3)) * scale  # (a_x, b_y, c_z) per ellipsoid
    y_lo = float((centers - axes[:, 1]).min()) + 1e-4
    y_hi = float((centers + axes[:, 1]).max()) - 1e-4
    ys = np.linspace(y_lo, y_hi, n_y)
    phi = np.linspace(0.0, 2 * np.pi, n_phi, endpoint=False)
    Y, PH = np.meshgrid(ys, phi, indexing="ij")
    r = np.zeros_like(Y)
    for (cy, (a, b, c)) in zip(centers, axes):
        s2 = 1.0 - ((Y - cy) / b) ** 2
        ok = s2 > 0
        s = np.sqrt(np.where(ok, s2, 0.0))
        with np.errstate(divide="ignore", invalid="ignore"):
            rk = 1.0 / np.sqrt(np.cos(PH) ** 2 / (a * s) ** 2 + np.sin(PH) ** 2 / (c * s) ** 2)
        r = np.maximum(r, np.where(ok, rk, 0.0))
    r = np.maximum(r, 0.01 * scale)
    ring = np.stack([r * np.cos(PH), Y, r * np.sin(PH)], -1).reshape(-1, 3)
    bottom_pole = np.array([[0.0, y_lo - 0.005 * scale, 0.0]])
    top_pole = np.array([[0.0, y_hi + 0.005 * scale, 0.0]])
    pos = np.concatenate([ring, bottom_pole, top_pole])
    ib, it = n_y * n_phi, n_y * n_phi + 1
    tris = []
    for j in range(n_y - 1):
        for k in range(n_phi):
            a = j * n_phi + k
            b = j * n_phi + (k + 1) % n_phi
            c = (j + 1) * n_phi + k
            d = (j + 1) * n_phi + (k + 1) % n_phi
            tris.append((a, c, b))
            tris.append((b, c, d))
    for k in range(n_phi):
        tris.append((ib, k, (k + 1) % n_phi))
        top = (n_y - 1) * n_phi
        tris.append((it, top + (k + 1) % n_phi, top + k))
    tris = np.array(tris, np.int64)
    # outward winding check: signed volume must be positive
    p = pos[tris]
    vol = np.einsum("ij,ij->i", np.cross(p[:, 0], p[:, 1]), p[:, 2]).sum() / 6.0
    if vol < 0:
        tris = tris[:, [0, 2, 1]]
    return pos.astype(np.float32), tris.astype(np.uint32), (centers, axes)


def sheath_on_torso(width: float = 0.6, height: float = 1.1, edge: float = 8.0e-3, seed: int = 1,
                    torso_seed: int = 11, torso_scale: float = 1.0, young: float = 1.0e5, poisson: float = 0.3,
                    thickness: float = 5.0e-4, bend: float = 1.0e-5, density: float = 0.2, dhat: float = 1.0e-3,
                    dt: float = 1.0 / 60.0, stitch_k: float = 1.0e3, seam_gap: float = 2.0e-3,
                    newton_tol_mps: float = 1.0e-3, torso_res=(100, 99), **kw):
    """Seamed sheath: two width x height panels (seeded Delaunay, mean edge `edge`) wrapped
    into the two halves of a vertical tube of circumference 2 * width, the side seams held by
    6-index stitches (rest length dhat, cap 10 * dhat, as the in-process transport builds
    them), hanging just above a static three-ellipsoid torso (20k triangles) it drapes onto.
    Materials as the sheet configuration.

    `stitch_k` is the seam's spring constant in N/m. The stitch energy
    k_raw (|t| - l0)^2 / (2 l0) (stitch.rs:42-46) has spring constant k_raw / l0, so the
    stitch carries k_raw = stitch_k * l0: 1.0 at 1e3 N/m and l0 = 1 mm, which is also the
    reference's default stitch stiffness (golden.rs read_stitches)."""
    rng = np.random.default_rng(seed)
    R = 2.0 * width / (2.0 * np.pi)
    tpos, ttris, _ = torso_mesh(torso_seed, torso_scale, *torso_res)
    y_top = float(tpos[:, 1].max())
    base_y = y_top + 0.01  # the tube hangs 1 cm above the torso and falls onto it
    panels, tris, seams, uvs, panel_of = [], [], [], [], []
    off = 0
    for k in range(2):
        uv, tr, left, right = _panel(width, height, edge, rng)
        uvs.append(uv)
        panel_of.append(np.full(tr.shape[0], k, np.uint8))
        th = (uv[:, 0] / width) * np.pi + k * np.pi
        p = np.stack([R * np.cos(th), base_y + uv[:, 1], R * np.sin(th)], 1)
        if k == 1:
            # back panel slightly larger so its seam edges sit seam_gap away from the front's
            p[:, [0, 2]] *= (R + seam_gap) / R
        panels.append(p)
        tris.append(tr + off)
        seams.append((left + off, right + off))
        off += p.shape[0]
    cloth = np.concatenate(panels)
    ctris = np.concatenate(tris)
    # seams: front left (theta=0) <-> back right (theta=2pi); front right (pi) <-> back left (pi)
    l0 = dhat
    sidx, sw, skl, seam_of = [], [], [], []
    for si_, (a_ids, b_ids) in enumerate(((seams[0][0], seams[1][1]), (seams[0][1], seams[1][0]))):
        for a, b in zip(a_ids, b_ids):
            sidx.append([a, a, a, b, b, b])
            sw.append([1, 0, 0, 1, 0, 0])
            skl.append([stitch_k * l0, l0, 10.0 * l0])
            seam_of.append(si_)
    nc = cloth.shape[0]
    pos = np.concatenate([cloth, tpos]).astype(np.float32)
    all_tris = np.concatenate([ctris, ttris.astype(np.int64) + nc]).astype(np.uint32)
    static = np.concatenate([np.zeros(nc, np.uint8), np.ones(tpos.shape[0], np.uint8)])
    m = uniform_mass(pos, all_tris, density)
    inv_mass = np.where(static > 0, 0.0, 1.0 / m).astype(np.float32)
    mu, lam = lame_from_young_poisson(young * thickness, poisson)
    params = default_params(dt=dt, bend_stiffness=bend, contact_dhat=dhat, shell_mu=mu, shell_lambda=lam,
                            newton_tol=newton_tol_mps * dt, **kw)
    return dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=inv_mass, tris=all_tris,
                shell_faces=ctris.astype(np.uint32), static_mask=static,
                stitch_idx=np.array(sidx, np.uint32), stitch_w=np.array(sw, np.float32),
                stitch_kl=np.array(skl, np.float32), colliders=np.zeros((0, 8), np.float32), params=params,
                # sewing pattern: panel coordinates of every shell face's corners (u along the
                # weft / circumference, v along the warp / height), its panel, and each
                # stitch's seam (0: front-left to back-right, 1: front-right to back-left)
                shell_uv=np.concatenate(uvs)[ctris].astype(np.float32), shell_panel=np.concatenate(panel_of),
                stitch_seam=np.array(seam_of, np.uint8),
                name=f"sheath {ctris.shape[0]} tris on torso {ttris.shape[0]} tris")


GRADE_WIDTHS = (0.50, 0.55, 0.60, 0.65, 0.70, 0.75)
GRADE_TORSO_SCALES = (0.9, 0.96, 1.02, 1.08, 1.14, 1.2)


def graded_sheath(i: int, widths=GRADE_WIDTHS, torso_scales=GRADE_TORSO_SCALES, **kw):
    """Size `i` (0 = XS) of the graded sheath."""
    return sheath_on_torso(width=widths[i], torso_scale=torso_scales[i], **kw)


def graded_sheaths(n: int = 6, widths=GRADE_WIDTHS, torso_scales=GRADE_TORSO_SCALES, **kw):
    """One pattern graded into `n` sizes XS..XXL (panel widths 0.50-0.75 m, torsos scaled
    0.9-1.2): the batched configuration."""
    return [graded_sheath(i, widths, torso_scales, **kw) for i in range(n)]
