#!/usr/bin/env python
"""Benchmark for the mguso implicit-step hot path on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mguso|reference] [--workload W]

Prints ONE JSON line (rank 0). Multi-GPU runs are independent replicas (one process per
GPU, no data-path collective): the workloads are independent drapes/operators, so per-GPU
work is fixed as N grows ("scaling": "weak") and `value` is the sum over ranks of the work
divided by the slowest rank's device time.

Workloads
  batch  The headline configuration (default): the seamed sheath below graded into 6 sizes
         (panel widths 0.50-0.75 m) on 6 torsos scaled 0.9-1.2, stepped as one batch in mixed
         precision, timed against the plain FP32 path stepping each size alone; the first
         step of the XS size is also checked against the FP64 oracle.
         Metric: drape steps (instance steps) per second.
  drape  Garment-scale drape: a seamed sheath of 41 400
         triangles (two 0.6 x 1.1 m panels, seeded Delaunay, 8 mm edges, 278 side-seam
         stitches, k = 1e3) dropped onto a static 19 800-triangle three-ellipsoid torso;
         StVK membrane (E = 1e5 Pa, nu = 0.3, h = 0.5 mm), hinge bending 1e-5, 0.2 kg/m^2,
         self and body contact at dhat = 1 mm, dt = 1/60 s. One step = one implicit step.
         Metric: drape steps per second.
  sheet  64 x 64 sheet (7 938 triangles) dropped onto an r = 0.3 m sphere, same materials.
  spmv   Operator microbenchmark: 3x3 BSR SpMV on the stiffness pattern of a 1024 x 1024
         cloth grid (1 048 576 block rows, 7 331 842 blocks, FP32 N(0,1) values made SPD).
         One step = one y = A x over the whole matrix. Metric: algorithmic HBM GB/s.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(REPO, "nguo-3d_b200"), os.path.join(REPO, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "drape steps/sec batched+mixed vs plain FP32 (same GPU, ≤1e-4 err); SpMV HBM GB/s"


def load_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = f"/tmp/mguso_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.device)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.proc is None:
            return out
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if sm:
            out = {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                   "samples": len(sm)}
        try:
            os.remove(self.path)
        except OSError:
            pass
        return out


# ---------------------------------------------------------------------------------------
# distributed plumbing (replicas only)
# ---------------------------------------------------------------------------------------
class Dist:
    def __init__(self, backend: str):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def __init_local__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        return self

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------------------
# workload: BSR SpMV + Schwarz apply on the 1024x1024 cloth grid
# ---------------------------------------------------------------------------------------
def spmv_bytes(nb: int, nnzb: int) -> int:
    """Algorithmic bytes of one FP32 BSR SpMV: values 36/block, column 4/block, row_ptr,
    x read once (12/row) and y written once (12/row)."""
    return 36 * nnzb + 4 * nnzb + 4 * (nb + 1) + 12 * nb + 12 * nb


def spmv_grid1024_side(steps: int) -> dict:
    """The operator benchmark's BSR SpMV measured beside the headline (the metric's "SpMV HBM
    GB/s"): the 1024 x 1024 cloth grid's pattern (1 048 576 block rows, 7 331 842 blocks,
    FP32 values N(0,1) made diagonally dominant), the variant the autotuner picks, `steps`
    launches after 3 untimed ones timed with CUDA events on one stream. The operator and its
    vectors (322.6 MB of algorithmic bytes) are larger than L2. No collectives: every rank
    measures its own GPU."""
    import torch

    import mguso
    from mguso import scenes

    ctx = mguso.Context(torch.cuda.current_device())
    a = None
    try:
        nb, rp, col, val = scenes.grid_bsr(1024, seed=2)
        a = mguso.Bsr(ctx, nb, rp, col, val)
        a.autotune()
        x = torch.from_numpy(np.random.default_rng(1).standard_normal(3 * nb).astype(np.float32)).cuda()
        y = torch.empty_like(x)
        stream = torch.cuda.current_stream()
        sp = stream.cuda_stream
        for _ in range(3):
            a.spmv(x.data_ptr(), y.data_ptr(), sp)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            a.spmv(x.data_ptr(), y.data_ptr(), sp)
        e1.record(stream)
        torch.cuda.synchronize()
        us = 1000.0 * e0.elapsed_time(e1) / steps
        nbytes = spmv_bytes(nb, a.nnzb)
        peak, peak_kind = load_peaks()
        gbs = nbytes / (us * 1e-6) / 1e9
        return {"workload": "BSR SpMV, 1024x1024 cloth grid (1048576 block rows, 7331842 blocks), FP32",
                "kernel": "autotuned BSR SpMV: " + json.dumps(a.kernel()), "us_per_launch": round(us, 2),
                "bytes_per_launch": int(nbytes), "GB/s": round(gbs, 1), "peak": peak,
                "frac": round(gbs / peak, 4), "peak_kind": f"{peak_kind} (burst copy)", "launches": steps}
    finally:
        if a is not None:
            a.close()
        ctx.close()


def cpu_spmv_sample(seconds: float = 10.0):
    """The oracle's scalar-CSR SpMV (csr.rs:98-111 restated, single thread) on a bounded
    sample of the same workload: a 256 x 256 grid of the same pattern and distribution."""
    import oracle_py as O
    from mguso import scenes

    nb, rp, col, val = scenes.grid_bsr(256, seed=2)
    n, srp, sci, svv = scenes.bsr_to_csr(nb, rp, col, val)
    x = np.random.default_rng(0).standard_normal(n).astype(np.float32)
    O.spmv(n, srp, sci, svv, x)
    t0 = time.perf_counter()
    reps = 0
    while time.perf_counter() - t0 < seconds:
        O.spmv(n, srp, sci, svv, x)
        reps += 1
    dt = (time.perf_counter() - t0) / reps
    gbs = spmv_bytes(nb, col.size) / dt / 1e9
    sample = f"oracle scalar-CSR SpMV, 256x256 grid ({nb} block rows, {col.size} blocks), {reps} applies"
    return gbs, sample


def run_spmv(args, dist: Dist):
    import torch

    import mguso
    from mguso import scenes

    torch.cuda.set_device(dist.local)
    ctx = mguso.Context(dist.local)
    nb, rp, col, val = scenes.grid_bsr(1024, seed=2)
    a = mguso.Bsr(ctx, nb, rp, col, val)
    tuned_us = a.autotune()
    nbytes = spmv_bytes(nb, a.nnzb)
    rng = np.random.default_rng(1 + dist.rank)
    x_h = torch.from_numpy(rng.standard_normal(3 * nb).astype(np.float32)).pin_memory()
    y_h = torch.empty(3 * nb, dtype=torch.float32).pin_memory()
    x = x_h.cuda()
    y = torch.empty_like(x)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream

    # Schwarz apply on the same matrix (reported alongside)
    sch = mguso.Schwarz(a, 32)
    sch.factor(sp)
    torch.cuda.synchronize()

    clocks = ClockSampler(dist.local)
    clocks.start()
    for _ in range(args.warmup):
        a.spmv(x.data_ptr(), y.data_ptr(), sp)
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        a.spmv(x.data_ptr(), y.data_ptr(), sp)
    e1.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    # keep the GPU busy (untimed) long enough for the clock sampler to see load
    t_end = time.time() + 1.0
    while time.time() < t_end:
        for _ in range(50):
            a.spmv(x.data_ptr(), y.data_ptr(), sp)
        torch.cuda.synchronize()
    clk = clocks.stop()
    ms_max = dist.max(ms)
    ms_step = ms_max / args.steps

    # Schwarz apply timing (same stream)
    zs = torch.empty_like(x)
    for _ in range(3):
        sch.apply(x.data_ptr(), zs.data_ptr(), sp)
    e0.record(stream)
    for _ in range(args.steps):
        sch.apply(x.data_ptr(), zs.data_ptr(), sp)
    e1.record(stream)
    torch.cuda.synchronize()
    sch_us = 1000.0 * e0.elapsed_time(e1) / args.steps
    # algorithmic bytes: each domain's triangular factor once (m (m + 1) / 2 floats), the
    # gathered residual, the scattered result and the domain vertex lists
    dsz = 3.0 * np.bincount(sch.domains().astype(np.int64))
    sch_bytes = int(4 * (dsz * (dsz + 1) / 2).sum() + 28 * nb)
    sch_stored = int(sch.factor_bytes + 28 * nb)

    # end to end through the C ABI with pinned host buffers
    xp, yp = x_h.numpy(), y_h.numpy()
    a.spmv_host(xp)
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        out = a.spmv_host(xp)
    e2e_s = dist.max(time.perf_counter() - t0) / args.steps
    del out, yp

    peak, peak_kind = load_peaks()
    achieved = nbytes / (ms_step * 1e-3) / 1e9
    res = {
        "metric": METRIC,
        "value": round(achieved * dist.world, 2),
        "unit": "GB/s",
        "n_gpus": dist.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_step, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded N(0,1) SPD blocks on the 1024^2 cloth-grid pattern)",
        "config": {
            "workload": "BSR SpMV, 1024x1024 cloth grid stiffness pattern",
            "block_rows": nb, "nnzb": a.nnzb, "bytes_per_apply": nbytes,
            "l2": "inputs larger than L2 (293 MB of blocks+columns streamed per step; x gathered from L2)",
            "parallelism": f"replicas x{dist.world}",
            "autotuned_us": round(tuned_us, 2),
        },
        "roofline": {
            "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": None, "peak_kind": f"{peak_kind} (burst copy)",
            "kernel": "autotuned BSR SpMV: " + json.dumps(a.kernel()),
        },
        "schwarz_apply": {
            "us": round(sch_us, 2), "GB/s": round(sch_bytes / (sch_us * 1e-6) / 1e9, 1),
            "domains": sch.ndomains, "bytes": sch_bytes, "stored_bytes": sch_stored,
        },
        "e2e": {"value": round(nbytes / e2e_s / 1e9 * dist.world, 2), "unit": "GB/s",
                "h2d_bytes_per_step": 12 * nb, "d2h_bytes_per_step": 12 * nb},
        "gpu_launches": args.steps,
        "clocks": {k: clk[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
    }
    if dist.rank == 0 and not args.no_cpu_baseline:
        gbs, sample = cpu_spmv_sample(args.cpu_seconds)
        res["cpu_baseline"] = {"value": round(gbs, 3), "unit": "GB/s", "cores": 1, "kind": "port",
                               "sample": sample}
    sch.close()
    a.close()
    ctx.close()
    return res


BATCH_WORKLOAD = ("sheath graded XS..XXL (panel widths 0.50-0.75 m) on 6 torsos scaled 0.9-1.2, one batch, "
                  "per-instance Newton/CCD/PCG convergence")
BATCH_UNIT = "drape-steps/s"


def drape_scene(which: str):
    from mguso import scenes

    if which == "batch":
        return scenes.graded_sheath(0), BATCH_WORKLOAD
    if which == "sheet":
        return scenes.sheet_on_sphere(64), "64x64 sheet (7938 tris) on r=0.3 m sphere, 36-step drape"
    sc = scenes.sheath_on_torso()
    return sc, "seamed sheath 41400 tris + 278 stitches on 19800-tri torso, 120-step drape"


def _instance_scene(which: str, i: int):
    from mguso import scenes

    return scenes.graded_sheath(i) if which == "batch" else drape_scene(which)[0]


def _oracle_window_worker(job):
    """One drape on the oracle's implicit step: `warmup` untimed steps from the scene's start
    (or the given state), then at least one timed step and more while `seconds` last.
    Returns (timed steps, seconds, Newton iterations per timed step, positions after the
    first timed step)."""
    which, i, precision, warmup, seconds, state = job
    import oracle_py as O

    sc = _instance_scene(which, i)
    o = O.OracleSolver(sc, precision)
    if state is not None:
        o.set_state(state[0], state[1])
    if warmup:
        o.step(warmup, check_intersection=False)
    t0 = time.perf_counter()
    n, newton, first = 0, [], None
    while n == 0 or time.perf_counter() - t0 < seconds:
        st = o.step(1, check_intersection=False)[0]
        newton.append(int(st["newton_iters"]))
        if first is None:
            first = o.positions()
        n += 1
    return n, time.perf_counter() - t0, newton, first


def _pool_map(jobs, workers):
    import multiprocessing as mp

    with mp.get_context("spawn").Pool(max(1, workers)) as pool:
        return pool.map(_oracle_window_worker, jobs)


def cpu_drape_window(which: str, warmup: int, seconds: float, states=None):
    """The oracle's f32 implicit step (implicit.rs:1951-2191 restated; one drape is one
    thread, as in the reference) on the same drape steps the GPU arm times: each drape runs
    `warmup` untimed steps (or starts from `states`, the GPU's state after its warm-up),
    then steps warmup+1, ... for at least `seconds`. The six graded sizes of the batch run
    concurrently, one process each. Returns (drape steps per second, sample description,
    cores, Newton iterations per timed step, positions after the first timed step)."""
    k = 6 if which == "batch" else 1
    workers = max(1, min(k, os.cpu_count() or 1))
    jobs = [(which, i, "f32", 0 if states is not None else warmup, seconds,
             None if states is None else states[i]) for i in range(k)]
    t0 = time.perf_counter()
    res = _pool_map(jobs, workers)
    wall = time.perf_counter() - t0
    steps = sum(n for n, _, _, _ in res)
    busy = max(dt for _, dt, _, _ in res)
    newton = [nw for _, _, nw, _ in res]
    start = "from the GPU's states before them" if states is not None else f"after {warmup} untimed oracle steps"
    desc = (f"oracle f32 implicit step, {'the 6 graded sizes' if k == 6 else 'the drape'} in {workers} concurrent "
            f"process{'es' if workers > 1 else ''}, steps {warmup + 1}..{warmup + max(n for n, _, _, _ in res)} "
            f"{start} ({busy:.1f} s timed, {wall:.1f} s wall); Newton iterations per timed step "
            f"{[x for nw in newton for x in nw]}")
    # each process times its own steps; the drapes run concurrently, so the rate is the
    # steps of all drapes over the longest timed span
    return steps / busy, desc, workers, newton, [f for _, _, _, f in res]


def count_launches(fn):
    """Kernel launches during fn(), from the CUDA activity trace (torch.profiler)."""
    try:
        from torch.profiler import ProfilerActivity, profile

        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            fn()
        n = 0
        for e in prof.events():
            if getattr(e, "device_type", None) is not None and str(e.device_type).endswith("CUDA"):
                n += 1
        return n
    except Exception:
        return None


def time_steps(solver, steps, stream, dist, name="timed"):
    """Device time (ms) of `steps` steps on the solver's stream, CUDA events, barrier-bracketed.
    The steps run inside an NVTX range `name` (a profiler can restrict itself to it)."""
    import torch

    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push(name)
    e0.record(stream)
    st = solver.step(steps)
    e1.record(stream)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    return dist.max(e0.elapsed_time(e1)), st


def e2e_steps(solver, p0, v0, k, dist, record=None):
    """End to end through the C ABI, the same steps as the timed region: every step uploads
    its state (positions, velocities) from pinned host memory, steps once and downloads the
    new state, which is the next step's input. Returns (seconds per step, h2d and d2h bytes
    per step). With `record` (a step index j of the window), the host state before step j and
    the positions after it are kept in record_out (copies made outside the timed span)."""
    import torch

    import mguso

    lib = solver.lib
    pin_p = torch.from_numpy(np.ascontiguousarray(p0, np.float32)).pin_memory()
    pin_v = torch.from_numpy(np.ascontiguousarray(v0, np.float32)).pin_memory()
    nbytes = pin_p.numel() * 4 + pin_v.numel() * 4
    torch.cuda.synchronize()
    dist.barrier()
    span, kept = 0.0, {}
    t0 = time.perf_counter()
    for j in range(k):
        if j == record:
            span += time.perf_counter() - t0
            kept["pre"] = (pin_p.numpy().copy(), pin_v.numpy().copy())
            t0 = time.perf_counter()
        mguso._lib.check(lib.mguso_write_positions(solver.h, pin_p.data_ptr()))
        mguso._lib.check(lib.mguso_write_velocities(solver.h, pin_v.data_ptr()))
        solver.step(1)
        mguso._lib.check(lib.mguso_read_positions(solver.h, pin_p.data_ptr()))
        mguso._lib.check(lib.mguso_read_velocities(solver.h, pin_v.data_ptr()))
        if j == record:
            span += time.perf_counter() - t0
            kept["post"] = pin_p.numpy().copy()
            t0 = time.perf_counter()
    span += time.perf_counter() - t0
    e2e_steps.kept = kept
    return dist.max(span) / k, nbytes, nbytes


def step_errors(x_start, x_test, x_ref):
    """Relative position error of one step against a reference result from the same start:
    max and RMS |x_test - x_ref| over max and RMS of the reference's step displacement, and
    the max over max |x_ref| (the positions)."""
    d = np.linalg.norm(x_test.astype(np.float64) - x_ref, axis=1)
    disp = np.linalg.norm(x_ref - x_start.astype(np.float64), axis=1)
    return {"max_rel_to_step_displacement": float(f"{d.max() / max(disp.max(), 1e-30):.3e}"),
            "rms_rel_to_step_displacement": float(f"{np.sqrt((d ** 2).mean() / max((disp ** 2).mean(), 1e-60)):.3e}"),
            "max_rel_to_positions": float(f"{d.max() / np.abs(x_ref).max():.3e}")}


def traffic_from_profiles(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summaries: a line
    `traffic_bytes_per_launch <kernel> = <bytes>` in profiles/*.md (None when absent)."""
    import glob
    import re

    pat = re.compile(r"traffic_bytes_per_launch\s+`?(.+?)`?\s*=\s*([0-9.eE+]+)")
    want = kernel.replace(" ", "")
    for f in sorted(glob.glob(os.path.join(REPO, "profiles", "*.md"))):
        for line in open(f):
            m = pat.search(line)
            if m and m.group(1).replace(" ", "") == want:
                return float(m.group(2)), os.path.basename(f)
    return None, None


def run_batch(args, dist: Dist):
    """The sheath graded into 6 sizes on 6 scaled torsos, stepped as one
    mixed-precision batch, against the plain FP32 path stepping each size alone."""
    import torch

    import mguso
    from mguso import scenes

    torch.cuda.set_device(dist.local)
    ctx = mguso.Context(dist.local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    scs = scenes.graded_sheaths()
    if args.pcg_variant:
        scs = [dict(sc, params=dict(sc["params"], pcg_variant=args.pcg_variant)) for sc in scs]
    ntri = [int(sc["shell_faces"].shape[0]) for sc in scs]
    clocks = ClockSampler(dist.local)
    clocks.start()
    # batched, mixed precision (FP16 Schwarz factor tiles): the headline
    b = mguso.ImplicitBatch(ctx, scs, "mixed")
    b.step(args.warmup)
    p_w, v_w = b.positions.copy(), b.velocities.copy()
    ms_b, st_b = time_steps(b, args.steps, stream, dist, "batch")
    clk = clocks.stop()
    # batched, mixed precision with FP32 factor tiles (the apply in FP32 storage), same steps
    scs32 = [dict(sc, params=dict(sc["params"], factor_storage=1)) for sc in scs]
    b32 = mguso.ImplicitBatch(ctx, scs32, "mixed")
    b32.step(args.warmup)
    ms_b32, st_b32 = time_steps(b32, args.steps, stream, dist)
    b32.close()
    # plain FP32 (FP32 storage everywhere, FP32 factor tiles), each size alone, same steps
    ms_p = 0.0
    newton_p = []
    for sc in scs:
        g = mguso.ImplicitSolver(ctx, sc, "fp32")
        g.step(args.warmup)
        ms, st = time_steps(g, args.steps, stream, dist)
        ms_p += ms
        newton_p += [s_["newton_iters"] for s_ in st]
        g.close()
    inst_steps = len(scs) * args.steps
    value = inst_steps / (ms_b * 1e-3) * dist.world
    value32 = inst_steps / (ms_b32 * 1e-3) * dist.world
    plain = inst_steps / (ms_p * 1e-3) * dist.world
    # the fused PCG kernels timed inside a solve of the last Newton system (CUDA events per
    # launch), and the other solver kernels timed alone
    fused = b.profile_pcg(64)
    prof = b.profile(100)
    dom = max(fused, key=lambda k: fused[k][0])
    us, nbytes = fused[dom]
    knames = b.pcg_kernel_names()
    kname = knames[dom]
    rv_, dv_ = b.pcg_kernels()
    pvar = 6 * rv_ + dv_ + 1  # the mguso_params.pcg_variant that fixes these kernels
    traffic, tsrc = traffic_from_profiles(kname)
    # the window's representative step: the one whose mean Newton count (over the sizes) is
    # the median of the window's; the CPU baseline and the FP64 error are taken there
    per_step = [float(np.mean([s_["newton_iters"] for s_ in step])) for step in st_b]
    j_med = int(np.argsort(per_step, kind="stable")[len(per_step) // 2])
    # end to end: the timed steps again from the same state, each step's state through host
    e2e_s, h2d, d2h = e2e_steps(b, p_w, v_w, args.steps, dist, record=j_med)
    kept = e2e_steps.kept
    nl = None if args.no_launch_count else count_launches(lambda: b.step(1))
    launches = None if nl is None else int(nl * args.steps)
    peak, peak_kind = load_peaks()
    achieved = nbytes / (us * 1e-6) / 1e9
    newton_b = [s_["newton_iters"] for step in st_b for s_ in step]
    res = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": BATCH_UNIT,
        "n_gpus": dist.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_b / args.steps, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 storage + f64 (dots, norms, SpMV/apply accumulation, barrier, CCD root); "
                 "Schwarz factor tiles f16 scaled per domain",
        "data": "synthetic (seeded meshes; no dataset)",
        "config": {
            "workload": BATCH_WORKLOAD,
            "unit_note": "instance steps per second: 6 graded sizes batched, mixed precision, steps "
                         f"{args.warmup + 1}..{args.warmup + args.steps} of each drape",
            "triangles_per_size": ntri, "vertices_total": int(b.nv),
            "drapes_per_s": round(value / 120.0, 4),
            "batched_mixed_fp32_tiles_drape_steps_per_s": round(value32, 3),
            "plain_fp32_per_size_drape_steps_per_s": round(plain, 3),
            "batched_mixed_over_plain_fp32": round(value / plain, 3),
            "batched_mixed_fp32_tiles_over_plain_fp32": round(value32 / plain, 3),
            "newton_iters_mean_batched": round(float(np.mean(newton_b)), 2),
            "newton_iters_mean_plain": round(float(np.mean(newton_p)), 2),
            "newton_iters_mean_batched_fp32_tiles": round(float(np.mean([s_["newton_iters"] for step in st_b32
                                                                          for s_ in step])), 2),
            "pcg_iters_max_batched": int(max(s_["max_cg_iters"] for step in st_b for s_ in step)),
            "l2": "working set L2-resident (latency-bound step); per-kernel GB/s reported, not graded",
            "parallelism": f"replicas x{dist.world}",
        },
        "roofline": {
            "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4),
            "traffic": None if traffic is None else int(traffic),
            "traffic_source": tsrc, "peak_kind": f"{peak_kind} (burst copy)",
            "kernel": kname + " (fused PCG, timed inside a solve of the last Newton system)",
            "us_per_launch": round(us, 2), "bytes_per_launch": int(nbytes),
            "fused": {k: {"kernel": knames[k], "us": round(v[0], 2), "bytes": int(v[1]),
                          "GB/s": round(v[1] / (v[0] * 1e-6) / 1e9, 1)} for k, v in fused.items()},
            "pcg_variant": int(pvar),
            "per_kernel_alone": {k: {"us": round(v[0], 2), "bytes": int(v[1]),
                                     "GB/s": round(v[1] / (v[0] * 1e-6) / 1e9, 1)} for k, v in prof.items()},
        },
        "e2e": {"value": round(len(scs) / e2e_s * dist.world, 3), "unit": BATCH_UNIT,
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": launches,
        "clocks": {k: clk[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        "status": sorted(set(int(s_["status"]) for step in st_b for s_ in step)),
    }
    step_no = args.warmup + 1 + j_med
    res["config"]["newton_iters_per_step_batched"] = [round(x, 2) for x in per_step]
    res["config"]["newton_iters_per_s_batched"] = round(float(np.sum(newton_b)) / (ms_b * 1e-3), 2)
    if dist.rank == 0 and not args.no_cpu_baseline:
        # the representative step of every size from the GPU's state before it: the batch's
        # result, the FP32 oracle's (timed: the CPU baseline) and the FP64 oracle's
        p_j, v_j = kept["pre"]
        x_gpu = kept["post"]
        off = b.offsets
        states = [(p_j[off[i]:off[i + 1]], v_j[off[i]:off[i + 1]]) for i in range(len(scs))]
        sps, sample, cores, newton_cpu, x32 = cpu_drape_window("batch", step_no - 1, args.cpu_seconds, states)
        res["cpu_baseline"] = {"value": round(sps, 4), "unit": BATCH_UNIT, "cores": cores, "kind": "port",
                               "sample": sample,
                               "newton_iters_per_s": round(sps * float(np.mean([n for nw in newton_cpu for n in nw])), 3)}
        if not args.no_fp64_check:
            jobs = [("batch", i, "f64", 0, 0.0, states[i]) for i in range(len(scs))]
            r64 = _pool_map(jobs, min(len(scs), os.cpu_count() or 1))
            table = []
            for i in range(len(scs)):
                x64 = r64[i][3]
                xs = p_j[off[i]:off[i + 1]]
                table.append({"size": i, "step": step_no,
                              "batch_mixed_vs_fp64": step_errors(xs, x_gpu[off[i]:off[i + 1]], x64),
                              "oracle_fp32_vs_fp64": step_errors(xs, x32[i], x64),
                              "newton_batch_fp64_fp32": [int(st_b[j_med][i]["newton_iters"]), r64[i][2][0],
                                                         newton_cpu[i][0]]})
            res["config"]["fp64_oracle_error_representative_step"] = table
    b.close()
    ctx.close()
    try:
        res["config"]["spmv_grid1024"] = spmv_grid1024_side(max(args.steps, 20))
    except Exception as e:  # reported, never fatal to the headline line
        res["config"]["spmv_grid1024"] = {"error": f"{type(e).__name__}: {e}"}
    return res


def run_drape(args, dist: Dist):
    import torch

    import mguso

    torch.cuda.set_device(dist.local)
    ctx = mguso.Context(dist.local)
    sc, desc = drape_scene(args.workload)
    solver = mguso.ImplicitSolver(ctx, sc, args.precision)
    nv = sc["positions"].shape[0]
    stream = torch.cuda.ExternalStream(ctx.stream)
    clocks = ClockSampler(dist.local)
    clocks.start()
    solver.step(args.warmup)
    p_w, v_w = solver.positions.copy(), solver.velocities.copy()
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    stats = solver.step(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = dist.max(e0.elapsed_time(e1))
    ms_step = ms / args.steps
    # live per-kernel times at the last assembled system (CUDA events, each kernel alone);
    # the SpMV and the preconditioner apply each run once per PCG iteration
    prof = solver.profile(100)
    dom = max(("spmv", "precond_apply"), key=lambda k: prof[k][0])
    us, nbytes = prof[dom]
    # end to end through the C ABI: the timed steps again, each step's state through host
    e2e_s, h2d, d2h = e2e_steps(solver, p_w, v_w, args.steps, dist)
    # launches per step from a short traced pass (not timed)
    nl = None if args.no_launch_count else count_launches(lambda: solver.step(2))
    launches = None if nl is None else int(round(nl / 2 * args.steps))
    peak, peak_kind = load_peaks()
    achieved = nbytes / (us * 1e-6) / 1e9
    newton = [s_["newton_iters"] for s_ in stats]
    res = {
        "metric": METRIC,
        "value": round(args.steps / (ms * 1e-3) * dist.world, 3),
        "unit": "steps/s",
        "n_gpus": dist.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_step, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32" if args.precision == "fp32" else "f32+f64(dots,barrier,ccd)",
        "data": "synthetic (seeded meshes; no dataset)",
        "config": {
            "workload": desc, "vertices": int(nv), "precision": args.precision,
            "newton_iters_mean": round(float(np.mean(newton)), 2), "cg_iters_max": int(max(s_["max_cg_iters"] for s_ in stats)),
            "stencils_max": int(max(s_["stencils"] for s_ in stats)),
            "l2": "working set L2-resident (drape step is latency-bound); per-kernel GB/s reported, not graded",
            "parallelism": f"replicas x{dist.world}",
        },
        "roofline": {
            "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": None, "peak_kind": f"{peak_kind} (burst copy)",
            "kernel": {"spmv": "k_system_spmv", "precond_apply": "k_schwarz_apply"}[dom]
            + " (once per PCG iteration; timed alone at the last Newton system)",
            "us_per_launch": round(us, 2), "bytes_per_launch": int(nbytes),
            "per_kernel": {k: {"us": round(v[0], 2), "bytes": int(v[1]),
                               "GB/s": round(v[1] / (v[0] * 1e-6) / 1e9, 1)} for k, v in prof.items()},
        },
        "e2e": {"value": round(1.0 / e2e_s * dist.world, 3), "unit": "steps/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": launches,
        "clocks": {k: clk[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        "status": sorted(set(int(s_["status"]) for s_ in stats)),
    }
    if dist.rank == 0 and not args.no_cpu_baseline:
        sps, sample, cores, _, _ = cpu_drape_window(args.workload, args.warmup, args.cpu_seconds, [(p_w, v_w)])
        res["cpu_baseline"] = {"value": round(sps, 4), "unit": "steps/s", "cores": cores, "kind": "port",
                               "sample": sample}
    solver.close()
    ctx.close()
    return res


def run_reference(args, dist: Dist):
    if dist.rank != 0:
        return None
    if args.workload == "spmv":
        gbs, sample = cpu_spmv_sample(max(1.0, min(args.cpu_seconds, 2.0 * args.steps)))
        return {
            "impl": "reference", "metric": METRIC, "value": round(gbs, 3), "unit": "GB/s",
            "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": "BSR SpMV, 1024x1024 cloth grid stiffness pattern"},
            "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": 1, "kind": "port", "sample": sample},
            "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
    sps, sample, cores, newton, _ = cpu_drape_window(args.workload, args.warmup, max(1.0, min(args.cpu_seconds, 30.0)))
    _, desc = drape_scene(args.workload)
    unit = BATCH_UNIT if args.workload == "batch" else "steps/s"
    nps = round(sps * float(np.mean([n for nw in newton for n in nw])), 3)
    return {
        "impl": "reference", "metric": METRIC, "value": round(sps, 4), "unit": unit, "n_gpus": dist.world,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": {"workload": desc},
        "cpu_baseline": {"value": round(sps, 4), "unit": unit, "cores": cores, "kind": "port", "sample": sample,
                         "newton_iters_per_s": nps},
        "e2e": {"value": round(sps, 4), "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="mguso", choices=["mguso", "reference"])
    ap.add_argument("--workload", default="batch", choices=["batch", "drape", "sheet", "spmv"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp32"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-check", action="store_true", help="skip the FP64-oracle error of the first timed step")
    ap.add_argument("--no-launch-count", action="store_true", help="skip the traced launch count (under ncu)")
    ap.add_argument("--pcg-variant", type=int, default=0,
                    help="fused PCG kernels (mguso_params.pcg_variant; 0 = the autotuner's choice), to profile "
                         "one variant reproducibly")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        # the reference's path is single-process CPU work: rank 0 runs it, other ranks
        # exit without work (no process group needed)
        os.environ.setdefault("WORLD_SIZE", "1")
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return
        res = run_reference(args, Dist.__new__(Dist).__init_local__())
        print(json.dumps(res), flush=True)
        return
    dist = Dist("nccl")
    try:
        if args.workload == "spmv":
            res = run_spmv(args, dist)
        elif args.workload == "batch":
            res = run_batch(args, dist)
        else:
            res = run_drape(args, dist)
        if dist.rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
