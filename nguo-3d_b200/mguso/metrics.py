"""The solver-invariant checker over a run's per-step stats (metrics.rs:84-170): the
acceptance gate the reference applies to a drape instead of per-vertex position matching.

``check_invariants(steps, cg_tol, cg_max_iter, strain_limit=0.0)`` takes the per-step stats
dicts ``ImplicitSolver.step`` returns (or the oracle's, which carry the same keys) and
returns an ``InvariantReport`` with the reference's six checks, in its order and with its
thresholds:

1. ``penetration_free``: every step free of penetration / CCD failure;
2. ``all_frames_finite``: every step finite;
3. ``strain_limit_respected``: peak ``max_sigma`` at most ``(1 + limit) 1.02``, auto-pass
   when strain limiting is off (``strain_limit <= 0``);
4. ``cg_converged``: worst ``max_reresid`` at most ``1.5 cg_tol``;
5. ``cg_iter_under_cap``: most PCG iterations in a step below ``cg_max_iter``;
6. ``zero_steady_state_alloc``: no device allocation or free in the second half of the run.
   The CUDA step keeps no such counters (its buffers are reused from step to step and grow
   only when a step needs more stencil or contact-block room than any before it), so its
   steps carry none and the check reports an auto-pass saying so, as the reference's CPU
   tier does.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Sequence


@dataclass
class Invariant:
    name: str
    ok: bool
    detail: str


@dataclass
class InvariantReport:
    checks: List[Invariant] = field(default_factory=list)

    def all_ok(self) -> bool:
        return all(c.ok for c in self.checks)

    def by_name(self, name: str) -> Invariant:
        return next(c for c in self.checks if c.name == name)


def _flatten(steps: Sequence) -> list:
    """Per-step dicts; a batch run's per-step lists of per-instance dicts are flattened."""
    out = []
    for s in steps:
        out.extend(s if isinstance(s, (list, tuple)) else [s])
    return out


def check_invariants(steps: Sequence, cg_tol: float, cg_max_iter: int, strain_limit: float = 0.0) -> InvariantReport:
    st = _flatten(steps)
    r = InvariantReport()
    bad = sum(1 for s in st if not s["penetration_free"])
    r.checks.append(Invariant("penetration_free", bad == 0, f"{bad} step(s) with penetration/CCD failure"))
    nonfinite = sum(1 for s in st if not s["all_finite"])
    r.checks.append(Invariant("all_frames_finite", nonfinite == 0, f"{nonfinite} non-finite step(s)"))
    if strain_limit <= 0:
        r.checks.append(Invariant("strain_limit_respected", True, "strain limiting disabled (auto-pass)"))
    else:
        peak = max([float(s.get("max_sigma", 0.0)) for s in st] + [0.0])
        ceiling = (1.0 + strain_limit) * 1.02
        r.checks.append(Invariant("strain_limit_respected", peak <= ceiling,
                                  f"peak sigma {peak:.4f} vs ceiling {ceiling:.4f}"))
    worst = max([float(s["max_reresid"]) for s in st] + [0.0])
    tol = float(cg_tol) * 1.5
    r.checks.append(Invariant("cg_converged", worst <= tol, f"worst reresid {worst:.3e} vs {tol:.3e}"))
    max_it = max([int(s["max_cg_iters"]) for s in st] + [0])
    r.checks.append(Invariant("cg_iter_under_cap", max_it < cg_max_iter, f"max cg iters {max_it} vs cap {cg_max_iter}"))
    half = st[len(st) // 2:]
    alloc = sum(int(s.get("device_alloc", 0)) for s in half)
    free = sum(int(s.get("device_free", 0)) for s in half)
    counted = any("device_alloc" in s or "device_free" in s for s in st)
    r.checks.append(Invariant("zero_steady_state_alloc", alloc == 0 and free == 0,
                              f"steady-state device alloc {alloc} free {free}" if counted else
                              "no device-pool counters recorded (auto-pass)"))
    return r
