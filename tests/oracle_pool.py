"""Oracle steps from given states in parallel processes (test infrastructure).

The oracle's implicit step is single-threaded; the configuration-size parity tests run one
oracle step per sampled state, each in its own process, started with `spawn` (a process
forked after the parent has touched the GPU would hang)."""
from __future__ import annotations

import multiprocessing as mp
import os


def _oracle_step_job(job):
    sc, precision, p, v, params, check = job
    import oracle_py as O

    if params:
        sc = dict(sc, params=dict(sc["params"], **params))
    o = O.OracleSolver(sc, precision)
    o.set_state(p, v)
    st = o.step(1, check_intersection=check)[0]
    return o.positions(), st


def oracle_steps_from(sc, states, precision="f32", params=None, check_intersection=False):
    """One oracle step of scene `sc` from each (positions, velocities) in `states`:
    a list of (positions after the step (f64), step stats); with check_intersection the
    stats' penetration_free includes the self-intersection scan."""
    jobs = [(sc, precision, p, v, params, check_intersection) for p, v in states]
    workers = max(1, min(len(jobs), os.cpu_count() or 1))
    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.map(_oracle_step_job, jobs)
