"""The oracle reproduces its committed golden trajectories bit for bit (FP32 and FP64
positions and per-step Newton counts of three small drapes, made by
tests/golden/make_oracle_trajectories.py), so any change to the restatement that moves a
trajectory is seen here before it can change a GPU parity result."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_oracle_trajectories as M  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "oracle_trajectories.npz"))


@pytest.mark.parametrize("case", [c[0] for c in M.cases()])
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_oracle_reproduces_its_golden_trajectory(case, prec):
    name, sc, steps = next(c for c in M.cases() if c[0] == case)
    x, it = M.run(sc, steps, prec)
    assert np.array_equal(it, GOLD[f"{name}_{prec}_newton"])
    assert np.array_equal(x, GOLD[f"{name}_{prec}"])
