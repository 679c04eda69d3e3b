"""The host-side callers of the step, on the CUDA step, against the oracle:

- the garment app's in-process drape loop (mguso.bridge.drape, the bridge's
  InProcessTransport::solve, ui/crates/nguo-engine-bridge/src/inproc.rs:85-143) draping the
  reference's sample bodice block sewn by mguso.garment (nguo-sewing's build), with the
  default stepper (mguso.ImplicitSolver);
- a recorded scene in the reference's capture format (engine-io/src/golden.rs) read by
  mguso.capture and stepped by mguso.ImplicitSolver.

Every GPU step is compared with the oracle's step from the same state (positions within 1e-3
of the step's displacement, Newton counts within +-1)."""
import numpy as np
import pytest

from mguso import ImplicitSolver, bridge
from mguso import capture as cap
from oracle_pool import oracle_steps_from
from test_capture import _sheet_capture
from test_garment import G, garment

pytestmark = pytest.mark.gpu


class Recording(ImplicitSolver):
    """ImplicitSolver that keeps the state before and the positions after every step."""

    def __init__(self, ctx, scene, precision="mixed"):
        super().__init__(ctx, scene, precision)
        self.pre, self.post, self.stats = [], [], []

    def step(self, n=1):
        out = []
        for _ in range(n):
            self.pre.append((self.positions.astype(np.float64), self.velocities.astype(np.float64)))
            st = super().step(1)
            self.post.append(self.positions.astype(np.float64))
            self.stats += st
            out += st
        return out


def _check_against_oracle(sc, rec):
    res = oracle_steps_from(sc, rec.pre)
    for k, ((p0, _), pg, sg, (po, so)) in enumerate(zip(rec.pre, rec.post, rec.stats, res)):
        disp = np.abs(po - p0).max()
        print(k, sg["newton_iters"], so["newton_iters"], disp, np.abs(pg - po).max())
        assert sg["status"] == 0 and abs(sg["newton_iters"] - so["newton_iters"]) <= 1, (k, sg, so)
        if so["t_min"] < 1e-6:
            # the CCD clamps the step to nothing (the sample garment starts with its panels
            # touching): both sides stay put, to within a micrometre
            assert disp < 1e-6 and np.abs(pg - p0).max() < 1e-6, (k, disp, np.abs(pg - p0).max())
        else:
            assert np.abs(pg - po).max() < 1e-3 * disp, (k, np.abs(pg - po).max() / disp)


def test_bridge_drapes_a_sewn_garment_on_the_cuda_step(ctx):
    g = garment(triangulate=G.T.Options(target_edge_mm=60.0))
    sc = g.scene(self_collision=1, bend_stiffness=1e-5, contact_dhat=1e-3)
    made = []

    def factory(ctx_, scene, precision):
        made.append(Recording(ctx_, scene, precision))
        return made[-1]

    class Sink(bridge.FrameSink):
        def __init__(self):
            self.frames = []

        def push(self, index, positions):
            self.frames.append((index, positions))
            return True

    sink = Sink()
    rep = bridge.drape(ctx, sc, 6, frame_stride=2, sink=sink, solver_factory=factory)
    # frames at steps 0, 2, 4 and the last step, 5
    assert rep["steps"] == 6 and rep["frames_emitted"] == 4 and [i for i, _ in sink.frames] == [0, 1, 2, 3]
    rec = made[0]
    assert np.array_equal(sink.frames[-1][1], rec.post[-1].astype(np.float32))
    idx, w = sc["stitch_idx"], sc["stitch_w"]
    x = rec.post[-1]
    gap = np.linalg.norm((x[idx[:, :3]] * w[:, :3, None]).sum(1) - (x[idx[:, 3:]] * w[:, 3:, None]).sum(1), axis=1)
    assert np.all(np.isfinite(x)) and gap.max() < 5e-3  # the seams hold
    _check_against_oracle(sc, rec)


def test_a_capture_steps_on_the_cuda_step(ctx, tmp_path):
    _sheet_capture(tmp_path)
    sc = cap.scene_from_capture(str(tmp_path), contact_dhat=1e-3)
    rec = Recording(ctx, sc, "mixed")
    rec.step(4)
    x = rec.post[-1]
    assert np.all(np.isfinite(x))
    assert np.array_equal(x[[30, 35]].astype(np.float32), sc["positions"][[30, 35]])  # pinned corners
    _check_against_oracle(sc, rec)
    (tmp_path / "checkpoints" / "vert_4.bin").write_bytes(x.astype("<f4").tobytes())
    assert cap.compare_frames(x, cap.load_checkpoint(str(tmp_path), 4)).passes()
