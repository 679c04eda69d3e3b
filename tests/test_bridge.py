"""The in-process drape loop (mguso.bridge) against the contract of the garment app's bridge
(ui/crates/nguo-engine-bridge/src/inproc.rs): frame stride with the last step always
published, cancellation, divergence, static scenes, stitch constants. The stepper is a fake
or the oracle wrapped as one (CPU)."""
import numpy as np
import pytest

import oracle_py as O
from mguso import bridge, scenes


def _sheet(n=4, pinned=True):
    pos = np.array([(i * 0.1, 0.5, j * 0.1) for j in range(n) for i in range(n)], np.float32)
    tris = []
    for j in range(n - 1):
        for i in range(n - 1):
            a = j * n + i
            tris += [(a, a + 1, a + n), (a + n, a + 1, a + n + 1)]
    im = np.full(n * n, 10.0, np.float32)
    if pinned:
        im[[0, n - 1]] = 0.0
    si, sw, skl = scenes._empty_stitches()
    return dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=im, tris=np.array(tris, np.uint32),
                shell_faces=np.zeros((0, 3), np.uint32), static_mask=None, stitch_idx=si, stitch_w=sw,
                stitch_kl=skl, colliders=np.zeros((0, 8), np.float32),
                params=scenes.default_params(self_collision=0, stiffness=1e3, bend_stiffness=0.0))


class Fake:
    """Moves every dynamic vertex down by 1 mm per step; NaN at step `nan_at`."""

    def __init__(self, ctx, scene, precision, nan_at=None):
        self.p = np.asarray(scene["positions"], np.float32).copy()
        self.dyn = np.asarray(scene["inv_mass"]) > 0
        self.k, self.nan_at, self.closed = 0, nan_at, False
        self.scene = scene

    def step(self, n):
        for _ in range(n):
            self.p[self.dyn, 1] -= 1e-3
            if self.nan_at is not None and self.k == self.nan_at:
                self.p[5, 0] = np.nan
            self.k += 1

    @property
    def positions(self):
        return self.p

    def close(self):
        self.closed = True


class Sink(bridge.FrameSink):
    def __init__(self, stop_at=None, cancel_after=None):
        self.frames, self.stop_at, self.cancel_after = [], stop_at, cancel_after

    def push(self, index, positions):
        self.frames.append((index, positions))
        return self.stop_at is None or index < self.stop_at

    def is_cancelled(self):
        return self.cancel_after is not None and len(self.frames) >= self.cancel_after


@pytest.mark.parametrize("steps, stride, want", [(10, 1, 10), (10, 3, 4), (10, 4, 4), (1, 5, 1)])
def test_frames_follow_the_stride_and_the_last_step_is_published(steps, stride, want):
    sink = Sink()
    rep = bridge.drape(None, _sheet(), steps, frame_stride=stride, sink=sink, solver_factory=Fake)
    assert rep["frames_emitted"] == want == len(sink.frames)
    assert [i for i, _ in sink.frames] == list(range(want))
    # the last frame is the state after the last step
    assert np.isclose(sink.frames[-1][1][5, 1], 0.5 - steps * 1e-3)


def test_the_sink_can_cancel_at_a_frame_or_between_steps():
    with pytest.raises(bridge.Cancelled):
        bridge.drape(None, _sheet(), 10, sink=Sink(stop_at=2), solver_factory=Fake)
    s = Sink(cancel_after=3)
    with pytest.raises(bridge.Cancelled):
        bridge.drape(None, _sheet(), 10, sink=s, solver_factory=Fake)
    assert len(s.frames) == 3


def test_a_non_finite_position_is_reported_with_its_step_and_vertex():
    made = []

    def factory(ctx, sc, prec):
        made.append(Fake(ctx, sc, prec, nan_at=4))
        return made[-1]

    with pytest.raises(bridge.Diverged) as e:
        bridge.drape(None, _sheet(), 10, solver_factory=factory)
    assert e.value.step == 4 and e.value.vertex == 5
    assert made[0].closed


def test_a_scene_with_nothing_dynamic_is_rejected():
    sc = _sheet()
    sc["inv_mass"] = np.zeros_like(sc["inv_mass"])
    with pytest.raises(bridge.Unsupported):
        bridge.drape(None, sc, 3, solver_factory=Fake)


def test_stitches_get_the_bridge_constants_and_are_validated():
    sc = _sheet()
    sewn = bridge.sew(sc, [([0, 0, 0, 5, 6, 6], [1, 0, 0, 0.5, 0.5, 0])])
    l0 = max(sc["params"]["contact_dhat"], 1e-4)
    assert np.allclose(sewn["stitch_kl"], [[1.0, l0, 10 * l0]])
    with pytest.raises(bridge.Unsupported):
        bridge.sew(sc, [([0, 0, 0, 5, 6, 6], [1, 0, 0, 0.7, 0.5, 0])])
    with pytest.raises(bridge.Unsupported):
        bridge.sew(sc, [([0, 0, 0, 99, 6, 6], [1, 0, 0, 1, 0, 0])])


class OracleStepper:
    """The oracle behind the stepper interface (a CPU stand-in for the GPU solver)."""

    def __init__(self, ctx, scene, precision):
        self.o = O.OracleSolver(scene)

    def step(self, n):
        self.o.step(n, check_intersection=False)

    @property
    def positions(self):
        return self.o.positions()


def test_a_sewn_drape_through_the_loop_closes_its_seam():
    sc = _sheet(4)
    sc["params"] = dict(sc["params"], gravity=(0.0, 0.0, 0.0))
    sink = Sink()
    rep = bridge.drape(None, sc, 60, stitches=[([3, 3, 3, 12, 12, 12], [1, 0, 0, 1, 0, 0])], frame_stride=20,
                       sink=sink, solver_factory=OracleStepper)
    assert rep["frames_emitted"] == 4 and rep["stitches"] == 1  # steps 0, 20, 40 and the last, 59
    first, last = sink.frames[0][1], sink.frames[-1][1]
    d0 = np.linalg.norm(sc["positions"][3] - sc["positions"][12])
    assert np.linalg.norm(last[3] - last[12]) < 0.5 * d0
    assert np.all(np.isfinite(last)) and np.array_equal(last[0], sc["positions"][0])


def test_a_sewn_garment_document_drapes_through_the_loop():
    """A garment document sewn by mguso.garment and submitted as the app does: the placed
    scene with its stitches handed to the loop, which attaches them at the bridge's
    constants and steps."""
    from mguso import garment as G

    g = G.build(G.sample_bodice_block(), G.SewOptions(triangulate=G.T.Options(target_edge_mm=90.0)))
    sc = g.scene(gravity=(0.0, -9.8, 0.0), self_collision=0, bend_stiffness=0.0, contact_dhat=1e-3)
    sc["stitch_idx"], sc["stitch_w"], sc["stitch_kl"] = scenes._empty_stitches()
    top = np.flatnonzero(np.abs(sc["positions"][:, 1] - sc["positions"][:, 1].max()) < 1e-6)
    sc["inv_mass"][top] = 0.0  # held by its waist
    sink = Sink()
    rep = bridge.drape(None, sc, 12, stitches=g.stitch_pairs(), frame_stride=4, sink=sink,
                       solver_factory=OracleStepper)
    assert rep["stitches"] == len(g.stitch_idx) > 0 and rep["frames_emitted"] == 4
    last = sink.frames[-1][1]
    assert np.all(np.isfinite(last))
    idx, w = g.stitch_idx, g.stitch_w
    a = (last[idx[:, :3]] * w[:, :3, None]).sum(1)
    b = (last[idx[:, 3:]] * w[:, 3:, None]).sum(1)
    assert np.linalg.norm(a - b, axis=1).max() < 0.01  # the seams hold while it hangs
    assert last[:, 1].min() < sc["positions"][:, 1].min()  # and it hangs
