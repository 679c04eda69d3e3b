"""The capture reader and OBJ writer (mguso.capture) on synthetic captures, with the
reference reader's own parsing tests (engine-io/src/golden.rs:1926-2062) restated."""
import os

import numpy as np
import pytest

import oracle_py as O
from mguso import capture as cap
from mguso import scenes


def _f64(vals):
    return np.asarray(vals, "<f8").tobytes()


def _f32(vals):
    return np.asarray(vals, "<f4").tobytes()


def _u64(vals):
    return np.asarray(vals, "<u8").tobytes()


def test_decodes_synthetic_buffers():  # golden.rs:1926-1949
    assert cap.decode_vec3_f64(_f64([1, 2, 3, -4, 5.5, 6.25])).tolist() == [[1, 2, 3], [-4, 5.5, 6.25]]
    assert cap.decode_vec3_f32(_f32([0.5, -0.25, 10.0])).tolist() == [[0.5, -0.25, 10.0]]
    assert cap.decode_tris_u64(_u64([0, 1, 2, 2, 1, 3])).tolist() == [[0, 1, 2], [2, 1, 3]]


def test_rejects_misaligned_and_oversized():  # golden.rs:2053-2061
    with pytest.raises(cap.CaptureError):
        cap.decode_vec3_f64(bytes(23))
    with pytest.raises(cap.CaptureError):
        cap.decode_vec3_f32(bytes(10))
    with pytest.raises(cap.CaptureError):
        cap.decode_tris_u64(_u64([2 ** 32]) + bytes(16))


def test_compare_identical_is_zero_and_passes():  # golden.rs:1951-1959
    f = [[0, 0, 0], [1, 0, 0], [0, 1, 0]]
    r = cap.compare_frames(f, f)
    assert r.max_rel == 0 and r.rms == 0 and r.centroid_rel == 0 and r.passes()


def test_compare_known_offset():  # golden.rs:1961-1977
    ref = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    g = cap.compare_frames(ref + [0.1, 0, 0], ref)
    d = np.sqrt(2.0)
    assert abs(g.diagonal - d) < 1e-5
    for v in (g.max_rel, g.rms, g.centroid_rel):
        assert abs(v - 0.1 / d) < 1e-5
    assert not g.passes()  # rms 0.0707 exceeds the 2e-2 gate


def test_compare_length_mismatch_errors():  # golden.rs:1979-1982
    with pytest.raises(cap.CaptureError):
        cap.compare_frames([[0, 0, 0]], [[0, 0, 0], [1, 1, 1]])


def test_parses_param_toml_from_text(tmp_path):  # golden.rs:1984-2001
    (tmp_path / "param.toml").write_text('[param]\ndt = 0.001\nfps = 60.0\nframes = 200\n'
                                         'gravity = [0.0, -9.8, 0.0]\nworld_scaling = 2.0\nbarrier = "cubic"\n'
                                         'friction_mode = "max"\ncg_tol = oops\n')
    p = cap.read_param_toml(str(tmp_path))
    assert p["dt"] == 0.001 and p["fps"] == 60.0 and p["frames"] == 200
    assert p["gravity"] == (0.0, -9.8, 0.0) and p["world_scaling"] == 2.0
    assert p["cubic_barrier"] and p["friction_mode"] == "max"
    assert p["cg_tol"] == 1.0e-3  # unparsable: the default stays


def test_u64_index_decoders_refuse_to_truncate():  # golden.rs:1410-1455 (the triangle and index-list decoders)
    poison = 0x1_0000_0005  # narrows to 5, a plausible in-range vertex
    tri = np.array([0, 1, poison], "<u8").tobytes()
    for decode in (cap.decode_tris_u64, cap.decode_u64_list):
        with pytest.raises(cap.CaptureError, match="exceeds u32"):
            decode(tri)
    ok = np.array([7, 8, 9, 10, 11, 12], "<u8").tobytes()
    assert cap.decode_tris_u64(ok).tolist() == [[7, 8, 9], [10, 11, 12]]
    assert cap.decode_u64_list(ok[:16]).tolist() == [7, 8]


def test_friction_mode_parsing_falls_back_to_the_reference_default(tmp_path):  # contact.rs:1144-1165
    """The spellings of FrictionMode::from_str_or_default's test as param.toml values (the
    reader trims the value and its quotes as golden.rs:514-522 does); the default is min."""
    for text, want in (("max", "max"), ('"max"', "max"), (" mean ", "mean"), ("min", "min"),
                       ("wobble", "min"), ("", "min")):
        (tmp_path / "param.toml").write_text(f"[param]\nfriction_mode = {text}\n")
        assert cap.read_param_toml(str(tmp_path))["friction_mode"] == want, text
    (tmp_path / "param.toml").write_text("[param]\ndt = 0.002\n")
    assert cap.read_param_toml(str(tmp_path))["friction_mode"] == "min"


def test_reads_material_means_from_synthetic(tmp_path):  # golden.rs:2003-2028
    d = tmp_path / "input_bin" / "param"
    d.mkdir(parents=True)
    (d / "tri-young-mod.bin").write_bytes(_f32([100, 100, 100]))
    (d / "tri-bend.bin").write_bytes(_f32([1, 3]))
    (d / "tri-density.bin").write_bytes(_f32([1]))
    (d / "tri-strain-limit.bin").write_bytes(_f32([0.01, 0.03]))
    m = cap.read_material(str(tmp_path))
    assert m["young_mod"] == 100 and abs(m["bend"] - 2) < 1e-6 and m["density"] == 1
    assert abs(m["strain_limit"] - 0.02) < 1e-6
    (d / "tri-young-mod.bin").unlink()
    assert cap.read_material(str(tmp_path)) is None


def test_reads_pin_list_from_synthetic(tmp_path):  # golden.rs:2030-2051
    ib = tmp_path / "input_bin"
    ib.mkdir()
    (ib / "pin-ind-0.bin").write_bytes(_u64([10, 13]))
    (ib / "pin-ind-1.bin").write_bytes(_u64([7]))
    assert cap.read_pin_indices(str(tmp_path)).tolist() == [10, 13, 7]
    (ib / "pin-ind-2.bin").write_bytes(bytes(12))
    with pytest.raises(cap.CaptureError):
        cap.read_pin_indices(str(tmp_path))


def _sheet_capture(root, n=6, with_disp=True, stitches=True):
    """A small captured sheet: n x n grid at y = 0 in the template, lifted by displacement
    group 1 (all but the first row), two pinned corners, two stitches."""
    ib = root / "input_bin"
    (ib / "param").mkdir(parents=True)
    v = np.array([(i * 0.1, 0.0, j * 0.1) for j in range(n) for i in range(n)], np.float64)
    tris = []
    for j in range(n - 1):
        for i in range(n - 1):
            a = j * n + i
            tris += [(a, a + 1, a + n), (a + n, a + 1, a + n + 1)]
    (ib / "vert.bin").write_bytes(_f64(v.ravel()))
    (ib / "tri.bin").write_bytes(_u64(np.ravel(tris)))
    (ib / "vel.bin").write_bytes(_f32(np.zeros(3 * n * n)))
    if with_disp:
        dmap = np.ones(n * n, np.uint32)
        dmap[:n] = 0
        (ib / "vert_dmap.bin").write_bytes(dmap.astype("<u4").tobytes())
        (ib / "displacement.bin").write_bytes(_f64([0, 0, 0, 0, 0.5, 0]))
    (ib / "pin-ind-0.bin").write_bytes(_u64([n * n - n, n * n - 1]))
    if stitches:
        (ib / "stitch_ind.bin").write_bytes(_u64([0, 0, 0, 2, 3, 3, 1, 1, 1, 4, 4, 4]))
        (ib / "stitch_w.bin").write_bytes(_f32([1, 0, 0, 0.5, 0.5, 0, 1, 0, 0, 1, 0, 0]))
    (ib / "param" / "tri-young-mod.bin").write_bytes(_f32(np.full(len(tris), 1e5)))
    (ib / "param" / "tri-density.bin").write_bytes(_f32(np.full(len(tris), 0.2)))
    (root / "param.toml").write_text("[param]\ndt = 0.004\ngravity = [0.0, -9.8, 0.0]\ncg_tol = 1e-4\n")
    ck = root / "checkpoints"
    ck.mkdir()
    return v, np.array(tris, np.uint32)


def test_capture_input_applies_the_displacement_groups(tmp_path):  # golden.rs:313-380, 600-640
    v, tris = _sheet_capture(tmp_path)
    inp = cap.load_capture_input(str(tmp_path))
    want = v.astype(np.float32)
    want[6:, 1] += np.float32(0.5)
    assert np.array_equal(inp["positions"], want)
    assert np.array_equal(inp["tris"], tris)
    assert inp["velocities"].shape == want.shape
    # without both displacement files the template is the initial state
    (tmp_path / "input_bin" / "displacement.bin").unlink()
    assert np.array_equal(cap.load_capture_input(str(tmp_path))["positions"], v.astype(np.float32))


def test_capture_input_rejects_inconsistent_files(tmp_path):
    _sheet_capture(tmp_path)
    ib = tmp_path / "input_bin"
    (ib / "vert_dmap.bin").write_bytes(np.full(36, 5, "<u4").tobytes())  # group 5 does not exist
    with pytest.raises(cap.CaptureError):
        cap.load_capture_input(str(tmp_path))
    (ib / "vert_dmap.bin").unlink()
    (ib / "tri.bin").write_bytes(_u64([0, 1, 99]))
    with pytest.raises(cap.CaptureError):
        cap.load_capture_input(str(tmp_path))
    (ib / "tri.bin").unlink()  # rod-only scenes ship no tri.bin
    assert cap.load_capture_input(str(tmp_path))["tris"].shape == (0, 3)
    (ib / "vel.bin").write_bytes(_f32(np.zeros(3 * 35)))
    with pytest.raises(cap.CaptureError):
        cap.load_capture_input(str(tmp_path))


def test_reads_stitches_with_default_stiffness(tmp_path):  # golden.rs:839-888
    _sheet_capture(tmp_path)
    idx, w, k = cap.read_stitches(str(tmp_path))
    assert idx.tolist() == [[0, 0, 0, 2, 3, 3], [1, 1, 1, 4, 4, 4]]
    assert w[0].tolist() == [1, 0, 0, 0.5, 0.5, 0] and k.tolist() == [1.0, 1.0]
    ib = tmp_path / "input_bin"
    (ib / "stitch_stiffness.bin").write_bytes(_f32([2.0, 3.0]))
    assert cap.read_stitches(str(tmp_path))[2].tolist() == [2.0, 3.0]
    (ib / "stitch_w.bin").write_bytes(_f32(np.zeros(6)))
    with pytest.raises(cap.CaptureError):
        cap.read_stitches(str(tmp_path))


def test_obj_round_trip_is_exact(tmp_path):
    rng = np.random.default_rng(0)
    p = rng.normal(size=(50, 3)).astype(np.float32)
    t = rng.integers(0, 50, size=(30, 3)).astype(np.uint32)
    path = str(tmp_path / "frame.obj")
    cap.write_obj(path, p, t)
    q, u = cap.read_obj(path)
    assert np.array_equal(p, q) and np.array_equal(t, u)


def test_a_capture_drives_the_step_and_compares_to_its_checkpoint(tmp_path):
    """scene_from_capture gives a description the solver interface takes: the oracle steps
    it, the pins hold, and compare_frames measures the result against a checkpoint written
    in the capture's own format."""
    _sheet_capture(tmp_path)
    sc = cap.scene_from_capture(str(tmp_path), contact_dhat=1e-3)
    assert sc["params"]["dt"] == 0.004 and sc["shell_faces"].shape[0] == 50
    assert np.allclose(sc["stitch_kl"], [[1.0, 1e-3, 1e-2]] * 2)
    assert (sc["inv_mass"] == 0).sum() == 2
    o = O.OracleSolver(sc)
    o.step(3, check_intersection=False)
    x = o.positions()
    assert np.all(np.isfinite(x))
    assert np.array_equal(x[[30, 35]], sc["positions"][[30, 35]])  # pinned corners
    (tmp_path / "checkpoints" / "vert_3.bin").write_bytes(x.astype("<f4").tobytes())
    ref = cap.load_checkpoint(str(tmp_path), 3)
    g = cap.compare_frames(x, ref)
    assert g.max_rel == 0 and g.passes()
    assert cap.compare_frames(sc["positions"], ref).max_rel > 0
    cap.write_obj(str(tmp_path / "frame_3.obj"), x, sc["tris"])
    q, _ = cap.read_obj(str(tmp_path / "frame_3.obj"))
    assert np.array_equal(q, x.astype(np.float32))


def _sched(kind, t0, t1, **kw):
    from mguso.capture import PinBlockSchedule, PinOp

    return PinBlockSchedule(np.array([0], np.uint32), 1.0, 0.0, [PinOp(kind, t0, t1, **kw)])


def test_spin_and_scale_ops_match_the_reference_laws():  # golden.rs:1544-1635
    def near(a, b):
        return np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max() < 1e-5

    spin = _sched("spin", 0.0, 2.0, center=(0.0, 0.0, 0.0), axis=(0.0, 0.0, 1.0), angular_velocity=90.0)
    x = [1.0, 0.0, 0.0]
    q, kin = spin.target_at(0, x, 1.0)
    assert near(q, [0, 1, 0]) and kin
    h, _ = spin.target_at(0, x, 0.5)
    r = np.float32(np.sqrt(0.5))
    assert near(h, [r, r, 0]) and abs(np.hypot(h[0], h[1]) - 1.0) < 1e-5
    e1, e2 = spin.target_at(0, x, 2.0)[0], spin.target_at(0, x, 50.0)[0]
    assert near(e1, [-1, 0, 0]) and near(e1, e2)
    later = _sched("spin", 5.0, 6.0, center=(0.0, 0.0, 0.0), axis=(0.0, 0.0, 1.0), angular_velocity=90.0)
    pre, pre_kin = later.target_at(0, x, 0.0)
    assert near(pre, x) and not pre_kin
    sc = _sched("scale", 0.0, 1.0, center=(1.0, 1.0, 1.0), factor=3.0)
    p = [2.0, 1.0, 1.0]
    assert near(sc.target_at(0, p, 0.0)[0], [2, 1, 1]) and near(sc.target_at(0, p, 0.5)[0], [3, 1, 1])
    assert near(sc.target_at(0, p, 1.0)[0], [4, 1, 1]) and near(sc.target_at(0, p, 9.0)[0], [4, 1, 1])
    assert near(sc.target_at(0, [1, 1, 1], 1.0)[0], [1, 1, 1])


def test_a_pin_schedule_decodes_from_info_toml_and_composes(tmp_path):  # golden.rs:1122-1200
    from mguso import capture

    d = tmp_path / "scene"
    ib = d / "input_bin"
    ib.mkdir(parents=True)
    (ib / "pin-ind-0.bin").write_bytes(np.array([3, 7], "<u8").tobytes())
    (ib / "pin-0-op-0.bin").write_bytes(np.array([[0.0, 0.1, 0.0], [0.0, 0.1, 0.0]], "<f8").tobytes())
    (d / "info.toml").write_text('[pin-0]\noperation_count = 2\nstiffness = 2.5\n\n'
                                 '[pin-0-op-0]\ntype = "move_by"\nt_start = 0.0\nt_end = 1.0\ntransition = "smooth"\n\n'
                                 '[pin-0-op-1]\ntype = "torque"\nt_start = 0.0\nt_end = 1.0\n')
    (s,) = capture.read_pin_schedule(str(d))
    assert s.indices.tolist() == [3, 7] and s.stiffness == 2.5
    assert [o.kind for o in s.ops] == ["move_by", "torque"]
    # smoothstep at a quarter of the window: 0.25^2 (3 - 0.5) = 0.15625 of the 0.1 delta
    q, kin = s.target_at(1, [1.0, 0.0, 0.0], 0.25)
    assert kin and abs(q[1] - 0.015625) < 1e-7 and q[0] == 1.0
    assert s.target_at(1, [1.0, 0.0, 0.0], 5.0)[0].tolist() == [1.0, np.float32(0.1), 0.0]
    (ib / "pin-0-op-0.bin").write_bytes(np.zeros((3, 3), "<f8").tobytes())
    with pytest.raises(capture.CaptureError):
        capture.read_pin_schedule(str(d))


def test_a_scheduled_pin_drags_its_vertex_in_the_oracle_step(tmp_path):
    """A move_by schedule driving kinematic pins between steps, as a capture replay does."""
    from mguso.capture import PinBlockSchedule, PinOp

    n = 4
    pos = np.array([(i * 0.1, 0.0, j * 0.1) for j in range(n) for i in range(n)], np.float32)
    tris = np.array([(j * n + i, j * n + i + 1, j * n + i + n) for j in range(n - 1) for i in range(n - 1)] +
                    [(j * n + i + n, j * n + i + 1, j * n + i + n + 1) for j in range(n - 1) for i in range(n - 1)],
                    np.uint32)
    si, sw, skl = scenes._empty_stitches()
    sc = dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=np.full(n * n, 10.0, np.float32), tris=tris,
              shell_faces=np.zeros((0, 3), np.uint32), static_mask=None, stitch_idx=si, stitch_w=sw, stitch_kl=skl,
              colliders=np.zeros((0, 8), np.float32),
              params=scenes.default_params(self_collision=0, stiffness=500.0, gravity=(0.0, 0.0, 0.0),
                                           bend_stiffness=0.0, newton_iters=4, precond=1))
    sched = PinBlockSchedule(np.array([0], np.uint32), 1.0, 0.0,
                             [PinOp("move_by", 0.0, 0.5, data=np.array([[0.0, 0.3, 0.0]], np.float32))])
    o = O.OracleSolver(sc)
    dt = sc["params"]["dt"]
    for k in range(1, 41):
        t, _ = sched.target_at(0, pos[0], k * dt)
        assert o.set_pins([(0, t.astype(np.float64), 0.02, True, sched.stiffness)])
        o.step(1, check_intersection=False)
    x = o.positions()
    assert np.all(np.isfinite(x)) and abs(x[0, 1] - 0.3) < 0.04 and x[0, 1] > 0.2


def test_obj_round_trip_quad(tmp_path):  # engine-io obj.rs:429-440
    pos, tris = cap.parse_obj("v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nf 1 2 3\nf 3 2 4\n")
    assert pos.shape == (4, 3) and tris.shape == (2, 3)
    cap.write_obj(str(tmp_path / "q.obj"), pos, tris)
    p2, t2 = cap.read_obj(str(tmp_path / "q.obj"))
    assert np.array_equal(p2, pos) and np.array_equal(t2, tris)


def test_obj_triangulates_quad_face():  # obj.rs:442-446
    assert cap.parse_obj("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3 4\n")[1].shape == (2, 3)


def test_obj_handles_slashed_and_negative_indices():  # obj.rs:448-458
    _, tris, uv = cap.parse_obj("v 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nvt 1 0\nvt 0 1\nvn 0 0 1\nvn 0 0 1\nvn 0 0 1\n"
                                "f -3/-3/-3 -2/-2/-2 -1/-1/-1\n", with_uvs=True)
    assert tris.tolist() == [[0, 1, 2]] and uv.tolist() == [[0, 0], [1, 0], [0, 1]]


def test_obj_rejects_out_of_range_index():  # obj.rs:459-464
    with pytest.raises(cap.CaptureError):
        cap.parse_obj("v 0 0 0\nf 1 2 3\n")
    with pytest.raises(cap.CaptureError):
        cap.parse_obj("v 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nf 1/1 2/2 3/1\n")


def test_obj_face_without_uv_index_drops_the_uv_array():  # obj.rs:477-484
    _, _, uv = cap.parse_obj("v 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nvt 1 0\nvt 0 1\nf 1/1 2/2 3\n", with_uvs=True)
    assert uv.shape == (0, 2)


def test_obj_comment_anywhere_on_the_line():  # obj.rs:103-107: '#' starts a comment anywhere
    pos, tris = cap.parse_obj("# header\nv 0 0 0 # a\nv 1 0 0\nv 0 1 0\nf 1 2 3 # trailing comment\n")
    assert pos.shape == (3, 3) and tris.tolist() == [[0, 1, 2]]


def test_obj_rejects_short_faces_empty_files_and_malformed_records():  # obj.rs:136-138, 195-197, 249-262
    with pytest.raises(cap.CaptureError):
        cap.parse_obj("v 0 0 0\nv 1 0 0\nf 1 2\n")
    with pytest.raises(cap.CaptureError):
        cap.parse_obj("# nothing here\n")
    with pytest.raises(cap.CaptureError):
        cap.parse_obj("v 0 0\n")
    with pytest.raises(cap.CaptureError):
        cap.parse_obj("v 0 0 0\nvt\n")
    with pytest.raises(cap.CaptureError):
        cap.parse_obj("v 0 0 x\n")
