"""The reference's scene-capture format and a per-frame OBJ writer: the data either side of
the implicit step when a recorded scene drives it (engine-io/src/golden.rs).

A capture directory holds little-endian binaries:

- ``input_bin/vert.bin``          f64 xyz per vertex, the template positions;
- ``input_bin/vert_dmap.bin``     u32 per vertex, its displacement group (optional);
- ``input_bin/displacement.bin``  f64 xyz per group, added to the template (optional);
- ``input_bin/tri.bin``           u64 x3 per triangle (optional: rod-only scenes omit it);
- ``input_bin/vel.bin``           f32 xyz per vertex, initial velocities;
- ``input_bin/pin-ind-<i>.bin``   u64 list of constrained vertices, one file per block;
- ``input_bin/stitch_ind.bin``    u64 x6 per stitch, ``stitch_w.bin`` f32 x6 per stitch,
  ``stitch_stiffness.bin`` f32 per stitch (optional, default 1);
- ``input_bin/param/tri-*.bin``   f32 per triangle material (young-mod, bend, density,
  strain-limit);
- ``param.toml``                  flat ``key = value`` run parameters;
- ``checkpoints/vert_<N>.bin``    f32 xyz per vertex, the recorded positions of frame N.

Readers here decode into numpy arrays, refuse misaligned buffers and indices that do not fit
u32 (a silently truncated index would build elements over the wrong vertices), and check
every index against the vertex count. ``scene_from_capture`` turns a capture into a scene
description for ``ImplicitSolver``; ``compare_frames`` measures a run against a checkpoint
with the reference's three scale-free gates; ``write_obj`` writes one frame as OBJ.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

__all__ = [
    "CaptureError", "decode_vec3_f64", "decode_vec3_f32", "decode_tris_u64", "decode_u64_list",
    "load_capture_input", "read_param_toml", "read_pin_indices", "read_stitches", "read_material",
    "load_checkpoint", "GateReport", "compare_frames", "scene_from_capture", "write_obj", "read_obj",
]


class CaptureError(ValueError):
    """A capture file that is missing, misaligned or inconsistent."""


def _read(path: str) -> bytes:
    try:
        with open(path, "rb") as f:
            return f.read()
    except OSError as e:
        raise CaptureError(f"reading capture file {path}: {e}") from e


def _aligned(buf: bytes, width: int, what: str):
    if len(buf) % width:
        raise CaptureError(f"{what} buffer length {len(buf)} is not a multiple of {width}")


def decode_vec3_f64(buf: bytes) -> np.ndarray:
    """f64 xyz records (24 bytes each) -> float32 (n, 3) (golden.rs:53-67)."""
    _aligned(buf, 24, "f64 vec3")
    return np.frombuffer(buf, "<f8").reshape(-1, 3).astype(np.float32)


def decode_vec3_f32(buf: bytes) -> np.ndarray:
    """f32 xyz records (12 bytes each) -> float32 (n, 3) (golden.rs:70-85)."""
    _aligned(buf, 12, "f32 vec3")
    return np.frombuffer(buf, "<f4").reshape(-1, 3).copy()


def _narrow(idx: np.ndarray, what: str) -> np.ndarray:
    if idx.size and int(idx.max()) > 0xFFFFFFFF:
        raise CaptureError(f"{what} index {int(idx.max())} exceeds u32")
    return idx.astype(np.uint32)


def decode_tris_u64(buf: bytes) -> np.ndarray:
    """u64 x3 triangles (24 bytes each) -> uint32 (n, 3), refusing indices above u32
    (golden.rs:89-110)."""
    _aligned(buf, 24, "u64 triangle")
    return _narrow(np.frombuffer(buf, "<u8").reshape(-1, 3), "triangle")


def decode_u64_list(buf: bytes, what: str = "u64 list") -> np.ndarray:
    """A flat u64 index list -> uint32 (n,)."""
    _aligned(buf, 8, what)
    return _narrow(np.frombuffer(buf, "<u8"), what)


def load_capture_input(scene_dir: str) -> dict:
    """Initial positions (template plus displacement group), triangles and velocities
    (golden.rs:313-380). The displacement is applied only when both its files exist."""
    ib = os.path.join(scene_dir, "input_bin")
    pos = np.frombuffer(_read(os.path.join(ib, "vert.bin")), "<f8")
    if pos.size % 3:
        raise CaptureError(f"vert.bin holds {pos.size} f64, not whole xyz records")
    pos = pos.reshape(-1, 3).copy()
    dmap_p, disp_p = os.path.join(ib, "vert_dmap.bin"), os.path.join(ib, "displacement.bin")
    if os.path.exists(dmap_p) and os.path.exists(disp_p):
        raw = _read(dmap_p)
        _aligned(raw, 4, "vert_dmap")
        dmap = np.frombuffer(raw, "<u4")
        if dmap.size != pos.shape[0]:
            raise CaptureError(f"vert_dmap has {dmap.size} entries but there are {pos.shape[0]} vertices")
        disp_raw = _read(disp_p)
        _aligned(disp_raw, 24, "displacement")
        disp = np.frombuffer(disp_raw, "<f8").reshape(-1, 3)
        if dmap.size and int(dmap.max()) >= disp.shape[0]:
            raise CaptureError(f"vert_dmap group {int(dmap.max())} exceeds the displacement table")
        # the group offset is added in f32, as the template's f64 is narrowed first
        pos32 = pos.astype(np.float32) + disp[dmap].astype(np.float32)
    else:
        pos32 = pos.astype(np.float32)
    tri_p = os.path.join(ib, "tri.bin")
    tris = decode_tris_u64(_read(tri_p)) if os.path.exists(tri_p) else np.zeros((0, 3), np.uint32)
    vel = decode_vec3_f32(_read(os.path.join(ib, "vel.bin")))
    nv = pos32.shape[0]
    if vel.shape[0] != nv:
        raise CaptureError(f"vel count {vel.shape[0]} != vert count {nv}")
    if tris.size and int(tris.max()) >= nv:
        raise CaptureError(f"a triangle references a vertex >= {nv}")
    return {"positions": pos32, "tris": tris, "velocities": vel}


_PARAM_DEFAULTS = dict(dt=1.0e-3, fps=60.0, frames=0, gravity=(0.0, -9.8, 0.0), world_scaling=1.0,
                       include_face_mass=False, air_density=1.0e-3, air_friction=0.0, isotropic_air_friction=0.0,
                       wind=(0.0, 0.0, 0.0), eiganalysis_eps=1.0e-2, cg_tol=1.0e-3, cg_max_iter=10000,
                       ccd_max_iter=4096, min_newton_steps=0, target_toi=0.25, max_dx=1.0, friction_eps=1.0e-5,
                       cubic_barrier=False, disable_contact=False, friction_mode="min", stitch_length_factor=10.0,
                       constraint_ghat=1.0e-3, constraint_tol=1.0e-2)


def _parse_param_text(text: str) -> dict:
    p = dict(_PARAM_DEFAULTS)
    for line in text.splitlines():
        if "=" not in line:
            continue
        key, val = (s.strip() for s in line.split("=", 1))
        if key not in p:
            continue
        cur = p[key]
        try:
            if key in ("gravity", "wind"):
                nums = [float(s) for s in val.strip("[]").split(",") if s.strip()]
                if len(nums) == 3:
                    p[key] = tuple(nums)
            elif key in ("include_face_mass", "disable_contact"):
                p[key] = val == "true"
            elif key == "friction_mode":
                v = val.strip('"')
                p[key] = v if v in ("max", "mean") else "min"
            elif isinstance(cur, bool):
                p[key] = val == "true"
            elif isinstance(cur, int):
                p[key] = int(val)
            else:
                p[key] = float(val)
        except ValueError:
            pass  # an unparsable value keeps its default, as the reference's reader does
    return p


def read_param_toml(scene_dir: str) -> dict:
    """The run parameters a driver needs from ``param.toml`` (golden.rs:448-540): defaults
    for missing or unparsable keys; ``barrier = "cubic"`` sets ``cubic_barrier``."""
    text = _read(os.path.join(scene_dir, "param.toml")).decode("utf-8", "replace")
    p = _parse_param_text(text)
    for line in text.splitlines():
        if "=" in line:
            key, val = (s.strip() for s in line.split("=", 1))
            if key == "barrier":
                p["cubic_barrier"] = val.strip('"') == "cubic"
    return p


def read_pin_indices(scene_dir: str) -> np.ndarray:
    """Constrained vertices: ``pin-ind-0.bin``, ``pin-ind-1.bin``, ... concatenated, each a
    u64 LIST (not a range) (golden.rs:562-597)."""
    ib = os.path.join(scene_dir, "input_bin")
    out, i = [], 0
    while os.path.exists(os.path.join(ib, f"pin-ind-{i}.bin")):
        out.append(decode_u64_list(_read(os.path.join(ib, f"pin-ind-{i}.bin")), f"pin-ind-{i}.bin"))
        i += 1
    return np.concatenate(out) if out else np.zeros(0, np.uint32)


def read_pin_blocks(scene_dir: str) -> list:
    """Each pin block's vertex list, in block order (golden.rs:880-913)."""
    ib = os.path.join(scene_dir, "input_bin")
    out, i = [], 0
    while os.path.exists(os.path.join(ib, f"pin-ind-{i}.bin")):
        out.append(decode_u64_list(_read(os.path.join(ib, f"pin-ind-{i}.bin")), f"pin-ind-{i}.bin"))
        i += 1
    return out


def _toml_section(text: str, want: str) -> dict:
    """key = value pairs of one [section] of a flat TOML text, quotes stripped
    (golden.rs:1205-1225)."""
    out, inside = {}, False
    for line in text.splitlines():
        t = line.strip()
        if t.startswith("[") and t.endswith("]"):
            inside = t[1:-1] == want
            continue
        if inside and "=" in t:
            k, v = (x.strip() for x in t.split("=", 1))
            out[k] = v.strip('"')
    return out


@dataclass
class PinOp:
    """One scheduled pin operation (golden.rs:930-1018): kind (move_by, move_to, spin, scale
    or an unsupported name), its window and easing, the spin / scale parameters and the
    per-vertex payload (a delta for move_by, a target for move_to)."""
    kind: str
    t_start: float
    t_end: float
    transition: str = "linear"   # linear, smooth, bezier (bezier eases linearly)
    center: tuple = (0.0, 0.0, 0.0)
    axis: tuple = (0.0, 0.0, 0.0)
    angular_velocity: float = 0.0  # degrees per second
    factor: float = 1.0
    data: Optional[np.ndarray] = None

    def progress_at(self, time: float) -> Optional[float]:
        """The eased ramp in [0, 1]; None before t_start (golden.rs:974-993)."""
        if time < self.t_start:
            return None
        if time >= self.t_end:
            return 1.0
        denom = self.t_end - self.t_start
        raw = (time - self.t_start) / denom if denom != 0.0 else 0.0
        return raw * raw * (3.0 - 2.0 * raw) if self.transition == "smooth" else raw


def _rodrigues(p, center, axis, angle):
    """p rotated by angle about the normalised axis through center, in f64, returned in f32
    (golden.rs:1088-1116); a zero axis does not rotate."""
    a = np.asarray(axis, np.float32).astype(np.float64)
    n = float(np.sqrt((np.float32(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]))))
    a = a * (1.0 / n if n > 0.0 else 0.0)
    c = np.asarray(center, np.float32)
    d = (np.asarray(p, np.float32) - c).astype(np.float64)
    ct, st = math.cos(angle), math.sin(angle)
    out = d * ct + np.cross(a, d) * st + a * float(d @ a) * (1.0 - ct)
    return out.astype(np.float32) + c


@dataclass
class PinBlockSchedule:
    """A pin block: its vertices, the FixPair stiffness and pull scalars, and its ordered
    operations (golden.rs:995-1083)."""
    indices: np.ndarray
    stiffness: float = 1.0
    pull: float = 0.0
    ops: list = field(default_factory=list)

    def target_at(self, slot: int, base, time: float):
        """(target, kinematic) of the block's slot-th vertex at time, composing every
        operation in order from its displaced initial position (golden.rs:1022-1082)."""
        p = np.asarray(base, np.float32).copy()
        kinematic = False
        for op in self.ops:
            if op.kind in ("move_by", "move_to"):
                prog = op.progress_at(time)
                if prog is None or op.data is None or slot >= len(op.data):
                    continue
                row = np.asarray(op.data[slot], np.float32)
                pr = np.float32(prog)
                p = p + row * pr if op.kind == "move_by" else p + (row - p) * pr
                kinematic = True
            elif op.kind == "spin":
                angle = math.radians(float(np.float32(op.angular_velocity))) * (min(time, op.t_end) - op.t_start)
                if angle <= 0.0:
                    continue
                p = _rodrigues(p, op.center, op.axis, angle)
                kinematic = True
            elif op.kind == "scale":
                if time < op.t_start:
                    continue
                if time >= op.t_end:
                    f = np.float32(op.factor)
                else:
                    f = np.float32(1.0 + (float(np.float32(op.factor)) - 1.0) * (op.progress_at(time) or 0.0))
                c = np.asarray(op.center, np.float32)
                p = (p - c) * f + c
                kinematic = True
        return p.astype(np.float32), kinematic


def read_pin_schedule(scene_dir: str) -> list:
    """Every pin block's schedule from info.toml's [pin-<i>] / [pin-<i>-op-<j>] tables and
    the op payloads pin-<i>-op-<j>.bin (golden.rs:1122-1200)."""
    blocks = read_pin_blocks(scene_dir)
    ip = os.path.join(scene_dir, "info.toml")
    info = open(ip, encoding="utf-8", errors="replace").read() if os.path.exists(ip) else ""
    ib = os.path.join(scene_dir, "input_bin")

    def num(sec, k, d):
        try:
            return float(sec[k])
        except (KeyError, ValueError):
            return d

    out = []
    for i, idx in enumerate(blocks):
        head = _toml_section(info, f"pin-{i}")
        ops = []
        for j in range(int(num(head, "operation_count", 0))):
            sec = _toml_section(info, f"pin-{i}-op-{j}")
            ty = sec.get("type", "")
            vec = tuple(float(np.float32(num(sec, f"center_{a}", 0.0))) for a in "xyz")
            axis = tuple(float(np.float32(num(sec, f"axis_{a}", 0.0))) for a in "xyz")
            path = os.path.join(ib, f"pin-{i}-op-{j}.bin")
            data = None
            if os.path.exists(path):
                data = decode_vec3_f64(_read(path)).astype(np.float32)
                if len(data) != len(idx):
                    raise CaptureError(f"pin-{i}-op-{j}.bin has {len(data)} rows but block {i} holds {len(idx)} vertices")
            tr = sec.get("transition")
            ops.append(PinOp(ty if ty in ("move_by", "move_to", "spin", "scale") else (ty or "unsupported"),
                             num(sec, "t_start", 0.0), num(sec, "t_end", 0.0),
                             tr if tr in ("smooth", "bezier") else "linear", vec, axis,
                             float(np.float32(num(sec, "angular_velocity", 0.0))),
                             float(np.float32(num(sec, "factor", 1.0))), data))
        out.append(PinBlockSchedule(idx, float(np.float32(num(head, "stiffness", 1.0))),
                                    float(np.float32(num(head, "pull", 0.0))), ops))
    return out


def read_stitches(scene_dir: str):
    """(index u32 (S, 6), weight f32 (S, 6), stiffness f32 (S,)) or empty arrays when the
    scene has no stitches (golden.rs:839-888); stiffness defaults to 1."""
    ib = os.path.join(scene_dir, "input_bin")
    ind_p = os.path.join(ib, "stitch_ind.bin")
    if not os.path.exists(ind_p):
        return np.zeros((0, 6), np.uint32), np.zeros((0, 6), np.float32), np.zeros(0, np.float32)
    raw = _read(ind_p)
    _aligned(raw, 48, "stitch_ind")
    idx = _narrow(np.frombuffer(raw, "<u8").reshape(-1, 6), "stitch")
    n = idx.shape[0]
    wraw = _read(os.path.join(ib, "stitch_w.bin"))
    _aligned(wraw, 24, "stitch_w")
    w = np.frombuffer(wraw, "<f4").reshape(-1, 6).copy()
    if w.shape[0] != n:
        raise CaptureError(f"stitch_w implies {w.shape[0]} stitches but stitch_ind implies {n}")
    st_p = os.path.join(ib, "stitch_stiffness.bin")
    if os.path.exists(st_p):
        sraw = _read(st_p)
        _aligned(sraw, 4, "stitch_stiffness")
        k = np.frombuffer(sraw, "<f4").copy()
        if k.size and k.size != n:
            raise CaptureError(f"stitch_stiffness has {k.size} entries but there are {n} stitches")
        if not k.size:
            k = np.ones(n, np.float32)
    else:
        k = np.ones(n, np.float32)
    return idx, w, k


def _f32_mean(path: str):
    if not os.path.exists(path):
        return None
    raw = _read(path)
    if not raw or len(raw) % 4:
        return None
    return float(np.frombuffer(raw, "<f4").astype(np.float64).mean())


def read_material(scene_dir: str):
    """Per-triangle material averaged to scalars (golden.rs:1254-1262): dict with
    young_mod, bend, density, strain_limit, or None without ``tri-young-mod.bin``."""
    p = os.path.join(scene_dir, "input_bin", "param")
    young = _f32_mean(os.path.join(p, "tri-young-mod.bin"))
    if young is None:
        return None
    bend = _f32_mean(os.path.join(p, "tri-bend.bin"))
    dens = _f32_mean(os.path.join(p, "tri-density.bin"))
    sl = _f32_mean(os.path.join(p, "tri-strain-limit.bin"))
    return {"young_mod": young, "bend": 0.0 if bend is None else bend, "density": 1.0 if dens is None else dens,
            "strain_limit": 0.0 if sl is None else sl}


def load_checkpoint(scene_dir: str, frame: int) -> np.ndarray:
    """Recorded positions of frame ``frame`` (frame 0 is the initial state)."""
    return decode_vec3_f32(_read(os.path.join(scene_dir, "checkpoints", f"vert_{frame}.bin")))


@dataclass
class GateReport:
    """Divergence from a checkpoint, each over the reference's bounding-box diagonal
    (golden.rs:1286-1304): worst vertex distance, RMS distance, centroid shift."""
    max_rel: float
    rms: float
    centroid_rel: float
    diagonal: float
    GATES = (8.0e-2, 2.0e-2, 6.0e-3)

    def passes(self) -> bool:
        return self.max_rel < self.GATES[0] and self.rms < self.GATES[1] and self.centroid_rel < self.GATES[2]


def compare_frames(ours, reference) -> GateReport:
    """Our positions against a checkpoint (golden.rs:1308-1371); a degenerate diagonal
    counts as 1 so the ratios stay finite."""
    a = np.asarray(ours, np.float64).reshape(-1, 3)
    b = np.asarray(reference, np.float64).reshape(-1, 3)
    if a.shape != b.shape:
        raise CaptureError(f"frame vertex count mismatch: ours {a.shape[0]} vs reference {b.shape[0]}")
    n = max(a.shape[0], 1)
    diag = float(np.linalg.norm(b.max(0) - b.min(0))) if b.size else 0.0
    diag = diag if diag > 1e-12 else 1.0
    d = np.linalg.norm(a - b, axis=1) if a.size else np.zeros(1)
    rms = float(np.sqrt((d * d).sum() / n))
    cen = float(np.linalg.norm((a.sum(0) - b.sum(0)) / n)) if a.size else 0.0
    return GateReport(float(d.max()) / diag, rms / diag, cen / diag, diag)


def scene_from_capture(scene_dir: str, poisson: float = 0.3, thickness: float = 5.0e-4, **params) -> dict:
    """A scene description for ``ImplicitSolver`` from a capture: the initial state,
    triangles as both contact and StVK membrane faces (Lamé parameters from the captured
    Young's modulus, ``poisson`` and ``thickness``), hinge stiffness from ``tri-bend``,
    uniform lumped mass from ``tri-density``, pinned vertices with zero inverse mass,
    stitches with ``l0`` the contact gap and ``l_cap = stitch_length_factor * l0`` (the
    reference driver's rule for uniform face gaps and zero contact offsets; per-face gap and
    offset arrays are not read), and ``dt``/gravity/CG limits from ``param.toml``. Keyword
    arguments override the resulting parameters (``contact_dhat`` also sets the stitches'
    gap)."""
    from . import scenes

    inp = load_capture_input(scene_dir)
    pos, tris = inp["positions"], inp["tris"]
    nv = pos.shape[0]
    prm = read_param_toml(scene_dir) if os.path.exists(os.path.join(scene_dir, "param.toml")) else dict(_PARAM_DEFAULTS)
    mat = read_material(scene_dir)
    if mat is not None and tris.size:
        mu, lam = scenes.lame_from_young_poisson(mat["young_mod"] * thickness, poisson)
        mass = scenes.uniform_mass(pos, tris, mat["density"])
        bend = mat["bend"]
    else:
        mu = lam = 0.0
        mass = 1.0
        bend = 0.0
    im = np.full(nv, 1.0 / mass, np.float32)
    pins = read_pin_indices(scene_dir)
    if pins.size and int(pins.max()) >= nv:
        raise CaptureError(f"a pin references a vertex >= {nv}")
    im[pins] = 0.0
    si, sw, sk = read_stitches(scene_dir)
    if si.size and int(si.max()) >= nv:
        raise CaptureError(f"a stitch references a vertex >= {nv}")
    gap = float(params.get("contact_dhat", 1.0e-3))
    kl = np.stack([sk, np.full_like(sk, gap), np.full_like(sk, gap * prm["stitch_length_factor"])], 1) \
        if sk.size else np.zeros((0, 3), np.float32)
    p = scenes.default_params(dt=float(prm["dt"]), gravity=tuple(float(g) for g in prm["gravity"]),
                              shell_mu=mu, shell_lambda=lam, bend_stiffness=bend, cg_tol=float(prm["cg_tol"]),
                              cg_max_iter=int(prm["cg_max_iter"]), ccd_max_iter=int(prm["ccd_max_iter"]),
                              friction_eps=float(prm["friction_eps"]), barrier_kind=1 if prm["cubic_barrier"] else 0,
                              self_collision=0 if prm["disable_contact"] else 1)
    p.update(params)
    return {"positions": pos, "velocities": inp["velocities"], "inv_mass": im, "tris": tris,
            "shell_faces": tris.copy(), "static_mask": None, "stitch_idx": si.astype(np.uint32),
            "stitch_w": sw.astype(np.float32), "stitch_kl": kl.astype(np.float32),
            "colliders": np.zeros((0, 8), np.float32), "params": p, "name": os.path.basename(scene_dir.rstrip("/"))}


def write_obj(path: str, positions, tris=None) -> None:
    """One frame as Wavefront OBJ: ``v x y z`` per vertex (9 significant digits, enough to
    read back every float32 exactly) and ``f a b c`` (1-based) per triangle."""
    p = np.asarray(positions, np.float32).reshape(-1, 3)
    with open(path, "w") as f:
        f.write(f"# {p.shape[0]} vertices\n")
        np.savetxt(f, p, fmt="v %.9g %.9g %.9g")
        if tris is not None and len(tris):
            t = np.asarray(tris, np.int64).reshape(-1, 3) + 1
            np.savetxt(f, t, fmt="f %d %d %d")


def parse_obj(text: str, with_uvs: bool = False):
    """(positions float32 (n, 3), triangles uint32 (m, 3)[, per-vertex uvs float32 (n, 2) or
    empty]) from Wavefront OBJ text (engine-io obj.rs): polygons are fan-triangulated,
    ``f a/b/c`` forms read the vertex (and texture) index, negative indices count back from
    the records read so far, and an index out of range is a CaptureError. UVs are kept only
    when every face corner names one (parallel or empty), a missing ``vt`` v reads as 0."""
    v, vt, fcs, fuv = [], [], [], []
    all_uv = True

    def num(tok, what, lineno):
        try:
            return float(tok)
        except ValueError:
            raise CaptureError(f"bad {what} on line {lineno}") from None

    def index(tok, what, lineno):
        try:
            return int(tok)
        except ValueError:
            raise CaptureError(f"bad {what} index {tok!r} on line {lineno}") from None

    for lineno, line in enumerate(text.splitlines(), 1):
        # '#' starts a comment anywhere on the line (obj.rs:103-107)
        s = line.split("#", 1)[0].split()
        if not s:
            continue
        if s[0] == "v":
            if len(s) < 4:
                raise CaptureError(f"vertex needs 3 coords on line {lineno}")
            v.append([num(x, "vertex", lineno) for x in s[1:4]])
        elif s[0] == "vt":
            if len(s) < 2:
                raise CaptureError(f"vt needs >=1 coord on line {lineno}")
            vt.append([num(s[1], "texcoord", lineno), num(s[2], "texcoord", lineno) if len(s) > 2 else 0.0])
        elif s[0] == "f":
            if len(s) < 4:
                raise CaptureError(f"face needs >=3 verts on line {lineno}")
            ids, uvs = [], []
            for tok in s[1:]:
                parts = tok.split("/")
                i = index(parts[0], "vertex", lineno)
                i = i - 1 if i > 0 else len(v) + i
                if not 0 <= i < len(v):
                    raise CaptureError(f"face index {parts[0]} is outside the {len(v)} vertices")
                ids.append(i)
                if len(parts) > 1 and parts[1]:
                    j = index(parts[1], "texture", lineno)
                    j = j - 1 if j > 0 else len(vt) + j
                    if not 0 <= j < len(vt):
                        raise CaptureError(f"texture index {parts[1]} is outside the {len(vt)} uvs")
                    uvs.append(j)
                else:
                    all_uv = False
            for k in range(1, len(ids) - 1):  # fan-triangulate polygons
                fcs.append([ids[0], ids[k], ids[k + 1]])
                if len(uvs) == len(ids):
                    fuv.append([uvs[0], uvs[k], uvs[k + 1]])
    if not v:
        raise CaptureError("OBJ contained no vertices")
    pos = np.asarray(v, np.float32).reshape(-1, 3)
    tris = np.asarray(fcs, np.uint32).reshape(-1, 3)
    if not with_uvs:
        return pos, tris
    uv = np.zeros((0, 2), np.float32)
    if all_uv and fcs and vt:
        uv = np.zeros((len(v), 2), np.float32)
        for t, tu in zip(fcs, fuv):
            for a, b in zip(t, tu):
                uv[a] = vt[b]
    return pos, tris, uv


def read_obj(path: str):
    """(positions float32 (n, 3), triangles uint32 (m, 3)) of an OBJ file (see parse_obj)."""
    with open(path) as f:
        return parse_obj(f.read())
