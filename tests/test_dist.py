"""The benchmark's multi-process plumbing on CPU: two ranks over gloo (barrier and the
max-over-ranks timing reduction), and the reference arm's rank handling under a launcher
(rank 0 prints one JSON line, other ranks exit 0 without work)."""
import json
import os
import socket
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

RANK_SCRIPT = r"""
import os, sys
sys.path.insert(0, {root!r})
import bench
d = bench.Dist("gloo")
d.barrier()
m = d.max(1.5 + d.rank)
d.barrier()
print("rank", d.rank, "world", d.world, "max", m, flush=True)
d.close()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_agree_on_the_max_over_ranks():
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_SCRIPT.format(root=ROOT)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=120) for p in procs]
    for p, (out, err) in zip(procs, outs):
        assert p.returncode == 0, err[-2000:]
    lines = sorted(o.strip().splitlines()[-1] for o, _ in outs)
    assert lines == ["rank 0 world 2 max 2.5", "rank 1 world 2 max 2.5"]


def test_the_reference_arm_runs_on_rank_zero_only():
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "spmv",
           "--steps", "1", "--warmup", "3", "--cpu-seconds", "1"]
    other = subprocess.run(cmd, env=dict(os.environ, RANK="1", WORLD_SIZE="2"), capture_output=True, text=True,
                           timeout=300)
    assert other.returncode == 0 and other.stdout.strip() == ""
    zero = subprocess.run(cmd, env=dict(os.environ, RANK="0", WORLD_SIZE="2"), capture_output=True, text=True,
                          timeout=300)
    assert zero.returncode == 0, zero.stderr[-2000:]
    line = json.loads(zero.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
