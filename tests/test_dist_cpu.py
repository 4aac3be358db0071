"""bench.py's multi-process path on CPU (gloo, two ranks on 127.0.0.1): the
max-over-ranks timing and barriers, and the reference arm under
torch.distributed.run, where rank 0 alone measures and prints one line."""
import json
import os
import socket
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def torchrun(*args, timeout=600):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), *args]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    return subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, cwd=ROOT, env=env)


def test_rank_plumbing_two_ranks_gloo():
    r = torchrun(os.path.join(HERE, "dist_probe.py"))
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.count("dist-ok") == 1


def test_reference_arm_under_torchrun_prints_one_line():
    r = torchrun("bench.py", "--impl", "reference", "--gpus", "2", "--steps", "2", "--warmup", "1")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["n_gpus"] == 2
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["cores"] >= 1
