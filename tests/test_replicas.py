"""The bench's N>1 path on CPU: two torchrun ranks over gloo on 127.0.0.1.

The path shards as replicas (every rank encodes its own frame; no collective on
the data path), so what crosses ranks is only the barrier around the timed
region, the max-over-ranks step time and the rank-0-only JSON line.  The
worker drives ``bench.Replicas`` exactly as ``bench.run_ours`` does, with a
host-side stand-in for the device step whose duration differs per rank."""
import json
import os
import socket
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = textwrap.dedent(
    """
    import json, os, sys, time
    sys.path.insert(0, {root!r})
    import bench

    ranks = bench.Replicas("gloo", timeout_s=30)
    assert ranks.world == int(os.environ["WORLD_SIZE"]) and ranks.rank == int(os.environ["RANK"])
    ranks.barrier()
    local_ms = 10.0 + 5.0 * ranks.rank  # rank r's step: 10 + 5 r ms
    step_ms = ranks.max(local_ms)
    ranks.emit({{"rank": ranks.rank, "step_ms": step_ms, "value": ranks.job_value(step_ms)}})
    with open(os.path.join({out!r}, "rank%d.json" % ranks.rank), "w") as f:
        json.dump({{"local_ms": local_ms, "step_ms": step_ms, "value": ranks.job_value(step_ms)}}, f)
    ranks.close()
    """
)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def torchrun(script, nproc, timeout=120):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={nproc}",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), script]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    return subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, env=env, cwd=ROOT)


def test_two_rank_max_over_ranks_and_rank0_line(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(WORKER.format(root=ROOT, out=str(tmp_path)))
    r = torchrun(str(script), 2)
    assert r.returncode == 0, r.stderr[-2000:]
    per_rank = [json.load(open(tmp_path / f"rank{i}.json")) for i in range(2)]
    # every rank reports the slowest rank's step
    assert [p["local_ms"] for p in per_rank] == [10.0, 15.0]
    assert all(p["step_ms"] == 15.0 for p in per_rank)
    # whole-job throughput: both ranks' frames over the slowest step
    import bench

    want = 2 * bench.MPIX / 0.015
    assert all(abs(p["value"] - want) < 1e-9 * want for p in per_rank)
    # exactly one JSON line on stdout, from rank 0
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1 and lines[0]["rank"] == 0 and lines[0]["step_ms"] == 15.0


def test_single_process_needs_no_group():
    import bench

    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK") if k in os.environ}
    try:
        ranks = bench.Replicas("gloo")
        assert ranks.world == 1 and ranks.dist is None
        assert ranks.max(3.5) == 3.5
        assert ranks.job_value(2.0) == pytest.approx(bench.MPIX / 0.002)
        ranks.barrier()
        ranks.close()
    finally:
        os.environ.update(env)


def test_reference_arm_nonzero_rank_exits_quietly():
    """Under torchrun only rank 0 times the reference; the others exit 0 without work."""
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "0"], capture_output=True, text=True, timeout=120, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
