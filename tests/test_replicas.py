"""CPU: the multi-GPU bench path. Each rank (one per GPU under torchrun) runs
its own replica of the workload; the only collectives are the barriers around
a timed region and the maximum over ranks of each measured time, and the
reported rate is every rank's units over the slowest rank's time. Checked here
with two gloo ranks on the host (the same calls run over NCCL on GPUs)."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = """
import json, sys
sys.path.insert(0, {root!r})
import bench
reps = bench.Replicas("gloo", device="cpu", timeout_s=60)
mine = 1.0 + 2.0 * reps.rank  # rank 1 is the slower one
reps.barrier()
slowest = reps.max(mine)
print(json.dumps({{"rank": reps.rank, "world": reps.world, "mine": mine, "max": slowest,
                  "rate": bench.whole_job_rate(1000, reps.world, slowest)}}))
reps.close()
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank: int, world: int, port: int) -> dict:
    env = dict(os.environ)
    env.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(port))
    return env


def test_two_gloo_ranks_take_the_slowest_time():
    port = _free_port()
    procs = [subprocess.Popen([sys.executable, "-c", RANK_SCRIPT.format(root=ROOT)], env=_env(r, 2, port),
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True) for r in range(2)]
    outs = [p.communicate(timeout=180) for p in procs]
    for p, (_, err) in zip(procs, outs):
        assert p.returncode == 0, err[-2000:]
    lines = [json.loads(out.strip().splitlines()[-1]) for out, _ in outs]
    assert sorted(line["rank"] for line in lines) == [0, 1]
    for line in lines:
        assert line["world"] == 2
        assert line["max"] == 3.0  # every rank sees the slowest rank's time
        assert line["rate"] == 1000 * 2 / 3.0


def test_one_rank_needs_no_process_group():
    env = _env(0, 1, _free_port())
    out = subprocess.run([sys.executable, "-c", RANK_SCRIPT.format(root=ROOT)], env=env, capture_output=True,
                         text=True, timeout=120)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["max"] == line["mine"] == 1.0 and line["rate"] == 1000.0


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun the reference arm is timed by rank 0; the other ranks
    exit 0 without work or output."""
    env = _env(1, 2, _free_port())
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.strip() == ""
