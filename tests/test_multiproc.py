"""The N>1 launch path on the CPU: two ranks over gloo (127.0.0.1).

bench.py runs one process per GPU as independent replicas (no collective on
the data path): a barrier around the timed region and the max of the ranks'
times.  These tests run that plumbing with two CPU processes, and the
reference arm under torchrun (rank 0 alone measures and prints one line;
the other rank exits 0 without work)."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.join(os.path.dirname(__file__), "..")


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist(world)
    d.barrier()
    m = d.max(float(10 * (rank + 1)))
    d.barrier()
    d.close()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"rank": d.rank, "world": d.world, "max": m}, f)


def test_dist_barrier_and_max_over_two_gloo_ranks(tmp_path):
    port = free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    got = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    assert [g["rank"] for g in got] == [0, 1]
    assert all(g["world"] == 2 and g["max"] == 20.0 for g in got)


def test_reference_arm_under_torchrun_two_ranks(tmp_path):
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--workload", "c2cc", "--steps", "1", "--warmup", "0", "--scale", "10"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["cpu_baseline"]["cores"] == len(os.sched_getaffinity(0))  # not torchrun's 1
