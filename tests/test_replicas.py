"""The multi-GPU path is "replicas only": bench.py --gpus N runs N independent
replicas, one process per GPU, with no collective on the data path; the only
collectives are the timing barrier and the max over ranks.  These tests run
that plumbing as world-size-2 gloo process groups on the CPU."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench

    w, r, _ = bench.dist_setup(world)
    bench.barrier(w)
    t = bench.max_over_ranks(1.0 + 2.0 * r, w)  # per-rank "times" 1 s and 3 s
    bench.barrier(w)
    with open(out + f".{r}", "w") as f:
        json.dump({"rank": r, "world": w, "max": t, "backend": dist.get_backend()}, f)
    dist.destroy_process_group()


def test_timing_is_max_over_ranks_on_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    out = str(tmp_path / "rank")
    mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    res = [json.load(open(out + f".{r}")) for r in range(2)]
    assert [x["rank"] for x in res] == [0, 1]
    assert all(x["world"] == 2 and x["backend"] == "gloo" for x in res)
    # every rank sees the slowest rank's time, so value = all ranks' units / max time
    assert all(x["max"] == 3.0 for x in res)


@pytest.mark.timeout(300)
def test_reference_arm_prints_one_line_from_rank_zero_under_torchrun():
    """bench.py --impl reference launched as the driver launches it for N=2:
    rank 0 alone times the CPU backprojector and prints; rank 1 exits 0."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "0"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    p = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=280)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
