"""The multi-GPU path's host logic on CPU: two gloo ranks.

bench.py runs one process per GPU with independent replicas (the Markov chain does not shard:
no collective on the data path).  The only cross-rank steps are the max over ranks of the timed
region and rank 0 printing the line; here they run as two gloo ranks on 127.0.0.1, and the
reference arm runs under torchrun with two ranks (rank 0 works, rank 1 exits 0)."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(WORLD_SIZE="2", RANK=str(rank), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", world_size=2, rank=rank,
                            timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, ROOT)
    import bench
    got = bench.max_over_ranks(1.5 + rank, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out, f"r{rank}"), "w") as f:
        f.write(repr(got))


def test_max_over_ranks_two_gloo_ranks(tmp_path):
    mp.spawn(_rank_main, args=(_free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        assert float(open(tmp_path / f"r{r}").read()) == 2.5


def test_replica_seeds_distinct():
    sys.path.insert(0, ROOT)
    import bench
    seeds = [bench.replica_seeds(rank, r) for rank in range(8) for r in range(148)]
    assert len(set(s[0] for s in seeds)) == len(seeds)
    assert len(set(s[1] for s in seeds)) == len(seeds)


def test_reference_arm_under_torchrun():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--ref-moves", "20",
           "--workload", "spce256"]
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [l for l in res.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port"
