"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (the replicas path), and the
reference arm under torchrun (rank 0 alone prints, the other rank exits 0 without work)."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parent.parent


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, str(REPO))
    import bench
    d = bench.Dist()
    d.init("gloo")
    d.barrier()
    # rank r moved (r + 1) GB in (r + 2) s: total 3 GB, slowest 3 s
    total, slowest = bench.aggregate_replicas((rank + 1) * 1e9, rank + 2.0, d)
    Path(out_dir, f"r{rank}.json").write_text(json.dumps({"total": total, "slowest": slowest}))
    d.close()


def test_replica_aggregation_two_gloo_ranks(tmp_path):
    port = free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    for r in range(2):
        got = json.loads((tmp_path / f"r{r}.json").read_text())
        assert got == {"total": 3e9, "slowest": 3.0}


def test_reference_arm_under_torchrun_prints_one_line():
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "1", "--scale", "0.004"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    p = subprocess.run(cmd, cwd=REPO, capture_output=True, text=True, timeout=600, env=env)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(x) for x in p.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["cores"] == 1
