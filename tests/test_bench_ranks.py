"""Host logic of bench.py's multi-GPU run (independent replicas, one process per
GPU) on the CPU: two `gloo` ranks launched as separate processes agree on the
whole-job figure, i.e. the slowest rank's seconds and the sum of the ranks' pair
counts, and a single process passes its own figures through unchanged."""
import os
import socket
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

RANK_SCRIPT = r"""
import datetime, json, os, sys
sys.path.insert(0, os.getcwd())
import torch.distributed as dist
import bench
rank, world, local = bench.dist_env()
dist.init_process_group("gloo", rank=rank, world_size=world,
                        timeout=datetime.timedelta(seconds=60))
sec, cnt = bench.whole_job(1.5 + rank, 100 * (rank + 1), world, device="cpu")
dist.barrier()
dist.destroy_process_group()
print(json.dumps({"rank": rank, "world": world, "local": local, "sec": sec, "cnt": cnt}))
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_whole_job_over_two_gloo_ranks():
    import json
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_SCRIPT], cwd=ROOT, env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    try:
        for p in procs:
            out, err = p.communicate(timeout=180)
            assert p.returncode == 0, err[-2000:]
            outs.append(json.loads(out.strip().splitlines()[-1]))
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    assert sorted(o["rank"] for o in outs) == [0, 1]
    for o in outs:
        assert o["world"] == 2 and o["local"] == o["rank"]
        assert o["sec"] == 2.5 and o["cnt"] == 300, o


def test_whole_job_single_process_is_identity():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.whole_job(0.75, 256, 1) == (0.75, 256)
