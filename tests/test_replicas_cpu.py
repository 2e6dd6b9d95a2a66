"""The N>1 path of bench.py on CPU: two replica ranks over gloo (one process
per rank, as torchrun launches them).  Each rank times its own independent
replica; the job's time is the slowest rank's (max over ranks) and its value
is the sum of the replicas' bytes over that time.  No data-path collective
exists: the only exchange is that timing scalar."""
import json
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out: str):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_setup("gloo")
    # each replica has its own seeded gauge field (bench uses SEED + rank)
    import iroiro_b200 as ib
    u = ib.synth_gauge([4, 4, 4, 4], bench.EPS, bench.SEED + r, gauge_transform=True)
    t_ms = 10.0 * (r + 1)  # rank 1 is the slower replica
    value = bench.replica_value(1e9, 100, t_ms, w)
    t_max = bench.reduce_max(t_ms, w)
    bench.barrier(w)
    Path(out, f"rank{r}.json").write_text(json.dumps(
        {"world": w, "value": value, "t_max": t_max, "u0": float(u[0])}))
    dist.destroy_process_group()


def test_two_replicas_gloo(tmp_path):
    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    res = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for d in res:
        assert d["world"] == world
        assert d["t_max"] == pytest.approx(20.0)
        # 2 replicas x 1 GB x 100 steps in the slowest rank's 20 ms
        assert d["value"] == pytest.approx(2 * 1e9 * 100 / 0.020 / 1e9)
    assert res[0]["u0"] != res[1]["u0"]  # independent replicas
