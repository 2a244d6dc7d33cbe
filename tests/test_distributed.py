"""The multi-rank host logic of bench.py on CPU with the gloo backend
(world size 2): config-5 scene sharding is identical on every rank and
balanced, and the batch numbers are the max (time) / sum (DOF) / gather
(latencies) over ranks; replica timings take the slowest rank."""
from __future__ import annotations

import os
import socket

import pytest

torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, costs, out_dir):
    import json
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    parts = bench.shard_by_cost(costs, world)
    mine = parts[rank]
    total_ms = float(sum(costs[k] for k in mine))   # stand-in device time of this rank's scenes
    dofs = 3 * len(mine)
    lat = [float(costs[k]) for k in mine]
    wall, dsum, lat_all = bench.reduce_batch_timings(total_ms, dofs, lat, torch.device("cpu"))
    slowest = bench.max_over_ranks(10.0 + rank, torch.device("cpu"))
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump(dict(parts=parts, wall=wall, dofs=dsum, lat=sorted(lat_all), slowest=slowest), f)
    dist.barrier()
    dist.destroy_process_group()


def test_sharding_and_reductions_two_ranks(tmp_path):
    import json
    import torch.multiprocessing as mp
    costs = [50, 7, 30, 30, 1, 12, 99, 3, 8, 20]
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), costs, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    r = [json.load(open(tmp_path / f"r{k}.json")) for k in range(world)]
    assert r[0]["parts"] == r[1]["parts"]                       # same assignment everywhere
    parts = r[0]["parts"]
    assert sorted(k for p in parts for k in p) == list(range(len(costs)))
    loads = [sum(costs[k] for k in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)               # greedy balance bound
    for q in r:
        assert q["wall"] == max(loads)
        assert q["dofs"] == 3 * len(costs)
        assert q["lat"] == sorted(float(c) for c in costs)
        assert q["slowest"] == 11.0
