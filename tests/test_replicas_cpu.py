"""Replica bookkeeping across processes (CPU, gloo, world size 2): the N-GPU
benchmark runs independent replicas whose step time is the slowest rank's
and whose seed-parallel work is split by `replicas.shard`."""
import json
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from hpsint_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, size, port, out_dir):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(size), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=size, timeout=datetime.timedelta(seconds=60))
    try:
        w = replicas.from_env()
        res = {
            "world": [w.rank, w.size, w.local_rank],
            "shard": replicas.shard(range(10), w.rank, w.size),
            "max": replicas.max_over_ranks(1.5 + rank, dist),
            "sum": replicas.sum_over_ranks(1.0 + rank, dist),
            "gather": replicas.gather({"rank": rank, "seeds": replicas.shard(range(5), rank, size)}, dist),
        }
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump(res, f)
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    size, port = 2, _free_port()
    mp.spawn(_rank_main, args=(size, port, str(tmp_path)), nprocs=size, join=True)
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(size)]
    assert res[0]["world"] == [0, 2, 0] and res[1]["world"] == [1, 2, 1]
    # every item on exactly one rank
    assert sorted(res[0]["shard"] + res[1]["shard"]) == list(range(10))
    assert res[0]["shard"] == [0, 2, 4, 6, 8]
    # the slowest rank's time, on every rank
    assert res[0]["max"] == res[1]["max"] == 2.5
    assert res[0]["sum"] == res[1]["sum"] == 3.0
    for r in res:
        assert r["gather"] == [{"rank": 0, "seeds": [0, 2, 4]}, {"rank": 1, "seeds": [1, 3]}]


def test_single_process_needs_no_group():
    assert replicas.max_over_ranks(3.0) == 3.0
    assert replicas.gather(7) == [7]
    assert replicas.shard("abc", 0, 1) == ["a", "b", "c"]
    with pytest.raises(ValueError):
        replicas.shard(range(3), 2, 2)
