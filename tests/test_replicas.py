"""Multi-rank host logic on CPU: region shards and the max-over-ranks timing reduction, run as two
gloo ranks (the same code runs over NCCL, one process per GPU)."""
import json
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_shard_covers_every_region_once_and_balances():
    import __graft_entry__ as ge

    ge.load_package()
    from vfwater import replicas

    w = [5, 1, 9, 3, 3, 7, 2, 8, 4, 6]
    for world in (1, 2, 3, 4):
        parts = [replicas.shard(w, r, world) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(w)))
        loads = [sum(w[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(w)
    with pytest.raises(ValueError):
        replicas.shard(w, 2, 2)


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    from datetime import timedelta

    import torch.distributed as dist

    import __graft_entry__ as ge

    ge.load_package()
    from vfwater import replicas

    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    try:
        mine = replicas.shard([10, 20, 30, 40, 50], rank, world)
        ms, cells = replicas.reduce_rate(100.0 + 50.0 * rank, 1000.0 * (rank + 1))
        dist.barrier()
    finally:
        dist.destroy_process_group()
    Path(out_dir, f"r{rank}.json").write_text(json.dumps({"mine": mine, "ms": ms, "cells": cells}))


def test_two_gloo_ranks_shard_and_reduce(tmp_path):
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r = [json.loads((tmp_path / f"r{k}.json").read_text()) for k in range(2)]
    assert sorted(r[0]["mine"] + r[1]["mine"]) == list(range(5))
    assert not set(r[0]["mine"]) & set(r[1]["mine"])
    for x in r:
        assert x["ms"] == 150.0  # the slowest rank's time
        assert x["cells"] == 3000.0  # every rank's cell-steps
