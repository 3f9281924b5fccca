"""The N > 1 path of bench.py (replicas: one independent solve per rank, device time as the max over
ranks), on the CPU with two gloo ranks."""
import json
import os

import pytest
import torch.multiprocessing as mp

from rayleighchebyshevgpgpu_b200 import replicas


def _rank_main(rank: int, world: int, out_dir: str):
    import datetime

    import torch.distributed as dist

    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank))
    env = replicas.rank_env()
    # rendezvous through a file in the test's directory: no ports to collide
    dist.init_process_group("gloo", init_method="file://" + os.path.join(out_dir, "store"), rank=env.rank,
                            world_size=env.world, timeout=datetime.timedelta(seconds=60))
    try:
        # each rank's own device time; the slowest sets the job's time
        mine = 1.5 + env.rank
        slowest = replicas.max_over_ranks(mine, env.world, device="cpu")
        again = replicas.max_over_ranks(0.25 * (env.rank + 1), env.world, device="cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"env": [env.world, env.rank, env.local], "slowest": slowest, "again": again,
                   "rate": replicas.job_rate(64, env.world, slowest)}, f)


def test_single_process_defaults(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    env = replicas.rank_env()
    assert (env.world, env.rank, env.local) == (1, 0, 0)
    assert replicas.max_over_ranks(3.5, 1) == 3.5  # no process group needed
    assert replicas.job_rate(64, 1, 1.6) == pytest.approx(40.0)


def test_two_gloo_ranks_take_the_slowest_time(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    rows = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r, d in enumerate(rows):
        assert d["env"] == [world, r, r]
        assert d["slowest"] == 2.5          # the max of 1.5 and 2.5, on every rank
        assert d["again"] == 0.5            # a second reduction in the same order
        assert d["rate"] == pytest.approx(64 * world / 2.5)
