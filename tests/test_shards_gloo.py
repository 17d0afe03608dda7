"""The multi-rank path on CPU: two gloo ranks shard the worlds (weak
scaling, a seed per rank), meet at barriers, and agree on the slowest
rank's time and the whole-job throughput; under torchrun the reference arm
runs on rank 0 only."""

import json
import os
import socket
import types

import pytest
import torch
import torch.multiprocessing as mp

from sap_warp_b200.shards import RankGroup, job_throughput, shard_of


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world_size, port, out_dir):
    import torch.distributed as dist

    from sap_warp_b200 import models

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world_size,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        group = RankGroup(dist, torch.device("cpu"))
        shard = shard_of(rank, world_size, 4, 2)
        _, state, _, contacts, _, _ = models.box_scene(shard.worlds, shard.seed, torch.device("cpu"), boxes=4,
                                                       sites=(2, 3))
        group.barrier()
        ms_local = 2.0 + rank  # rank 1 is the slow one
        ms_max = group.max_over_ranks(ms_local)
        worlds_total = group.sum_over_ranks(shard.worlds)
        res = dict(rank=rank, first=shard.first_world, seed=shard.seed, ms_max=ms_max, worlds_total=worlds_total,
                   value=job_throughput(shard.worlds, world_size, ms_max),
                   q_sum=float(state.joint_q.double().sum()), contacts=int(contacts.rigid_contact_count.item()))
        group.barrier()
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump(res, f)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_time(tmp_path):
    mp.spawn(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    r = [json.loads((tmp_path / f"rank{k}.json").read_text()) for k in range(2)]
    assert (r[0]["first"], r[1]["first"]) == (0, 4)  # disjoint world ranges
    assert r[0]["seed"] != r[1]["seed"] and r[0]["q_sum"] != r[1]["q_sum"]  # each rank its own scene
    assert r[0]["ms_max"] == r[1]["ms_max"] == 3.0  # the slowest rank's time on every rank
    assert r[0]["worlds_total"] == r[1]["worlds_total"] == 8.0
    assert r[0]["value"] == r[1]["value"] == pytest.approx(8 / 3.0e-3)


def test_shards_are_weak_scaling_and_checked():
    s = [shard_of(k, 4, 4096, 2) for k in range(4)]
    assert [x.first_world for x in s] == [0, 4096, 8192, 12288]
    assert len({x.seed for x in s}) == 4
    with pytest.raises(ValueError):
        shard_of(4, 4, 4096, 2)
    with pytest.raises(ValueError):
        job_throughput(4096, 1, 0.0)
    one = RankGroup()  # no process group: one rank
    assert one.max_over_ranks(1.5) == 1.5 and one.sum_over_ranks(3) == 3.0


def test_reference_arm_runs_on_rank_zero_only(capsys):
    import bench

    args = types.SimpleNamespace(gpus=2, steps=1, warmup=0)
    bench.run_reference(args, rank=1, world_size=2)
    assert capsys.readouterr().out == ""
