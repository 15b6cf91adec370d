"""Host logic of the multi-GPU bench: independent replicas, max over ranks.

Two gloo ranks on the CPU stand in for two GPUs: each replica draws its own
load seeds, the timed region is reduced with MAX, and the reference arm runs
on rank 0 only.
"""
import json
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    res = {"seeds": bench.replica_seeds(rank),
           "max": bench.reduce_max(1.5 * (rank + 1), dist, "cpu")}
    if rank != 0:
        # the reference arm prints and runs nothing off rank 0
        res["ref_arm"] = bench.reference_arm(bench.parse_args([]))
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump(res, f)


@pytest.mark.timeout(120)
def test_two_replicas_gloo(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    r = [json.load(open(tmp_path / f"r{i}.json")) for i in range(world)]
    assert r[0]["max"] == r[1]["max"] == 3.0
    assert r[0]["seeds"] != r[1]["seeds"]
    assert r[1]["ref_arm"] == 0
