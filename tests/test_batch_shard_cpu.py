"""Multi-rank plumbing of the batched workload, on CPU with gloo.

The 64 scenes are independent, so N ranks split them with no per-step
exchange: every rank computes the same greedy partition, steps its share, and
the ranks only meet for the max of their timings.  Here two gloo ranks check
that the partition is identical on every rank, covers every scene exactly
once and is balanced, and that the max-over-ranks reduction the benchmark
uses returns the slowest rank's time.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, sizes, out_dir):
    import torch

    from pbf_b200.batch import partition_scenes
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    parts = partition_scenes(sizes, world)
    mine = parts[rank]
    load = torch.tensor([float(sum(sizes[k] for k in mine))], dtype=torch.float64)
    gathered = [torch.zeros(64, dtype=torch.int64) - 1 for _ in range(world)]
    t = torch.full((64,), -1, dtype=torch.int64)
    t[:len(mine)] = torch.tensor(mine, dtype=torch.int64)
    dist.all_gather(gathered, t)
    fake_ms = torch.tensor([10.0 + rank], dtype=torch.float64)  # rank 1 is the slow one
    dist.all_reduce(fake_ms, op=dist.ReduceOp.MAX)
    dist.all_reduce(load, op=dist.ReduceOp.MAX)
    np.save(os.path.join(out_dir, f"r{rank}.npy"),
            np.concatenate([g.numpy() for g in gathered] + [fake_ms.numpy().astype(np.int64),
                                                            load.numpy().astype(np.int64)]))
    dist.barrier()
    dist.destroy_process_group()


def test_partition_is_rank_consistent_complete_and_balanced(tmp_path):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "realtime-fsi-engine_b200"))
    from pbf_b200.scenes import c3_sizes
    sizes = [int(v) for v in c3_sizes()]
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), sizes, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    res = [np.load(tmp_path / f"r{r}.npy") for r in range(world)]
    assert np.array_equal(res[0], res[1])  # every rank saw the same gathered partition
    lists = [res[0][64 * r:64 * (r + 1)] for r in range(world)]
    scenes = sorted(int(k) for l in lists for k in l if k >= 0)
    assert scenes == list(range(64))
    loads = [sum(sizes[int(k)] for k in l if k >= 0) for l in lists]
    assert max(loads) - min(loads) <= max(sizes)  # greedy: within one scene of even
    assert res[0][128] == 11  # max over ranks of (10 + rank)
    assert res[0][129] == max(loads)


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition_properties(world):
    from pbf_b200.batch import partition_scenes
    rng = np.random.default_rng(world)
    sizes = rng.integers(4096, 131073, size=64)
    parts = partition_scenes(sizes, world)
    assert sorted(k for p in parts for k in p) == list(range(64))
    loads = [int(sum(int(sizes[k]) for k in p)) for p in parts]
    assert max(loads) - min(loads) <= int(sizes.max())
    assert parts == partition_scenes(sizes, world)
