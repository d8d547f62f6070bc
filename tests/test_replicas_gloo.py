"""The multi-GPU mode is N independent replicas. Two gloo ranks on CPU run the replica bookkeeping
of bench.py (disjoint seeds, per-rank detection, max-over-ranks time) with the CPU oracle standing in
for the device, and the union of their results must equal one process doing all frames."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from compactcnncascade_b200.replicas import job_throughput, rank_seeds, reduce_max, shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import time
    import compactcnncascade_b200 as ccnn
    from oracle import oracle as orc
    seeds = rank_seeds(rank, 2, stride=1000)
    t0 = time.perf_counter()
    res = {}
    for s in seeds:
        img, _ = ccnn.synth_frame(320, 240, s, 3, 40, 100)
        res[s] = orc.detect(img, orc.params(max_w=320, max_h=240))["final"]
    t = time.perf_counter() - t0
    tmax = reduce_max(t, dist)
    gathered = [None] * world
    dist.all_gather_object(gathered, res)
    if rank == 0:
        q.put((gathered, tmax, t))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas_cover_the_stream():
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, tmax, t0 = q.get()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    import compactcnncascade_b200 as ccnn
    from oracle import oracle as orc
    merged = {k: v for part in gathered for k, v in part.items()}
    assert sorted(merged) == sorted(rank_seeds(0, 2, 1000) + rank_seeds(1, 2, 1000))
    for s, faces in merged.items():
        img, _ = ccnn.synth_frame(320, 240, s, 3, 40, 100)
        assert faces == orc.detect(img, orc.params(max_w=320, max_h=240))["final"]
    assert tmax >= t0 > 0


def test_replica_helpers():
    assert shard(list(range(10)), 1, 3) == [1, 4, 7]
    assert set(rank_seeds(0, 5)).isdisjoint(rank_seeds(1, 5))
    assert job_throughput([10, 10], [1.0, 2.0]) == pytest.approx(10.0)
