"""Host logic of the serving loop: request stream, sharding, merging (CPU).

The multi-rank path is exercised with world_size 2 over gloo on 127.0.0.1:
each rank takes its shard of the request stream and the per-rank completions
are gathered on rank 0, which must see every request exactly once.
"""
import os
import socket

import numpy as np
import pytest

from rheon_b200 import serving as S


def test_request_stream_follows_the_workload_definition():
    reqs = S.make_requests(2000, rate_hz=50.0, seed=5)
    edges = np.array([r.edge for r in reqs])
    steps = np.array([r.steps for r in reqs])
    arrivals = np.array([r.arrival for r in reqs])
    assert np.all(edges % 8 == 0) and edges.min() >= 32 and edges.max() <= 256
    assert steps.min() >= 1 and steps.max() <= 20
    assert np.all(np.diff(arrivals) >= 0) and arrivals[0] == 0.0
    # log-uniform edges: the geometric middle of [32, 256] splits the mass
    assert 0.4 < np.mean(edges <= 90) < 0.6
    # Poisson: mean gap 1/rate
    assert abs(np.mean(np.diff(arrivals)) - 1 / 50.0) < 0.1 / 50.0
    again = S.make_requests(2000, rate_hz=50.0, seed=5)
    assert [r.__dict__ for r in reqs] == [r.__dict__ for r in again]


def test_shards_partition_the_stream():
    reqs = S.make_requests(101, rate_hz=10.0)
    parts = [S.shard_requests(reqs, r, 3) for r in range(3)]
    ids = sorted(r.rid for p in parts for r in p)
    assert ids == list(range(101))


def test_percentiles_and_summary():
    lat = [0.1 * i for i in range(1, 101)]
    p = S.percentiles(lat)
    assert abs(p["p50"] - 5.05) < 1e-9 and p["p99"] > p["p95"] > p["p50"]
    comps = [S.Completion(i, 32, 2, 0.0, 0.0, 1.0 + i, 0) for i in range(10)]
    summ = S.summarize(comps, 10.0)
    assert summ["accepted"] == 10 and summ["cell_steps_per_s"] == 10 * 32 ** 3 * 2 / 10.0
    assert summ["rejected"] == {} and summ["rejections"] == []
    # a rejected request is counted by status and listed for a rerun alone
    bad = S.Completion(77, 168, 14, 0.0, 0.0, 3.0, 7, iterations=[16, 17], kind="step")
    summ = S.summarize(comps + [bad], 10.0)
    assert summ["accepted"] == 10 and summ["rejected"] == {"IterationLimit": 1}
    assert summ["rejections"] == [{"rid": 77, "edge": 168, "kind": "step", "steps_done": 14, "status": 7,
                                   "iterations": [16, 17]}]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}")
    reqs = S.make_requests(37, rate_hz=20.0, seed=11)
    mine = S.shard_requests(reqs, rank, world)
    comps = [S.Completion(r.rid, r.edge, r.steps, r.arrival, r.arrival, r.arrival + 0.5, 0) for r in mine]
    gathered = [None] * world
    dist.all_gather_object(gathered, comps)
    if rank == 0:
        merged = S.merge_completions(gathered)
        out_q.put([c.rid for c in merged])
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharding_over_gloo_covers_every_request_once():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    rids = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert rids == list(range(37))
