"""The N>1 bench path's host logic on CPU: two ranks over gloo (127.0.0.1).

On several GPUs every rank runs its shard of one event list, split by sorted-multiplicity
round-robin (itsu.shard; no collective on the data path); the only collectives are the barrier
and the reductions of the timing: the step time is the max over ranks and the throughput counts
the events of all ranks. The reference arm prints on rank 0 only; the other ranks leave without
work. Not measured on more than one GPU here: the runs of this build have one GPU.
"""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import json
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench

    w, r, local = bench.dist_env()
    dist = bench.init_dist(w, "gloo")
    try:
        res = {}
        # rank r's step took 10 ms * (r + 1) for 128 events
        rate, ms, units = bench.whole_job_rate(dist, 128 * 40, 10.0 * (r + 1) * 40, None)
        res.update(rate=rate, ms=ms, units=units)
        res["max"] = bench.max_over_ranks(dist, float(r), None)
        res["sum"] = bench.sum_over_ranks(dist, float(r + 1), None)
        res["seed"] = bench.shard_seed(2024, r)
        # one uneven list of 2 x 64 events (log-uniform 20-8000 tracks), this rank's shard of it
        events, mine, imb = bench.rank_events("uneven", 2024, 64, w, r)
        shards = [None] * w
        dist.all_gather_object(shards, mine)
        res["shards"] = shards
        res["imbalance"] = imb
        res["my_clusters"] = [int(sum(len(l) for l in ev.layers)) for ev in events]
        pb, pb_mine, pb_imb = bench.rank_events("pbpb", 7, 2, w, r)
        res["pbpb_shard"] = pb_mine

        class Args:
            seed, steps, warmup, events = 2024, 1, 3, 4

        res["reference_line"] = bench.run_reference(Args) if r != 0 else "skipped on rank 0"
        dist.barrier()
        with open(os.path.join(out_dir, "rank%d.json" % r), "w") as f:
            json.dump(res, f)
    finally:
        dist.destroy_process_group()


def test_two_ranks_over_gloo(tmp_path):
    import json

    import torch.multiprocessing as mp

    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        if p.is_alive():
            p.kill()
            pytest.fail("rank did not finish")
        assert p.exitcode == 0
    res = [json.load(open(tmp_path / ("rank%d.json" % r))) for r in range(world)]
    for r in res:
        assert r["ms"] == 800.0  # the slowest rank
        assert r["units"] == 2 * 128 * 40
        assert r["rate"] == pytest.approx(2 * 128 * 40 / 0.8)
        assert r["max"] == 1.0 and r["sum"] == 3.0
    assert res[0]["seed"] != res[1]["seed"]
    assert res[1]["reference_line"] is None  # the reference arm runs on rank 0 only
    # both ranks see the same split of the one list: every event exactly once
    assert res[0]["shards"] == res[1]["shards"]
    shards = res[0]["shards"]
    assert sorted(shards[0] + shards[1]) == list(range(128))
    assert res[0]["shards"][0] != res[0]["shards"][1]
    # balanced by N^2 cost within 10% (measured on the generated events' cluster counts too)
    from itsu import gen, shard

    mults = gen.batch_multiplicities(2024, n_events=128)
    assert shard.imbalance(shard.event_cost(mults), shards) < 0.10
    assert res[0]["imbalance"] == res[1]["imbalance"] < 0.10
    loads = [sum(c * c for c in r["my_clusters"]) for r in res]
    assert max(loads) / (sum(loads) / 2) - 1 < 0.10
    # central events all cost the same: dealt evenly
    assert sorted(res[0]["pbpb_shard"] + res[1]["pbpb_shard"]) == [0, 1, 2, 3] and len(res[0]["pbpb_shard"]) == 2


def test_partition_edge_cases():
    from itsu import shard

    assert shard.partition([], 3) == [[], [], []]
    assert shard.partition([5.0], 2) == [[0], []]
    # snake order: costs 9 8 7 6 5 4 over 3 ranks -> rank 0 gets 9 and 4, rank 2 gets 7 and 6
    assert shard.partition([9, 8, 7, 6, 5, 4], 3) == [[0, 5], [1, 4], [2, 3]]
    with pytest.raises(ValueError):
        shard.partition([1.0], 0)
