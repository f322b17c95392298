"""A fixed batched workload for profilers: ``python -m itsu.profile_run [--gate FILE] [--events N]``.

Builds one device-resident batch of seeded central Pb-Pb-like events (the bench's generator and
seeds: ``gen.pbpb_event(2024 * 100000 + i, 6000)``), then calls ``itsu_batch_run`` ``--runs``
times, in the plain form or, with ``--gate``, with that tracklet-gate checkpoint enabled. Nothing
is timed; the kernels of each run are launched in the same order, so a profiler can pick a run's
launches by their index (``ncu -s/-c``). Prints the road count of the last run.
"""
from __future__ import annotations

import argparse

from . import capi, gen, prefilter


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("--events", type=int, default=32)
    p.add_argument("--runs", type=int, default=2)
    p.add_argument("--gate", default=None, help="tracklet-gate checkpoint to enable (default: the plain form)")
    args = p.parse_args(argv)
    import torch

    dev = torch.device("cuda", 0)
    events = [gen.pbpb_event(2024 * 100000 + i, 6000) for i in range(args.events)]
    ctx = capi.Context(device=0)
    try:
        batch = prefilter.DeviceBatch(ctx, events, dev)
        if args.gate:
            ctx.gate_set_model(capi.gate_load(args.gate))
            ctx.gate_enable(True)
        for _ in range(args.runs):
            ctx.batch_run(batch.batch)
        roads = sum(int(ctx.counts(e).roads) for e in range(batch.n_runs))
        print("events %d runs %d form %s roads %d" % (len(events), args.runs, "gate" if args.gate else "plain", roads))
    finally:
        ctx.close()


if __name__ == "__main__":
    main()
