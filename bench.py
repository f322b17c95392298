#!/usr/bin/env python
"""Benchmark of the ITS CA track finder on B200: Pb-Pb-like events/s.

Workload (one "step"): a batch of central Pb-Pb-like events (6000 tracks, pT mean 0.6 GeV/c,
|eta| < 1, 5% noise; seeded synthetic, each event its own vertex) through the plain path:
clustering, tracklets, cells, neighbours/levels, roads and labels, every event in one batched
pass of every kernel, replayed as one CUDA graph. The batch's inputs and intermediates (about
200 MB of raw clusters, 1.3 GB of tracklets) are larger than the 126 MB L2, so there is no L2
flush between steps.

  value  events/s with the inputs already resident in HBM (device-side batch API)
  e2e    events/s through the host-facing C ABI call (itsu_batch_run_host_tracks): pinned host
         clusters (16-byte input records: coordinates and MC id) in, roads out, every copy inside
         the timed region (modes.e2e_compact: the same with the 24-byte records)
  roofline  the dominant kernel's own compulsory bytes / its CUDA-event duration, against the
         measured HBM copy bandwidth (every main kernel's figure under roofline.kernels)
  cpu_baseline  the reference CPU Tracker (oracle/_ref, compiled from the reference's sources)
         on a bounded sample of the same events, one process per host core
  modes  the learned forms (tracklet gate, pair prefilter, both) on the same batch, the road
         report, and the other configurations: a 256-event uneven batch and a 1024-frame pile-up
         stream

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU (torchrun, one rank per GPU): one event list of events-per-GPU x N events, split by
sorted-multiplicity round-robin (weak scaling, no collective on the data path); the step time is
the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "tracking-itsu_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

from itsu import gen  # noqa: E402

METRIC = "Pb-Pb-like events/s on 1 B200: plain vs batched vs learned-prefilter @≥99.5% roads"
UNIT = "events/s"
TRACKS = 6000
WORKLOAD = "pbpb_central_6000trk_5pct_noise"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--events", type=int, default=128, help="events per step per GPU (pbpb, uneven)")
    ap.add_argument("--workload", choices=("pbpb", "uneven", "pileup"), default="pbpb",
                    help="pbpb: central Pb-Pb-like events, 6000 tracks (the headline); uneven: log-uniform "
                         "20-8000 tracks; pileup: frames of 5 collisions of ~1500 tracks, 10%% noise")
    ap.add_argument("--frames", type=int, default=32, help="pile-up frames per step per GPU")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other configurations' legs (the 256-event uneven batch and the 1024-frame pile-up stream)")
    ap.add_argument("--uneven-events", type=int, default=256, help="events of the uneven-batch leg")
    ap.add_argument("--stream-frames", type=int, default=1024, help="frames of the pile-up stream leg")
    ap.add_argument("--stream-chunk", type=int, default=32, help="frames per call of the pile-up stream leg")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shape")
    ap.add_argument("--no-prefilter", action="store_true", help="skip the learned-prefilter modes")
    ap.add_argument("--prefilter", default=None,
                    help="checkpoint of the learned pair prefilter (default: the one trained for the workload)")
    ap.add_argument("--gate", default=None,
                    help="checkpoint of the learned tracklet gate (default: the one trained for the workload)")
    args = ap.parse_args()
    if args.prefilter is None:
        own = os.path.join(PKG, "weights", "prefilter_%s.itsumlp" % args.workload)
        args.prefilter = own if os.path.exists(own) else os.path.join(PKG, "weights", "prefilter_pbpb.itsumlp")
    if args.gate is None:
        own = os.path.join(PKG, "weights", "gate_%s.itsugate" % args.workload)
        args.gate = own if os.path.exists(own) else os.path.join(PKG, "weights", "gate_pbpb.itsugate")
    return args


# ------------------------------------------------------------------------------------------
# distributed plumbing (one process per GPU, weak scaling)


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def init_dist(world, backend):
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
        return dist
    return None


def max_over_ranks(dist, value, device=None):
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(dist, value, device=None):
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def shard_seed(seed, rank):
    """A per-rank seed for the legs whose streams are generated rank by rank (the pile-up stream)."""
    return seed + 7919 * rank


def rank_events(workload, seed, per_rank, world, rank):
    """This rank's share of ONE event list of per_rank * world events (weak scaling), split by
    sorted-multiplicity round-robin (itsu.shard): central events all cost the same and are dealt
    evenly; an uneven batch's events are balanced by N^2 cost. Returns (events, shard indices,
    imbalance of the split)."""
    from itsu import shard

    n = per_rank * world
    if workload == "uneven":
        mults = gen.batch_multiplicities(seed, n_events=n)
    else:
        mults = np.full(n, TRACKS)
    shards = shard.partition(shard.event_cost(mults), world)
    mine = shards[rank]
    if workload == "uneven":
        events = gen.batch_events(seed, n_events=n, indices=mine)
    else:
        events = [gen.pbpb_event(seed * 100000 + i, TRACKS) for i in mine]
    return events, mine, shard.imbalance(shard.event_cost(mults), shards)


def whole_job_rate(dist, units_local, ms_local, device=None):
    """Units of all ranks / the slowest rank's time: (units per second, max ms, total units)."""
    ms = max_over_ranks(dist, ms_local, device)
    units = sum_over_ranks(dist, units_local, device)
    return units / (ms * 1e-3), ms, units


# ------------------------------------------------------------------------------------------
# workload


def make_events(n, seed):
    return [gen.pbpb_event(seed * 100000 + i, TRACKS) for i in range(n)]


WORKLOADS = {
    "pbpb": "pbpb_central_6000trk_5pct_noise",
    "uneven": "uneven_batch_loguniform_20_8000trk_5pct_noise",
    "pileup": "pileup_frames_5x1500trk_10pct_noise",
}


def algorithmic_bytes(counts) -> dict:
    """Compulsory bytes per stage from one event's output sizes (one touch of every object in
    the reference layouts: 36 B clusters, 16 B tracklets, 40 B cells, 32 B roads, 4 B indices)."""
    N, T, C, E, R = counts["N"], counts["T"], counts["C"], counts["E"], counts["R"]
    b = {}
    b["cluster_sort"] = sum(72 * n for n in N) + 6 * 401 * 4
    b["tracklets"] = sum(36 * (N[l] + N[l + 1]) + 16 * T[l] for l in range(6)) + sum(4 * N[l] for l in range(1, 6))
    b["cells"] = sum(16 * (T[l] + T[l + 1]) + 36 * (N[l] + N[l + 1] + N[l + 2]) + 40 * C[l] for l in range(5)) + sum(
        4 * T[l] for l in range(1, 5))
    b["neighbours"] = sum(40 * (C[l] + C[l + 1]) + 4 * E[l] + 4 * C[l + 1] for l in range(4))
    b["roads"] = 40 * C[4] + 4 * sum(E) + 32 * R
    b["event"] = sum(b.values())
    return b


def kernel_bytes(counts) -> dict:
    """Each main kernel's own share of the compulsory bytes (the stage sums above split by which
    kernel reads or writes each object): the tracklet count pass reads both layers' clusters, the
    tracklet write pass writes the tracklets and their lookup table, the cell count pass reads the
    tracklets of both layers and the three layers' clusters, the cell scatter writes the cells and
    their lookup table."""
    N, T, C = counts["N"], counts["T"], counts["C"]
    b = algorithmic_bytes(counts)
    return {
        "cluster_sort": b["cluster_sort"],
        "tracklets_count": sum(36 * (N[l] + N[l + 1]) for l in range(6)),
        "tracklets_write": sum(16 * T[l] for l in range(6)) + sum(4 * N[l] for l in range(1, 6)),
        "cells_count": sum(16 * (T[l] + T[l + 1]) + 36 * (N[l] + N[l + 1] + N[l + 2]) for l in range(5)),
        "cells_scatter": sum(40 * C[l] for l in range(5)) + sum(4 * T[l] for l in range(1, 5)),
        "neighbours_write": b["neighbours"],
        "roads_write": b["roads"],
    }


# ------------------------------------------------------------------------------------------
# clocks during the timed region


class ClockSampler:
    """nvidia-smi samples (every 100 ms) of SM clock, power and throttle reasons; only samples
    taken inside the timed window (mark_start/mark_end) are summarised."""

    QUERY = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.device_index = device_index
        self.proc = None
        self.path = None
        self.t0 = self.t1 = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + self.QUERY, "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.device_index), "-f", self.path],
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.5)
        return self

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        import datetime

        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 10:
                    continue
                try:
                    ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                    rows.append((ts, float(f[2]), float(f[3]), f[4], f[6:10]))
                except ValueError:
                    continue
        except OSError:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        lo, hi = (self.t0 or 0) - 0.05, (self.t1 or 1e18) + 0.05
        inside = [r for r in rows if lo <= r[0] <= hi]
        used = inside if inside else rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in used for n, v in zip(names, r[4]) if v.lower().startswith("active")})
        power = [float(r[3]) for r in used if r[3].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(r[1] for r in used), "sm_max_mhz": used[0][2], "reasons": reasons,
                "samples": len(used), "samples_in_window": len(inside), "power_w_max": max(power) if power else None}


# ------------------------------------------------------------------------------------------
# CPU baseline: the reference tracker (or the oracle port) on all host cores


def cpu_workers():
    return max(1, min(os.cpu_count() or 1, 64))


def _reference_binary():
    from oracle import oracle

    return oracle.ref_binary("cr") if oracle.ref_available("cr") else None


def run_reference_sample(events, workers, per_worker, repeats=1):
    """Runs the reference harness in `workers` parallel processes, each timing `per_worker`
    events of the file (after its own warm-up event). Returns (events, seconds = max worker)."""
    binary = _reference_binary()
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "events.bin")
        gen.write_binary_events(events, path)
        n = len(events)
        procs = []
        for w in range(workers):
            first = (w * per_worker) % max(n - per_worker + 1, 1)
            procs.append(subprocess.Popen([binary, "timebin", path, str(repeats), str(first), str(per_worker)],
                                          stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
        results = []
        for p in procs:
            out, err = p.communicate(timeout=900)
            if p.returncode != 0:
                raise RuntimeError("reference harness failed: %s" % err.strip())
            results.append(json.loads(out.strip().splitlines()[-1]))
    total = sum(r["events"] for r in results)
    return total, max(r["seconds"] for r in results)


def _port_worker(args):
    clusters, offsets, vertices, n = args
    from oracle import oracle

    t0 = time.perf_counter()
    oracle.lib().oracle_run_batch(clusters.ctypes.data, offsets.ctypes.data, vertices.ctypes.data, n)
    return time.perf_counter() - t0


def run_port_sample(events, workers, per_worker):
    import multiprocessing as mp

    jobs = []
    for w in range(workers):
        sub = [events[(w * per_worker + k) % len(events)] for k in range(per_worker)]
        c, o, v = gen.pack_batch(sub)
        jobs.append((c, o, v, len(sub)))
    with mp.get_context("spawn").Pool(workers) as pool:
        secs = pool.map(_port_worker, jobs)
    return workers * per_worker, max(secs)


def cpu_baseline(events, budget_s):
    """Bounded sample of the workload on every host core (one single-threaded process each)."""
    workers = cpu_workers()
    ref = _reference_binary() is not None
    # calibrate: one event on one core, then size the per-worker share to the budget
    if ref:
        n1, s1 = run_reference_sample(events[:1], 1, 1)
    else:
        n1, s1 = run_port_sample(events[:1], 1, 1)
    per_event = s1 / max(n1, 1)
    per_worker = max(1, min(len(events), int(budget_s / max(per_event, 1e-6))))
    if ref:
        n, s = run_reference_sample(events, workers, per_worker)
    else:
        n, s = run_port_sample(events, workers, per_worker)
    return {"value": n / s, "unit": UNIT, "cores": workers, "kind": "reference" if ref else "port",
            "value_1_core": 1.0 / per_event,  # the calibration event alone on one core
            "sample": "%d Pb-Pb-like events (%d per process, %d single-threaded processes, one per core) of the "
                      "benchmark workload; %s" % (n, per_worker, workers,
                                                  "reference CPU Tracker built from its sources (oracle/_ref/ref_cr)"
                                                  if ref else "oracle C port")}


# ------------------------------------------------------------------------------------------
# our implementation


def run_ours(args):
    import torch

    world, rank, local = dist_env()
    dist = init_dist(world, "nccl")
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    from itsu import capi

    seed = shard_seed(args.seed, rank)
    frames = None
    shard_info = None
    if args.workload == "pileup":
        frames = gen.pileup_stream(seed, args.frames, collisions=5, n_tracks=1500)
        events = [ev for ev in frames for _ in ev.vertices]
        f_clusters, f_offsets, f_vertices, f_vertex_frame = gen.pack_frames(frames)
        clusters, offsets, vertices = gen.pack_batch(events, [iv for ev in frames for iv in range(len(ev.vertices))])
    else:
        # one event list of events-per-GPU x world events, this rank's shard of it
        events, mine, imb = rank_events(args.workload, args.seed, args.events, world, rank)
        shard_info = {"events_total": args.events * world, "split": "sorted-multiplicity round-robin (N^2 cost, snake)",
                      "cost_imbalance": imb}
        clusters, offsets, vertices = gen.pack_batch(events)
    n_events, n_clusters = len(events), len(clusters)

    # device-resident inputs (torch owns the memory; the library only reads it)
    d_clusters = torch.from_numpy(clusters.view(np.uint8)).to(device)
    d_offsets = torch.from_numpy(offsets).to(device)
    d_vertices = torch.from_numpy(vertices).to(device)
    stream = torch.cuda.Stream(device=device)
    ctx = capi.Context(device=local)
    ctx.set_stream(stream.cuda_stream)
    batch = ctx.batch_device(d_clusters.data_ptr(), d_offsets.data_ptr(), d_vertices.data_ptr(), n_events, n_clusters)
    if frames is not None:
        # frames: the raw clusters of a frame are resident once and shared by its vertices
        ctx.frames_run_host(f_clusters, f_offsets, f_vertices, f_vertex_frame)
        launch = ctx.relaunch
    else:
        ctx.batch_run(batch)  # sizes the arena, validates the inputs, captures the graph
        launch = lambda: ctx.batch_launch(batch)  # noqa: E731
    tune = None
    if not args.no_autotune:
        # the batched form's autotuner: launch shape for this multiplicity band (untimed)
        tune = ctx.autotune(repeats=2)
    counts = []
    for e in range(n_events):
        c = ctx.counts(e)
        counts.append(dict(N=list(c.clusters), T=list(c.tracklets), C=list(c.cells), E=list(c.neighbours), R=c.roads))
    total_roads = sum(c["R"] for c in counts)

    for _ in range(args.warmup):
        launch()
    stream.synchronize()
    kernels = ctx.lib.itsu_kernels_per_run()

    # ---- value: device-resident batch, K graph replays ----
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        clocks.mark_start()
        start.record(stream)
        for _ in range(args.steps):
            launch()
        end.record(stream)
        torch.cuda.synchronize()
        clocks.mark_end()
    ctx.batch_status()
    if dist:
        dist.barrier()
    ms_local = start.elapsed_time(end)
    value, ms, total_events = whole_job_rate(dist, n_events * args.steps, ms_local, device)
    clock_summary = clocks.summary()

    # ---- e2e: host in / host out through the C ABI ----
    # the host-facing call takes the 16-byte input records (itsu_cluster_track): what the roads
    # and their labels need of each cluster, 4/9 of the 36-byte Cluster; the 24-byte records
    # (itsu_cluster_in, all the raw constructor's arguments) are timed beside it
    from itsu import capi as _capi

    def pinned(records):
        t = torch.empty(records.nbytes, dtype=torch.uint8, pin_memory=True)
        t.numpy()[:] = records.view(np.uint8)
        return t

    clusters_in = _capi.track_clusters(clusters)
    h_clusters = pinned(clusters_in)
    h_compact = pinned(_capi.compact_clusters(clusters)) if frames is None else None
    host_fn = "itsu_batch_run_host_tracks"
    h_offsets = torch.empty(len(offsets), dtype=torch.int32, pin_memory=True)
    h_offsets.numpy()[:] = offsets
    h_vertices = torch.empty(len(vertices), dtype=torch.float32, pin_memory=True)
    h_vertices.numpy()[:] = vertices
    roads_cap = int(total_roads * 1.1) + 1024
    h_roads = torch.empty(roads_cap * 32, dtype=torch.uint8, pin_memory=True)
    h_road_off = torch.empty(n_events + 1, dtype=torch.int32, pin_memory=True)
    import ctypes

    # the host-facing call streams: chunks of events, each upload overlapping the work on the
    # chunk before (its own context, so the device-resident arena above stays as it is)
    ctx_e2e = None
    if frames is None:
        ctx_e2e = capi.Context(device=local, flags=capi.FLAG_STREAM_HOST)
        ctx_e2e.set_stream(stream.cuda_stream)
        if tune is not None:
            ctx_e2e.set_tune(tune["band"], tune["threads_per_block"], tune["blocks_per_sm"], tune["prune"], tune["events_per_group"])

    def host_run():
        st = getattr(ctx_e2e.lib, host_fn)(ctx_e2e.h, ctypes.c_void_p(h_clusters.data_ptr()), ctypes.c_void_p(h_offsets.data_ptr()),
                                           ctypes.c_void_p(h_vertices.data_ptr()), n_events, ctypes.c_void_p(h_roads.data_ptr()),
                                           roads_cap, ctypes.c_void_p(h_road_off.data_ptr()))
        ctx_e2e._check(st)

    if frames is not None:
        from itsu.capi import Frames

        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).pin_memory()  # noqa: E731
        hf = [pin(f_clusters), pin(f_offsets), pin(f_vertices), pin(f_vertex_frame)]
        fr = Frames()
        fr.clusters, fr.frame_offsets, fr.vertices, fr.vertex_frame = (t.data_ptr() for t in hf)
        fr.n_frames, fr.n_vertices = len(frames), n_events
        h_clusters = hf[0]
        h2d_bytes = sum(t.numel() for t in hf)

        def host_run():  # noqa: F811
            st = ctx.lib.itsu_frames_run_host(ctx.h, ctypes.byref(fr), ctypes.c_void_p(h_roads.data_ptr()), roads_cap,
                                              ctypes.c_void_p(h_road_off.data_ptr()))
            ctx._check(st)
    else:
        h2d_bytes = int(clusters_in.nbytes + offsets.nbytes + vertices.nbytes)

    for _ in range(max(1, args.warmup)):
        host_run()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for _ in range(args.steps):
        host_run()
    e_end.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(dist, e_start.elapsed_time(e_end), device)
    assert int(h_road_off[-1]) == total_roads, "host path road count differs from the device path"
    e2e_compact_ms = None
    if ctx_e2e is not None:
        # the same call with the 24-byte records, timed the same way
        host_fn, h_clusters = "itsu_batch_run_host_compact", h_compact
        for _ in range(max(1, args.warmup)):
            host_run()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e_start.record(stream)
        for _ in range(args.steps):
            host_run()
        e_end.record(stream)
        torch.cuda.synchronize()
        e2e_compact_ms = max_over_ranks(dist, e_start.elapsed_time(e_end), device)
        assert int(h_road_off[-1]) == total_roads, "compact host path road count differs from the device path"
        ctx_e2e.close()

    # ---- learned forms: same inputs, same timing rules ----
    # the tracklet gate alone, the pair prefilter alone, and both (where their checkpoints exist)
    learned = {}
    if not args.no_prefilter:
        from itsu import capi as _capi

        pair = _capi.prefilter_load(args.prefilter) if os.path.exists(args.prefilter) else None
        gate = _capi.gate_load(args.gate) if os.path.exists(args.gate) else None
        windows = None  # the gate's first stage alone: its windows, no layer scored by the network
        if gate is not None:
            windows = _capi.GateModel.from_buffer_copy(bytes(gate))
            windows.mlp_layers = 0
        forms = (("tracklet_gate", None, gate), ("gate_windows_only", None, windows), ("pair_prefilter", pair, None),
                 ("gate_and_pair", pair, gate))
        for name, p_model, g_model in forms:
            if (name != "pair_prefilter" and g_model is None) or (name in ("pair_prefilter", "gate_and_pair") and p_model is None):
                continue
            if name == "gate_windows_only" and gate.mlp_layers == 0:
                continue  # the committed gate is its windows already
            l_ms, l_cmp, l_prof = learned_mode(ctx, launch, args, stream, dist, device, p_model, g_model)
            learned[name] = dict(ms=l_ms, cmp=l_cmp, prof=l_prof,
                                 pair_threshold=None if p_model is None else float(p_model.logit_threshold),
                                 gate_threshold=None if g_model is None else float(g_model.logit_threshold),
                                 gate_mlp_layers=None if g_model is None else int(g_model.mlp_layers))
        launch()  # back to the plain graph (the profile below times the plain kernels)
        ctx.batch_status()

    # ---- road report (IOUtils::writeRoadsReport) on the device, over the roads left resident ----
    report = road_report_mode(ctx, events, frames, args, rank, world)
    configs = None
    if not args.no_configs and args.workload == "pbpb":
        configs = {"uneven_batch": uneven_leg(args, stream, dist, device, local, peak_hbm()),
                   "pileup_stream": pileup_stream_leg(args, stream, dist, device, local)}
    usage = ctx.memory_usage()
    arena = dict(usage, occupancy={k: (usage["used"][k] / usage["capacity"][k]) if usage["capacity"][k] else None
                                   for k in usage["capacity"]},
                 note="itsu_memory_usage_get after the step: the arena sized by the count passes (exact totals, grown "
                      "once), against the reference's per-vertex coefficient reservations (itsu.io.MemoryModel)")

    # ---- live per-kernel timing for the roofline ----
    prof = ctx.profile(repeats=3)
    step_bytes = {}
    for c in counts:
        for k, v in algorithmic_bytes(c).items():
            step_bytes[k] = step_bytes.get(k, 0) + v
    own_bytes = {}
    for c in counts:
        for k, v in kernel_bytes(c).items():
            own_bytes[k] = own_bytes.get(k, 0) + v
    top_name, top_ms = max(prof, key=lambda x: x[1])
    peak, peak_src = peak_hbm_with_source()
    achieved = (own_bytes[top_name] / (top_ms * 1e-3) / 1e9) if top_name in own_bytes else None
    per_kernel = {name: {"ms": round(t, 4), "own_bytes": own_bytes[name],
                         "gbs": own_bytes[name] / (t * 1e-3) / 1e9, "frac": own_bytes[name] / (t * 1e-3) / 1e9 / peak}
                  for name, t in prof if name in own_bytes and t > 0}
    # DRAM bytes of the kernel from an ncu capture of this same workload (profiles/traffic.json,
    # per event, scaled to this launch's events); none for a workload that was not captured
    traffic = None
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        if tr.get("workload") == args.workload:
            per_event = tr.get("kernels", {}).get(top_name, {}).get("dram_bytes_per_event")
            if per_event is not None:
                traffic = per_event * n_events
    except (OSError, ValueError):
        pass

    # plain path, one vertex per call (itsu_clusters_to_tracks, host in / host out, synchronous),
    # the way the reference's Tracker::clustersToTracks is driven event by event
    single = events[: min(16, len(events))]
    ctx1 = capi.Context(device=local)
    ctx1.set_stream(stream.cuda_stream)
    for ev in single[:2]:
        ctx1.clusters_to_tracks(ev.layers, ev.vertices[0])
    t0 = time.perf_counter()
    for ev in single:
        ctx1.clusters_to_tracks(ev.layers, ev.vertices[0])
    single_eps = len(single) / (time.perf_counter() - t0)
    ctx1.close()

    e2e_value = total_events / (e2e_ms * 1e-3)
    line = None
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            cpu = cpu_baseline(events, args.cpu_seconds)
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded helix generator, reference geometry; no public dataset)",
            "config": {
                "workload": WORKLOADS[args.workload],
                "events_per_step_per_gpu": n_events,
                "tracks_per_event": TRACKS if args.workload == "pbpb" else ("log-uniform 20-8000" if args.workload == "uneven" else "5 collisions x 1050-1950"),
                "frames_per_step_per_gpu": len(frames) if frames is not None else None,
                "clusters_per_step_per_gpu": n_clusters,
                "tracklets_per_step_per_gpu": int(sum(sum(c["T"]) for c in counts)),
                "cells_per_step_per_gpu": int(sum(sum(c["C"]) for c in counts)),
                "roads_per_step_per_gpu": int(total_roads),
                "mode": "batched plain path, one CUDA graph per step" + ("; frames: raw clusters resident once per frame" if frames is not None else ""),
                "launch_shape": tune if tune is not None else "default (256 threads, 8 blocks/SM, pruning on)",
                "parallelism": "event shards, one rank per GPU" if world > 1 else "single GPU",
                "sharding": shard_info,
                "l2": "inputs larger than L2 (%.0f MB raw clusters, %.0f MB tracklets per step), no flush" % (
                    clusters.nbytes / 1e6, 16 * sum(sum(c["T"]) for c in counts) / 1e6),
            },
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d_bytes),
                    "d2h_bytes_per_step": int(32 * total_roads + 4 * (n_events + 1)),
                    "api": "itsu_frames_run_host (pinned host buffers)" if frames is not None else
                           "itsu_batch_run_host_tracks (16-byte input records: coordinates and MC id) with ITSU_FLAG_STREAM_HOST (chunks of events, uploads overlapping the work; pinned host buffers)"},
            "gpu_launches": kernels * args.steps,
            "roofline": {"bound": "hbm", "kernel": top_name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "algorithmic_bytes_per_launch": own_bytes.get(top_name), "launch_ms": top_ms,
                         "bytes_note": "the kernel's own compulsory bytes: the objects it must read or write once, "
                                       "in the reference layouts (bench.py kernel_bytes)",
                         "kernels": per_kernel,
                         "peak_source": "%s (MEASURED_PEAKS.json hbm_gbs)" % peak_src if peak_src == "measured" else "fallback 6.65 TB/s"},
            "modes": {
                "batched_plain_events_per_s": value,
                "e2e_compact": None if e2e_compact_ms is None else {
                    "value": total_events / (e2e_compact_ms * 1e-3), "unit": UNIT,
                    "h2d_bytes_per_step": int(24 * len(clusters) + offsets.nbytes + vertices.nbytes),
                    "api": "itsu_batch_run_host_compact (24-byte input records), otherwise as e2e"},
                "plain_single_event_events_per_s": single_eps,
                "plain_single_event_note": "itsu_clusters_to_tracks, one vertex per synchronous call, host in/out, wall clock",
                "learned_prefilter": learned_summary(learned, total_events, value, args),
                "road_report": report,
                "configurations": configs,
            },
            "arena": arena,
            "kernel_ms": {name: round(t, 4) for name, t in prof},
            "algorithmic_bytes_per_step": step_bytes.get("event"),
            "achieved_gbs_whole_step": step_bytes.get("event") / (ms / args.steps * 1e-3) / 1e9,
            "clocks": clock_summary,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return line


def peak_hbm_with_source():
    """The HBM roofline denominator: MEASURED_PEAKS.json's copy bandwidth, else the fallback."""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def peak_hbm():
    return peak_hbm_with_source()[0]


def timed_replays(launch, stream, steps, warmup, dist, device):
    """CUDA-event time of `steps` launches after `warmup` untimed ones (max over ranks), in ms."""
    import torch

    for _ in range(warmup):
        launch()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(steps):
        launch()
    end.record(stream)
    torch.cuda.synchronize()
    return max_over_ranks(dist, start.elapsed_time(end), device)


def uneven_leg(args, stream, dist, device, local, peak):
    """Configuration 3: one batch of `--uneven-events` events of log-uniform 20-8000 tracks (5%
    noise, each its own vertex) per step, device-resident, one CUDA graph, the autotuner's shape
    for the batch's band; its dominant kernel against its own compulsory bytes."""
    import torch

    from itsu import capi

    world, rank, _ = dist_env()
    evs = gen.batch_events(shard_seed(args.seed, rank) + 31, n_events=args.uneven_events)
    clusters, offsets, vertices = gen.pack_batch(evs)
    d = [torch.from_numpy(a.view(np.uint8) if a is clusters else a).to(device) for a in (clusters, offsets, vertices)]
    ctx = capi.Context(device=local)
    try:
        ctx.set_stream(stream.cuda_stream)
        batch = ctx.batch_device(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), len(evs), len(clusters))
        ctx.batch_run(batch)
        tune = None if args.no_autotune else ctx.autotune(repeats=2)
        ms = timed_replays(lambda: ctx.batch_launch(batch), stream, args.steps, args.warmup, dist, device)
        ctx.batch_status()
        counts = []
        for e in range(len(evs)):
            c = ctx.counts(e)
            counts.append(dict(N=list(c.clusters), T=list(c.tracklets), C=list(c.cells), E=list(c.neighbours), R=c.roads))
        prof = ctx.profile(repeats=3)
    finally:
        ctx.close()
    value, ms, total = whole_job_rate(dist, len(evs) * args.steps, ms, device)
    own = {}
    for c in counts:
        for k, v in kernel_bytes(c).items():
            own[k] = own.get(k, 0) + v
    top, top_ms = max(prof, key=lambda x: x[1])
    achieved = own[top] / (top_ms * 1e-3) / 1e9 if top in own else None
    return {
        "workload": "uneven_batch_loguniform_20_8000trk_5pct_noise", "events_per_step_per_gpu": len(evs),
        "clusters_per_step_per_gpu": int(len(clusters)), "events_per_s": value, "clusters_per_s": value * len(clusters) / len(evs),
        "ms_per_step": ms / args.steps, "launch_shape": tune, "roads_per_step_per_gpu": int(sum(c["R"] for c in counts)),
        "roofline": {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if achieved else None, "algorithmic_bytes_per_launch": own.get(top),
                     "launch_ms": top_ms, "traffic": None},
        "kernel_ms": {k: round(t, 4) for k, t in prof},
        "note": "configuration 3 at its stated size; the per-event parity against single runs is tests/test_gpu_parity.py",
    }


def pileup_stream_leg(args, stream, dist, device, local):
    """Configuration 5: a stream of `--stream-frames` frames of 5 overlapping collisions
    (1050-1950 tracks each, vertices z ~ N(0, 5 cm), 10% noise), fed from pinned host memory
    through itsu_frames_run_host in calls of `--stream-chunk` frames (each frame's clusters uploaded
    once and tracked from each of its 5 vertices), roads back to the host: one step is the whole
    stream. The plain form, and the learned form with the pile-up checkpoints where they exist."""
    import ctypes
    import multiprocessing as mp

    import torch

    from itsu import capi, prefilter
    from itsu.capi import Frames

    world, rank, _ = dist_env()
    seed = shard_seed(args.seed, rank) + 57
    rng = np.random.default_rng(seed)
    mults = [int(rng.integers(1050, 1951)) for _ in range(args.stream_frames)]
    jobs = [(seed * 1000003 + f, mults[f]) for f in range(args.stream_frames)]
    with mp.get_context("spawn").Pool(min(32, os.cpu_count() or 1)) as pool:
        frames = pool.map(_pileup_frame_job, jobs, chunksize=8)
    chunks = []
    for k in range(0, len(frames), args.stream_chunk):
        fr = frames[k:k + args.stream_chunk]
        c, o, v, vf = gen.pack_frames(fr)
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).pin_memory()  # noqa: E731
        t = [pin(c), pin(o), pin(v), pin(vf)]
        f = Frames()
        f.clusters, f.frame_offsets, f.vertices, f.vertex_frame = (x.data_ptr() for x in t)
        f.n_frames, f.n_vertices = len(fr), len(vf)
        chunks.append(dict(t=t, f=f, runs=len(vf), clusters=len(c)))
    runs = sum(ch["runs"] for ch in chunks)
    frame_clusters = sum(ch["clusters"] for ch in chunks)
    cap = 4 * max(ch["clusters"] for ch in chunks)  # roads per call: well below one per cluster
    h_roads = torch.empty(cap * 32, dtype=torch.uint8, pin_memory=True)
    h_off = torch.empty(max(ch["runs"] for ch in chunks) + 1, dtype=torch.int32, pin_memory=True)
    ctx = capi.Context(device=local)
    out = {"workload": "pileup_stream_5x1050_1950trk_10pct_noise", "frames_per_step_per_gpu": len(frames),
           "frames_per_call": args.stream_chunk, "vertex_runs_per_step_per_gpu": runs,
           "frame_clusters_per_step_per_gpu": int(frame_clusters),
           "api": "itsu_frames_run_host per call (pinned host frames in, roads and road offsets out)", "forms": {}}
    try:
        ctx.set_stream(stream.cuda_stream)
        n_roads = [0]

        def one_step():
            n_roads[0] = 0
            for ch in chunks:
                st = ctx.lib.itsu_frames_run_host(ctx.h, ctypes.byref(ch["f"]), ctypes.c_void_p(h_roads.data_ptr()), cap,
                                                  ctypes.c_void_p(h_off.data_ptr()))
                ctx._check(st)
                n_roads[0] += int(h_off[ch["runs"]])

        pair_path = os.path.join(PKG, "weights", "prefilter_pileup.itsumlp")
        gate_path = os.path.join(PKG, "weights", "gate_pileup.itsugate")
        pair = capi.prefilter_load(pair_path) if os.path.exists(pair_path) else None
        gate = capi.gate_load(gate_path) if os.path.exists(gate_path) else None
        forms = [("plain", None, None)]
        if not args.no_prefilter and gate is not None:
            # the tracklet gate alone: with the pair prefilter as well the frames keep under 99.5% of their roads
            forms.append(("learned", None, gate))
        elif not args.no_prefilter and pair is not None:
            forms.append(("learned", pair, None))
        steps = max(1, min(args.steps, 3))
        for name, p_model, g_model in forms:
            if p_model is not None:
                ctx.prefilter_set_model(p_model)
            if g_model is not None:
                ctx.gate_set_model(g_model)
            prefilter.set_learned(ctx, p_model is not None, g_model is not None)
            ms = timed_replays(one_step, stream, steps, 1, dist, device)
            value, ms, _ = whole_job_rate(dist, runs * steps, ms, device)
            out["forms"][name] = {"vertex_runs_per_s": value, "frames_per_s": value / 5.0, "ms_per_step": ms / steps,
                                  "roads_per_step_per_gpu": n_roads[0], "steps": steps,
                                  "networks": [k for k, m in (("pair_prefilter", p_model), ("tracklet_gate", g_model))
                                               if m is not None]}
        prefilter.set_learned(ctx, False, False)
    finally:
        ctx.close()
    if "learned" in out["forms"]:
        out["forms"]["learned"]["vs_plain"] = out["forms"]["learned"]["vertex_runs_per_s"] / out["forms"]["plain"]["vertex_runs_per_s"]
        out["forms"]["learned"]["road_fraction_of_plain"] = (out["forms"]["learned"]["roads_per_step_per_gpu"] /
                                                             max(out["forms"]["plain"]["roads_per_step_per_gpu"], 1))
    return out


def _pileup_frame_job(job):
    seed, n_tracks = job
    return gen.make_event(seed, n_tracks, pt_mean=0.6, noise=0.10, n_vertices=5)


def road_report_mode(ctx, events, frames, args, rank, world):
    """itsu_roads_report over the step's roads, left on the device by the last graph replay: the
    correct / duplicate / fake classification of IOUtils::writeRoadsReport against each event's
    labels map (the particles with |pdg| == 211 and 7 clusters). Timed per call (labels up, road
    classes and counts down, wall clock around the synchronous call), next to the reference's own
    writeRoadsReport on a sample of the same events (oracle/_ref/ref_cr report)."""
    import tempfile

    from itsu import io

    owners = frames if frames is not None else events
    maps = [np.ascontiguousarray(ev.labels[(np.abs(ev.labels["pdg"]) == io.PION_CODE) & (ev.labels["ncl"] == 7)], io.LABEL_DTYPE)
            for ev in owners]
    run_event = None
    if frames is not None:
        run_event = np.concatenate([np.full(len(f.vertices), k, np.int32) for k, f in enumerate(frames)])
    n_runs = len(events)
    for _ in range(2):
        ctx.roads_report(maps, run_event=run_event, n_runs=n_runs)
    reps = 5
    t0 = time.perf_counter()
    for _ in range(reps):
        cls, counts = ctx.roads_report(maps, run_event=run_event, n_runs=n_runs)
    call_ms = (time.perf_counter() - t0) / reps * 1e3
    labels = int(counts["labels"].sum())
    out = {"ms_per_step": call_ms, "events_per_s": len(owners) / (call_ms * 1e-3), "events": len(owners),
           "roads": int(len(cls)), "labels": labels, "correct": int(counts["correct"].sum()),
           "duplicate": int(counts["duplicate"].sum()), "fake": int(counts["fake"].sum()),
           "efficiency": (int(counts["correct"].sum()) / labels) if labels else None,
           "api": "itsu_roads_report on the device-resident roads (labels uploaded, classes and counts downloaded per call)",
           "reference": None}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import oracle

            if oracle.ref_available("cr"):
                sample = owners[: min(8, len(owners))]
                with tempfile.TemporaryDirectory() as tmp:
                    gen.write_reference_events(sample, os.path.join(tmp, "data.txt"))
                    gen.write_reference_labels(sample, os.path.join(tmp, "labels.txt"))
                    r = oracle.run_reference_report(os.path.join(tmp, "data.txt"), os.path.join(tmp, "labels.txt"), tmp)
                out["reference"] = {"events_per_s": r["events"] / r["report_seconds"] if r["report_seconds"] > 0 else None,
                                    "sample_events": r["events"], "report_seconds": r["report_seconds"], "cores": 1,
                                    "kind": "reference",
                                    "note": "IOUtils::writeRoadsReport of the reference build (ref_cr report), one core, "
                                            "steady_clock around each call, roads from its own Tracker"}
        except Exception as exc:  # the baseline is reported, not required
            out["reference"] = {"error": str(exc)}
    return out


def learned_summary(learned, total_events, plain_value, args):
    """The learned forms' bench entries: each form's rate against the batched plain path on the
    same resident batch, its road reproduction and what it kept; the headline form is the fastest
    one that reproduces at least 99.5% of the plain roads with no extra road."""
    if not learned:
        return None
    out = {}
    for name, r in learned.items():
        eps = total_events / (r["ms"] * 1e-3)
        out[name] = {
            "events_per_s": eps, "ms_per_step": r["ms"] / args.steps, "vs_batched_plain": eps / plain_value,
            "road_reproduction": r["cmp"]["road_reproduction"], "plain_roads": r["cmp"]["plain_roads"],
            "learned_roads": r["cmp"]["learned_roads"], "extra_roads": r["cmp"]["extra"], "extra_fakes": r["cmp"]["extra_fakes"],
            "tracklets_kept": r["cmp"]["tracklets_kept"], "cells_kept": r["cmp"]["cells_kept"],
            "gate_logit_threshold": r["gate_threshold"], "gate_mlp_layers": r["gate_mlp_layers"],
            "pair_logit_threshold": r["pair_threshold"],
            "kernel_ms": {k: round(t, 4) for k, t in r["prof"]},
        }
    ok = [k for k, v in out.items() if v["road_reproduction"] >= 0.995 and v["extra_roads"] == 0]
    best = max(ok, key=lambda k: out[k]["events_per_s"]) if ok else None
    return {
        "headline_form": best,
        "vs_batched_plain": out[best]["vs_batched_plain"] if best else None,
        "road_reproduction": out[best]["road_reproduction"] if best else None,
        "forms": out,
        "checkpoints": {"pair_prefilter": os.path.relpath(args.prefilter, ROOT) if os.path.exists(args.prefilter) else None,
                        "tracklet_gate": os.path.relpath(args.gate, ROOT) if os.path.exists(args.gate) else None},
        "note": "same resident batch and timing as the plain value; tracklet gate: learned per-layer |dphi| and |dz| "
                "windows in the tracklet count pass, then an 8-16-16-1 ReLU MLP on the tracklets inside them (of the "
                "layers in its mlp_layers) before the tracklet scan; gate_windows_only: the same gate's windows with no "
                "layer scored; pair prefilter: 8-64-64-1 GELU MLP on the cell stage's pairs; BF16 MMAs, FP32 accumulation",
    }


def learned_mode(ctx, launch, args, stream, dist, device, pair_model, gate_model):
    """One learned form on the same resident inputs: K timed graph replays (max over ranks), and its
    roads against the plain run's (exported just before)."""
    import torch

    from itsu import prefilter

    prefilter.set_learned(ctx, False, False)
    launch()
    ctx.batch_status()
    plain_keys, plain_fake = prefilter.export_roads(ctx, device)
    plain_cells = ctx.prefilter_export()[0]
    plain_tracklets = ctx.gate_export()[0]
    if pair_model is not None:
        ctx.prefilter_set_model(pair_model)
    if gate_model is not None:
        ctx.gate_set_model(gate_model)
    prefilter.set_learned(ctx, pair_model is not None, gate_model is not None)
    try:
        launch()  # captures the learned graph
        ctx.batch_status()
        learned_cells = ctx.prefilter_export()[0]
        learned_tracklets = ctx.gate_export()[0]
        keys, fake = prefilter.export_roads(ctx, device)
        for _ in range(args.warmup):
            launch()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        start.record(stream)
        for _ in range(args.steps):
            launch()
        end.record(stream)
        torch.cuda.synchronize()
        ctx.batch_status()
        ms = max_over_ranks(dist, start.elapsed_time(end), device)
        prof = ctx.profile(repeats=3)
    finally:
        prefilter.set_learned(ctx, False, False)
    cmp = prefilter.compare_roads(plain_keys, plain_fake, keys, fake)
    cmp["road_reproduction"] = cmp["reproduced"] / max(cmp["plain_roads"], 1)
    cmp["cells_kept"] = learned_cells / max(plain_cells, 1)
    cmp["tracklets_kept"] = learned_tracklets / max(plain_tracklets, 1)
    return ms, cmp, prof


# ------------------------------------------------------------------------------------------
# the reference's own CPU implementation of the path


def run_reference(args):
    world, rank, local = dist_env()
    if rank != 0:
        return None
    if _reference_binary() is None:
        impl = "oracle C port (the reference build oracle/_ref is not present)"
    else:
        impl = "reference CPU Tracker built from its own sources (oracle/_ref/ref_cr, patched P1-P5)"
    workers = cpu_workers()
    events = make_events(max(workers, 8), args.seed)
    per_worker = 1
    total_events = 0
    total_s = 0.0
    for step in range(args.warmup + args.steps):
        if _reference_binary() is not None:
            n, s = run_reference_sample(events, workers, per_worker)
        else:
            n, s = run_port_sample(events, workers, per_worker)
        if step >= args.warmup:
            total_events += n
            total_s += s
    value = total_events / total_s
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_s / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded helix generator, reference geometry; no public dataset)",
        "config": {"workload": WORKLOAD, "events_per_step": workers * per_worker, "tracks_per_event": TRACKS,
                   "mode": "reference CPU Tracker::clustersToTracks, one single-threaded process per host core"},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers,
                         "kind": "reference" if _reference_binary() else "port",
                         "sample": "%d events per step (%d processes x %d), %s" % (workers * per_worker, workers, per_worker, impl)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return line


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
