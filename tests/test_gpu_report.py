"""The road report on the device (itsu_roads_report): road classes and per-event counts equal
the oracle's restatement of IOUtils::writeRoadsReport, and the report files written from them
equal the reference's own (tests/golden/report/), byte for byte."""
import numpy as np
import pytest

from itsu import capi, gen, io
from oracle import oracle
from test_report import REPORT_FILES, _golden, _unpack, maps_for, oracle_roads, write_report

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(device=0)
    yield c
    c.close()


def _runs_batch(events):
    """Every vertex of every event as one run of a batch (runs share their event's clusters)."""
    runs = [(ev, iv, e) for e, ev in enumerate(events) for iv in range(len(ev.vertices))]
    clusters, offsets, vertices = gen.pack_batch([ev for ev, _, _ in runs], [iv for _, iv, _ in runs])
    return clusters, offsets, vertices, np.array([e for _, _, e in runs], np.int32)


def test_device_report_writes_the_reference_files(ctx, tmp_path):
    _unpack(tmp_path, "mixed", ("data.txt", "labels.txt"))
    events = io.read_reference_events(str(tmp_path / "data.txt"))
    maps = maps_for(str(tmp_path / "labels.txt"), len(events))
    clusters, offsets, vertices, run_event = _runs_batch(events)
    roads, road_off = ctx.batch_run_host(clusters, offsets, vertices)
    cls, counts = ctx.roads_report(maps, roads, road_off, run_event)
    want_cls, want_counts = oracle.roads_report(roads, road_off, maps, run_event)
    assert np.array_equal(cls, want_cls)
    assert np.array_equal(counts, want_counts.astype(capi.REPORT_COUNTS_DTYPE))
    got = write_report(tmp_path, roads, road_off, cls, maps, run_event)
    for n in REPORT_FILES:
        assert got[n] == _golden("mixed." + n), n
    # the same classes from the roads left on the device by that run
    cls_dev, counts_dev = ctx.roads_report(maps, run_event=run_event, n_runs=len(run_event))
    assert np.array_equal(cls_dev, cls) and np.array_equal(counts_dev, counts)
    # and the roads the oracle finds for the same runs are the ones the device found
    o_roads, o_off, _ = oracle_roads(events)
    assert np.array_equal(o_off, road_off) and np.array_equal(o_roads.view(np.uint8), roads.view(np.uint8))


def test_device_report_on_pbpb_and_jet_batch(ctx):
    """Thousands of labels and roads per event: the hash tables against the oracle's sorted ids."""
    events = [gen.pbpb_event(s, n_tracks=4000) for s in (91, 92)] + [gen.jet_event(93), gen.pbpb_event(94, n_tracks=300)]
    maps = []
    for ev in events:
        lab = ev.labels[(np.abs(ev.labels["pdg"]) == io.PION_CODE) & (ev.labels["ncl"] == 7)]
        maps.append(np.ascontiguousarray(lab, io.LABEL_DTYPE))
    maps[3] = maps[3][:0]  # an event with an empty labels map
    clusters, offsets, vertices = gen.pack_batch(events)
    roads, road_off = ctx.batch_run_host(clusters, offsets, vertices)
    cls, counts = ctx.roads_report(maps, roads, road_off)
    want_cls, want_counts = oracle.roads_report(roads, road_off, maps)
    assert np.array_equal(cls, want_cls)
    assert np.array_equal(counts, want_counts.astype(capi.REPORT_COUNTS_DTYPE))
    assert counts[0]["correct"] > 0.8 * counts[0]["labels"] and counts[2]["duplicate"] + counts[2]["fake"] > 0
    assert counts[3]["labels"] == 0


def test_device_report_on_pileup_frames(ctx):
    frames = [gen.pileup_frame(95 + f, collisions=3, n_tracks=600) for f in range(2)]
    clusters, frame_off, vertices, vertex_frame = gen.pack_frames(frames)
    roads, road_off = ctx.frames_run_host(clusters, frame_off, vertices, vertex_frame)
    maps = [np.ascontiguousarray(ev.labels[(np.abs(ev.labels["pdg"]) == 211) & (ev.labels["ncl"] == 7)], io.LABEL_DTYPE)
            for ev in frames]
    cls, counts = ctx.roads_report(maps, roads, road_off, vertex_frame)
    want_cls, want_counts = oracle.roads_report(roads, road_off, maps, vertex_frame)
    assert np.array_equal(cls, want_cls)
    assert np.array_equal(counts, want_counts.astype(capi.REPORT_COUNTS_DTYPE))
    cls_dev, _ = ctx.roads_report(maps, run_event=vertex_frame, n_runs=len(vertex_frame))
    assert np.array_equal(cls_dev, cls)


def test_device_report_rejects_bad_arguments(ctx):
    lab = np.zeros(1, io.LABEL_DTYPE)
    road = np.zeros(1, oracle.ROAD_DTYPE)
    with pytest.raises(capi.ItsuError) as e:
        ctx.roads_report([lab, lab], road, np.array([0, 1, 1], np.int32), np.array([1, 0], np.int32))
    assert e.value.status == capi.ERR_INVALID
    bad = lab.copy()
    bad["mc"] = np.iinfo(np.int32).min
    with pytest.raises(capi.ItsuError) as e:
        ctx.roads_report([bad], road, np.array([0, 1], np.int32))
    assert e.value.status == capi.ERR_INVALID
    fresh = capi.Context(device=0)
    try:
        with pytest.raises(capi.ItsuError) as e:
            fresh.roads_report([lab], n_runs=1)
        assert e.value.status == capi.ERR_STATE
    finally:
        fresh.close()


def test_facade_driver_writes_the_reference_report(tmp_path):
    """The C++ facade's driver with a labels file, as the reference's main.cpp: the three report
    files in the events file's folder equal the reference's."""
    import os
    import subprocess

    main = os.path.join(os.path.dirname(capi.LIB_PATH), "itsu_tracker_main")
    _unpack(tmp_path, "mixed", ("data.txt", "labels.txt"))
    proc = subprocess.run([main, str(tmp_path / "data.txt"), str(tmp_path / "labels.txt")], capture_output=True, text=True,
                          timeout=300)
    assert proc.returncode == 0, proc.stderr
    for n in REPORT_FILES:
        assert (tmp_path / n).read_text() == _golden("mixed." + n), n


def test_memory_occupancy_and_arena_usage(tmp_path):
    """The reference's MemoryOccupancy.txt from the device's per-run counts, and the arena's own
    occupancy (itsu_memory_usage_get): capacities hold the counted totals, bytes follow growth."""
    _unpack(tmp_path, "mixed", ("data.txt",))
    events = io.read_reference_events(str(tmp_path / "data.txt"))
    clusters, offsets, vertices, _ = _runs_batch(events)
    c = capi.Context(device=0)
    try:
        c.batch_run_host(clusters, offsets, vertices)
        runs = []
        for r in range(len(vertices) // 3):
            n = c.counts(r)
            runs.append((list(n.clusters), list(n.tracklets), list(n.cells), n.roads))
        assert io.memory_occupancy(runs[: len(events[0].vertices)], runs) == _golden("mixed.MemoryOccupancy.txt")
        small = c.memory_usage()
        totals = dict(tracklets=sum(sum(r[1]) for r in runs), cells=sum(sum(r[2]) for r in runs),
                      roads=sum(r[3] for r in runs))
        for k, v in totals.items():
            assert small["used"][k] == v and small["capacity"][k] >= v, k
        assert small["device_bytes"] > 0 and small["clusters_capacity"] >= len(clusters)
        big = [gen.pbpb_event(s, n_tracks=3000) for s in (71, 72, 73, 74)]
        c.batch_run_host(*gen.pack_batch(big))
        grown = c.memory_usage()
        assert grown["device_bytes"] > small["device_bytes"]
        for k in ("tracklets", "cells", "neighbours", "roads"):
            assert grown["capacity"][k] >= grown["used"][k] > 0, k
    finally:
        c.close()
