"""Parity of the sm_100a path (through the C ABI) with the reference and the oracle.

Bit-exact equality is required for every output: sorted clusters, index tables, tracklets and
their lookup tables, cells (including CA levels) and their lookup tables, neighbour rows, and
roads with their labels.
"""
import numpy as np
import pytest

from helpers import CASES, beyond_z_event, load_case, vertex_runs
from itsu import capi, gen
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(device=0)
    yield c
    c.close()


def _assert_same(got, want, what):
    mismatches = oracle.diff(got, want)
    assert mismatches == [], "%s: %s" % (what, mismatches[:6])


@pytest.mark.parametrize("case", CASES)
def test_stage_api_matches_reference_fixture(ctx, case):
    """PrimaryVertexContext::initialize + each Tracker stage, one C ABI call per stage."""
    events, expected = load_case(case)
    for k, ((ev, iv), exp) in enumerate(zip(vertex_runs(events), expected)):
        _assert_same(ctx.run_vertex(ev.layers, ev.vertices[iv]), exp, "%s vertex %d" % (case, k))


@pytest.mark.parametrize("case", CASES)
def test_whole_path_roads_match_reference_fixture(ctx, case):
    events, expected = load_case(case)
    for (ev, iv), exp in zip(vertex_runs(events), expected):
        roads = ctx.clusters_to_tracks(ev.layers, ev.vertices[iv])
        assert np.array_equal(roads.view(np.uint8), exp["roads"].view(np.uint8))


@pytest.mark.parametrize("case", CASES)
def test_batch_matches_reference_fixture(ctx, case):
    """Every vertex of the fixture as one event of a single batch."""
    events, expected = load_case(case)
    runs = vertex_runs(events)
    clusters, offsets, vertices = gen.pack_batch([ev for ev, _ in runs], [iv for _, iv in runs])
    roads, road_off = ctx.batch_run_host(clusters, offsets, vertices)
    for e, exp in enumerate(expected):
        _assert_same(ctx.results(e), exp, "%s batch event %d" % (case, e))
        assert np.array_equal(roads[road_off[e]:road_off[e + 1]].view(np.uint8), exp["roads"].view(np.uint8))


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_pbpb_event_matches_oracle(ctx, seed):
    ev = gen.pbpb_event(seed)
    want = oracle.run_vertex(ev.layers, ev.vertices[0])
    _assert_same(ctx.run_vertex(ev.layers, ev.vertices[0]), want, "Pb-Pb stages")
    roads = ctx.clusters_to_tracks(ev.layers, ev.vertices[0])
    assert np.array_equal(roads.view(np.uint8), want["roads"].view(np.uint8))
    assert len(want["roads"]) > 1000


def test_jet_event_crowded_paths_match_oracle(ctx):
    """A dense jet-like cone: inner clusters with more tracklets than the count pass keeps (48)
    and middle clusters with more outgoing tracklets than the cell pass's pair mask holds (64)
    take the crowded kernels. Stage by stage, whole path and batched beside a Pb-Pb event, the
    results equal the oracle's."""
    jet = gen.jet_event(5)
    want = oracle.run_vertex(jet.layers, jet.vertices[0])
    per_inner = [np.bincount(t["c1"]) for t in want["tracklets"]]
    assert sum(int((p > 48).sum()) for p in per_inner) > 0
    assert sum(int((p > 64).sum()) for p in per_inner[1:]) > 0
    _assert_same(ctx.run_vertex(jet.layers, jet.vertices[0]), want, "jet stages")
    roads = ctx.clusters_to_tracks(jet.layers, jet.vertices[0])
    assert np.array_equal(roads.view(np.uint8), want["roads"].view(np.uint8))
    bg = gen.pbpb_event(4)
    want_bg = oracle.run_vertex(bg.layers, bg.vertices[0])
    clusters, offsets, vertices = gen.pack_batch([bg, jet, bg])
    roads, road_off = ctx.batch_run_host(clusters, offsets, vertices)
    for e, exp in enumerate([want_bg, want, want_bg]):
        _assert_same(ctx.results(e), exp, "jet batch event %d" % e)
        assert np.array_equal(roads[road_off[e]:road_off[e + 1]].view(np.uint8), exp["roads"].view(np.uint8))


def test_bins_above_128_clusters_match_oracle(ctx):
    """A 150-track jet puts about 150 clusters into one index-table bin on every layer: the
    tracklet walk's pruned columns then need the four-word pass mask (layers of smaller bins use
    one or two words). Stage by stage and batched beside a Pb-Pb event."""
    jet = gen.jet_event(3, 150)
    want = oracle.run_vertex(jet.layers, jet.vertices[0])
    largest = [int(np.bincount(c["bin"][(c["bin"] >= 0) & (c["bin"] < 400)], minlength=400).max()) for c in want["clusters"][1:]]
    assert min(largest) > 128
    _assert_same(ctx.run_vertex(jet.layers, jet.vertices[0]), want, "dense jet stages")
    bg = gen.pbpb_event(5)
    clusters, offsets, vertices = gen.pack_batch([jet, bg])
    roads, road_off = ctx.batch_run_host(clusters, offsets, vertices)
    _assert_same(ctx.results(0), want, "dense jet batched")
    _assert_same(ctx.results(1), oracle.run_vertex(bg.layers, bg.vertices[0]), "Pb-Pb beside the jet")


def test_pileup_frame_matches_oracle(ctx):
    ev = gen.pileup_frame(7)
    clusters, offsets, vertices = gen.pack_batch([ev] * 5, list(range(5)))
    roads, road_off = ctx.batch_run_host(clusters, offsets, vertices)
    for iv in range(5):
        want = oracle.run_vertex(ev.layers, ev.vertices[iv])
        _assert_same(ctx.results(iv), want, "pile-up vertex %d" % iv)


def test_uneven_batch_matches_per_event_runs(ctx):
    """A batch of uneven multiplicity (20-8000 tracks, log-uniform) equals event-by-event runs
    and the oracle, event by event."""
    events = gen.batch_events(11, n_events=24)
    clusters, offsets, vertices = gen.pack_batch(events)
    roads, road_off = ctx.batch_run_host(clusters, offsets, vertices)
    batch_results = [ctx.results(e) for e in range(len(events))]
    for e, ev in enumerate(events):
        want = oracle.run_vertex(ev.layers, ev.vertices[0])
        _assert_same(batch_results[e], want, "batch event %d" % e)
        single = ctx.clusters_to_tracks(ev.layers, ev.vertices[0])
        assert np.array_equal(single.view(np.uint8), roads[road_off[e]:road_off[e + 1]].view(np.uint8))


def test_arena_growth_gives_identical_results():
    """Tiny initial capacities force every growth path; results must not change."""
    ev = gen.pbpb_event(4, n_tracks=2000)
    want = oracle.run_vertex(ev.layers, ev.vertices[0])
    small = capi.Context(device=0, max_clusters=16, max_tracklets=16, max_cells=16, max_neighbours=16, max_roads=16, max_events=1)
    try:
        roads = small.clusters_to_tracks(ev.layers, ev.vertices[0])
        assert np.array_equal(roads.view(np.uint8), want["roads"].view(np.uint8))
        _assert_same(small.results(0), want, "after growth")
    finally:
        small.close()
    # a fixed arena (ITSU_FLAG_NO_GROW) reports the overflow instead of growing, for the inputs
    # and for every output class, and stays usable for work that fits
    clusters, offsets, vertices = gen.pack_batch([ev])
    for caps in (dict(max_clusters=64), dict(max_tracklets=1000), dict(max_cells=100), dict(max_neighbours=10), dict(max_roads=10)):
        full = dict(max_clusters=100000, max_tracklets=10**6, max_cells=10**6, max_neighbours=10**6, max_roads=10**6, max_events=4)
        full.update(caps)
        fixed = capi.Context(device=0, flags=capi.FLAG_NO_GROW, **full)
        try:
            with pytest.raises(capi.ItsuError) as err:
                fixed.batch_run_host(clusters, offsets, vertices, roads_capacity=100000)
            assert err.value.status == capi.ERR_CAPACITY, caps
            pp = gen.pp_event(3)
            roads = fixed.clusters_to_tracks(pp.layers, pp.vertices[0]) if "max_clusters" not in caps else None
            if roads is not None:
                want_pp = oracle.run_vertex(pp.layers, pp.vertices[0])["roads"]
                if len(want_pp) <= full["max_roads"]:
                    assert np.array_equal(roads.view(np.uint8), want_pp.view(np.uint8))
        except capi.ItsuError as e:
            assert e.status == capi.ERR_CAPACITY, caps
        finally:
            fixed.close()


def test_malformed_input_is_rejected(ctx):
    ev = gen.pp_event(5)
    bad = [l.copy() for l in ev.layers]
    bad[2]["z"][3] = np.nan
    with pytest.raises(capi.ItsuError) as err:
        ctx.run_vertex(bad, ev.vertices[0])
    assert err.value.status == capi.ERR_INVALID
    with pytest.raises(capi.ItsuError) as err:
        ctx.clusters_to_tracks(ev.layers, (np.inf, 0.0, 0.0))
    assert err.value.status == capi.ERR_INVALID
    # the context stays usable after a rejected input
    want = oracle.run_vertex(ev.layers, ev.vertices[0])
    _assert_same(ctx.run_vertex(ev.layers, ev.vertices[0]), want, "after rejection")


def test_stage_order_is_enforced():
    fresh = capi.Context(device=0)
    try:
        with pytest.raises(capi.ItsuError) as err:
            fresh._check(fresh.lib.itsu_compute_layer_cells(fresh.h))
        assert err.value.status == capi.ERR_STATE
    finally:
        fresh.close()


def test_results_after_each_stage(ctx):
    """The PrimaryVertexContext getters after each stage hold that stage's results and empty
    later ones, like the reference between its Tracker stages (Tracker.cxx:253-259)."""
    ev = gen.pp_event(9)
    want = oracle.run_vertex(ev.layers, ev.vertices[0])
    stages = [ctx.lib.itsu_compute_layer_tracklets, ctx.lib.itsu_compute_layer_cells, ctx.lib.itsu_find_cells_neighbours,
              ctx.lib.itsu_find_tracks]
    fresh = capi.Context(device=0)
    try:
        fresh.initialize(ev.layers, ev.vertices[0])
        got = fresh.results(0)
        for l in range(7):
            assert np.array_equal(got["clusters"][l].view(np.uint8), want["clusters"][l].view(np.uint8))
        assert np.array_equal(got["index_tables"], want["index_tables"])
        assert all(len(t) == 0 for t in got["tracklets"]) and len(got["roads"]) == 0
        assert all((lk == -1).all() for lk in got["trk_lookup"])
        for k, stage in enumerate(stages):
            fresh._check(stage(fresh.h))
            got = fresh.results(0)
            if k == 0:
                for l in range(6):
                    assert np.array_equal(got["tracklets"][l].view(np.uint8), want["tracklets"][l].view(np.uint8))
                assert all(len(c) == 0 for c in got["cells"])
            if k == 1:
                for l in range(4):
                    assert np.array_equal(got["cell_lookup"][l], want["cell_lookup"][l])
        _assert_same(got, want, "all stages")
    finally:
        fresh.close()


def test_pileup_frames_share_their_clusters(ctx):
    """Frames API: every vertex of a frame runs over the frame's clusters uploaded once; each run
    equals the oracle on that vertex and the roads equal the duplicated-batch path's."""
    frames = gen.pileup_stream(17, n_frames=3, collisions=3, n_tracks=250)
    clusters, offsets, vertices, vertex_frame = gen.pack_frames(frames)
    roads, road_off = ctx.frames_run_host(clusters, offsets, vertices, vertex_frame)
    runs = [(ev, iv) for ev in frames for iv in range(len(ev.vertices))]
    assert len(road_off) == len(runs) + 1
    for v, (ev, iv) in enumerate(runs):
        want = oracle.run_vertex(ev.layers, ev.vertices[iv])
        _assert_same(ctx.results(v), want, "frame run %d" % v)
    b_clusters, b_offsets, b_vertices = gen.pack_batch([ev for ev, _ in runs], [iv for _, iv in runs])
    b_roads, b_off = ctx.batch_run_host(b_clusters, b_offsets, b_vertices)
    assert np.array_equal(b_off, road_off)
    assert np.array_equal(b_roads.view(np.uint8), roads.view(np.uint8))
    # the device-resident replay of the same frames gives the same roads
    ctx.frames_run_host(clusters, offsets, vertices, vertex_frame)
    ctx.relaunch()
    ctx.batch_status()
    again = ctx.results(len(runs) - 1)
    _assert_same(again, oracle.run_vertex(runs[-1][0].layers, runs[-1][0].vertices[runs[-1][1]]), "replay")


def test_launch_shapes_and_autotuner_keep_results(ctx):
    """The batch results do not depend on the launch shape; the autotuner's pick neither."""
    events = gen.batch_events(5, n_events=6)
    clusters, offsets, vertices = gen.pack_batch(events)
    base_roads, base_off = ctx.batch_run_host(clusters, offsets, vertices)
    want = [ctx.results(e) for e in range(len(events))]
    band = ctx.lib.itsu_multiplicity_band(len(clusters), len(events))
    try:
        for block, per_sm, prune, group in [(128, 4, 0, 0), (512, 16, 1, 0), (64, 2, 1, 0), (256, 8, 1, 2), (64, 4, 1, 4),
                                            (256, 8, 2, 0), (512, 4, 2, 0)]:
            ctx.set_tune(band, block, per_sm, prune, group)
            assert ctx.get_tune(band)["threads_per_block"] == block and ctx.get_tune(band)["events_per_group"] == group
            roads, off = ctx.batch_run_host(clusters, offsets, vertices)
            assert np.array_equal(off, base_off) and np.array_equal(roads.view(np.uint8), base_roads.view(np.uint8))
            for e in range(len(events)):
                _assert_same(ctx.results(e), want[e], "shape %d/%d/%d/%d event %d" % (block, per_sm, prune, group, e))
        best = ctx.autotune(repeats=1)
        assert best["band"] == band and best["threads_per_block"] in (64, 128, 256, 512) and best["ms"] > 0
        assert best["events_per_group"] in (0, 8, 16, 32)
        roads, off = ctx.batch_run_host(clusters, offsets, vertices)
        assert np.array_equal(roads.view(np.uint8), base_roads.view(np.uint8))
    finally:
        ctx.set_tune(band, 256, 8, 1)


def test_uneven_batch_of_256_events(ctx):
    """The batched form at its stated size: 256 events of log-uniform 20-8000 tracks in one pass.
    Every event's roads equal its own single-vertex run (itsu_clusters_to_tracks) byte for byte
    and its counts equal that run's; a stratified sample (the 8 largest and 8 random events) equals
    the oracle in every output."""
    events = gen.batch_events(31, n_events=256)
    clusters, offsets, vertices = gen.pack_batch(events)
    roads, road_off = ctx.batch_run_host(clusters, offsets, vertices)
    sizes = np.array([sum(len(l) for l in ev.layers) for ev in events])
    rng = np.random.default_rng(31)
    largest = list(np.argsort(sizes)[-8:])
    sample = sorted(set(largest) | set(rng.choice(np.setdiff1d(np.arange(256), largest), 8, replace=False)))
    batch_results = {int(e): ctx.results(int(e)) for e in sample}
    batch_counts = [ctx.counts(e) for e in range(len(events))]
    for e in sample:
        ev = events[e]
        _assert_same(batch_results[e], oracle.run_vertex(ev.layers, ev.vertices[0]), "256-event batch, event %d" % e)
    for e, ev in enumerate(events):
        single = ctx.clusters_to_tracks(ev.layers, ev.vertices[0])
        assert np.array_equal(single.view(np.uint8), roads[road_off[e]:road_off[e + 1]].view(np.uint8)), e
        c = ctx.counts(0)
        b = batch_counts[e]
        assert list(c.tracklets) == list(b.tracklets) and list(c.cells) == list(b.cells), e
        assert list(c.neighbours) == list(b.neighbours) and c.roads == b.roads, e
    assert sizes.max() > 50000 and sizes.min() < 1000  # the log-uniform span


def test_pileup_frames_at_stated_size(ctx):
    """Pile-up frames of 5 collisions of 1500 tracks with 10% noise through the frames API (each
    frame's clusters uploaded once, every vertex run over them): each run equals the oracle."""
    frames = [gen.pileup_frame(7), gen.pileup_frame(8)]
    clusters, offsets, vertices, vertex_frame = gen.pack_frames(frames)
    roads, road_off = ctx.frames_run_host(clusters, offsets, vertices, vertex_frame)
    runs = [(ev, iv) for ev in frames for iv in range(len(ev.vertices))]
    assert len(runs) == 10 and len(road_off) == 11
    for v, (ev, iv) in enumerate(runs):
        want = oracle.run_vertex(ev.layers, ev.vertices[iv])
        _assert_same(ctx.results(v), want, "frame run %d" % v)
        assert np.array_equal(roads[road_off[v]:road_off[v + 1]].view(np.uint8), want["roads"].view(np.uint8))


def test_clusters_beyond_z_range_match_oracle(ctx):
    """Hundreds of clusters per layer beyond the z range, most with negative bins (sorted apart
    from the index table, stably, by the clustering's merge sort), many tied: stage by stage and
    batched beside a Pb-Pb event, equal to the oracle."""
    ev = beyond_z_event(4244)
    want = oracle.run_vertex(ev.layers, ev.vertices[0])
    assert sum(int((c["bin"] < 0).sum()) for c in want["clusters"]) > 1500
    _assert_same(ctx.run_vertex(ev.layers, ev.vertices[0]), want, "beyond-z stages")
    bg = gen.pbpb_event(6)
    clusters, offsets, vertices = gen.pack_batch([bg, ev])
    roads, road_off = ctx.batch_run_host(clusters, offsets, vertices)
    _assert_same(ctx.results(1), want, "beyond-z batched")
    assert np.array_equal(roads[road_off[1]:road_off[2]].view(np.uint8), want["roads"].view(np.uint8))


def test_event_groups_keep_results():
    """The tracklet write and cell count passes run event group by event group (groups of 1, 3, 7
    and 16 events, so group ends fall inside the 32-cluster and 32-tracklet blocks of the passes'
    warps), whole runs and streamed chunks: the results equal the run without groups bit for bit."""
    events = gen.batch_events(19, n_events=40) + [gen.jet_event(9), gen.pp_event(10)]
    clusters, offsets, vertices = gen.pack_batch(events)
    plain = capi.Context(device=0)
    grouped = capi.Context(device=0)
    streamed = capi.Context(device=0, flags=capi.FLAG_STREAM_HOST, stream_chunk_clusters=150000)
    try:
        want_roads, want_off = plain.batch_run_host(clusters, offsets, vertices)
        want = [plain.results(e) for e in range(len(events))]
        band = plain.lib.itsu_multiplicity_band(len(clusters), len(events))
        for group in (1, 3, 7, 16):
            grouped.set_tune(band, 256, 8, 1, group)
            roads, off = grouped.batch_run_host(clusters, offsets, vertices)
            assert np.array_equal(off, want_off) and np.array_equal(roads.view(np.uint8), want_roads.view(np.uint8)), group
            for e in range(len(events)):
                _assert_same(grouped.results(e), want[e], "groups of %d, event %d" % (group, e))
            prof = grouped.profile(repeats=1)
            assert any(name == "write_count_by_event_group" for name, _ in prof)
            assert not any(name == "cells_count" for name, _ in prof)
        for b in range(32):
            streamed.set_tune(b, 256, 8, 1, 3)  # every chunk's band
        roads, off = streamed.batch_run_host(clusters, offsets, vertices)
        assert np.array_equal(off, want_off) and np.array_equal(roads.view(np.uint8), want_roads.view(np.uint8))
    finally:
        plain.close()
        grouped.close()
        streamed.close()


def test_staged_walk_matches_oracle(ctx):
    """The staged tracklet walk (prune 2: each block's rows of the next layer copied into shared
    memory by one bulk copy) on central events, a dense jet (bins above 128 clusters) and an
    uneven batch: every output equals the oracle's."""
    events = [gen.pbpb_event(3), gen.jet_event(3, 150)] + gen.batch_events(23, n_events=10)
    clusters, offsets, vertices = gen.pack_batch(events)
    band = ctx.lib.itsu_multiplicity_band(len(clusters), len(events))
    try:
        ctx.set_tune(band, 256, 8, 2)
        ctx.batch_run_host(clusters, offsets, vertices)
        for e, ev in enumerate(events):
            _assert_same(ctx.results(e), oracle.run_vertex(ev.layers, ev.vertices[0]), "staged walk, event %d" % e)
    finally:
        ctx.set_tune(band, 256, 8, 1)


def _without_layer3_tracklets(seed, n_tracks):
    """An event whose layer-3 clusters are moved 100 cm along the beam, past the layer's end: no
    tracklet reaches them from layer 2 or leaves them for layer 4 (the z cut), while the tracklet
    layers 4 and 5 keep theirs. Cell layer 0 runs; cell layers 1-4 do not (Tracker.cxx:124-128),
    although cell layer 4's first tracklets exist."""
    ev = gen.pbpb_event(seed, n_tracks)
    l3 = ev.layers[3].copy()
    l3["z"] = l3["z"] + 100.0
    ev.layers[3] = l3
    return ev


def test_inactive_cell_layers_match_oracle(ctx):
    """Cell layers that do not run although their first tracklets exist: per vertex and inside a
    batch beside ordinary events, against the oracle."""
    odd = _without_layer3_tracklets(11, 1500)
    want = oracle.run_vertex(odd.layers, odd.vertices[0])
    sizes = [len(t) for t in want["tracklets"]]
    assert sizes[2] == 0 and sizes[3] == 0 and sizes[4] > 0 and sizes[5] > 0, sizes
    assert len(want["cells"][0]) > 0 and all(len(c) == 0 for c in want["cells"][1:])
    _assert_same(ctx.run_vertex(odd.layers, odd.vertices[0]), want, "inactive cell layers")
    events = [gen.pbpb_event(12, 1500), odd, gen.pbpb_event(13, 1500)]
    clusters, offsets, vertices = gen.pack_batch(events)
    roads, road_off = ctx.batch_run_host(clusters, offsets, vertices)
    for e, ev in enumerate(events):
        exp = oracle.run_vertex(ev.layers, ev.vertices[0])
        _assert_same(ctx.results(e), exp, "batch event %d" % e)
        assert np.array_equal(roads[road_off[e]:road_off[e + 1]].view(np.uint8), exp["roads"].view(np.uint8))
