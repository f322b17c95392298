"""Streamed host batches (ITSU_FLAG_STREAM_HOST): the batch runs as consecutive chunks of events
whose uploads overlap the work on earlier chunks. The roads and road offsets must be the ones of
the one-pass run, byte for byte; the per-event intermediates are not kept."""
import numpy as np
import pytest

from itsu import capi, gen
from oracle import oracle

pytestmark = pytest.mark.gpu


def _pinned(a):
    import torch

    t = torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).pin_memory()
    return t.numpy().view(a.dtype)


def _both(events, chunk, prefilter=None):
    clusters, offsets, vertices = gen.pack_batch(events)
    one = capi.Context(device=0)
    streamed = capi.Context(device=0, flags=capi.FLAG_STREAM_HOST, stream_chunk_clusters=chunk)
    try:
        if prefilter is not None:
            for c in (one, streamed):
                c.prefilter_set_model(prefilter)
                c.prefilter_enable(True)
        want = one.batch_run_host(clusters, offsets, vertices)
        got = streamed.batch_run_host(_pinned(clusters), _pinned(offsets), _pinned(vertices))
        got_again = streamed.batch_run_host(clusters, offsets, vertices)  # pageable buffers, arena reused
        with pytest.raises(capi.ItsuError) as e:
            streamed.results(0)
        assert e.value.status == capi.ERR_STATE
        return want, got, got_again
    finally:
        one.close()
        streamed.close()


def _same(a, b):
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(a[0].view(np.uint8), b[0].view(np.uint8))


def test_streamed_pbpb_batch_equals_one_pass():
    import torch

    torch.cuda.init()
    events = [gen.pbpb_event(s, n_tracks=2000) for s in range(60, 66)]
    want, got, again = _both(events, chunk=30000)
    assert want[1][-1] > 0
    _same(want, got)
    _same(want, again)


def test_streamed_uneven_batch_equals_one_pass():
    events = gen.batch_events(61, n_events=24, hi=4000)
    want, got, again = _both(events, chunk=20000)
    _same(want, got)
    _same(want, again)


def test_streamed_learned_batch_equals_one_pass():
    events = [gen.pbpb_event(s, n_tracks=2000) for s in range(70, 74)]
    model = capi.prefilter_init(4)
    model.logit_threshold = -0.5
    want, got, _ = _both(events, chunk=30000, prefilter=model)
    _same(want, got)


def test_streamed_malformed_cluster_reports_its_batch_index():
    events = [gen.pbpb_event(s, n_tracks=800) for s in range(80, 86)]
    clusters, offsets, vertices = gen.pack_batch(events)
    bad = int(offsets[4 * 7 + 2]) + 3  # a cluster of event 4, layer 2: in a later chunk
    clusters = clusters.copy()
    clusters["x"][bad] = np.nan
    ctx = capi.Context(device=0, flags=capi.FLAG_STREAM_HOST, stream_chunk_clusters=8000)
    try:
        with pytest.raises(capi.ItsuError) as e:
            ctx.batch_run_host(clusters, offsets, vertices)
        assert e.value.status == capi.ERR_INVALID
        assert "cluster %d " % bad in str(e.value)
    finally:
        ctx.close()


def test_streamed_roads_into_pinned_host_buffer():
    """Pinned host buffers in and out (the benchmark's e2e call): same bytes as the one-pass run,
    and a too small road buffer is reported."""
    import ctypes

    import torch

    events = [gen.pbpb_event(s, n_tracks=2000) for s in range(90, 96)]
    clusters, offsets, vertices = gen.pack_batch(events)
    one = capi.Context(device=0)
    ctx = capi.Context(device=0, flags=capi.FLAG_STREAM_HOST, stream_chunk_clusters=30000)
    try:
        want = one.batch_run_host(clusters, offsets, vertices)
        cap = len(want[0]) + 16
        h_roads = torch.zeros(cap * capi.ROAD_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
        h_off = torch.zeros(len(events) + 1, dtype=torch.int32).pin_memory()
        hc, ho, hv = _pinned(clusters), _pinned(offsets), _pinned(vertices)
        st = ctx.lib.itsu_batch_run_host(ctx.h, hc.ctypes.data_as(ctypes.c_void_p), ho.ctypes.data_as(ctypes.c_void_p),
                                         hv.ctypes.data_as(ctypes.c_void_p), len(events), ctypes.c_void_p(h_roads.data_ptr()), cap,
                                         ctypes.c_void_p(h_off.data_ptr()))
        assert st == capi.OK, ctx.lib.itsu_last_error(ctx.h)
        got_off = h_off.numpy().copy()
        got = h_roads.numpy().view(capi.ROAD_DTYPE)[: got_off[-1]].copy()
        got["pad"] = 0
        assert np.array_equal(got_off, want[1])
        assert np.array_equal(got.view(np.uint8), want[0].view(np.uint8))
        # too small a pinned buffer: the call reports the shortfall
        st = ctx.lib.itsu_batch_run_host(ctx.h, hc.ctypes.data_as(ctypes.c_void_p), ho.ctypes.data_as(ctypes.c_void_p),
                                         hv.ctypes.data_as(ctypes.c_void_p), len(events), ctypes.c_void_p(h_roads.data_ptr()),
                                         len(want[0]) // 2, ctypes.c_void_p(h_off.data_ptr()))
        assert st == capi.ERR_CAPACITY
    finally:
        one.close()
        ctx.close()


def test_streamed_batch_outgrowing_the_arena_falls_back_and_grows():
    """Tiny starting capacities: the first chunk overflows, the call runs the batch in one pass
    (which grows the arena) and returns the same roads; the next call streams in the grown arena."""
    events = [gen.pbpb_event(s, n_tracks=2000) for s in range(100, 106)]
    clusters, offsets, vertices = gen.pack_batch(events)
    one = capi.Context(device=0)
    small = capi.Context(device=0, flags=capi.FLAG_STREAM_HOST, stream_chunk_clusters=30000, max_tracklets=1000,
                         max_cells=1000, max_neighbours=1000, max_roads=100)
    try:
        want = one.batch_run_host(clusters, offsets, vertices)
        _same(want, small.batch_run_host(clusters, offsets, vertices))
        _same(want, small.batch_run_host(clusters, offsets, vertices))
    finally:
        one.close()
        small.close()


@pytest.mark.parametrize("streamed", [False, True])
def test_compact_input_records_give_the_same_run(streamed):
    """itsu_batch_run_host_compact (24-byte input records, the fields clustering computes left out)
    gives the 36-byte call's roads and every per-event result bit for bit, one pass and streamed
    (chunks on two arenas), with malformed input reported at the same cluster."""
    events = [gen.pbpb_event(s, n_tracks=3000) for s in (81, 82)] + gen.batch_events(83, n_events=12) + [gen.jet_event(7)]
    clusters, offsets, vertices = gen.pack_batch(events)
    # streamed: small chunks, so that the batch splits
    kw = dict(flags=capi.FLAG_STREAM_HOST, stream_chunk_clusters=60000) if streamed else {}
    full = capi.Context(device=0, **kw)
    comp = capi.Context(device=0, **kw)
    try:
        want_roads, want_off = full.batch_run_host(clusters, offsets, vertices)
        got_roads, got_off = comp.batch_run_host_compact(capi.compact_clusters(clusters), offsets, vertices)
        assert np.array_equal(want_off, got_off)
        assert np.array_equal(want_roads.view(np.uint8), got_roads.view(np.uint8))
        if not streamed:
            for e in range(len(events)):
                assert oracle.diff(comp.results(e), full.results(e)) == [], e
        bad = capi.compact_clusters(clusters)
        bad["x"][offsets[7 * 3 + 2] + 5] = np.nan
        with pytest.raises(capi.ItsuError) as err:
            comp.batch_run_host_compact(bad, offsets, vertices)
        assert err.value.status == capi.ERR_INVALID and str(offsets[7 * 3 + 2] + 5) in str(err.value)
    finally:
        full.close()
        comp.close()


@pytest.mark.parametrize("streamed", [False, True])
def test_track_input_records_give_the_same_roads(streamed):
    """itsu_batch_run_host_tracks (16-byte records: coordinates and MC id) gives the 36-byte call's
    roads, labels and fake flags bit for bit, one pass and streamed; its sorted clusters are the
    full call's with each cluster's index in its layer's input order as the id and alpha 0, and
    every other per-event result is the full call's."""
    events = [gen.pbpb_event(s, n_tracks=3000) for s in (84, 85)] + gen.batch_events(86, n_events=12) + [gen.jet_event(8)]
    clusters, offsets, vertices = gen.pack_batch(events)
    kw = dict(flags=capi.FLAG_STREAM_HOST, stream_chunk_clusters=60000) if streamed else {}
    full = capi.Context(device=0, **kw)
    trk = capi.Context(device=0, **kw)
    try:
        want_roads, want_off = full.batch_run_host(clusters, offsets, vertices)
        got_roads, got_off = trk.batch_run_host_tracks(capi.track_clusters(clusters), offsets, vertices)
        assert np.array_equal(want_off, got_off)
        assert np.array_equal(want_roads.view(np.uint8), got_roads.view(np.uint8))
        if not streamed:
            for e in range(len(events)):
                want, got = full.results(e), trk.results(e)
                for layer in range(7):
                    w, g = want["clusters"][layer], got["clusters"][layer]
                    base = offsets[7 * e + layer]
                    # the full call's ids are its input indices here: the id is the input position
                    order = w["id"] - clusters["id"][base] if len(w) else w["id"]
                    assert np.array_equal(g["id"], np.asarray(order, np.int32)), (e, layer)
                    assert np.all(g["alpha"] == 0)
                    for k in ("x", "y", "z", "phi", "r", "mc", "bin"):
                        assert np.array_equal(g[k].view(np.uint32), w[k].view(np.uint32)), (e, layer, k)
                    want["clusters"][layer] = g
                assert oracle.diff(got, want) == [], e
        bad = capi.track_clusters(clusters)
        bad["z"][offsets[7 * 4 + 3] + 2] = np.inf
        with pytest.raises(capi.ItsuError) as err:
            trk.batch_run_host_tracks(bad, offsets, vertices)
        assert err.value.status == capi.ERR_INVALID and str(offsets[7 * 4 + 3] + 2) in str(err.value)
    finally:
        full.close()
        trk.close()
