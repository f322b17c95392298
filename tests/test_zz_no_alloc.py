"""The no-allocation clustering entry point (itsu_pvc_initialize_noalloc).

It exists for callers that cannot call cudaMalloc: a process whose memory pool owns the
device's memory, or a latency-critical loop that cannot afford an allocation's implicit
synchronisation. It must give exactly what the allocating entry point (itsu_pvc_initialize)
gives: the stably sorted clusters and the six index tables, bit for bit. Two calls in a row
check that the scratch array the calls share (it keeps the previous call's contents) does not
leak into the next result. This file is collected last, so a failure here comes after every
other test has run.
"""
import ctypes

import numpy as np
import pytest

from itsu import capi, gen

pytestmark = pytest.mark.gpu


def _noalloc_call(lib, clusters, offsets, vertex, stream):
    """One call on device copies of the given host arrays: (status, sorted clusters, tables)."""
    import torch

    dev = torch.device("cuda", 0)
    d_clusters = torch.from_numpy(clusters.view(np.uint8).copy()).to(dev)
    d_offsets = torch.from_numpy(np.asarray(offsets, np.int32)).to(dev)
    d_vertex = torch.tensor(np.asarray(vertex, np.float32), device=dev)
    d_sorted = torch.full((max(len(clusters), 1) * 36,), 0xAB, dtype=torch.uint8, device=dev)
    d_tables = torch.full((6 * 401,), -7, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    st = lib.itsu_pvc_initialize_noalloc(
        ctypes.c_void_p(d_clusters.data_ptr()), ctypes.c_void_p(d_offsets.data_ptr()), ctypes.c_void_p(d_vertex.data_ptr()),
        len(clusters), ctypes.c_void_p(d_sorted.data_ptr()), ctypes.c_void_p(d_tables.data_ptr()), ctypes.c_void_p(stream))
    return st, d_sorted, d_tables


def _noalloc(lib, ev, vertex, stream):
    import torch

    clusters = np.concatenate(ev.layers)
    offsets = np.zeros(8, np.int32)
    offsets[1:] = np.cumsum([len(l) for l in ev.layers])
    dev = torch.device("cuda", 0)
    d_clusters = torch.from_numpy(clusters.view(np.uint8).copy()).to(dev)
    d_offsets = torch.from_numpy(offsets).to(dev)
    d_vertex = torch.tensor(np.asarray(vertex, np.float32), device=dev)
    d_sorted = torch.full((len(clusters) * 36,), 0xAB, dtype=torch.uint8, device=dev)
    d_tables = torch.full((6 * 401,), -7, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    st = lib.itsu_pvc_initialize_noalloc(
        ctypes.c_void_p(d_clusters.data_ptr()), ctypes.c_void_p(d_offsets.data_ptr()), ctypes.c_void_p(d_vertex.data_ptr()),
        len(clusters), ctypes.c_void_p(d_sorted.data_ptr()), ctypes.c_void_p(d_tables.data_ptr()), ctypes.c_void_p(stream))
    assert st == capi.OK, lib.itsu_last_error(None).decode()
    sorted_ = d_sorted.cpu().numpy().view(gen.CLUSTER_DTYPE)
    return [sorted_[offsets[l]:offsets[l + 1]] for l in range(7)], d_tables.cpu().numpy().reshape(6, 401)


def test_noalloc_clustering_matches_the_allocating_entry_point():
    import torch

    torch.cuda.init()
    stream = torch.cuda.Stream()
    ctx = capi.Context(device=0)
    lib = ctx.lib
    try:
        # a larger event first, then a smaller one: stale scratch from the first must not matter
        for ev in (gen.pbpb_event(21, n_tracks=3000), gen.pp_event(22)):
            got_clusters, got_tables = _noalloc(lib, ev, ev.vertices[0], stream.cuda_stream)
            ctx.initialize(ev.layers, ev.vertices[0])
            want = ctx.results(0)
            for l in range(7):
                assert np.array_equal(got_clusters[l].view(np.uint8), want["clusters"][l].view(np.uint8)), l
            assert np.array_equal(got_tables, want["index_tables"])
    finally:
        ctx.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = capi.load()
    limit = 65536  # ITSU_NOALLOC_MAX_CLUSTERS
    st = lib.itsu_pvc_initialize_noalloc(None, None, None, limit + 1, None, None, None)
    assert st == capi.ERR_CAPACITY
    assert b"65536" in lib.itsu_last_error(None)


def test_noalloc_reports_malformed_inputs():
    """A non-finite vertex and a cluster beyond 1e6 cm are found on the device, decreasing layer
    offsets on the host before anything is launched; each is ITSU_ERR_INVALID with its reason,
    and a well-formed call right after still gives the allocating entry point's result (the
    status word in the shared scratch is cleared by every call)."""
    import torch

    torch.cuda.init()
    stream = torch.cuda.Stream()
    lib = capi.load()
    ev = gen.pp_event(23)
    clusters = np.concatenate(ev.layers)
    offsets = np.zeros(8, np.int32)
    offsets[1:] = np.cumsum([len(l) for l in ev.layers])

    st, _, _ = _noalloc_call(lib, clusters, offsets, [0.0, float("nan"), 0.0], stream.cuda_stream)
    assert st == capi.ERR_INVALID
    assert b"primary vertex" in lib.itsu_last_error(None)

    far = clusters.copy()
    far["z"][offsets[3] + 1] = 2.0e6
    st, _, _ = _noalloc_call(lib, far, offsets, ev.vertices[0], stream.cuda_stream)
    assert st == capi.ERR_INVALID
    msg = lib.itsu_last_error(None)
    assert b"cluster" in msg and str(offsets[3] + 1).encode() in msg

    bad = offsets.copy()
    bad[2], bad[3] = bad[3], bad[2]  # layer 2 ends before it starts
    st, _, _ = _noalloc_call(lib, clusters, bad, ev.vertices[0], stream.cuda_stream)
    assert st == capi.ERR_INVALID
    assert b"decrease" in lib.itsu_last_error(None)

    ctx = capi.Context(device=0)
    try:
        got_clusters, got_tables = _noalloc(lib, ev, ev.vertices[0], stream.cuda_stream)
        ctx.initialize(ev.layers, ev.vertices[0])
        want = ctx.results(0)
        for l in range(7):
            assert np.array_equal(got_clusters[l].view(np.uint8), want["clusters"][l].view(np.uint8)), l
        assert np.array_equal(got_tables, want["index_tables"])
    finally:
        ctx.close()
