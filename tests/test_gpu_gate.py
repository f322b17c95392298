"""The learned tracklet gate on the GPU: sample export, the gate pass of the tracklet stage, the
scorer, training gradients and the committed checkpoint.

The plain path is the yardstick: a gated run must keep exactly the plain tracklets the gate scores at
or above its threshold (inner clusters with more than 48 tracklets keep all of theirs), in the
plain run's order; it must equal the plain run when the threshold keeps everything; and its roads
must be exactly the plain roads whose 6 tracklets all survive.
"""
import os

import numpy as np
import pytest

from itsu import capi, gen, prefilter
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_dev():
    import torch

    torch.cuda.init()
    return torch.device("cuda", 0)


@pytest.fixture(scope="module")
def ctx(torch_dev):
    c = capi.Context(device=0)
    yield c
    c.close()


def _gate(features, seed=3, threshold=0.0):
    m = capi.gate_init(seed)
    f = features[np.isfinite(features).all(axis=1)]
    mean, std = f.mean(axis=0), f.std(axis=0)
    std[std == 0] = 1.0
    for k in range(8):
        m.mean[k], m.inv_std[k] = float(mean[k]), float(1.0 / std[k])
    m.logit_threshold = threshold
    return m


def _score(ctx, features, torch_dev):
    import torch

    f = features if hasattr(features, "data_ptr") else torch.from_numpy(np.ascontiguousarray(features)).to(torch_dev)
    out = torch.empty(max(len(f), 1), dtype=torch.float32, device=torch_dev)
    ctx.gate_score(f.data_ptr(), len(f), out.data_ptr())
    return out[:len(f)].cpu().numpy()


def _plain(ctx, torch_dev, events):
    b = prefilter.DeviceBatch(ctx, events, torch_dev)
    prefilter.set_learned(ctx, False, False)
    ctx.batch_run(b.batch)
    f, l, r = prefilter.export_gate_samples(ctx, torch_dev)
    return b, f, l, r


def test_gate_export_matches_oracle_tracklets(ctx, torch_dev):
    """Features equal to the float32 restatement on the oracle's tracklets (bit for bit where the
    device uses IEEE operations; the slope, dz and curvature use the hardware's fast division and
    reciprocal square root, within 1e-5 relative + 1e-6 absolute); labels and road rows from the
    oracle's roads."""
    ev = gen.pbpb_event(61, n_tracks=1500)
    want = oracle.run_vertex(ev.layers, ev.vertices[0])
    ctx.run_vertex(ev.layers, ev.vertices[0])
    f, l, r = prefilter.export_gate_samples(ctx, torch_dev)
    feats = prefilter.tracklet_features(want)
    got = f.cpu().numpy()
    assert got.shape[0] == len(feats) > 0
    exact = [0, 4, 5, 7]
    assert np.array_equal(got[:, exact].view(np.uint32), feats[:, exact].view(np.uint32))
    # the slope and the curvature: a few units in the last place
    for col in (3, 6):
        assert np.all(np.abs(got[:, col] - feats[:, col]) <= 1e-7 + 1e-5 * np.abs(feats[:, col])), col
    # dz = slope * (r2 - r1) + z1 - z2: the slope's error times the radius step, against terms of
    # tens of cm (the cut it is compared with is 0.1-0.3 cm)
    for col in (1, 2):
        assert np.all(np.abs(got[:, col] - feats[:, col]) <= 2e-5), col
    rows = prefilter.road_tracklets(want)
    assert np.array_equal(r.cpu().numpy(), rows)
    labels = np.zeros(len(feats), np.uint8)
    labels[rows.ravel()] = 1
    assert np.array_equal(l.cpu().numpy(), labels)


def test_gate_scorer_matches_numpy_reference(ctx, torch_dev):
    """Tensor-core logits vs a float64 restatement with the same BF16 roundings (ReLU is exact; a
    different FP32 summation order can move a BF16 activation by one unit): 0.02 absolute + 1%
    relative on the logit."""
    ev = gen.pbpb_event(62, n_tracks=1500)
    feats = prefilter.tracklet_features(oracle.run_vertex(ev.layers, ev.vertices[0]))
    m = _gate(feats)
    rng = np.random.default_rng(5)
    m.b3 = 0.3
    for k in range(16):
        m.b1[k], m.b2[k] = float(rng.normal(0, 0.2)), float(rng.normal(0, 0.2))
    ctx.gate_set_model(m)
    got = _score(ctx, feats, torch_dev)
    ref = prefilter.mlp_forward(m.arrays(), feats, act="relu")["z"]
    err = np.abs(got - ref)
    assert np.all(err <= 0.02 + 0.01 * np.abs(ref)), (err.max(), np.argmax(err))
    assert np.corrcoef(got, ref)[0, 1] > 0.9999
    assert np.std(ref) > 0.05


def test_gate_threshold_minus_infinity_gives_the_plain_run(ctx, torch_dev):
    events = [gen.pbpb_event(s, n_tracks=2000) for s in (63, 64)] + [gen.pp_event(65), gen.jet_event(5)]
    b, f, _, _ = _plain(ctx, torch_dev, events)
    plain = [ctx.results(e) for e in range(len(events))]
    ctx.gate_set_model(_gate(f.cpu().numpy(), threshold=float("-inf")))
    prefilter.set_learned(ctx, False, True)
    try:
        ctx.batch_run(b.batch)
        for e in range(len(events)):
            assert oracle.diff(ctx.results(e), plain[e]) == [], e
    finally:
        prefilter.set_learned(ctx, False, False)


def _windows_at(features, q):
    """Per inner layer, the q-quantiles of the plain tracklets' |dphi| and |dz| (features 0 and 2),
    as float32."""
    wphi = np.full(6, np.pi, np.float32)
    wz = np.full(6, np.inf, np.float32)
    for layer in range(6):
        on = features[:, 4] == layer
        if on.any():
            wphi[layer] = np.float32(np.quantile(features[on, 0], q))
            wz[layer] = np.float32(np.quantile(features[on, 2], q))
    return wphi, wz


def _set_windows(m, wphi, wz):
    for layer in range(6):
        m.dphi_window[layer] = float(wphi[layer])
        m.dz_window[layer] = float(wz[layer])


@pytest.mark.parametrize("window_q,mlp_layers", [(None, 0x3f), (0.9, 0x3f), (0.9, 0x2b)])
def test_gate_keeps_exactly_what_the_scorer_keeps(ctx, torch_dev, window_q, mlp_layers):
    """Threshold at the 12% quantile of an untrained gate's logits, on central events and a dense
    jet (inner clusters with more than 48 tracklets): the gated run's tracklets are the plain
    tracklets scored at or above it (all of a crowded cluster's), in order; its roads are exactly
    the plain roads whose 6 tracklets all survive, with the same labels. With the cascade's first
    stage (window_q: per layer, |dphi| and |dz| windows at that quantile of the layer's plain
    tracklets),
    only the tracklets inside the window are scored or kept, and a cluster is crowded by the
    tracklets inside it. mlp_layers: the layers the network scores (the others keep every tracklet
    inside the windows)."""
    events = [gen.pbpb_event(s, n_tracks=2500) for s in (66, 67)] + [gen.jet_event(5)]
    b, f, l, r = _plain(ctx, torch_dev, events)
    pkeys, pfake = prefilter.export_roads(ctx, torch_dev)
    plain = [ctx.results(e) for e in range(len(events))]
    fn = f.cpu().numpy()
    m = _gate(fn, seed=11)
    inside = np.ones(len(fn), bool)
    if window_q is not None:
        wphi, wz = _windows_at(fn, window_q)
        _set_windows(m, wphi, wz)
        inside = prefilter.window_pass(fn, wphi, wz)
        assert 0.7 < inside.mean() < 0.9
    m.mlp_layers = mlp_layers
    ctx.gate_set_model(m)
    logits = _score(ctx, f, torch_dev)
    scored = inside & (((mlp_layers >> fn[:, 4].astype(np.int64)) & 1) == 1)
    thr = float(np.quantile(logits[scored], 0.12))  # keeps about 88%: some roads keep all 6 tracklets
    m.logit_threshold = thr
    ctx.gate_set_model(m)
    keep = (~(logits < thr) | ~scored) & inside
    # inner clusters with more than 48 tracklets (inside the window) keep all of them
    row = 0
    crowded = 0
    for e in range(len(events)):
        for layer in range(6):
            t = plain[e]["tracklets"][layer]
            ins = inside[row:row + len(t)]
            per = np.bincount(t["c1"][ins], minlength=len(plain[e]["clusters"][layer]))
            big = (per[t["c1"]] > 48) & ins
            keep[row:row + len(t)] |= big
            crowded += int(big.sum())
            row += len(t)
    assert row == len(keep)
    if window_q is None:
        assert crowded > 0
        assert 0.8 < keep.mean() < 0.95
    else:
        assert 0.55 < keep.mean() < 0.85
    prefilter.set_learned(ctx, False, True)
    try:
        ctx.batch_run(b.batch)
        lkeys, lfake = prefilter.export_roads(ctx, torch_dev)
        row = 0
        for e in range(len(events)):
            got = ctx.results(e)
            for layer in range(6):
                pt = plain[e]["tracklets"][layer]
                kept = pt[keep[row:row + len(pt)]]
                row += len(pt)
                assert np.array_equal(got["tracklets"][layer].view(np.uint8), kept.view(np.uint8)), (e, layer)
    finally:
        prefilter.set_learned(ctx, False, False)
    rows = r.cpu().numpy().astype(np.int64)
    survives = np.append(keep, True)[rows].all(axis=1)  # row -1: no tracklet in that layer
    cmp = prefilter.compare_roads(pkeys, pfake, lkeys, lfake)
    assert cmp["extra"] == 0 and cmp["extra_fakes"] == 0
    assert cmp["reproduced"] == int(survives.sum()) == cmp["learned_roads"]
    assert 0 < cmp["reproduced"] < cmp["plain_roads"]
    # the surviving roads keep their Monte Carlo labels and fake flags (same 7 clusters)
    lab = {bytes(k): fk for k, fk in zip(np.ascontiguousarray(pkeys), pfake)}
    assert all(lab[bytes(k)] == fk for k, fk in zip(np.ascontiguousarray(lkeys), lfake))


def test_gate_window_alone_keeps_the_tracklets_inside_it(ctx, torch_dev):
    """The cascade's first stage alone (threshold -inf), the windows at each layer's median |dphi|
    and |dz|: the gated run's tracklets are the plain tracklets inside their layer's windows, in
    order, on central, pp and jet events and across the phi wrap; a zero window keeps only exact
    zeros, and the other layers' windows do not change."""
    events = [gen.pbpb_event(s, n_tracks=2000) for s in (68, 69)] + [gen.pp_event(70), gen.jet_event(5)]
    b, f, _, _ = _plain(ctx, torch_dev, events)
    plain = [ctx.results(e) for e in range(len(events))]
    fn = f.cpu().numpy()
    m = _gate(fn, threshold=float("-inf"))
    wphi, wz = _windows_at(fn, 0.5)
    _set_windows(m, wphi, wz)
    inside = prefilter.window_pass(fn, wphi, wz)
    assert 0.15 < inside.mean() < 0.5
    # some kept tracklets cross phi = 0 (their clusters on both sides of the wrap)
    wraps = 0
    row = 0
    for e in range(len(events)):
        for layer in range(6):
            t = plain[e]["tracklets"][layer]
            p1 = plain[e]["clusters"][layer]["phi"][t["c1"]]
            p2 = plain[e]["clusters"][layer + 1]["phi"][t["c2"]]
            wraps += int((inside[row:row + len(t)] & (np.abs(p1 - p2) > np.pi)).sum())
            row += len(t)
    assert wraps > 0
    ctx.gate_set_model(m)
    prefilter.set_learned(ctx, False, True)
    try:
        ctx.batch_run(b.batch)
        row = 0
        layer3 = []
        for e in range(len(events)):
            got = ctx.results(e)
            layer3.append(got["tracklets"][3].copy())
            for layer in range(6):
                pt = plain[e]["tracklets"][layer]
                kept = pt[inside[row:row + len(pt)]]
                row += len(pt)
                assert np.array_equal(got["tracklets"][layer].view(np.uint8), kept.view(np.uint8)), (e, layer)
        # zero windows keep only the tracklets at exactly zero |dphi| (layer 2) or |dz| (layer 4)
        wphi[2], wz[4] = 0.0, 0.0
        _set_windows(m, wphi, wz)
        inside = prefilter.window_pass(fn, wphi, wz)
        ctx.gate_set_model(m)
        ctx.batch_run(b.batch)
        row = 0
        for e in range(len(events)):
            got = ctx.results(e)["tracklets"]
            for layer in range(6):
                pt = plain[e]["tracklets"][layer]
                kept = pt[inside[row:row + len(pt)]]
                row += len(pt)
                assert np.array_equal(got[layer].view(np.uint8), kept.view(np.uint8)), (e, layer)
            assert np.array_equal(got[3].view(np.uint8), layer3[e].view(np.uint8)), e
        assert sum(len(t) for t in layer3) > 0
    finally:
        prefilter.set_learned(ctx, False, False)


def test_gate_and_pair_prefilter_together(ctx, torch_dev):
    """Both learned networks on: the result is the gated run's cells filtered by the pair scores,
    and every road is a plain road."""
    events = [gen.pbpb_event(s, n_tracks=2000) for s in (68, 69)]
    b, f, _, _ = _plain(ctx, torch_dev, events)
    pkeys, pfake = prefilter.export_roads(ctx, torch_dev)
    gm = _gate(f.cpu().numpy(), seed=12)
    ctx.gate_set_model(gm)
    logits = _score(ctx, f, torch_dev)
    gm.logit_threshold = float(np.quantile(logits, 0.3))
    ctx.gate_set_model(gm)
    prefilter.set_learned(ctx, False, True)
    ctx.batch_run(b.batch)
    pf, _, _ = prefilter.export_samples(ctx, torch_dev)
    pm = capi.prefilter_init(13)
    ff = pf.cpu().numpy()
    mean, std = ff.mean(axis=0), ff.std(axis=0)
    std[std == 0] = 1.0
    for k in range(8):
        pm.mean[k], pm.inv_std[k] = float(mean[k]), float(1.0 / std[k])
    ctx.prefilter_set_model(pm)
    pl = prefilter.score(ctx, pf, torch_dev).cpu().numpy()
    pm.logit_threshold = float(np.quantile(pl, 0.3))
    ctx.prefilter_set_model(pm)
    gated = [ctx.results(e) for e in range(len(events))]
    prefilter.set_learned(ctx, True, True)
    try:
        ctx.batch_run(b.batch)
        both = [ctx.results(e) for e in range(len(events))]
        lkeys, lfake = prefilter.export_roads(ctx, torch_dev)
    finally:
        prefilter.set_learned(ctx, False, False)
    keep = ~(pl < pm.logit_threshold)
    row = 0
    for e in range(len(events)):
        assert all(np.array_equal(both[e]["tracklets"][l].view(np.uint8), gated[e]["tracklets"][l].view(np.uint8))
                   for l in range(6)), e
        for layer in range(5):
            gc = gated[e]["cells"][layer]
            kept = gc[keep[row:row + len(gc)]]
            row += len(gc)
            assert np.array_equal(both[e]["cells"][layer]["c3"], kept["c3"]), (e, layer)
    cmp = prefilter.compare_roads(pkeys, pfake, lkeys, lfake)
    assert cmp["extra"] == 0 and 0 < cmp["learned_roads"] < cmp["plain_roads"]


def test_gate_gradient_matches_numpy_reference(ctx, torch_dev):
    """Device minibatch gradient of the gate vs the float64 restatement: relative error of each
    parameter block below 3%, loss within 1e-3."""
    import torch

    ev = gen.pbpb_event(70, n_tracks=1500)
    feats = prefilter.tracklet_features(oracle.run_vertex(ev.layers, ev.vertices[0]))[:1000]
    labels = np.zeros(len(feats), np.uint8)
    labels[::4] = 1
    m = _gate(feats, seed=13)
    rng = np.random.default_rng(6)
    for k in range(16):
        m.b1[k], m.b2[k] = float(rng.normal(0, 0.2)), float(rng.normal(0, 0.2))
    ctx.gate_set_model(m)
    df = torch.from_numpy(feats).to(torch_dev)
    dl = torch.from_numpy(labels).to(torch_dev)
    g, loss = ctx.gate_gradient(df.data_ptr(), dl.data_ptr(), len(feats), 2.0)
    gr, lr = prefilter.mlp_gradient(m.arrays(), feats, labels, 2.0, act="relu")
    assert abs(loss - lr) <= 1e-3 * max(1.0, abs(lr))
    bounds = [0, 128, 144, 400, 416, 432, 433]
    for a, b in zip(bounds[:-1], bounds[1:]):
        rel = np.linalg.norm(g[a:b] - gr[a:b]) / max(np.linalg.norm(gr[a:b]), 1e-12)
        assert rel < 0.03, (a, b, rel)


def test_gate_training_lowers_the_loss(ctx, torch_dev):
    events = [gen.pbpb_event(s, n_tracks=3000) for s in (71, 72)]
    _, f, l, _ = _plain(ctx, torch_dev, events)
    ctx.gate_set_model(_gate(f.cpu().numpy(), seed=17))
    before = ctx.gate_get_model().params()
    cfg = capi.train_config(steps=400, batch=4096, lr=3e-3, lr_final=3e-4, seed=5)
    losses = ctx.gate_train(f.data_ptr(), l.data_ptr(), len(f), cfg)
    after = ctx.gate_get_model()
    assert np.isfinite(losses).all()
    assert losses[-50:].mean() < 0.85 * losses[:50].mean()
    assert not np.array_equal(before, after.params())


@pytest.mark.skipif(not os.path.exists(prefilter.GATE_CHECKPOINTS["pbpb"]), reason="no trained gate checkpoint")
def test_committed_gate_reproduces_plain_roads(ctx, torch_dev):
    """Held-out central Pb-Pb-like events (seeds after the evaluation set): the gate alone keeps at
    least 99.5% of the plain roads and no road the plain path lacks, with fewer tracklets."""
    gate = capi.gate_load(prefilter.GATE_CHECKPOINTS["pbpb"])
    seeds = range(prefilter.EVAL_SEED0 + 1000, prefilter.EVAL_SEED0 + 1008)
    res = prefilter.evaluate(ctx, None, seeds, torch_dev, chunk=8, workers=1, log=lambda *a: None, gate=gate)
    assert res["extra"] == 0
    assert res["road_reproduction"] >= 0.995, res
    assert res["tracklets_kept"] < 0.5, res


def test_gate_windows_on_pileup_frames(ctx, torch_dev):
    """Frames of 3 collisions (every vertex of a frame is one run over the frame's clusters): the
    windows apply per run, about that run's vertex; each run's gated tracklets are its plain
    tracklets inside the windows, in order, and the gated roads are plain roads."""
    frames = gen.pileup_stream(19, n_frames=2, collisions=3, n_tracks=400)
    clusters, offsets, vertices, vertex_frame = gen.pack_frames(frames)
    prefilter.set_learned(ctx, False, False)
    ctx.frames_run_host(clusters, offsets, vertices, vertex_frame)
    n_runs = len(vertex_frame)
    plain = [ctx.results(v) for v in range(n_runs)]
    f, _, _ = prefilter.export_gate_samples(ctx, torch_dev)
    pkeys, _ = prefilter.export_roads(ctx, torch_dev)
    fn = f.cpu().numpy()
    m = _gate(fn, threshold=float("-inf"))
    wphi, wz = _windows_at(fn, 0.6)
    _set_windows(m, wphi, wz)
    inside = prefilter.window_pass(fn, wphi, wz)
    ctx.gate_set_model(m)
    prefilter.set_learned(ctx, False, True)
    try:
        ctx.frames_run_host(clusters, offsets, vertices, vertex_frame)
        lkeys, _ = prefilter.export_roads(ctx, torch_dev)
        row = 0
        for v in range(n_runs):
            got = ctx.results(v)
            for layer in range(6):
                pt = plain[v]["tracklets"][layer]
                kept = pt[inside[row:row + len(pt)]]
                row += len(pt)
                assert np.array_equal(got["tracklets"][layer].view(np.uint8), kept.view(np.uint8)), (v, layer)
        assert row == len(fn)
    finally:
        prefilter.set_learned(ctx, False, False)
    p = {bytes(r) for r in np.ascontiguousarray(pkeys)}
    assert all(bytes(r) in p for r in np.ascontiguousarray(lkeys))
    assert 0 < len(lkeys) < len(pkeys)


def test_gate_through_the_streamed_host_call(ctx, torch_dev):
    """The learned form through the streamed host call (chunks on two arenas, the context's gate
    serving both): the same roads as the one-pass call with the same gate."""
    events = [gen.pbpb_event(s, n_tracks=2500) for s in (74, 75)] + gen.batch_events(76, n_events=10)
    clusters, offsets, vertices = gen.pack_batch(events)
    _, f, _, _ = _plain(ctx, torch_dev, events)
    m = _gate(f.cpu().numpy(), threshold=float("-inf"))
    wphi, wz = _windows_at(f.cpu().numpy(), 0.7)
    _set_windows(m, wphi, wz)
    one = capi.Context(device=0)
    streamed = capi.Context(device=0, flags=capi.FLAG_STREAM_HOST, stream_chunk_clusters=40000)
    try:
        plain_roads, _ = one.batch_run_host(clusters, offsets, vertices)
        for c in (one, streamed):
            c.gate_set_model(m)
            c.gate_enable(True)
        want_roads, want_off = one.batch_run_host(clusters, offsets, vertices)
        got_roads, got_off = streamed.batch_run_host_tracks(capi.track_clusters(clusters), offsets, vertices)
        assert np.array_equal(want_off, got_off)
        assert np.array_equal(want_roads.view(np.uint8), got_roads.view(np.uint8))
        assert 0 < len(want_roads) < len(plain_roads)
    finally:
        one.close()
        streamed.close()
