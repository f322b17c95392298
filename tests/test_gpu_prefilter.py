"""The learned prefilter on the GPU: sample export, the fused inference in the cell stage, the
scorer, training gradients and the committed checkpoint.

The plain path is the yardstick: a learned run must keep exactly the plain cells its model scores at
or above the threshold (the fused kernel and the scorer share their device code), it must equal
the plain run when the threshold keeps everything, and its roads must be plain roads.
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


def _model(features, seed=3, threshold=0.0):
    m = capi.prefilter_init(seed)
    f = features[np.isfinite(features).all(axis=1)]
    mean, std = f.mean(axis=0), f.std(axis=0)
    std[std == 0] = 1.0
    for k in range(8):
        m.mean[k], m.inv_std[k] = float(mean[k]), float(1.0 / std[k])
    m.logit_threshold = threshold
    return m


def _plain_samples(ctx, torch_dev, events):
    b = prefilter.DeviceBatch(ctx, events, torch_dev)
    ctx.prefilter_enable(False)
    ctx.batch_run(b.batch)
    f, l, r = prefilter.export_samples(ctx, torch_dev)
    return b, f, l, r


def test_export_matches_oracle_cells_and_roads(ctx, torch_dev):
    """Features bit-exact to the float32 restatement on the oracle's cells; labels and road rows
    from the oracle's roads; road keys are the roads' 7 clusters."""
    ev = gen.pbpb_event(41, n_tracks=1500)
    want = oracle.run_vertex(ev.layers, ev.vertices[0])
    ctx.run_vertex(ev.layers, ev.vertices[0])
    f, l, r = prefilter.export_samples(ctx, torch_dev)
    feats = prefilter.pair_features(want)
    assert f.shape[0] == len(feats) > 0
    assert np.array_equal(f.cpu().numpy().view(np.uint32), feats.view(np.uint32))
    rows = prefilter.road_cells(want)
    assert np.array_equal(r.cpu().numpy(), rows)
    labels = np.zeros(len(feats), np.uint8)
    labels[rows.ravel()] = 1
    assert np.array_equal(l.cpu().numpy(), labels)
    keys, fake = prefilter.export_roads(ctx, torch_dev)
    c0 = want["cells"][0][want["roads"]["cells"][:, 0]]
    expect = np.stack([np.zeros(len(rows), np.int32), c0["c1"], c0["c2"]] +
                      [want["cells"][k][want["roads"]["cells"][:, k]]["c3"] for k in range(5)], axis=1)
    assert np.array_equal(keys, expect)
    assert np.array_equal(fake, want["roads"]["fake"])


def test_scorer_matches_numpy_reference(ctx, torch_dev):
    """Tensor-core logits vs a float64 restatement with the same BF16 roundings. The device's
    GELU uses the hardware tanh approximation (about 2^-11 relative), which can move a BF16
    activation by one unit: the tolerance is 0.02 absolute + 1% relative on the logit."""
    import torch

    ev = gen.pbpb_event(42, n_tracks=1500)
    want = oracle.run_vertex(ev.layers, ev.vertices[0])
    feats = prefilter.pair_features(want)
    m = _model(feats)
    rng = np.random.default_rng(5)
    m.b3 = 0.3
    for k in range(64):
        m.b1[k], m.b2[k] = float(rng.normal(0, 0.2)), float(rng.normal(0, 0.2))
    ctx.prefilter_set_model(m)
    got = prefilter.score(ctx, torch.from_numpy(feats).to(torch_dev), torch_dev).cpu().numpy()
    ref = prefilter.mlp_forward(m.arrays(), feats)["z"]
    err = np.abs(got - ref)
    assert np.all(err <= 0.02 + 0.01 * np.abs(ref)), (err.max(), np.argmax(err))
    assert np.corrcoef(got, ref)[0, 1] > 0.9999
    # a wrong row, column or layer layout in the MMA fragments would be far off
    assert np.std(ref) > 0.05


def test_threshold_minus_infinity_gives_the_plain_run(ctx, torch_dev):
    events = [gen.pbpb_event(s, n_tracks=2000) for s in (43, 44)] + [gen.pp_event(45)]
    b, f, _, _ = _plain_samples(ctx, torch_dev, events)
    plain = [ctx.results(e) for e in range(len(events))]
    ctx.prefilter_set_model(_model(f.cpu().numpy(), threshold=float("-inf")))
    ctx.prefilter_enable(True)
    try:
        ctx.batch_run(b.batch)
        for e in range(len(events)):
            assert oracle.diff(ctx.results(e), plain[e]) == [], e
    finally:
        ctx.prefilter_enable(False)


def test_fused_inference_keeps_exactly_what_the_scorer_keeps(ctx, torch_dev):
    """Threshold at the median logit: the learned run's cells are the plain cells scored at or
    above it, in order; its roads are the plain roads whose 5 cells all survive."""
    events = [gen.pbpb_event(s, n_tracks=2500) for s in (46, 47, 48)]
    b, f, l, r = _plain_samples(ctx, torch_dev, events)
    pkeys, pfake = prefilter.export_roads(ctx, torch_dev)
    plain = [ctx.results(e) for e in range(len(events))]
    m = _model(f.cpu().numpy(), seed=11)
    ctx.prefilter_set_model(m)
    logits = prefilter.score(ctx, f, torch_dev).cpu().numpy()
    thr = float(np.median(logits))
    m.logit_threshold = thr
    ctx.prefilter_set_model(m)
    keep = ~(logits < thr)
    assert 0.3 < keep.mean() < 0.7
    ctx.prefilter_enable(True)
    try:
        ctx.batch_run(b.batch)
        lkeys, lfake = prefilter.export_roads(ctx, torch_dev)
        row = 0
        for e in range(len(events)):
            got = ctx.results(e)
            for layer in range(5):
                pc = plain[e]["cells"][layer]
                k = keep[row:row + len(pc)]
                row += len(pc)
                kept = pc[k]
                gc = got["cells"][layer]
                assert len(gc) == len(kept), (e, layer)
                for field in ("c1", "c2", "c3", "nx", "ny", "nz", "curvature"):
                    assert np.array_equal(gc[field], kept[field]), (e, layer, field)
        assert row == len(keep)
    finally:
        ctx.prefilter_enable(False)
    rows = r.cpu().numpy()
    survives = keep[rows].all(axis=1)
    cmp = prefilter.compare_roads(pkeys, pfake, lkeys, lfake)
    assert cmp["extra"] == 0
    assert cmp["reproduced"] == int(survives.sum()) == cmp["learned_roads"]


def test_gradient_matches_numpy_reference(ctx, torch_dev):
    """Device minibatch gradient (tensor-core backward, BF16 operands, FP32 accumulation) vs the
    float64 restatement: relative error of each parameter block below 3%, loss within 1e-3."""
    import torch

    ev = gen.pbpb_event(49, n_tracks=1500)
    want = oracle.run_vertex(ev.layers, ev.vertices[0])
    feats = prefilter.pair_features(want)[:1000]
    labels = np.zeros(len(feats), np.uint8)
    labels[::3] = 1
    m = _model(feats, seed=13)
    rng = np.random.default_rng(6)
    for k in range(64):
        m.b1[k], m.b2[k] = float(rng.normal(0, 0.2)), float(rng.normal(0, 0.2))
    ctx.prefilter_set_model(m)
    df = torch.from_numpy(feats).to(torch_dev)
    dl = torch.from_numpy(labels).to(torch_dev)
    g, loss = ctx.prefilter_gradient(df.data_ptr(), dl.data_ptr(), len(feats), 1.5)
    gr, lr = prefilter.mlp_gradient(m.arrays(), feats, labels, 1.5)
    assert abs(loss - lr) <= 1e-3 * max(1.0, abs(lr))
    bounds = [0, 512, 576, 4672, 4736, 4800, 4801]
    for a, b in zip(bounds[:-1], bounds[1:]):
        rel = np.linalg.norm(g[a:b] - gr[a:b]) / max(np.linalg.norm(gr[a:b]), 1e-12)
        assert rel < 0.03, (a, b, rel)


def test_training_lowers_the_loss(ctx, torch_dev):
    events = [gen.pbpb_event(s, n_tracks=3000) for s in (50, 51)]
    _, f, l, _ = _plain_samples(ctx, torch_dev, events)
    m = _model(f.cpu().numpy(), seed=17)
    ctx.prefilter_set_model(m)
    before = ctx.prefilter_get_model().params()
    cfg = capi.train_config(steps=400, batch=4096, lr=3e-3, lr_final=3e-4, seed=5)
    losses = ctx.prefilter_train(f.data_ptr(), l.data_ptr(), len(f), cfg)
    after = ctx.prefilter_get_model()
    assert np.isfinite(losses).all()
    assert losses[-50:].mean() < 0.85 * losses[:50].mean()
    assert not np.array_equal(before, after.params())
    # the device model follows the master: the scorer sees the trained weights
    _, loss_now = ctx.prefilter_gradient(f.data_ptr(), l.data_ptr(), min(len(f), 1 << 20), 1.0)
    assert loss_now < losses[:50].mean()


@pytest.mark.skipif(not os.path.exists(prefilter.CHECKPOINT), reason="no trained checkpoint")
def test_committed_checkpoint_reproduces_plain_roads(ctx, torch_dev):
    """Held-out central Pb-Pb-like events (seeds after the evaluation set): at least 99.5% of the
    plain roads, and no road the plain path lacks."""
    model = capi.prefilter_load(prefilter.CHECKPOINT)
    seeds = range(prefilter.EVAL_SEED0 + 1000, prefilter.EVAL_SEED0 + 1008)
    res = prefilter.evaluate(ctx, model, seeds, torch_dev, chunk=8, workers=1, log=lambda *a: None)
    assert res["extra"] == 0
    assert res["road_reproduction"] >= 0.995, res
    assert res["cells_kept"] < 1.0


@pytest.mark.skipif(not os.path.exists(prefilter.CHECKPOINTS["pileup"]), reason="no trained pile-up checkpoint")
def test_committed_pileup_checkpoint_reproduces_plain_roads(ctx, torch_dev):
    """Held-out pile-up frames (5 collisions each, every vertex a run): at least 99.5% of the plain
    roads, and no road the plain path lacks."""
    model = capi.prefilter_load(prefilter.CHECKPOINTS["pileup"])
    seeds = range(prefilter.EVAL_SEED0 + 2000, prefilter.EVAL_SEED0 + 2006)
    res = prefilter.evaluate(ctx, model, seeds, torch_dev, chunk=6, workers=1, log=lambda *a: None, workload="pileup")
    assert res["extra"] == 0
    assert res["road_reproduction"] >= 0.995, res

