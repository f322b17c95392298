"""Host-side parts of the learned prefilter (no GPU): the checkpoint format, the seeded
initialisation, the numpy restatements the GPU tests compare against, threshold calibration and
road-set comparison."""
import ctypes
import os

import numpy as np
import pytest

from itsu import capi, gen, prefilter
from oracle import oracle


def test_model_layout_matches_the_header():
    assert ctypes.sizeof(capi.PrefilterModel) == 4 * (capi.MLP_PARAMS + 2 * 8 + 1)
    assert capi.MLP_PARAMS == 4801
    assert ctypes.sizeof(capi.PrefilterSamples) == 72
    assert ctypes.sizeof(capi.TrainConfig) == 56


def test_init_is_seeded():
    a, b, c = capi.prefilter_init(1), capi.prefilter_init(1), capi.prefilter_init(2)
    assert bytes(a) == bytes(b) and bytes(a) != bytes(c)
    p = a.params()
    assert np.all(np.abs(p[:512]) <= np.sqrt(6 / 72) + 1e-7)
    assert np.all(p[512:576] == 0) and a.logit_threshold == 0.0
    assert list(a.inv_std) == [1.0] * 8


def test_checkpoint_round_trip_and_corruption(tmp_path):
    m = capi.prefilter_init(9)
    m.logit_threshold = -1.25
    m.mean[3] = 0.5
    path = str(tmp_path / "m.itsumlp")
    capi.prefilter_save(m, path)
    assert bytes(capi.prefilter_load(path)) == bytes(m)
    raw = bytearray(open(path, "rb").read())
    # a flipped byte anywhere fails the checksum
    bad = bytearray(raw)
    bad[100] ^= 1
    open(path, "wb").write(bytes(bad))
    with pytest.raises(capi.ItsuError) as e:
        capi.prefilter_load(path)
    assert e.value.status == capi.ERR_INVALID and "checksum" in str(e.value)
    # truncated
    open(path, "wb").write(bytes(raw[:-9]))
    with pytest.raises(capi.ItsuError):
        capi.prefilter_load(path)
    # master weights edited and the checksum recomputed: the BF16 copies no longer match
    bad = bytearray(raw[:-8])
    off = 24  # header: 8-byte magic + 4 uint32
    w = np.frombuffer(bytes(bad[off:off + 4]), np.float32)[0]
    bad[off:off + 4] = np.float32(w + 0.5).tobytes()
    h = 0xcbf29ce484222325
    for byte in bad:
        h = ((h ^ byte) * 0x100000001b3) & 0xFFFFFFFFFFFFFFFF
    open(path, "wb").write(bytes(bad) + h.to_bytes(8, "little"))
    with pytest.raises(capi.ItsuError) as e:
        capi.prefilter_load(path)
    assert "BF16" in str(e.value)
    with pytest.raises(capi.ItsuError):
        capi.prefilter_load(str(tmp_path / "missing"))


def test_committed_checkpoint_loads():
    if not os.path.exists(prefilter.CHECKPOINT):
        pytest.skip("no trained checkpoint")
    m = capi.prefilter_load(prefilter.CHECKPOINT)
    assert np.isfinite(m.params()).all() and np.isfinite(m.logit_threshold)


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 3.0e38], np.float32)
    got = prefilter.bf16_round(x)
    assert list(got[:5]) == [1.0, 1.0, 1.0 + 2 ** -6, 1.0, -2.5]  # ties to even, exact values kept
    assert np.isfinite(got[5])


def test_numpy_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    m = capi.prefilter_init(3).arrays()
    m["b1"], m["b2"], m["b3"] = rng.normal(0, 0.1, 64), rng.normal(0, 0.1, 64), 0.1
    f = rng.normal(0, 1, (64, 8)).astype(np.float32)
    y = (rng.random(64) < 0.6).astype(np.float64)
    g, _ = prefilter.mlp_gradient(m, f, y, 1.5, rounding=False)
    flat = np.concatenate([m["w1"].ravel(), m["b1"], m["w2"].ravel(), m["b2"], m["w3"], [m["b3"]]]).astype(np.float64)
    shapes = (("w1", (64, 8)), ("b1", (64,)), ("w2", (64, 64)), ("b2", (64,)), ("w3", (64,)), ("b3", ()))

    def loss_at(v):
        mm, o = dict(m), 0
        for k, shp in shapes:
            n = int(np.prod(shp)) if shp else 1
            mm[k] = v[o:o + n].reshape(shp) if shp else v[o]
            o += n
        return prefilter.mlp_gradient(mm, f, y, 1.5, rounding=False)[1]

    for i in list(rng.choice(len(flat), 30, replace=False)) + [0, 512, 600, 4700, 4750, 4800]:
        up, dn = flat.copy(), flat.copy()
        up[i] += 1e-6
        dn[i] -= 1e-6
        assert abs((loss_at(up) - loss_at(dn)) / 2e-6 - g[i]) < 1e-7 + 1e-5 * abs(g[i])


def test_pair_features_of_oracle_cells():
    """Features of the plain path's cells respect the cuts that made them."""
    ev = gen.pbpb_event(5, n_tracks=800)
    res = oracle.run_vertex(ev.layers, ev.vertices[0])
    f = prefilter.pair_features(res)
    assert len(f) == sum(len(c) for c in res["cells"]) > 0 and np.isfinite(f).all()
    layer = f[:, 6].astype(int)
    assert np.all(f[:, 0] < 0.14) and np.all(f[:, 2] < 0.025)
    assert np.all(f[:, 1] < np.array([0.2, 0.4, 0.5, 0.6, 3.0], np.float32)[layer])
    assert np.all(f[:, 5] <= prefilter.CELL_MAX_DCA[layer])
    rows = prefilter.road_cells(res)
    assert np.all(f[rows, 6] == np.arange(5)[None, :])


def test_calibrate_keeps_the_target_fraction_of_roads():
    rng = np.random.default_rng(1)
    logits = rng.normal(0, 1, 5000).astype(np.float32)
    logits[7] = np.nan  # NaN keeps its cell
    rows = rng.integers(0, 5000, (997, 5))
    for target in (0.9, 0.995, 1.0):
        thr = prefilter.calibrate(logits, rows, target)
        kept = ~(logits < thr)
        assert kept[rows].all(axis=1).mean() >= target
    assert prefilter.calibrate(logits, rows[:0], 0.99) == float("-inf")


def test_compare_roads():
    p = np.array([[0, 1, 2, 3, 4, 5, 6, 7], [1, 1, 2, 3, 4, 5, 6, 7], [1, 2, 2, 3, 4, 5, 6, 7]], np.int32)
    l = np.array([[1, 1, 2, 3, 4, 5, 6, 7], [2, 0, 0, 0, 0, 0, 0, 0]], np.int32)
    c = prefilter.compare_roads(p, np.array([0, 1, 0]), l, np.array([1, 1]))
    assert c == dict(plain_roads=3, learned_roads=2, reproduced=1, extra=1, extra_fakes=1, plain_fakes=1, learned_fakes=2)


# ---- the tracklet gate (8 -> 16 -> 16 -> 1, ReLU) ----


def test_gate_model_layout_and_init():
    assert ctypes.sizeof(capi.GateModel) == 4 * (capi.GATE_PARAMS + 2 * 8 + 1 + 12 + 1)
    assert capi.GATE_PARAMS == 433
    assert ctypes.sizeof(capi.GateSamples) == 56
    a, b, c = capi.gate_init(1), capi.gate_init(1), capi.gate_init(2)
    assert bytes(a) == bytes(b) and bytes(a) != bytes(c)
    p = a.params()
    assert np.all(np.abs(p[:128]) <= np.sqrt(6 / 24) + 1e-7)
    assert np.all(p[128:144] == 0) and a.logit_threshold == 0.0
    assert list(a.dphi_window) == [np.float32(np.pi)] * 6  # no first stage until trained
    assert list(a.dz_window) == [np.inf] * 6
    assert a.mlp_layers == 0x3f


def test_gate_windows_fit_the_road_tracklets():
    """The cascade's first stage: per layer, the margin times the largest |dphi| and |dz| of the
    tracklets on roads (|dphi| at most the tracklet cut's 0.3); a layer without road tracklets
    keeps no window; the test is inclusive."""
    rng = np.random.default_rng(3)
    f = np.zeros((600, 8), np.float32)
    f[:, 4] = np.repeat(np.arange(6), 100)
    f[:, 0] = rng.uniform(0, 0.3, 600)
    f[:, 2] = rng.uniform(0, 0.2, 600)
    on_road = np.flatnonzero((f[:, 4] != 5) & (rng.random(600) < 0.2))
    f[on_road[0], 0] = 0.29  # its window would pass the cut
    rows = np.full((len(on_road), 6), -1, np.int64)
    rows[:, 0] = on_road
    wphi, wz = prefilter.fit_windows(f, rows, margin=1.25)
    for layer in range(5):
        r = on_road[f[on_road, 4] == layer]
        assert wphi[layer] == np.float32(min(0.3, 1.25 * f[r, 0].astype(np.float64).max()))
        assert wz[layer] == np.float32(1.25 * f[r, 2].astype(np.float64).max())
    assert wphi[5] == np.float32(0.3) and wz[5] == np.inf
    assert wphi[int(f[on_road[0], 4])] == np.float32(0.3)
    ok = prefilter.window_pass(f, wphi, wz)
    assert ok[on_road].all()
    edge = f.copy()
    edge[:, 0] = wphi[edge[:, 4].astype(int)]
    edge[:, 2] = wz[edge[:, 4].astype(int)]
    assert prefilter.window_pass(edge, wphi, wz).all()
    edge[:, 2] = np.nextafter(edge[:, 2], np.float32(np.inf))
    assert not prefilter.window_pass(edge, wphi, wz)[:500].any()


def test_gate_checkpoint_round_trip_and_kinds(tmp_path):
    """The gate's checkpoint has its own magic: neither kind loads as the other."""
    g = capi.gate_init(4)
    g.logit_threshold = -2.5
    g.dphi_window[3] = 0.0625
    g.dz_window[1] = 0.03125
    g.mlp_layers = 0x2d
    path = str(tmp_path / "g.itsugate")
    capi.gate_save(g, path)
    assert bytes(capi.gate_load(path)) == bytes(g)
    with pytest.raises(capi.ItsuError):
        capi.prefilter_load(path)
    pair = str(tmp_path / "p.itsumlp")
    capi.prefilter_save(capi.prefilter_init(4), pair)
    with pytest.raises(capi.ItsuError):
        capi.gate_load(pair)
    raw = bytearray(open(path, "rb").read())
    raw[60] ^= 1
    open(path, "wb").write(bytes(raw))
    with pytest.raises(capi.ItsuError) as e:
        capi.gate_load(path)
    assert "checksum" in str(e.value)


def test_gate_numpy_gradient_matches_finite_differences():
    rng = np.random.default_rng(2)
    m = capi.gate_init(3).arrays()
    m["b1"], m["b2"], m["b3"] = rng.normal(0, 0.1, 16), rng.normal(0, 0.1, 16), 0.1
    f = rng.normal(0, 1, (64, 8)).astype(np.float32)
    y = (rng.random(64) < 0.3).astype(np.float64)
    g, _ = prefilter.mlp_gradient(m, f, y, 2.0, rounding=False, act="relu")
    flat = np.concatenate([m["w1"].ravel(), m["b1"], m["w2"].ravel(), m["b2"], m["w3"], [m["b3"]]]).astype(np.float64)
    assert len(flat) == capi.GATE_PARAMS
    shapes = (("w1", (16, 8)), ("b1", (16,)), ("w2", (16, 16)), ("b2", (16,)), ("w3", (16,)), ("b3", ()))

    def loss_at(v):
        mm, o = dict(m), 0
        for k, shp in shapes:
            n = int(np.prod(shp)) if shp else 1
            mm[k] = v[o:o + n].reshape(shp) if shp else v[o]
            o += n
        return prefilter.mlp_gradient(mm, f, y, 2.0, rounding=False, act="relu")[1]

    for i in list(rng.choice(len(flat), 30, replace=False)) + [0, 128, 150, 400, 420, 432]:
        up, dn = flat.copy(), flat.copy()
        up[i] += 1e-6
        dn[i] -= 1e-6
        assert abs((loss_at(up) - loss_at(dn)) / 2e-6 - g[i]) < 1e-7 + 1e-5 * abs(g[i])


def test_tracklet_features_of_oracle_tracklets():
    """The gate's features of the plain path's tracklets respect the tracklet cuts that made them
    (Tracker.cxx:93-100), and each road's 6 tracklet rows run through layers 0..5."""
    ev = gen.pbpb_event(6, n_tracks=800)
    res = oracle.run_vertex(ev.layers, ev.vertices[0])
    f = prefilter.tracklet_features(res)
    assert len(f) == sum(len(t) for t in res["tracklets"]) > 0 and np.isfinite(f).all()
    layer = f[:, 4].astype(int)
    assert np.all(f[:, 2] < np.array([0.1, 0.1, 0.3, 0.3, 0.3, 0.3], np.float32)[layer])
    assert np.all(f[:, 0] < 0.3) and np.all(f[:, 0] == np.abs(f[:, 7])) and np.all(f[:, 2] == np.abs(f[:, 1]))
    rows = prefilter.road_tracklets(res)
    assert len(rows) == len(res["roads"]) > 0
    assert np.all(f[rows, 4] == np.arange(6)[None, :])


def test_committed_gate_checkpoint_loads():
    path = prefilter.GATE_CHECKPOINTS["pbpb"]
    if not os.path.exists(path):
        pytest.skip("no trained gate checkpoint")
    m = capi.gate_load(path)
    assert np.isfinite(m.params()).all() and np.isfinite(m.logit_threshold)
