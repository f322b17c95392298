"""The learned form's two networks: training pipelines, threshold calibration, evaluation, and
numpy restatements of their arithmetic (the tests' references).

The tracklet gate (include/itsu.h, itsu_gate_model) is a cascade before the tracklet scan:
learned per-layer windows on |dphi| and |dz| (fit_windows), tested in the tracklet count pass,
then a network (8 -> 16 -> 16 -> 1, ReLU) on the tracklets inside them; a tracklet outside a
window or whose logit is below the gate's threshold is not kept, so the cell stage enumerates only
pairs of kept tracklets. It is trained on one sample per tracklet of plain runs (label 1: a found
road uses it) and calibrated on road reproduction (a road survives iff its 6 tracklets are kept):
``python -m itsu.prefilter --model gate``.

The pair prefilter (itsu_prefilter_model; 8 -> 64 -> 64 -> 1, GELU) scores, inside the cell stage,
each tracklet pair that passes the exact cell cuts; a pair whose logit is below the model's
threshold does not become a cell. Everything below runs through the C ABI on one GPU:

1. ``collect``: plain batched runs over seeded central Pb-Pb-like events (6000 tracks, 5% noise);
   ``itsu_prefilter_export`` gives one sample per cell (its 8 pair features; label 1 when a
   found road uses the cell) and each road's 5 cells as sample rows.
2. ``train``: feature standardisation from the training samples, then ``itsu_prefilter_train``
   (hand-written CUDA forward/backward on the tensor cores, Adam on FP32 master weights).
3. ``calibrate``: the largest logit threshold that keeps all 5 cells of at least ``target`` of
   the training roads (a plain road survives the learned form iff all its cells are kept).
4. ``evaluate``: learned and plain batched runs over held-out events; the fraction of plain
   roads the learned runs reproduce, and the learned roads that the plain runs lack (zero by
   construction: a learned run's cells are a subset of the plain run's, and roads are the
   complete 5-cell chains of the cell graph).

Run ``python -m itsu.prefilter [--workload pbpb|pileup]`` (from tracking-itsu_b200/) on a GPU
machine; it writes ``weights/prefilter_<workload>.itsumlp`` and a JSON report beside it. The
pile-up model learns from frames of 5 collisions (every vertex of a frame is one run).
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing
import os
import time

import numpy as np

from . import capi, gen

TRAIN_SEED0 = 7_000_000  # training events: seeds TRAIN_SEED0 .. + n_train - 1
EVAL_SEED0 = 8_000_000   # held-out events
WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "weights")
CHECKPOINT = os.path.join(WEIGHTS, "prefilter_pbpb.itsumlp")
CHECKPOINTS = {"pbpb": CHECKPOINT, "pileup": os.path.join(WEIGHTS, "prefilter_pileup.itsumlp")}
GATE_CHECKPOINTS = {"pbpb": os.path.join(WEIGHTS, "gate_pbpb.itsugate"), "pileup": os.path.join(WEIGHTS, "gate_pileup.itsugate")}
TWO_PI_F = np.float32(6.28318530717958647692)
CELL_MAX_DCA = np.array([0.05, 0.04, 0.05, 0.2, 0.4], np.float32)

# ---------------------------------------------------------------------------------------------
# numpy restatements (float32 ops in the device's order; BF16 by round-to-nearest-even)


def bf16_round(x) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32)


def gelu(x):
    x = np.asarray(x, np.float64)
    return 0.5 * x * (1.0 + np.tanh(0.7978845608028654 * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    x = np.asarray(x, np.float64)
    th = np.tanh(0.7978845608028654 * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + th) + 0.5 * x * (1.0 - th * th) * 0.7978845608028654 * (1.0 + 3.0 * 0.044715 * x * x)


def relu(x):
    return np.maximum(np.asarray(x, np.float64), 0.0)


def relu_grad(x):
    return (np.asarray(x, np.float64) > 0).astype(np.float64)


ACTIVATIONS = {"gelu": (gelu, gelu_grad), "relu": (relu, relu_grad)}


def mlp_forward(m: dict, features, rounding: bool = True, act: str = "gelu"):
    """Logits as the device computes them (BF16 inputs, weights and activations; wide
    accumulation). rounding=False gives the same network in plain float64. act: "gelu" (the pair
    prefilter) or "relu" (the tracklet gate)."""
    fn = ACTIVATIONS[act][0]
    rnd = (lambda a: bf16_round(np.asarray(a, np.float32)).astype(np.float64)) if rounding else (lambda a: np.asarray(a, np.float64))
    f = np.asarray(features, np.float32)
    x = rnd((f - m["mean"].astype(np.float32)) * m["inv_std"].astype(np.float32))
    w1, w2, w3 = (rnd(m[k]) for k in ("w1", "w2", "w3"))
    a1 = x @ w1.T + m["b1"]
    h1 = rnd(fn(a1))
    a2 = h1 @ w2.T + m["b2"]
    h2 = rnd(fn(a2))
    z = h2 @ w3 + m["b3"]
    return dict(x=x, a1=a1, h1=h1, a2=a2, h2=h2, z=z, w2=w2, w3=w3)


def mlp_gradient(m: dict, features, labels, pos_weight: float = 1.0, rounding: bool = True, act: str = "gelu"):
    """Mean weighted binary cross-entropy and its gradient (itsu_prefilter_model parameter order),
    in float64 through the forward values (straight-through for the BF16 rounding)."""
    dact = ACTIVATIONS[act][1]
    fw = mlp_forward(m, features, rounding, act)
    y = np.asarray(labels, np.float64)
    n = len(y)
    w = np.where(y > 0, pos_weight, 1.0)
    z = fw["z"]
    loss = float(np.sum(w * (np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))))) / n)
    dz = w * (1.0 / (1.0 + np.exp(-z)) - y) / n
    g_w3 = fw["h2"].T @ dz
    g_b3 = dz.sum()
    d2 = dz[:, None] * fw["w3"][None, :] * dact(fw["a2"])
    g_w2 = d2.T @ fw["h1"]
    g_b2 = d2.sum(0)
    d1 = (d2 @ fw["w2"]) * dact(fw["a1"])
    g_w1 = d1.T @ fw["x"]
    g_b1 = d1.sum(0)
    grad = np.concatenate([g_w1.ravel(), g_b1, g_w2.ravel(), g_b2, g_w3, [g_b3]])
    return grad, loss


def _curvature(ax, ay, bx, by, cx, cy):
    ux, uy, vx, vy, wx, wy = bx - ax, by - ay, cx - ax, cy - ay, cx - bx, cy - by
    cross = ux * vy - uy * vx
    d = np.sqrt((ux * ux + uy * uy) * (vx * vx + vy * vy) * (wx * wx + wy * wy))
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(d > 0, np.float32(2.0) * cross / d, np.float32(0.0)).astype(np.float32)


def _dca(layer, c1, c2, c3, vx, vy):
    """Tracker.cxx:175-210 in float32: the DCA of the circle through three clusters."""
    f = np.float32
    r1sq, r2sq, r3sq = c1["r"] * c1["r"], c2["r"] * c2["r"], c3["r"] * c3["r"]
    d1x, d1y, d1z = c2["x"] - c1["x"], c2["y"] - c1["y"], r2sq - r1sq
    d2x, d2y, d2z = c3["x"] - c1["x"], c3["y"] - c1["y"], r3sq - r1sq
    nx = (d1y * d2z) - (d1z * d2y)
    ny = (d1z * d2x) - (d1x * d2z)
    nz = (d1x * d2y) - (d1y * d2x)
    with np.errstate(all="ignore"):
        norm = np.sqrt(nx * nx + ny * ny + nz * nz)
        inv = f(1.0) / norm
        unx, uny, unz = nx * inv, ny * inv, nz * inv
        plane_d = -unx * (c2["x"] - vx) - (uny * c2["y"] - vy) - unz * r2sq
        nzsq = unz * unz
        radius = np.sqrt((f(1.0) - nzsq - f(4.0) * plane_d * unz) / (f(4.0) * nzsq))
        ccx = f(-0.5) * unx / unz
        ccy = f(-0.5) * uny / unz
        return np.abs(radius - np.sqrt(ccx * ccx + ccy * ccy)).astype(np.float32)


def pair_features(res: dict) -> np.ndarray:
    """The 8 features of every cell of one vertex's results (oracle canonical form), in the
    export's row order (layer by layer, cells in order)."""
    out = []
    vx, vy, vz = (np.float32(v) for v in res["vertex"])
    for layer in range(5):
        cells = res["cells"][layer]
        if len(cells) == 0:
            continue
        t1 = res["tracklets"][layer][cells["t1"]]
        t2 = res["tracklets"][layer + 1][cells["t2"]]
        c1 = res["clusters"][layer][cells["c1"]]
        c2 = res["clusters"][layer + 1][cells["c2"]]
        c3 = res["clusters"][layer + 2][cells["c3"]]
        f = np.zeros((len(cells), 8), np.float32)
        dphi = np.abs(t1["phi"] - t2["phi"])
        f[:, 0] = np.minimum(dphi, np.abs(dphi - TWO_PI_F))
        f[:, 1] = np.abs(-(np.float32(0.5) * (t1["tan_lambda"] + t2["tan_lambda"])) * c1["r"] + c1["z"] - vz)
        f[:, 2] = np.abs(t1["tan_lambda"] - t2["tan_lambda"])
        f[:, 3] = _curvature(vx, vy, c1["x"], c1["y"], c2["x"], c2["y"])
        f[:, 4] = _curvature(vx, vy, c2["x"], c2["y"], c3["x"], c3["y"])
        f[:, 5] = _dca(layer, c1, c2, c3, vx, vy)
        f[:, 6] = np.float32(layer)
        f[:, 7] = c1["r"]
        out.append(f)
    return np.concatenate(out) if out else np.zeros((0, 8), np.float32)


def tracklet_features(res: dict) -> np.ndarray:
    """The tracklet gate's 8 features of every tracklet of one vertex's results (oracle canonical
    form), float32 in the device's order, in the export's row order (layer by layer)."""
    out = []
    vx, vy, vz = (np.float32(v) for v in res["vertex"])
    pi_f, two_pi_f = np.float32(3.14159265358979323846), TWO_PI_F
    for layer in range(6):
        t = res["tracklets"][layer]
        if len(t) == 0:
            continue
        c1 = res["clusters"][layer][t["c1"]]
        c2 = res["clusters"][layer + 1][t["c2"]]
        dphi = c1["phi"] - c2["phi"]
        dphi = np.where(dphi > pi_f, dphi - two_pi_f, np.where(dphi < -pi_f, dphi + two_pi_f, dphi)).astype(np.float32)
        tan_lambda = (c1["z"] - vz) / c1["r"]
        dz = tan_lambda * (c2["r"] - c1["r"]) + c1["z"] - c2["z"]
        f = np.zeros((len(t), 8), np.float32)
        f[:, 0] = np.abs(dphi)
        f[:, 1] = dz
        f[:, 2] = np.abs(dz)
        f[:, 3] = _curvature(vx, vy, c1["x"], c1["y"], c2["x"], c2["y"])
        f[:, 4] = np.float32(layer)
        f[:, 5] = c1["r"]
        f[:, 6] = tan_lambda
        f[:, 7] = dphi
        out.append(f)
    return np.concatenate(out) if out else np.zeros((0, 8), np.float32)


def road_tracklets(res: dict) -> np.ndarray:
    """Each road's 6 tracklets as rows of tracklet_features(res)."""
    base = np.concatenate([[0], np.cumsum([len(t) for t in res["tracklets"]])])[:6]
    rows = np.zeros((len(res["roads"]), 6), np.int64)
    for k, road in enumerate(res["roads"]):
        for l in range(5):
            cell = res["cells"][l][road["cells"][l]]
            rows[k, l] = base[l] + cell["t1"]
            rows[k, l + 1] = base[l + 1] + cell["t2"]
    return rows


def road_cells(res: dict) -> np.ndarray:
    """Each road's 5 cells as rows of pair_features(res)."""
    base = np.concatenate([[0], np.cumsum([len(c) for c in res["cells"]])])[:5]
    return res["roads"]["cells"].astype(np.int64) + base[None, :]


def calibrate(logits: np.ndarray, road_rows: np.ndarray, target: float) -> float:
    """Largest threshold t such that at least `target` of the roads keep all their cells
    (logit >= t; NaN logits keep their cell)."""
    lg = np.where(np.isnan(logits), np.inf, logits.astype(np.float64))
    lg = np.append(lg, np.inf)  # row -1 (no object in that layer) never drops its road
    road_min = lg[road_rows].min(axis=1) if len(road_rows) else np.zeros(0)
    if len(road_min) == 0:
        return float("-inf")
    s = np.sort(road_min)
    k = int(math.floor((1.0 - target) * len(s)))
    k = min(max(k, 0), len(s) - 1)
    return float(np.float32(s[k]))


def compare_roads(plain_keys, plain_fake, learned_keys, learned_fake) -> dict:
    """Road sets of a plain and a learned run of the same events, keyed by (event, 7 clusters)."""
    p = {bytes(r) for r in np.ascontiguousarray(plain_keys, np.int32)}
    lk = np.ascontiguousarray(learned_keys, np.int32)
    reproduced = extra = extra_fakes = 0
    for r, fk in zip(lk, learned_fake):
        if bytes(r) in p:
            reproduced += 1
        else:
            extra += 1
            extra_fakes += int(fk != 0)
    return dict(plain_roads=len(plain_keys), learned_roads=len(learned_keys), reproduced=reproduced, extra=extra,
                extra_fakes=extra_fakes, plain_fakes=int(np.count_nonzero(plain_fake)),
                learned_fakes=int(np.count_nonzero(learned_fake)))


# ---------------------------------------------------------------------------------------------
# pipeline (GPU)


def pileup_frame(seed: int) -> gen.Event:
    """A pile-up frame as the pile-up stream makes them: 5 collisions of 1050-1950 tracks (drawn
    from the seed), 10% noise."""
    rng = np.random.default_rng(seed)
    return gen.make_event(seed, int(rng.integers(1050, 1951)), pt_mean=0.6, noise=0.10, n_vertices=5)


MAKERS = {"pbpb": gen.pbpb_event, "pileup": pileup_frame}


def make_events(seeds, workers: int | None = None, workload: str = "pbpb") -> list:
    """Central Pb-Pb-like events (6000 tracks, 5% noise), or pile-up frames, for the given seeds,
    generated in parallel worker processes (spawned, so that no CUDA state is forked)."""
    seeds = list(seeds)
    make = MAKERS[workload]
    workers = workers or min(32, os.cpu_count() or 1)
    if workers <= 1 or len(seeds) < 8:
        return [make(s) for s in seeds]
    with multiprocessing.get_context("spawn").Pool(workers) as pool:
        return pool.map(make, seeds, chunksize=max(1, len(seeds) // (4 * workers)))


class DeviceBatch:
    """A batch of runs resident on the device (torch owns the memory): every vertex of every
    event is one run."""

    def __init__(self, ctx, events, device):
        import torch

        runs = [(ev, iv) for ev in events for iv in range(len(ev.vertices))]
        clusters, offsets, vertices = gen.pack_batch([ev for ev, _ in runs], [iv for _, iv in runs])
        self.n_runs = len(runs)
        self.clusters = torch.from_numpy(clusters.view(np.uint8)).to(device)
        self.offsets = torch.from_numpy(offsets).to(device)
        self.vertices = torch.from_numpy(vertices).to(device)
        self.batch = ctx.batch_device(self.clusters.data_ptr(), self.offsets.data_ptr(), self.vertices.data_ptr(), len(runs),
                                      len(clusters))


def export_samples(ctx, device):
    """Samples and road rows of the context's last run, as device tensors."""
    import torch

    n_cells, n_roads = ctx.prefilter_export()
    feats = torch.empty((max(n_cells, 1), 8), dtype=torch.float32, device=device)
    labels = torch.empty(max(n_cells, 1), dtype=torch.uint8, device=device)
    rcells = torch.empty((max(n_roads, 1), 5), dtype=torch.int32, device=device)
    ctx.prefilter_export(features=feats.data_ptr(), labels=labels.data_ptr(), capacity=n_cells, road_cells=rcells.data_ptr(),
                         road_capacity=n_roads)
    return feats[:n_cells], labels[:n_cells], rcells[:n_roads]


def export_roads(ctx, device):
    import torch

    _, n_roads = ctx.prefilter_export()
    keys = torch.empty((max(n_roads, 1), 8), dtype=torch.int32, device=device)
    fake = torch.empty(max(n_roads, 1), dtype=torch.uint8, device=device)
    ctx.prefilter_export(road_keys=keys.data_ptr(), road_fake=fake.data_ptr(), road_capacity=n_roads)
    return keys[:n_roads].cpu().numpy(), fake[:n_roads].cpu().numpy()


def collect(ctx, seeds, device, chunk: int = 100, workers: int | None = None, log=print, workload: str = "pbpb") -> dict:
    """Plain runs over the events of `seeds`; all their samples, concatenated on the device."""
    import torch

    feats, labels, rows = [], [], []
    base = 0
    seeds = list(seeds)
    for k in range(0, len(seeds), chunk):
        events = make_events(seeds[k:k + chunk], workers, workload)
        b = DeviceBatch(ctx, events, device)
        set_learned(ctx, False, False)
        ctx.batch_run(b.batch)
        f, l, r = export_samples(ctx, device)
        feats.append(f.clone())
        labels.append(l.clone())
        rows.append(r.to(torch.int64) + base)
        base += len(f)
        log("collect: events %d..%d, %d cells, %d roads" % (k, k + len(events) - 1, len(f), len(r)))
    return dict(features=torch.cat(feats), labels=torch.cat(labels), road_rows=torch.cat(rows))


def standardisation(features) -> tuple:
    import torch

    ok = torch.isfinite(features).all(dim=1)
    f = features[ok].double()
    mean = f.mean(dim=0)
    std = f.std(dim=0)
    std = torch.where(std > 0, std, torch.ones_like(std))
    return mean.float().cpu().numpy(), (1.0 / std).float().cpu().numpy()


def score(ctx, features, device):
    import torch

    n = len(features)
    logits = torch.empty(max(n, 1), dtype=torch.float32, device=device)
    ctx.prefilter_score(features.data_ptr(), n, logits.data_ptr())
    return logits[:n]


def train(ctx, data: dict, device, seed: int = 1, target: float = 0.997, log=print, **train_kw) -> tuple:
    """Trains a model on `data` (from collect) and calibrates its threshold; returns
    (model, report dict)."""
    import torch

    model = capi.prefilter_init(seed)
    mean, inv_std = standardisation(data["features"])
    for k in range(8):
        model.mean[k], model.inv_std[k] = float(mean[k]), float(inv_std[k])
    ctx.prefilter_set_model(model)
    ok = torch.isfinite(data["features"]).all(dim=1)
    f = data["features"][ok].contiguous()
    y = data["labels"][ok].contiguous()
    cfg = capi.train_config(**train_kw)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = ctx.prefilter_train(f.data_ptr(), y.data_ptr(), len(f), cfg)
    train_s = time.perf_counter() - t0
    model = ctx.prefilter_get_model()
    logits = score(ctx, data["features"], device).cpu().numpy()
    rows = data["road_rows"].cpu().numpy()
    thr = calibrate(logits, rows, target)
    model.logit_threshold = thr
    ctx.prefilter_set_model(model)
    labels = data["labels"].cpu().numpy()
    kept = ~(logits < thr)
    report = dict(
        samples=int(len(f)), positives=int(y.sum().item()), steps=int(cfg.steps), batch=int(cfg.batch), lr=float(cfg.lr),
        lr_final=float(cfg.lr_final), train_seconds=train_s, loss_first=float(np.mean(losses[:100])) if len(losses) else None,
        loss_last=float(np.mean(losses[-100:])) if len(losses) else None, threshold=thr, calibration_target=target,
        train_cells_kept=float(kept.mean()), train_positive_cells_kept=float(kept[labels == 1].mean()),
        train_negative_cells_kept=float(kept[labels == 0].mean()),
        train_road_reproduction=float((np.where(np.isnan(logits), np.inf, logits)[rows].min(axis=1) >= thr).mean()),
    )
    log("train: %s" % json.dumps(report))
    return model, report


def export_gate_samples(ctx, device):
    """Tracklet samples and road rows of the context's last run, as device tensors."""
    import torch

    n, n_roads = ctx.gate_export()
    feats = torch.empty((max(n, 1), 8), dtype=torch.float32, device=device)
    labels = torch.empty(max(n, 1), dtype=torch.uint8, device=device)
    rows = torch.empty((max(n_roads, 1), 6), dtype=torch.int32, device=device)
    ctx.gate_export(features=feats.data_ptr(), labels=labels.data_ptr(), capacity=n, road_tracklets=rows.data_ptr(),
                    road_capacity=n_roads)
    return feats[:n], labels[:n], rows[:n_roads]


def collect_gate(ctx, seeds, device, chunk: int = 50, workers: int | None = None, log=print, workload: str = "pbpb") -> dict:
    """Plain runs over the events of `seeds`; one sample per tracklet (label 1: a found road uses
    it) and each road's 6 tracklets as sample rows, concatenated on the device."""
    import torch

    feats, labels, rows = [], [], []
    base = 0
    seeds = list(seeds)
    for k in range(0, len(seeds), chunk):
        events = make_events(seeds[k:k + chunk], workers, workload)
        b = DeviceBatch(ctx, events, device)
        set_learned(ctx, False, False)
        ctx.batch_run(b.batch)
        f, l, r = export_gate_samples(ctx, device)
        feats.append(f.clone())
        labels.append(l.clone())
        r = r.to(torch.int64)
        rows.append(torch.where(r >= 0, r + base, r))
        base += len(f)
        log("collect gate: events %d..%d, %d tracklets (%d on roads), %d roads" % (k, k + len(events) - 1, len(f),
                                                                                   int(l.sum().item()), len(r)))
    return dict(features=torch.cat(feats), labels=torch.cat(labels), road_rows=torch.cat(rows))


def ctx_has_gate(ctx) -> bool:
    try:
        ctx.gate_get_model()
        return True
    except capi.ItsuError:
        return False


PHI_CUT = 0.3  # the tracklet cut's phi window (the reference's kPhiCoordinateCut, Constants.h)


def fit_windows(features: np.ndarray, road_rows: np.ndarray, margin: float = 1.25, quantile: float = 1.0) -> tuple:
    """The cascade's first stage: per inner layer, `margin` times the `quantile` (1: the largest) of
    |dphi| (feature 0) and of |dz| (feature 2) over the tracklets on the training roads; the |dphi|
    window at most the tracklet cut's own (a layer without a road tracklet keeps no window).
    Returns (dphi, dz) windows."""
    rows = np.unique(road_rows[road_rows >= 0])
    layer = features[rows, 4]
    wphi = np.full(6, PHI_CUT, np.float32)
    wz = np.full(6, np.inf, np.float32)
    for l in range(6):
        on = layer == l
        dphi = features[rows[on], 0].astype(np.float64)
        dz = features[rows[on], 2].astype(np.float64)
        dphi, dz = dphi[np.isfinite(dphi)], dz[np.isfinite(dz)]
        if len(dphi):
            wphi[l] = np.float32(min(PHI_CUT, margin * float(np.quantile(dphi, quantile))))
        if len(dz):
            wz[l] = np.float32(margin * float(np.quantile(dz, quantile)))
    return wphi, wz


def window_pass(features: np.ndarray, dphi_window: np.ndarray, dz_window: np.ndarray | None = None) -> np.ndarray:
    """The first stage's verdict per tracklet: |dphi| and |dz| within its layer's windows (the
    device tests the same values, features 0 and 2, in float32)."""
    layer = np.clip(features[:, 4], 0, 5).astype(np.int64)
    ok = ~(features[:, 0] > dphi_window[layer])
    if dz_window is not None:
        ok &= ~(features[:, 2] > dz_window[layer])
    return ok


def per_layer_fractions(layer: np.ndarray, inside: np.ndarray, kept: np.ndarray) -> list:
    """Per inner layer: its share of the tracklets, and the fractions inside the windows and kept
    by both stages."""
    out = []
    for l in range(6):
        on = layer == l
        n = int(on.sum())
        out.append(dict(layer=l, tracklets=n, share=n / max(len(layer), 1),
                        inside_window=float(inside[on].mean()) if n else None,
                        kept=float(kept[on].mean()) if n else None))
    return out


def train_gate(ctx, data: dict, device, seed: int = 1, target: float = 0.997, log=print, window_margin: float = 1.0,
               window_quantile: float = 0.9999, mlp_layers: int = 0x04, **train_kw) -> tuple:
    """Trains a tracklet gate on `data` (from collect_gate): the first stage's per-layer |dphi| and
    |dz| windows from the road tracklets (fit_windows), then the network on the tracklets inside them
    of the inner layers in `mlp_layers` (bit l), its threshold calibrated on road reproduction (a
    road survives the gate iff all its 6 tracklets pass both stages); returns (model, report)."""
    import torch

    model = capi.gate_init(seed)
    feats_np = data["features"].cpu().numpy()
    rows = data["road_rows"].cpu().numpy()
    wphi, wz = fit_windows(feats_np, rows, window_margin, window_quantile)
    inside = window_pass(feats_np, wphi, wz)
    for l in range(6):
        model.dphi_window[l] = float(wphi[l])
        model.dz_window[l] = float(wz[l])
    model.mlp_layers = mlp_layers
    layer = np.clip(feats_np[:, 4], 0, 5).astype(np.int64)
    scored = inside & (((mlp_layers >> layer) & 1) == 1)
    mean, inv_std = standardisation(data["features"][torch.from_numpy(scored).to(data["features"].device)])
    for k in range(8):
        model.mean[k], model.inv_std[k] = float(mean[k]), float(inv_std[k])
    ctx.gate_set_model(model)
    ok = torch.isfinite(data["features"]).all(dim=1) & torch.from_numpy(scored).to(data["features"].device)
    f = data["features"][ok].contiguous()
    y = data["labels"][ok].contiguous()
    cfg = capi.train_config(**train_kw)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = ctx.gate_train(f.data_ptr(), y.data_ptr(), len(f), cfg) if len(f) else np.zeros(0)  # no layer scored: no network
    train_s = time.perf_counter() - t0
    model = ctx.gate_get_model()
    n = len(data["features"])
    logits_t = torch.empty(max(n, 1), dtype=torch.float32, device=device)
    ctx.gate_score(data["features"].data_ptr(), n, logits_t.data_ptr())
    logits = logits_t[:n].cpu().numpy()
    logits = np.where(scored, logits, np.inf)  # layers the network does not score: kept
    logits = np.where(inside, logits, -np.inf)  # outside the windows: dropped by stage 1
    thr = calibrate(logits, rows, target)
    if not np.isfinite(thr):  # only the windows drop tracklets: the threshold is never used
        thr = float("-inf")
    model.logit_threshold = thr
    ctx.gate_set_model(model)
    labels = data["labels"].cpu().numpy()
    kept = ~(logits < thr)
    report = dict(
        dphi_window=[float(w) for w in wphi], dz_window=[float(w) for w in wz], window_margin=window_margin,
        window_quantile=window_quantile, mlp_layers=mlp_layers,
        train_tracklets_inside_window=float(inside.mean()),
        samples=int(len(f)), positives=int(y.sum().item()), steps=int(cfg.steps), batch=int(cfg.batch), lr=float(cfg.lr),
        lr_final=float(cfg.lr_final), train_seconds=train_s, loss_first=float(np.mean(losses[:100])) if len(losses) else None,
        loss_last=float(np.mean(losses[-100:])) if len(losses) else None, threshold=thr, calibration_target=target,
        train_tracklets_kept=float(kept.mean()), train_positive_tracklets_kept=float(kept[labels == 1].mean()),
        train_negative_tracklets_kept=float(kept[labels == 0].mean()),
        per_layer=per_layer_fractions(feats_np[:, 4], inside, kept),
    )
    log("train gate: %s" % json.dumps(report))
    return model, report


def evaluate(ctx, model, seeds, device, chunk: int = 100, workers: int | None = None, log=print, workload: str = "pbpb",
             gate=None) -> dict:
    """Learned vs plain batched runs over the events of `seeds`: the learned form runs the pair
    prefilter `model` (None: not used) and the tracklet gate `gate` (None: not used)."""
    if model is not None:
        ctx.prefilter_set_model(model)
    if gate is not None:
        ctx.gate_set_model(gate)
    tot = dict(plain_roads=0, learned_roads=0, reproduced=0, extra=0, extra_fakes=0, plain_fakes=0, learned_fakes=0,
               plain_cells=0, learned_cells=0, events=0)
    seeds = list(seeds)
    for k in range(0, len(seeds), chunk):
        events = make_events(seeds[k:k + chunk], workers, workload)
        b = DeviceBatch(ctx, events, device)
        set_learned(ctx, False, False)
        ctx.batch_run(b.batch)
        plain_cells, _ = ctx.prefilter_export()
        plain_tracklets = ctx.gate_export()[0]
        pk, pf = export_roads(ctx, device)
        set_learned(ctx, model is not None, gate is not None)
        ctx.batch_run(b.batch)
        learned_cells, _ = ctx.prefilter_export()
        learned_tracklets = ctx.gate_export()[0]
        lk, lf = export_roads(ctx, device)
        set_learned(ctx, False, False)
        c = compare_roads(pk, pf, lk, lf)
        for key in c:
            tot[key] += c[key]
        tot["plain_cells"] += plain_cells
        tot["learned_cells"] += learned_cells
        tot["plain_tracklets"] = tot.get("plain_tracklets", 0) + plain_tracklets
        tot["learned_tracklets"] = tot.get("learned_tracklets", 0) + learned_tracklets
        tot["events"] += len(events)
        tot["runs"] = tot.get("runs", 0) + b.n_runs
        log("evaluate: events %d..%d %s" % (k, k + len(events) - 1, json.dumps(c)))
    tot["road_reproduction"] = tot["reproduced"] / max(tot["plain_roads"], 1)
    tot["cells_kept"] = tot["learned_cells"] / max(tot["plain_cells"], 1)
    tot["tracklets_kept"] = tot.get("learned_tracklets", 0) / max(tot.get("plain_tracklets", 0), 1)
    tot["learned_form"] = "+".join(k for k, v in (("tracklet gate", gate), ("pair prefilter", model)) if v is not None)
    return tot


def set_learned(ctx, pair: bool, gate: bool):
    """The learned form's networks on or off (a network must have a model to be turned on)."""
    if pair or ctx_has_pair(ctx):
        ctx.prefilter_enable(pair)
    if gate or ctx_has_gate(ctx):
        ctx.gate_enable(gate)


def ctx_has_pair(ctx) -> bool:
    try:
        ctx.prefilter_get_model()
        return True
    except capi.ItsuError:
        return False


def main(argv=None):
    p = argparse.ArgumentParser(description="Train, calibrate and evaluate a learned network of the learned form on one GPU.")
    p.add_argument("--model", choices=("pair", "gate"), default="pair",
                   help="pair: the tracklet-pair prefilter of the cell stage; gate: the tracklet gate of the tracklet stage")
    p.add_argument("--workload", choices=("pbpb", "pileup"), default="pbpb",
                   help="pbpb: central Pb-Pb-like events; pileup: frames of 5 collisions (every vertex is a run)")
    p.add_argument("--out", default=None, help="checkpoint to write (default: weights/<model>_<workload>.itsu{mlp,gate})")
    p.add_argument("--report", default=None, help="JSON report (default: the checkpoint path with .json)")
    p.add_argument("--train-events", type=int, default=None, help="default: 2000 (pair), 300 (gate)")
    p.add_argument("--eval-events", type=int, default=500)
    p.add_argument("--steps", type=int, default=20000)
    p.add_argument("--batch", type=int, default=8192)
    p.add_argument("--lr", type=float, default=2e-3)
    p.add_argument("--target", type=float, default=None,
                   help="road reproduction the threshold keeps on the training events (default: 0.997)")
    p.add_argument("--with-pair", default=None,
                   help="gate: also evaluate the learned form with this pair-prefilter checkpoint enabled")
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--window-margin", type=float, default=1.0,
                   help="gate: its windows are this times the training roads' --window-quantile of |dphi| and |dz| per layer")
    p.add_argument("--window-quantile", type=float, default=0.9999,
                   help="gate: the quantile of the road tracklets' |dphi| and |dz| its windows start from (1: the largest)")
    p.add_argument("--mlp-layers", type=lambda v: int(v, 0), default=0x04,
                   help="gate: the inner layers its network scores, as a bit mask (0x3f: all six; default: layer 2, "
                        "where the windows keep the most)")
    p.add_argument("--chunk", type=int, default=None)
    args = p.parse_args(argv)
    gate_mode = args.model == "gate"
    args.out = args.out or (GATE_CHECKPOINTS[args.workload] if gate_mode else CHECKPOINTS[args.workload])
    args.train_events = args.train_events or (300 if gate_mode else 2000)
    args.target = args.target or 0.997
    args.chunk = args.chunk or (50 if gate_mode else 100)
    import torch

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    ctx = capi.Context(device=0)
    t0 = time.perf_counter()
    train_seeds = range(TRAIN_SEED0, TRAIN_SEED0 + args.train_events)
    eval_seeds = range(EVAL_SEED0, EVAL_SEED0 + args.eval_events)
    if gate_mode:
        data = collect_gate(ctx, train_seeds, device, chunk=args.chunk, workload=args.workload)
    else:
        data = collect(ctx, train_seeds, device, chunk=args.chunk, workload=args.workload)
    collect_s = time.perf_counter() - t0
    trainer = train_gate if gate_mode else train
    extra = dict(window_margin=args.window_margin, window_quantile=args.window_quantile,
                 mlp_layers=args.mlp_layers) if gate_mode else {}
    model, report = trainer(ctx, data, device, seed=args.seed, target=args.target, steps=args.steps, batch=args.batch,
                            lr=args.lr, **extra)
    del data
    if gate_mode:
        ev = evaluate(ctx, None, eval_seeds, device, chunk=args.chunk, workload=args.workload, gate=model)
        if args.with_pair:
            pair = capi.prefilter_load(args.with_pair)
            ev_both = evaluate(ctx, pair, eval_seeds, device, chunk=args.chunk, workload=args.workload, gate=model)
            ev = dict(gate_only=ev, gate_and_pair=ev_both, pair_checkpoint=os.path.basename(args.with_pair))
        capi.gate_save(model, os.path.abspath(args.out))
    else:
        ev = evaluate(ctx, model, eval_seeds, device, chunk=args.chunk, workload=args.workload)
        capi.prefilter_save(model, os.path.abspath(args.out))
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    full = dict(model=args.model, workload=args.workload, train_events=args.train_events,
                train_seeds=[TRAIN_SEED0, TRAIN_SEED0 + args.train_events - 1], eval_events=args.eval_events,
                eval_seeds=[EVAL_SEED0, EVAL_SEED0 + args.eval_events - 1], collect_seconds=collect_s, train=report,
                evaluation=ev)
    with open(args.report or os.path.splitext(args.out)[0] + ".json", "w") as fh:
        json.dump(full, fh, indent=1)
    print(json.dumps(full))
    ctx.close()


if __name__ == "__main__":
    main()
