"""Seeded synthetic ITS events (helix tracks through 7 cylindrical layers).

The reference ships no event data (its CI downloads files that are not available here), so
every workload is generated: 7 layers at radii 2.3/3.1/3.9/19.6/24.5/34.4/39.3 cm with
half-lengths 13.5/13.5/13.5/42/42/73.5/73.5 cm in a 0.5 T solenoid; primary vertex
x, y ~ N(0, 0.005 cm), z ~ N(0, 5 cm); pT ~ 0.1 + Exp(mean) GeV/c (an exponential truncated at
0.1 is memoryless), |eta| < 1, phi uniform, charge +-1. Each helix is intersected with each
layer (hits beyond the layer half-length are dropped), smeared by N(0, 5 um) in r-phi and z,
and uniform noise is added at a fixed fraction of each layer's signal count.

Clusters use the reference's raw Cluster record (Cluster.h:36-44, 36 bytes) with phi, r and
bin left at zero, the way Layer::addCluster builds them (Layer.cxx:38-42). Cluster ids are a
running per-event index in file order, exactly as IOUtils::loadEventData assigns them
(IOUtils.cxx:44,63,71). Pile-up frames merge collisions with the Monte Carlo id offset of the
reference's pile-up merger (benchmarks/scripts/root/generatePileUpData.cxx:31, 100000).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

CLUSTER_DTYPE = np.dtype(
    [
        ("x", "<f4"),
        ("y", "<f4"),
        ("z", "<f4"),
        ("phi", "<f4"),
        ("r", "<f4"),
        ("id", "<i4"),
        ("alpha", "<f4"),
        ("mc", "<i4"),
        ("bin", "<i4"),
    ]
)
assert CLUSTER_DTYPE.itemsize == 36

LAYERS = 7
RADII_CM = (2.3, 3.1, 3.9, 19.6, 24.5, 34.4, 39.3)
HALF_LENGTHS_CM = (13.5, 13.5, 13.5, 42.0, 42.0, 73.5, 73.5)
FIELD_T = 0.5
SMEAR_CM = 5e-4
PILEUP_MC_OFFSET = 100000


@dataclasses.dataclass
class Event:
    """One reference Event: primary vertices plus 7 layers of raw clusters."""

    vertices: np.ndarray  # (nv, 3) float32
    layers: list  # 7 arrays of CLUSTER_DTYPE
    labels: np.ndarray  # structured: mc, pt, phi, eta, pdg, ncl

    @property
    def n_clusters(self) -> int:
        return int(sum(len(l) for l in self.layers))

    def counts(self) -> list:
        return [len(l) for l in self.layers]


LABEL_DTYPE = np.dtype(
    [("mc", "<i4"), ("pt", "<f4"), ("phi", "<f4"), ("eta", "<f4"), ("pdg", "<i4"), ("ncl", "<i4")]
)


def _collision(rng, n_tracks, pt_mean, vertex, mc_offset, eta_range=(-1.0, 1.0), phi_range=(0.0, 2.0 * math.pi)):
    """Hits of one collision: returns per-layer (x, y, z, mc) lists and the label table."""
    vx, vy, vz = (float(v) for v in vertex)
    pt = 0.1 + rng.exponential(pt_mean, n_tracks)
    eta = rng.uniform(eta_range[0], eta_range[1], n_tracks)
    phi0 = rng.uniform(phi_range[0], phi_range[1], n_tracks)
    q = np.where(rng.random(n_tracks) < 0.5, -1.0, 1.0)
    radius = pt / (0.3 * FIELD_T) * 100.0  # cm
    # circle centre: left of the direction for q = +1 (counter-clockwise), right for q = -1
    cx = vx - q * radius * np.sin(phi0)
    cy = vy + q * radius * np.cos(phi0)
    cmod = np.hypot(cx, cy)
    gamma = np.arctan2(cy, cx)
    sinh_eta = np.sinh(eta)
    hits = []
    ncl = np.zeros(n_tracks, np.int32)
    mc = np.arange(n_tracks, dtype=np.int32) + mc_offset
    for layer in range(LAYERS):
        rho = RADII_CM[layer]
        kk = (rho * rho - cmod * cmod - radius * radius) / (2.0 * radius)
        ratio = q * kk / cmod  # sin(beta - gamma), sign folded by charge
        ok = np.abs(ratio) <= 1.0
        ratio = np.clip(ratio, -1.0, 1.0)
        a1 = np.arcsin(ratio)
        alphas = []
        for branch in (a1, math.pi - a1):
            beta = gamma + branch
            alpha = np.where(q > 0, beta - phi0, phi0 - beta)
            alphas.append(np.mod(alpha, 2.0 * math.pi))
        alpha = np.minimum(alphas[0], alphas[1])
        beta = np.where(q > 0, phi0 + alpha, phi0 - alpha)
        px = np.where(q > 0, cx + radius * np.sin(beta), cx - radius * np.sin(beta))
        py = np.where(q > 0, cy - radius * np.cos(beta), cy + radius * np.cos(beta))
        z = vz + radius * alpha * sinh_eta
        # smear: rotate by N(0, 5 um)/rho about the beam axis, shift z by N(0, 5 um)
        dphi = rng.normal(0.0, SMEAR_CM, n_tracks) / rho
        cphi, sphi = np.cos(dphi), np.sin(dphi)
        px, py = px * cphi - py * sphi, px * sphi + py * cphi
        z = z + rng.normal(0.0, SMEAR_CM, n_tracks)
        keep = ok & (np.abs(z) <= HALF_LENGTHS_CM[layer]) & (alpha < math.pi)
        ncl += keep
        hits.append((px[keep], py[keep], z[keep], mc[keep]))
    labels = np.zeros(n_tracks, LABEL_DTYPE)
    labels["mc"] = mc
    labels["pt"] = pt
    labels["phi"] = phi0
    labels["eta"] = eta
    labels["pdg"] = (211 * q).astype(np.int32)
    labels["ncl"] = ncl
    return hits, labels


def make_event(
    seed: int,
    n_tracks: int,
    pt_mean: float = 0.6,
    noise: float = 0.05,
    n_vertices: int = 1,
    eta_range=(-1.0, 1.0),
    phi_range=(0.0, 2.0 * math.pi),
) -> Event:
    """One event with ``n_vertices`` overlapping collisions of ``n_tracks`` tracks each, their
    directions uniform in ``eta_range`` x ``phi_range``."""
    rng = np.random.default_rng(seed)
    vertices = np.zeros((n_vertices, 3), np.float32)
    per_layer = [[] for _ in range(LAYERS)]
    labels = []
    for iv in range(n_vertices):
        v = (rng.normal(0.0, 0.005), rng.normal(0.0, 0.005), rng.normal(0.0, 5.0))
        vertices[iv] = v
        hits, lab = _collision(rng, n_tracks, pt_mean, v, PILEUP_MC_OFFSET * iv, eta_range, phi_range)
        labels.append(lab)
        for layer in range(LAYERS):
            per_layer[layer].append(hits[layer])
    layers = []
    next_id = 0
    for layer in range(LAYERS):
        xs = np.concatenate([h[0] for h in per_layer[layer]])
        ys = np.concatenate([h[1] for h in per_layer[layer]])
        zs = np.concatenate([h[2] for h in per_layer[layer]])
        mcs = np.concatenate([h[3] for h in per_layer[layer]])
        n_noise = int(round(noise * len(xs)))
        nphi = rng.uniform(0.0, 2.0 * math.pi, n_noise)
        rho = RADII_CM[layer]
        xs = np.concatenate([xs, rho * np.cos(nphi)])
        ys = np.concatenate([ys, rho * np.sin(nphi)])
        zs = np.concatenate([zs, rng.uniform(-HALF_LENGTHS_CM[layer], HALF_LENGTHS_CM[layer], n_noise)])
        mcs = np.concatenate([mcs, np.full(n_noise, -1, np.int32)])
        perm = rng.permutation(len(xs))
        arr = np.zeros(len(xs), CLUSTER_DTYPE)
        arr["x"] = xs[perm]
        arr["y"] = ys[perm]
        arr["z"] = zs[perm]
        arr["mc"] = mcs[perm]
        arr["alpha"] = np.arctan2(arr["y"].astype(np.float64), arr["x"].astype(np.float64)).astype(np.float32)
        arr["id"] = np.arange(next_id, next_id + len(arr), dtype=np.int32)
        next_id += len(arr)
        layers.append(arr)
    return Event(vertices=vertices, layers=layers, labels=np.concatenate(labels))


# Workload presets (sizes of the benchmark configurations).
def pp_event(seed: int) -> Event:
    """pp-like: 60 tracks, pT mean 0.5 GeV/c, 1% noise."""
    return make_event(seed, 60, pt_mean=0.5, noise=0.01)


def pbpb_event(seed: int, n_tracks: int = 6000) -> Event:
    """Central Pb-Pb-like: 6000 tracks, pT mean 0.6 GeV/c, 5% noise."""
    return make_event(seed, n_tracks, pt_mean=0.6, noise=0.05)


def batch_multiplicities(seed: int, n_events: int = 256, lo: int = 20, hi: int = 8000) -> np.ndarray:
    """The track counts of an uneven batch: log-uniform over [lo, hi]."""
    rng = np.random.default_rng(seed)
    return np.rint(np.exp(rng.uniform(math.log(lo), math.log(hi), n_events))).astype(int)


def batch_event(seed: int, index: int, n_tracks: int) -> Event:
    """Event `index` of the uneven batch of `seed` (its own vertex, 5% noise)."""
    return make_event(seed * 100003 + index, int(n_tracks), pt_mean=0.6, noise=0.05)


def batch_events(seed: int, n_events: int = 256, lo: int = 20, hi: int = 8000, indices=None) -> list:
    """Uneven batch: multiplicity log-uniform over [lo, hi] tracks, own vertex per event; only the
    events at `indices` when given (a rank's shard of the batch)."""
    mults = batch_multiplicities(seed, n_events, lo, hi)
    idx = range(n_events) if indices is None else indices
    return [batch_event(seed, i, mults[i]) for i in idx]


def jet_event(seed: int, n_tracks: int = 100) -> Event:
    """A dense jet-like cone: ``n_tracks`` stiff tracks within 0.06 rad of azimuth and 0.06 of
    pseudorapidity, no noise. Inner clusters there have more tracklets than the count pass keeps
    per cluster, and tracklets more outgoing tracklets than the cell pass's pair mask holds."""
    return make_event(seed, n_tracks, pt_mean=3.0, noise=0.0, eta_range=(0.0, 0.06), phi_range=(1.0, 1.06))


def pileup_frame(seed: int, collisions: int = 5, n_tracks: int = 1500) -> Event:
    """Pile-up frame: 5 overlapping 1500-track collisions, 10% noise."""
    return make_event(seed, n_tracks, pt_mean=0.6, noise=0.10, n_vertices=collisions)


def write_reference_events(events, path: str) -> None:
    """Write events in the reference text format read by IOUtils::loadEventData
    (IOUtils.cxx:38-78): one "-1 x y z" line per vertex, then one
    "layer x y z _ _ _ alpha mc" line per cluster. Nine significant digits make every
    binary32 value round-trip exactly through the reference's float parser."""
    with open(path, "w") as f:
        for ev in events:
            for v in ev.vertices:
                f.write("-1\t%.9g\t%.9g\t%.9g\n" % (float(v[0]), float(v[1]), float(v[2])))
            for layer, arr in enumerate(ev.layers):
                for c in arr:
                    f.write(
                        "%d\t%.9g\t%.9g\t%.9g\t0\t0\t0\t%.9g\t%d\n"
                        % (layer, float(c["x"]), float(c["y"]), float(c["z"]), float(c["alpha"]), int(c["mc"]))
                    )


def write_reference_labels(events, path: str) -> None:
    """Labels in the format of IOUtils::loadLabels (IOUtils.cxx:80-123): a header line,
    then "mc pT phi eta pdg nClusters" per particle and "-1" after each event."""
    with open(path, "w") as f:
        f.write("mc\tpt\tphi\teta\tpdg\tncl\n")
        for ev in events:
            for lab in ev.labels:
                f.write(
                    "%d\t%.9g\t%.9g\t%.9g\t%d\t%d\n"
                    % (int(lab["mc"]), float(lab["pt"]), float(lab["phi"]), float(lab["eta"]), int(lab["pdg"]), int(lab["ncl"]))
                )
            f.write("-1\n")


def pack_batch(events, vertex_index=None):
    """Flatten events (one vertex each) into the batch layout of the C ABI:
    clusters event-major then layer-major, layer_offsets[n_events*7+1], vertices[n_events*3].
    ``vertex_index`` picks the vertex of multi-vertex events (default 0); to run every vertex,
    list an event once per vertex."""
    if vertex_index is None:
        vertex_index = [0] * len(events)
    counts = []
    for ev in events:
        counts.extend(len(l) for l in ev.layers)
    offsets = np.zeros(len(counts) + 1, np.int32)
    np.cumsum(counts, out=offsets[1:])
    clusters = np.concatenate([l for ev in events for l in ev.layers]) if counts else np.zeros(0, CLUSTER_DTYPE)
    vertices = np.stack([ev.vertices[vi] for ev, vi in zip(events, vertex_index)]).astype(np.float32)
    return clusters, offsets, vertices.reshape(-1)


def write_binary_events(events, path: str) -> None:
    """Binary event file "ITSUEVT1" read by the reference harness (oracle/ref_harness.cpp):
    int32 n_events; per event int32 n_vertices, float32 xyz per vertex, int32 counts[7], then per
    cluster float32 x, y, z, alpha and int32 mc, layer by layer (cluster ids are implied by order,
    as in the reference's text loader)."""
    rec = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("alpha", "<f4"), ("mc", "<i4")])
    with open(path, "wb") as f:
        f.write(b"ITSUEVT1")
        f.write(np.array([len(events)], np.int32).tobytes())
        for ev in events:
            f.write(np.array([len(ev.vertices)], np.int32).tobytes())
            f.write(np.ascontiguousarray(ev.vertices, np.float32).tobytes())
            f.write(np.array([len(l) for l in ev.layers], np.int32).tobytes())
            for l in ev.layers:
                r = np.zeros(len(l), rec)
                for k in ("x", "y", "z", "alpha", "mc"):
                    r[k] = l[k]
                f.write(r.tobytes())


def pack_frames(frames):
    """Flatten pile-up frames for itsu_frames_run_host: clusters frame-major then layer-major,
    frame_offsets[n_frames*7+1], vertices[n_vertices*3] and each vertex's frame index."""
    counts = []
    for ev in frames:
        counts.extend(len(l) for l in ev.layers)
    offsets = np.zeros(len(counts) + 1, np.int32)
    np.cumsum(counts, out=offsets[1:])
    clusters = np.concatenate([l for ev in frames for l in ev.layers]) if counts else np.zeros(0, CLUSTER_DTYPE)
    vertices = np.concatenate([ev.vertices for ev in frames]).astype(np.float32).reshape(-1)
    vertex_frame = np.concatenate([np.full(len(ev.vertices), f, np.int32) for f, ev in enumerate(frames)])
    return clusters, offsets, vertices, vertex_frame


def pileup_stream(seed: int, n_frames: int, collisions: int = 5, n_tracks: int = 1500, spread: float = 0.3) -> list:
    """Pile-up frames of uneven size: each collision's multiplicity is drawn uniformly within
    +-spread of n_tracks."""
    rng = np.random.default_rng(seed)
    out = []
    for f in range(n_frames):
        m = int(rng.integers(int(n_tracks * (1 - spread)), int(n_tracks * (1 + spread)) + 1))
        out.append(make_event(seed * 1000003 + f, m, pt_mean=0.6, noise=0.10, n_vertices=collisions))
    return out
