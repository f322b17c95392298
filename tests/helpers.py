"""Shared test helpers: golden fixtures and the reference event-file reader."""
from __future__ import annotations

import gzip
import os
import tempfile

import numpy as np

from itsu import gen
from oracle import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ("pp", "mid", "empty_layers", "one_bin", "phi_wrap", "z_edges", "phi_boundary", "duplicates", "pileup_small")


def load_reference_events(text: str) -> list:
    """Parse the reference event format the way IOUtils::loadEventData does (IOUtils.cxx:38-78):
    a "-1 x y z" line opens a new event unless it directly follows another vertex line; cluster
    lines are "layer x y z _ _ _ alpha mc"; cluster ids run per event in file order."""
    events = []
    cluster_id = -1
    rows = None
    for line in text.splitlines():
        tok = line.split()
        if len(tok) < 4:
            continue
        try:
            layer = int(tok[0])
            x, y, z = (np.float32(float(t)) for t in tok[1:4])
        except ValueError:
            continue
        if layer == -1:
            if cluster_id != 0:
                rows = [[] for _ in range(7)]
                events.append(([], rows))
            events[-1][0].append((x, y, z))
            cluster_id = 0
        elif len(tok) >= 9:
            rows[layer].append((x, y, z, 0.0, 0.0, cluster_id, np.float32(float(tok[7])), int(tok[8]), 0))
            cluster_id += 1
    out = []
    for vertices, per_layer in events:
        layers = [np.array(r, dtype=gen.CLUSTER_DTYPE) if r else np.zeros(0, gen.CLUSTER_DTYPE) for r in per_layer]
        out.append(gen.Event(vertices=np.array(vertices, np.float32), layers=layers, labels=np.zeros(0, gen.LABEL_DTYPE)))
    return out


def load_case(name: str):
    """(events, expected per-vertex results) of one golden fixture."""
    with gzip.open(os.path.join(GOLDEN, name + ".events.txt.gz"), "rt") as f:
        events = load_reference_events(f.read())
    with tempfile.NamedTemporaryFile(suffix=".bin") as tmp:
        with gzip.open(os.path.join(GOLDEN, name + ".ref.bin.gz"), "rb") as f:
            tmp.write(f.read())
        tmp.flush()
        expected = oracle.parse_dump(tmp.name)
    return events, expected


def vertex_runs(events):
    """(event, vertex index) pairs in the reference's loop order (Tracker.cxx:251)."""
    return [(ev, iv) for ev in events for iv in range(len(ev.vertices))]


def beyond_z_event(seed: int, n_beyond: int = 700):
    """A 2000-track event plus ``n_beyond`` clusters in each of layers 1, 2 and 5 whose z lies
    beyond the tracker's half-length of that layer, most of them in phi bin 0, where that gives a
    negative bin (sorted apart from the index table, PrimaryVertexContext.cxx:52-54), many of them
    sharing a bin so that the stable order of ties matters, and a few beyond +z (bin 400)."""
    rng = np.random.default_rng(seed)
    ev = gen.make_event(seed, 2000)
    half = {1: 16.333, 2: 16.333, 5: 73.745}
    radius = {1: 3.1, 2: 3.9, 5: 34.4}
    layers = list(ev.layers)
    for layer in (1, 2, 5):
        extra = np.zeros(n_beyond, gen.CLUSTER_DTYPE)
        # a bin is phi bin * 20 + z bin: negative only in phi bin 0 (phi < 2 pi / 20)
        phi = rng.uniform(0.0, 0.3, n_beyond)
        phi[: n_beyond // 2] = rng.choice([0.05, 0.2], n_beyond // 2)  # shared phi values
        phi[-n_beyond // 10:] = rng.uniform(0.0, 2.0 * np.pi, n_beyond // 10)  # the rest elsewhere
        z = -half[layer] - rng.uniform(0.0, 400.0, n_beyond)
        z[: n_beyond // 3] = -half[layer] - 5.0  # shared z bin as well: exact ties
        z[-10:] = half[layer] + rng.uniform(1.0, 5.0, 10)  # beyond +z: bin 400
        extra["x"] = (radius[layer] * np.cos(phi)).astype(np.float32)
        extra["y"] = (radius[layer] * np.sin(phi)).astype(np.float32)
        extra["z"] = z.astype(np.float32)
        extra["mc"] = -1
        # interleave with the layer's own clusters so that input order is not bin order
        merged = np.concatenate([layers[layer], extra])
        layers[layer] = merged[rng.permutation(len(merged))]
    # cluster ids run in file order, as the reference's loader numbers them (IOUtils.cxx:38-78)
    first = 0
    for l in layers:
        l["id"] = np.arange(first, first + len(l))
        first += len(l)
    return gen.Event(vertices=ev.vertices, layers=layers, labels=ev.labels)
