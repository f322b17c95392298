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
