"""Generates the golden fixtures under tests/golden/ from the reference tracker itself.

Run in a checkout where oracle/build_ref.sh has built oracle/_ref/ref_cr (it needs the
reference sources):  python tests/golden/make_golden.py
For each case it writes <case>.events.txt.gz, the reference-format event file the reference
read, and <case>.ref.bin.gz, the reference harness dump (every intermediate list of every
vertex). The cases are seeded synthetic events plus hand-built edge cases; nothing is taken
from the reference's (absent) data files.
"""
from __future__ import annotations

import gzip
import math
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tracking-itsu_b200"))

from itsu import gen  # noqa: E402
from oracle import oracle  # noqa: E402


def _event_from_points(vertex, per_layer, seed=0):
    """Event from explicit (x, y, z, mc) points per layer (7 lists of tuples)."""
    rng = np.random.default_rng(seed)
    layers = []
    next_id = 0
    for pts in per_layer:
        arr = np.zeros(len(pts), gen.CLUSTER_DTYPE)
        if pts:
            p = np.array(pts, dtype=np.float64)
            arr["x"], arr["y"], arr["z"] = p[:, 0], p[:, 1], p[:, 2]
            arr["mc"] = p[:, 3].astype(np.int32)
            arr["alpha"] = np.arctan2(arr["y"], arr["x"]).astype(np.float32)
        arr = arr[rng.permutation(len(arr))]
        arr["id"] = np.arange(next_id, next_id + len(arr), dtype=np.int32)
        next_id += len(arr)
        layers.append(arr)
    labels = np.zeros(0, gen.LABEL_DTYPE)
    return gen.Event(vertices=np.array([vertex], np.float32), layers=layers, labels=labels)


def _clear_layer(ev, layer):
    ev.layers[layer] = ev.layers[layer][:0]
    # keep ids running in file order, as the reference loader assigns them
    nid = 0
    for l in ev.layers:
        l["id"] = np.arange(nid, nid + len(l), dtype=np.int32)
        nid += len(l)
    return ev


def one_bin_event(seed):
    """A narrow jet: every cluster of a layer falls into one phi-z bin."""
    rng = np.random.default_rng(seed)
    per_layer = [[] for _ in range(7)]
    for t in range(40):
        phi = 1.0 + rng.uniform(-0.02, 0.02)
        tl = rng.uniform(-0.01, 0.01)
        for l, r in enumerate(gen.RADII_CM):
            per_layer[l].append((r * math.cos(phi), r * math.sin(phi), 0.2 + tl * r, t))
    return _event_from_points((0.0, 0.0, 0.0), per_layer, seed)


def phi_wrap_event(seed):
    """Straight tracks straddling phi = 0 / 2 pi."""
    rng = np.random.default_rng(seed)
    per_layer = [[] for _ in range(7)]
    for t in range(60):
        phi = rng.uniform(-0.25, 0.25)
        tl = rng.uniform(-0.3, 0.3)
        for l, r in enumerate(gen.RADII_CM):
            per_layer[l].append((r * math.cos(phi), r * math.sin(phi), 0.1 + tl * r, t))
    return _event_from_points((0.0, 0.0, 0.1), per_layer, seed)


def z_edge_event(seed):
    """Clusters at and beyond the tracker's z half-lengths (16.333/42.14/73.745 cm): bins of
    the last z column and z bins of 20 and more, which spill into the next phi row."""
    rng = np.random.default_rng(seed)
    zhalf = (16.333, 16.333, 16.333, 42.140, 42.140, 73.745, 73.745)
    per_layer = [[] for _ in range(7)]
    for l, r in enumerate(gen.RADII_CM):
        for k in range(30):
            phi = rng.uniform(0, 2 * math.pi)
            z = zhalf[l] * rng.choice([-1.0, 1.0]) * rng.uniform(0.97, 1.4)
            per_layer[l].append((r * math.cos(phi), r * math.sin(phi), z, k))
        per_layer[l].append((r, 0.0, zhalf[l], 99))
        per_layer[l].append((0.0, r, -zhalf[l], 98))
        # phi row 0 with a negative z bin: a negative index-table bin, sorted before bin 0
        for k in range(4):
            phi = 0.05 + 0.06 * k
            per_layer[l].append((r * math.cos(phi), r * math.sin(phi), -zhalf[l] * (1.15 + 0.1 * k), 90 + k))
    # straight tracks towards the edges
    for t in range(20):
        phi = rng.uniform(0, 2 * math.pi)
        tl = rng.choice([-1.0, 1.0]) * rng.uniform(1.5, 1.9)
        for l, r in enumerate(gen.RADII_CM):
            per_layer[l].append((r * math.cos(phi), r * math.sin(phi), tl * r, 1000 + t))
    return _event_from_points((0.0, 0.0, 0.0), per_layer, seed)


def _transform_phi(layer, vertex, x, y):
    raw = np.zeros(1, gen.CLUSTER_DTYPE)
    raw["x"], raw["y"] = x, y
    import ctypes

    out = np.zeros(1, gen.CLUSTER_DTYPE)
    v = (ctypes.c_float * 3)(*vertex)
    L = oracle.lib()
    L.oracle_transform_cluster(ctypes.c_int(layer), v, ctypes.c_void_p(raw.ctypes.data), ctypes.c_void_p(out.ctypes.data))
    return float(out["phi"][0]), int(out["bin"][0])


def phi_boundary_event(seed):
    """Clusters whose phi is exactly 2 pi (bin 400) and inner clusters whose phi window edge
    normalises to exactly 2 pi (phi bin 20: the P5 case), next to ordinary tracks."""
    rng = np.random.default_rng(seed)
    two_pi = np.float32(2.0) * np.float32(3.14159265359)
    per_layer = [[] for _ in range(7)]
    vertex = (0.0, 0.0, 0.0)
    # phi == 2 pi: y a hair below the +x axis
    for l, r in enumerate(gen.RADII_CM):
        for k in range(3):
            per_layer[l].append((r, -1e-8 * (k + 1), 0.5 * k, 500 + k))
    # windows ending exactly at 2 pi: search points on layer 0-2 near phi = 2pi - 0.3
    targets = [(lambda p: np.float32(np.float32(p) + np.float32(0.3)) == two_pi),
               (lambda p: np.float32(np.float32(p) - np.float32(0.3)) < 0 and np.float32(np.float32(p) - np.float32(0.3)) + two_pi == two_pi)]
    centres = [2 * math.pi - 0.3, 0.3]
    found = 0
    for l in range(3):
        r = gen.RADII_CM[l]
        for want, centre in zip(targets, centres):
            hits = 0
            for _ in range(400000):
                a = centre + rng.uniform(-2e-6, 2e-6)
                x, y = r * math.cos(a), r * math.sin(a)
                x32, y32 = float(np.float32(x)), float(np.float32(y))
                phi, _ = _transform_phi(l, vertex, x32, y32)
                if want(phi):
                    per_layer[l].append((x32, y32, rng.uniform(-1, 1), 700 + found))
                    found += 1
                    hits += 1
                    if hits >= 2:
                        break
    # ordinary straight tracks around phi ~ 0 so the windows have candidates
    for t in range(30):
        phi = rng.uniform(-0.4, 0.4)
        tl = rng.uniform(-0.2, 0.2)
        for l, r in enumerate(gen.RADII_CM):
            per_layer[l].append((r * math.cos(phi), r * math.sin(phi), tl * r, t))
    return _event_from_points(vertex, per_layer, seed), found


def duplicate_event(seed):
    """Every cluster of a pp event twice (equal bins and coordinates: the stable order)."""
    ev = gen.pp_event(seed)
    nid = 0
    for l in range(7):
        arr = np.concatenate([ev.layers[l], ev.layers[l]])
        arr["id"] = np.arange(nid, nid + len(arr), dtype=np.int32)
        nid += len(arr)
        ev.layers[l] = arr
    return ev


def cases():
    out = {}
    out["pp"] = [gen.pp_event(s) for s in range(1, 9)]
    out["mid"] = [gen.make_event(11, 400, pt_mean=0.6, noise=0.05)]
    out["empty_layers"] = [_clear_layer(gen.pp_event(21), 0), _clear_layer(gen.pp_event(22), 3),
                           _clear_layer(gen.pp_event(23), 6), _clear_layer(_clear_layer(gen.pp_event(24), 2), 5)]
    out["one_bin"] = [one_bin_event(31)]
    out["phi_wrap"] = [phi_wrap_event(32)]
    out["z_edges"] = [z_edge_event(33)]
    ev, found = phi_boundary_event(34)
    print("phi boundary clusters found:", found)
    out["phi_boundary"] = [ev]
    out["duplicates"] = [duplicate_event(35)]
    out["pileup_small"] = [gen.make_event(36, 150, pt_mean=0.6, noise=0.10, n_vertices=3)]
    return out


def main():
    if not oracle.ref_available("cr"):
        raise SystemExit("build the reference first: oracle/build_ref.sh")
    with tempfile.TemporaryDirectory() as d:
        for name, events in cases().items():
            txt = os.path.join(d, name + ".events.txt")
            dump = os.path.join(d, name + ".ref.bin")
            gen.write_reference_events(events, txt)
            subprocess.check_call([oracle.ref_binary("cr"), "dump", txt, dump])
            for src in (txt, dump):
                with open(src, "rb") as fi, gzip.GzipFile(os.path.join(HERE, os.path.basename(src) + ".gz"), "wb", mtime=0) as fo:
                    shutil.copyfileobj(fi, fo)
            recs = oracle.parse_dump(dump)
            print(name, "vertices", len(recs), "tracklets", sum(len(t) for r in recs for t in r["tracklets"]),
                  "cells", sum(len(c) for r in recs for c in r["cells"]), "roads", sum(len(r["roads"]) for r in recs))


if __name__ == "__main__":
    main()
