"""Python side of the oracle: the C restatement (liboracle.so) and the reference harness.

TEST INFRASTRUCTURE ONLY. Imported by tests/, by __graft_entry__.smoke() and by bench.py's
CPU-baseline leg, as the checker. Results of both sources are returned in one canonical form
(a dict of numpy arrays per vertex) so they compare field by field and bit by bit.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "tracking-itsu_b200"))

from itsu.gen import CLUSTER_DTYPE  # noqa: E402

TRACKLET_DTYPE = np.dtype([("c1", "<i4"), ("c2", "<i4"), ("tan_lambda", "<f4"), ("phi", "<f4")])
CELL_DTYPE = np.dtype(
    [
        ("c1", "<i4"),
        ("c2", "<i4"),
        ("c3", "<i4"),
        ("t1", "<i4"),
        ("t2", "<i4"),
        ("nx", "<f4"),
        ("ny", "<f4"),
        ("nz", "<f4"),
        ("curvature", "<f4"),
        ("level", "<i4"),
    ]
)
ROAD_DTYPE = np.dtype([("cells", "<i4", (5,)), ("size", "<i4"), ("label", "<i4"), ("fake", "u1"), ("pad", "u1", (3,))])
assert TRACKLET_DTYPE.itemsize == 16 and CELL_DTYPE.itemsize == 40 and ROAD_DTYPE.itemsize == 32

LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_KINDS = dict(clusters=0, index_table=1, tracklets=2, trk_lookup=3, cells=4, cell_lookup=5, nb_offsets=6, nb=7, roads=8)


def build(force: bool = False) -> str:
    """Compile the C restatement (gcc, no FMA contraction)."""
    src = os.path.join(HERE, "itsu_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(
        os.path.getmtime(src), os.path.getmtime(os.path.join(ROOT, "include", "itsu_atan2f.h"))
    ):
        subprocess.check_call(
            ["gcc", "-std=c99", "-O2", "-Wall", "-ffp-contract=off", "-fPIC", "-shared", src, "-o", LIB_PATH, "-lm"]
        )
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()  # rebuilt when the sources are newer
        L = ctypes.CDLL(LIB_PATH)
        L.oracle_run_vertex.restype = ctypes.c_void_p
        L.oracle_run_vertex.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_size.restype = ctypes.c_int64
        L.oracle_size.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.oracle_data.restype = ctypes.c_void_p
        L.oracle_data.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.oracle_free.argtypes = [ctypes.c_void_p]
        L.oracle_atan2f.restype = ctypes.c_float
        L.oracle_atan2f.argtypes = [ctypes.c_float, ctypes.c_float]
        L.oracle_atan2f_n.restype = None
        L.oracle_atan2f_n.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
        L.oracle_run_batch.restype = ctypes.c_int64
        L.oracle_run_batch.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32]
        L.oracle_roads_report.restype = ctypes.c_int
        L.oracle_roads_report.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int32] + [ctypes.c_void_p] * 2 + [ctypes.c_int32] + [ctypes.c_void_p] * 2
        _lib = L
    return _lib


def _array(ptr, n, dtype):
    if n <= 0:
        return np.zeros(0, dtype)
    buf = (ctypes.c_char * (n * np.dtype(dtype).itemsize)).from_address(ptr)
    return np.frombuffer(buf, dtype=dtype, count=n).copy()


def run_vertex(layers, vertex) -> dict:
    """Run the C restatement on one vertex; layers = 7 CLUSTER_DTYPE arrays."""
    L = lib()
    layers = [np.ascontiguousarray(l, dtype=CLUSTER_DTYPE) for l in layers]
    ptrs = (ctypes.c_void_p * 7)(*[l.ctypes.data if len(l) else 0 for l in layers])
    counts = (ctypes.c_int32 * 7)(*[len(l) for l in layers])
    v = (ctypes.c_float * 3)(*[float(x) for x in vertex])
    h = L.oracle_run_vertex(ptrs, counts, v)
    if not h:
        raise MemoryError("oracle_run_vertex failed")
    try:
        get = lambda kind, layer, dt: _array(L.oracle_data(h, _KINDS[kind], layer), L.oracle_size(h, _KINDS[kind], layer), dt)
        res = dict(
            vertex=np.array(vertex, np.float32),
            clusters=[get("clusters", l, CLUSTER_DTYPE) for l in range(7)],
            index_tables=np.stack([get("index_table", l, np.int32) for l in range(6)]),
            tracklets=[get("tracklets", l, TRACKLET_DTYPE) for l in range(6)],
            trk_lookup=[get("trk_lookup", l, np.int32) for l in range(5)],
            cells=[get("cells", l, CELL_DTYPE) for l in range(5)],
            cell_lookup=[get("cell_lookup", l, np.int32) for l in range(4)],
            nb_offsets=[get("nb_offsets", l, np.int32) for l in range(4)],
            nb=[get("nb", l, np.int32) for l in range(4)],
            roads=get("roads", 0, ROAD_DTYPE),
        )
    finally:
        L.oracle_free(h)
    return canonical(res)


def canonical(res: dict) -> dict:
    """Canonical form: cells lookup L has one entry per tracklet of layer L+1 (-1 when absent);
    road padding bytes zeroed."""
    for l in range(4):
        n = len(res["tracklets"][l + 1])
        lk = np.full(n, -1, np.int32)
        src = res["cell_lookup"][l]
        m = min(n, len(src))
        lk[:m] = src[:m]
        if len(src) > n:
            assert np.all(src[n:] == -1), "cells lookup has entries beyond the tracklets"
        res["cell_lookup"][l] = lk
    roads = res["roads"].copy()
    roads["pad"] = 0
    res["roads"] = roads
    return res


# ---- reference harness (oracle/_ref, built by build_ref.sh) ----


def ref_binary(variant: str = "cr") -> str:
    return os.path.join(REF_DIR, "ref_" + variant)


def ref_available(variant: str = "cr") -> bool:
    return os.access(ref_binary(variant), os.X_OK)


def run_reference(events, workdir: str, variant: str = "cr") -> list:
    """Write events in the reference text format, run the patched reference, parse its dump."""
    from itsu.gen import write_reference_events

    txt = os.path.join(workdir, "events.txt")
    out = os.path.join(workdir, "dump_%s.bin" % variant)
    write_reference_events(events, txt)
    subprocess.check_call([ref_binary(variant), "dump", txt, out])
    return parse_dump(out)


def parse_dump(path: str) -> list:
    data = open(path, "rb").read()
    assert data[:8] == b"ITSUREF1", "not a reference dump"
    pos = 8

    def i32():
        nonlocal pos
        v = int(np.frombuffer(data, np.int32, 1, pos)[0])
        pos += 4
        return v

    def arr(n, dt):
        nonlocal pos
        a = np.frombuffer(data, dt, n, pos).copy() if n else np.zeros(0, dt)
        pos += n * np.dtype(dt).itemsize
        return a

    records = i32()
    out = []
    road_raw = np.dtype([("cells", "<i4", (5,)), ("size", "<i4"), ("label", "<i4"), ("fake", "<i4")])
    for _ in range(records):
        event, vertex = i32(), i32()
        pv = arr(3, np.float32)
        clusters = [arr(i32(), CLUSTER_DTYPE) for _ in range(7)]
        tables = np.stack([arr(401, np.int32) for _ in range(6)])
        tracklets = [arr(i32(), TRACKLET_DTYPE) for _ in range(6)]
        trk_lookup = [arr(i32(), np.int32) for _ in range(5)]
        cells = [arr(i32(), CELL_DTYPE) for _ in range(5)]
        cell_lookup = [arr(i32(), np.int32) for _ in range(4)]
        nb_offsets, nb = [], []
        for l in range(4):
            k = i32()
            lists = [arr(i32(), np.int32) for _ in range(k)]
            rows = len(cells[l + 1])
            assert k in (0, rows), "neighbour table size %d for %d cells" % (k, rows)
            offs = np.zeros(rows + 1, np.int32)
            if k:
                offs[1:] = np.cumsum([len(x) for x in lists])
            nb_offsets.append(offs)
            nb.append(np.concatenate(lists).astype(np.int32) if k and offs[-1] else np.zeros(0, np.int32))
        rr = arr(i32(), road_raw)
        roads = np.zeros(len(rr), ROAD_DTYPE)
        roads["cells"] = rr["cells"]
        roads["size"] = rr["size"]
        roads["label"] = rr["label"]
        roads["fake"] = rr["fake"].astype(np.uint8)
        out.append(
            canonical(
                dict(
                    event=event,
                    vertex_index=vertex,
                    vertex=pv,
                    clusters=clusters,
                    index_tables=tables,
                    tracklets=tracklets,
                    trk_lookup=trk_lookup,
                    cells=cells,
                    cell_lookup=cell_lookup,
                    nb_offsets=nb_offsets,
                    nb=nb,
                    roads=roads,
                )
            )
        )
    assert pos == len(data), "trailing bytes in dump"
    return out


FIELDS = ("clusters", "index_tables", "tracklets", "trk_lookup", "cells", "cell_lookup", "nb_offsets", "nb", "roads")


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint8).reshape(-1)


def diff(a: dict, b: dict) -> list:
    """Bitwise comparison of two canonical results; returns a list of mismatch descriptions."""
    out = []
    for f in FIELDS:
        x, y = a[f], b[f]
        if isinstance(x, list):
            for l, (xl, yl) in enumerate(zip(x, y)):
                if len(xl) != len(yl):
                    out.append("%s[%d]: size %d vs %d" % (f, l, len(xl), len(yl)))
                elif not np.array_equal(_bits(xl), _bits(yl)):
                    out.append("%s[%d]: contents differ" % (f, l))
        else:
            if x.shape != y.shape or not np.array_equal(_bits(x), _bits(y)):
                out.append("%s: contents differ" % f)
    return out


def canonical_sets(res: dict) -> dict:
    """Order-free form keyed by cluster ids: tracklets (L, id1, id2), cells (L, id1, id2, id3),
    roads as tuples of 7 cluster ids. Used to compare runs whose sort order differs."""
    ids = [c["id"] for c in res["clusters"]]
    trk = []
    for l, t in enumerate(res["tracklets"]):
        trk.extend((l, int(ids[l][a]), int(ids[l + 1][b])) for a, b in zip(t["c1"], t["c2"]))
    cel = []
    for l, c in enumerate(res["cells"]):
        cel.extend((l, int(ids[l][a]), int(ids[l + 1][b]), int(ids[l + 2][d])) for a, b, d in zip(c["c1"], c["c2"], c["c3"]))
    roads = []
    for r in res["roads"]:
        cl = []
        for l in range(5):
            ci = r["cells"][l]
            if ci < 0:
                continue
            cell = res["cells"][l][ci]
            if not cl:
                cl.extend([int(ids[l][cell["c1"]]), int(ids[l + 1][cell["c2"]])])
            cl.append(int(ids[l + 2][cell["c3"]]))
        roads.append(tuple(cl))
    return dict(tracklets=sorted(trk), cells=sorted(cel), roads=sorted(roads))


# ---- road report (IOUtils::writeRoadsReport) ----

COUNTS_DTYPE = np.dtype([("labels", "<i4"), ("correct", "<i4"), ("duplicate", "<i4"), ("fake", "<i4")])


def roads_report(roads, run_offsets, label_maps, run_event=None):
    """The C restatement's road classes (ITSU_ROAD_*) and per-event counts for the roads of the
    runs (vertices) in run_offsets and one labels map per event (itsu.io.read_reference_labels)."""
    from itsu import io

    roads = np.ascontiguousarray(roads, ROAD_DTYPE)
    run_offsets = np.ascontiguousarray(run_offsets, np.int32)
    labels, label_offsets = io.labels_for_report(label_maps)
    n_runs, n_events = len(run_offsets) - 1, len(label_maps)
    rev = None if run_event is None else np.ascontiguousarray(run_event, np.int32)
    cls = np.zeros(max(len(roads), 1), np.uint8)
    counts = np.zeros(max(n_events, 1), COUNTS_DTYPE)
    ptr = lambda a: None if a is None or len(a) == 0 else a.ctypes.data  # noqa: E731
    rc = lib().oracle_roads_report(ptr(roads), run_offsets.ctypes.data, ptr(rev), n_runs, ptr(labels), label_offsets.ctypes.data,
                                   n_events, cls.ctypes.data, counts.ctypes.data)
    if rc != 0:
        raise MemoryError("oracle_roads_report failed")
    return cls[:len(roads)], counts[:n_events]


def run_reference_report(events_txt: str, labels_txt: str, outdir: str) -> dict:
    """The reference's own road report (oracle/_ref/ref_cr report): loadEventData + loadLabels,
    clustersToTracks per event and writeRoadsReport into outdir/{Correct,Duplicate,Fake}Roads.txt.
    Returns the harness's JSON line (events, roads, seconds spent in writeRoadsReport)."""
    import json

    out = subprocess.run([ref_binary("cr"), "report", events_txt, labels_txt, outdir], check=True, capture_output=True, text=True)
    return json.loads(out.stdout.strip().splitlines()[-1])
