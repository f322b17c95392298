"""Event and label files of the reference, the road report and the pile-up merger.

Same formats and semantics as the reference's tools:
  read_reference_events  IOUtils::loadEventData   (src/CA/IOUtils.cxx:38-78)
  read_reference_labels  IOUtils::loadLabels      (src/CA/IOUtils.cxx:80-123)
  write_roads_report     IOUtils::writeRoadsReport (src/CA/IOUtils.cxx:125-170), from the road
                         classes the library computes on the device (itsu_roads_report)
  merge_pileup           mergeEvents / mergeLabels of benchmarks/scripts/root/generatePileUpData.cxx
  read_binary_events     the binary event format of itsu.gen.write_binary_events (no parsing)
The writers of the input formats are itsu.gen.write_reference_events / _labels / write_binary_events.
"""
from __future__ import annotations

import ctypes
import math
import os
import re

import numpy as np

from . import gen

PRIMARY_VERTEX_LAYER = -1   # IOUtils.cxx:28 (a "-1 x y z" line is a primary vertex)
LABELS_SEPARATOR = -1       # IOUtils.cxx:29 (a "-1" line ends an event's labels)
PION_CODE = 211             # Constants::PDGCodes::PionCode
MONTE_CARLO_OFFSET = 100000  # generatePileUpData.cxx:31

ROAD_UNREPORTED, ROAD_CORRECT, ROAD_DUPLICATE, ROAD_FAKE = 0, 1, 2, 3

# itsu_label (include/itsu.h), the reference's Label layout: the generator's label records
LABEL_DTYPE = gen.LABEL_DTYPE

_INT = re.compile(r"[+-]?\d+")
_libc = None


def _strtof(token: str) -> np.float32:
    global _libc
    if _libc is None:
        _libc = ctypes.CDLL(None)
        _libc.strtof.restype = ctypes.c_float
        _libc.strtof.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    return np.float32(_libc.strtof(token.encode(), None))


def parse_floats(tokens) -> np.ndarray:
    """Tokens to binary32 exactly as the C library's strtof (what `stream >> float` uses): a
    float64 parse, then a float64 -> float32 rounding, redone with strtof for the values where
    rounding twice can differ (a float64 exactly halfway between two float32)."""
    if len(tokens) == 0:
        return np.zeros(0, np.float32)
    d = np.array(tokens, dtype=np.float64)
    f = d.astype(np.float32)
    with np.errstate(invalid="ignore", over="ignore"):
        back = f.astype(np.float64)
        half = np.spacing(np.abs(f)).astype(np.float64) / 2
        tie = np.isfinite(d) & (np.abs(d - back) == half)
    for i in np.nonzero(tie)[0]:
        f[i] = _strtof(tokens[i])
    return f


def _leading_int(token: str):
    m = _INT.match(token)
    return int(m.group(0)) if m else None


def read_reference_events(path: str) -> list:
    """IOUtils::loadEventData: a "-1 x y z" line adds a primary vertex, opening a new event unless
    it follows another vertex line; a cluster line "layer x y z _ _ _ alpha mc" adds a cluster to
    its layer with the next cluster id of the event (ids run over the event in file order)."""
    raw = []  # per event: [vertices, [per layer: (ids, x, y, z, alpha, mc) token lists]]
    cluster_id = LABELS_SEPARATOR
    with open(path) as f:
        for line in f:
            tok = line.split()
            if len(tok) < 4:
                continue
            layer = _leading_int(tok[0])
            if layer is None:
                continue
            if layer == PRIMARY_VERTEX_LAYER:
                if cluster_id != 0:
                    raw.append([[], [[[], [], [], [], [], []] for _ in range(gen.LAYERS)]])
                raw[-1][0].append(tok[1:4])
                cluster_id = 0
            elif len(tok) >= 9:
                if not raw:
                    raise ValueError("%s: a cluster line before any primary vertex" % path)
                if not 0 <= layer < gen.LAYERS:
                    raise ValueError("%s: cluster on layer %d" % (path, layer))
                cols = raw[-1][1][layer]
                mc = _leading_int(tok[8])
                if mc is None:
                    continue
                cols[0].append(cluster_id)
                for k, t in enumerate((tok[1], tok[2], tok[3], tok[7])):
                    cols[1 + k].append(t)
                cols[5].append(mc)
                cluster_id += 1
    events = []
    for vertices, layers in raw:
        v = parse_floats([t for vx in vertices for t in vx]).reshape(-1, 3)
        arrays = []
        for cols in layers:
            a = np.zeros(len(cols[0]), gen.CLUSTER_DTYPE)
            a["id"] = cols[0]
            a["x"], a["y"], a["z"], a["alpha"] = (parse_floats(c) for c in cols[1:5])
            a["mc"] = cols[5]
            arrays.append(a)
        events.append(gen.Event(vertices=v, layers=arrays, labels=np.zeros(0, gen.LABEL_DTYPE)))
    return events


BINARY_MAGIC = b"ITSUEVT1"
_BINARY_RECORD = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("alpha", "<f4"), ("mc", "<i4")])


def read_binary_events(path: str) -> list:
    """The binary event file written by itsu.gen.write_binary_events (and read by the reference
    harness): the events of the text format without parsing, cluster ids implied by order as in
    loadEventData. A fast loader for large samples; read_reference_events(f) and
    read_binary_events(g) give the same events when g was written from f's events."""
    buf = np.fromfile(path, np.uint8)
    if buf[:8].tobytes() != BINARY_MAGIC:
        raise ValueError("%s: not an ITSUEVT1 file" % path)
    pos = 8

    def take(dtype, count):
        nonlocal pos
        a = np.frombuffer(buf, dtype, count, pos)
        pos += a.nbytes
        return a

    n_events = int(take(np.int32, 1)[0])
    events = []
    for _ in range(n_events):
        nv = int(take(np.int32, 1)[0])
        vertices = take(np.float32, 3 * nv).reshape(nv, 3).copy()
        counts = take(np.int32, gen.LAYERS)
        layers, next_id = [], 0
        for n in counts:
            r = take(_BINARY_RECORD, int(n))
            a = np.zeros(int(n), gen.CLUSTER_DTYPE)
            for k in ("x", "y", "z", "alpha", "mc"):
                a[k] = r[k]
            a["id"] = np.arange(next_id, next_id + int(n), dtype=np.int32)
            next_id += int(n)
            layers.append(a)
        events.append(gen.Event(vertices=vertices, layers=layers, labels=np.zeros(0, gen.LABEL_DTYPE)))
    return events


def read_reference_labels(path: str) -> list:
    """IOUtils::loadLabels: the first line is a header; "mc pT phi eta pdg nClusters" lines are
    kept when |pdg| == 211 and nClusters == 7 (a repeated id keeps its first entry); a "-1" line
    closes an event's map, and the maps end with the one open at the end of the file (empty
    after a final "-1"). Returns one LABEL_DTYPE array per map, entries in file order."""
    maps, current, seen = [], [], set()
    with open(path) as f:
        f.readline()
        for line in f:
            tok = line.split()
            if not tok:
                continue
            mc = _leading_int(tok[0])
            if mc is None:
                continue
            if mc == LABELS_SEPARATOR:
                maps.append(current)
                current, seen = [], set()
            elif len(tok) >= 6:
                pdg, ncl = _leading_int(tok[4]), _leading_int(tok[5])
                if pdg is not None and ncl is not None and abs(pdg) == PION_CODE and ncl == 7 and mc not in seen:
                    seen.add(mc)
                    current.append((mc, tok[1], tok[2], tok[3], pdg, ncl))
    maps.append(current)
    out = []
    for m in maps:
        a = np.zeros(len(m), LABEL_DTYPE)
        if m:
            a["mc"] = [r[0] for r in m]
            for k, name in ((1, "pt"), (2, "phi"), (3, "eta")):
                a[name] = parse_floats([r[k] for r in m])
            a["pdg"] = [r[4] for r in m]
            a["ncl"] = [r[5] for r in m]
        out.append(a)
    return out


def labels_for_report(label_maps) -> tuple:
    """The per-event maps as the itsu_roads_report arguments: labels (LABEL_DTYPE, event-major) and
    label_offsets[n_events + 1]."""
    offsets = np.zeros(len(label_maps) + 1, np.int32)
    np.cumsum([len(m) for m in label_maps], out=offsets[1:])
    labels = np.concatenate(list(label_maps)) if len(label_maps) and offsets[-1] else np.zeros(0, LABEL_DTYPE)
    return np.ascontiguousarray(labels, LABEL_DTYPE), offsets


def _g(x: float) -> str:
    """A float as `std::ostream << float` prints it: %g, 6 significant digits."""
    v = float(x)
    if math.isnan(v):
        return "-nan" if math.copysign(1.0, v) < 0 else "nan"
    return "%g" % v


def format_label(row) -> str:
    """operator<<(std::ostream&, const Label&) (src/CA/Label.cxx:32-37)."""
    return "%d\t%s\t%s\t%s\t%d\t%d" % (int(row["mc"]), _g(row["pt"]), _g(row["phi"]), _g(row["eta"]), int(row["pdg"]),
                                       int(row["ncl"]))


def write_roads_report(streams, roads, run_offsets, road_class, label_maps, run_event=None) -> None:
    """IOUtils::writeRoadsReport for every event in turn, as main.cpp calls it (main.cpp:131-135),
    label_maps holding one map per event (the loaded maps cut to the events' count):
    streams = (correct, duplicate, fake) open text files; "-1" opens each event in the correct and
    fake streams (not the duplicate one); each reported road writes its label to the stream of
    its class (road_class from itsu_roads_report or the oracle), in road order."""
    correct, duplicate, fake = streams
    out = {ROAD_CORRECT: correct, ROAD_DUPLICATE: duplicate, ROAD_FAKE: fake}
    n_runs = len(run_offsets) - 1
    r = 0
    for e, m in enumerate(label_maps):
        correct.write("%d\n" % LABELS_SEPARATOR)
        fake.write("%d\n" % LABELS_SEPARATOR)
        by_id = {int(row["mc"]): row for row in m}
        while r < n_runs and (run_event[r] if run_event is not None else r) == e:
            for i in range(int(run_offsets[r]), int(run_offsets[r + 1])):
                cls = int(road_class[i])
                if cls != ROAD_UNREPORTED:
                    out[cls].write(format_label(by_id[int(roads[i]["label"])]) + "\n")
            r += 1


def _merge(pile_up: int, src: str, dst: str, columns: int, mc_column: int, labels: bool) -> None:
    """The shared loop of mergeEvents / mergeLabels (generatePileUpData.cxx:44-207), as text: lines
    whose first token is not an integer are dropped; from the second vertex of a frame on, the
    Monte Carlo id column is offset by (vertex - 1) * 100000 and the line re-joined with tabs."""
    held = []
    vertices = 0
    with open(src) as f, open(dst, "w") as out:
        for line in f:
            line = line.rstrip("\n")
            tok = line.split()
            first = _leading_int(tok[0]) if tok else None
            if first is None:
                continue
            if first == PRIMARY_VERTEX_LAYER:
                if vertices == pile_up:
                    if labels:
                        out.write(line + "\n")
                    for h in held:
                        out.write(h + "\n")
                    vertices = 0
                    held = []
                if not labels:
                    out.write(line + "\n")
                vertices += 1
            else:
                data = [str(first)] + tok[1:columns] + [""] * max(0, columns - len(tok))
                if vertices > 1:
                    mc = _leading_int(data[mc_column])
                    data[mc_column] = str(mc + (vertices - 1) * MONTE_CARLO_OFFSET)
                    held.append("\t".join(data[:columns]))
                else:
                    held.append(line)
        if labels:
            out.write("%d\n" % PRIMARY_VERTEX_LAYER)
        for h in held:
            out.write(h + "\n")


def merge_pileup(pile_up: int, input_folder: str, output_folder: str = None) -> None:
    """generatePileUpData(pileUp, inputFolder, outputFolder): data.txt -> merged_data.txt (frames of
    pile_up vertices, cluster Monte Carlo ids of the k-th vertex offset by (k-1)*100000) and
    labels.txt -> merged_labels.txt (same offsets; the reference's label grouping, including its
    first frame, is kept as it is)."""
    output_folder = input_folder if output_folder is None else output_folder
    _merge(pile_up, os.path.join(input_folder, "data.txt"), os.path.join(output_folder, "merged_data.txt"), 10, 8, False)
    _merge(pile_up, os.path.join(input_folder, "labels.txt"), os.path.join(output_folder, "merged_labels.txt"), 6, 0, True)


# ---- memory occupancy (Tracker::clustersToTracksMemoryBenchmark, src/CA/Tracker.cxx:304-363) ----

# Constants::Memory (include/ITSReconstruction/CA/Constants.h:87-92): the reference's preallocation
# coefficients, reserve = ceil(coefficient * N_L * N_L+1 (* N_L+2 for cells)) in binary32
TRACKLETS_MEMORY_COEFFICIENTS = np.array([0.0016353, 0.0013627, 0.000984, 0.00078135, 0.00057934, 0.00052217], np.float32)
CELLS_MEMORY_COEFFICIENTS = np.array([2.3208e-08, 2.104e-08, 1.6432e-08, 1.2412e-08, 1.3543e-08], np.float32)


def _reserve(capacity: int, size_f: np.float32) -> int:
    """`if (size > v.capacity()) v.reserve(size)` with a float size (PrimaryVertexContext.cxx:60-64,
    125-130): the comparison in binary32, reserve() of the truncated value."""
    return int(size_f) if size_f > np.float32(capacity) else capacity


def _grow(capacity: int, size: int) -> int:
    """The capacity after `size` emplace_backs into a cleared vector (libstdc++: a full vector of n
    elements reallocates to n + max(n, 1))."""
    while capacity < size:
        capacity = capacity + max(capacity, 1)
    return capacity


class MemoryModel:
    """The reference tracker's per-layer vectors (tracklets, cells) across the vertices it runs:
    cleared and reserved from the coefficients at each initialize, grown by push_back, never
    shrunk. run() takes one vertex's counts and returns its MemoryOccupancy.txt lines (the CPU
    build's six lines)."""

    def __init__(self):
        self.trk_cap = [0] * (gen.LAYERS - 1)
        self.cell_cap = [0] * 5

    def run(self, n, t, c, roads: int) -> str:
        n = [int(x) for x in n]
        nf = [np.float32(x) for x in n]
        for l in range(5):
            size = np.float32(np.ceil(np.float32(np.float32(CELLS_MEMORY_COEFFICIENTS[l] * nf[l]) * nf[l + 1]) * nf[l + 2]))
            self.cell_cap[l] = _reserve(self.cell_cap[l], size)
        for l in range(gen.LAYERS - 1):
            size = np.float32(np.ceil(np.float32(TRACKLETS_MEMORY_COEFFICIENTS[l] * nf[l]) * nf[l + 1]))
            self.trk_cap[l] = _reserve(self.trk_cap[l], size)
        lines = ["".join("%d\t" % x for x in n), "".join("%d\t" % x for x in self.trk_cap)]
        for l in range(gen.LAYERS - 1):
            self.trk_cap[l] = _grow(self.trk_cap[l], int(t[l]))
        lines += ["".join("%d\t" % int(x) for x in t), "".join("%d\t" % x for x in self.cell_cap)]
        for l in range(5):
            self.cell_cap[l] = _grow(self.cell_cap[l], int(c[l]))
        lines += ["".join("%d\t" % int(x) for x in c), "%d" % int(roads)]
        return "\n".join(lines) + "\n"


def memory_occupancy(warmup_runs, runs) -> str:
    """MemoryOccupancy.txt as the reference's MEMORY_BENCHMARK build writes it (main.cpp:67-70,
    85-86): the warm-up event's vertices first (not written), then one six-line block per vertex.
    Each run is (clusters[7], tracklets[6], cells[5], roads), e.g. from itsu_get_counts."""
    model = MemoryModel()
    for n, t, c, r in warmup_runs:
        model.run(n, t, c, r)
    return "".join(model.run(n, t, c, r) for n, t, c, r in runs)
