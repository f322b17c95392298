"""The road report (IOUtils::writeRoadsReport), the event and label loaders (IOUtils::loadEventData,
IOUtils::loadLabels) and the pile-up merger (generatePileUpData.cxx), on the CPU: the oracle's
classification and itsu.io's readers, writer and merger against the reference's own output,
byte for byte (fixtures in tests/golden/report/ made by tests/golden/make_report_golden.py; a
fresh seeded case through the reference harness when oracle/_ref is built)."""
import ctypes
import gzip
import os
import subprocess

import numpy as np
import pytest

from itsu import gen, io
from oracle import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "report")
REPORT_FILES = ("CorrectRoads.txt", "DuplicateRoads.txt", "FakeRoads.txt")


def _golden(name: str) -> str:
    with gzip.open(os.path.join(GOLDEN, name + ".gz"), "rt") as f:
        return f.read()


def _unpack(tmp_path, case: str, names) -> None:
    for n in names:
        (tmp_path / n).write_text(_golden(case + "." + n))


def events_dump(events) -> str:
    """The reference harness's `events` dump format (oracle/ref_harness.cpp run_events)."""
    out = []
    for k, ev in enumerate(events):
        out.append("event %d vertices %d" % (k, len(ev.vertices)))
        out += ["v %.9g %.9g %.9g" % tuple(float(x) for x in v) for v in ev.vertices]
        for l, a in enumerate(ev.layers):
            out += ["c %d %d %.9g %.9g %.9g %.9g %d" % (l, c["id"], c["x"], c["y"], c["z"], c["alpha"], c["mc"]) for c in a]
    return "\n".join(out) + "\n"


def labels_dump(maps) -> str:
    """The harness's `labels` dump: each map's entries by ascending id, "-1" after each map."""
    out = []
    for m in maps:
        out += ["%d %.9g %.9g %.9g %d %d" % (r["mc"], r["pt"], r["phi"], r["eta"], r["pdg"], r["ncl"]) for r in sorted(m, key=lambda r: int(r["mc"]))]
        out.append("-1")
    return "\n".join(out) + "\n"


def runs_of(events):
    """Every vertex of every event as one run (the reference's vertex loop, Tracker.cxx:251-262)."""
    return [(ev, iv, e) for e, ev in enumerate(events) for iv in range(len(ev.vertices))]


def oracle_roads(events):
    roads, offsets, run_event = [], [0], []
    for ev, iv, e in runs_of(events):
        r = oracle.run_vertex(ev.layers, ev.vertices[iv])["roads"]
        roads.append(r)
        offsets.append(offsets[-1] + len(r))
        run_event.append(e)
    return np.concatenate(roads), np.array(offsets, np.int32), np.array(run_event, np.int32)


def write_report(tmp_path, roads, offsets, cls, maps, run_event) -> dict:
    paths = [tmp_path / n for n in REPORT_FILES]
    with open(paths[0], "w") as c, open(paths[1], "w") as d, open(paths[2], "w") as f:
        io.write_roads_report((c, d, f), roads, offsets, cls, maps, run_event)
    return {n: p.read_text() for n, p in zip(REPORT_FILES, paths)}


def maps_for(labels_path: str, n_events: int) -> list:
    maps = io.read_reference_labels(labels_path)[:n_events]
    return maps + [np.zeros(0, io.LABEL_DTYPE)] * (n_events - len(maps))


def test_loaders_match_the_reference_parse(tmp_path):
    _unpack(tmp_path, "mixed", ("data.txt", "labels.txt"))
    events = io.read_reference_events(str(tmp_path / "data.txt"))
    assert [len(ev.vertices) for ev in events] == [1, 1, 3]
    assert events_dump(events) == _golden("mixed.events.dump")
    maps = io.read_reference_labels(str(tmp_path / "labels.txt"))
    assert len(maps) == len(events) + 1 and len(maps[-1]) == 0  # the map open after the last "-1"
    assert labels_dump(maps) == _golden("mixed.labels.dump")


def test_oracle_report_matches_the_reference_files(tmp_path):
    _unpack(tmp_path, "mixed", ("data.txt", "labels.txt"))
    events = io.read_reference_events(str(tmp_path / "data.txt"))
    maps = maps_for(str(tmp_path / "labels.txt"), len(events))
    roads, offsets, run_event = oracle_roads(events)
    cls, counts = oracle.roads_report(roads, offsets, maps, run_event)
    got = write_report(tmp_path, roads, offsets, cls, maps, run_event)
    for n in REPORT_FILES:
        assert got[n] == _golden("mixed." + n), n
    assert counts["duplicate"].sum() > 0 and counts["fake"].sum() > 0 and counts["correct"].sum() > 0
    assert np.array_equal(counts["labels"], [len(m) for m in maps])
    assert [int(counts[k].sum()) for k in ("correct", "duplicate", "fake")] == [int((cls == c).sum()) for c in (1, 2, 3)]


def test_merge_pileup_matches_the_reference_merger(tmp_path):
    _unpack(tmp_path, "merge", ("data.txt", "labels.txt"))
    io.merge_pileup(3, str(tmp_path))
    assert (tmp_path / "merged_data.txt").read_text() == _golden("merge.merged_data.txt")
    assert (tmp_path / "merged_labels.txt").read_text() == _golden("merge.merged_labels.txt")


def test_parse_floats_rounds_like_strtof():
    libc = ctypes.CDLL(None)
    libc.strtof.restype = ctypes.c_float
    libc.strtof.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    rng = np.random.default_rng(5)
    bits = rng.integers(0, 2**32, 20000, dtype=np.uint64).astype(np.uint32)
    vals = bits.view(np.float32)
    vals = vals[np.isfinite(vals)]
    tokens = []
    for k, v in enumerate(vals[:4000]):
        tokens.append(("%.9g", "%.6g", "%.3e", "%.17g")[k % 4] % float(v))
    # decimal strings exactly halfway between two binary32 values (float64 parses them exactly)
    for v in vals[:500]:
        a = np.float32(v)
        b = np.nextafter(a, np.float32(np.inf))
        if np.isfinite(b):
            tokens.append(repr((float(a) + float(b)) / 2))
    got = io.parse_floats(tokens)
    want = np.array([libc.strtof(t.encode(), None) for t in tokens], np.float32)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_report_edge_cases():
    """Unlabelled roads are skipped, a repeated id keeps one map entry, events without runs or
    labels, and runs mapped to events."""
    road = np.zeros(6, oracle.ROAD_DTYPE)
    road["label"] = [7, 9, 7, -1, 7, 9]
    road["fake"] = [0, 0, 0, 0, 1, 1]
    lab = np.zeros(3, io.LABEL_DTYPE)
    lab["mc"] = [7, 7, 9]
    maps = [lab, np.zeros(0, io.LABEL_DTYPE), lab[:1]]
    offsets = np.array([0, 3, 3, 6], np.int32)  # run 0 -> event 0; runs 1, 2 -> event 2
    cls, counts = oracle.roads_report(road, offsets, maps, np.array([0, 2, 2], np.int32))
    assert list(cls) == [1, 1, 2, 0, 3, 0]
    assert counts.tolist() == [(2, 2, 1, 0), (0, 0, 0, 0), (1, 0, 0, 1)]


@pytest.mark.skipif(not oracle.ref_available("cr"), reason="oracle/_ref not built (needs the reference sources)")
def test_fresh_case_through_the_reference(tmp_path):
    events = [gen.jet_event(81, 50), gen.make_event(82, 150, noise=0.1, n_vertices=2)]
    gen.write_reference_events(events, str(tmp_path / "data.txt"))
    gen.write_reference_labels(events, str(tmp_path / "labels.txt"))
    ref_dir = tmp_path / "ref"
    ref_dir.mkdir()
    oracle.run_reference_report(str(tmp_path / "data.txt"), str(tmp_path / "labels.txt"), str(ref_dir))
    loaded = io.read_reference_events(str(tmp_path / "data.txt"))
    maps = maps_for(str(tmp_path / "labels.txt"), len(loaded))
    roads, offsets, run_event = oracle_roads(loaded)
    cls, _ = oracle.roads_report(roads, offsets, maps, run_event)
    got = write_report(tmp_path, roads, offsets, cls, maps, run_event)
    for n in REPORT_FILES:
        assert got[n] == (ref_dir / n).read_text(), n
    merger = os.path.join(oracle.REF_DIR, "merge_pileup")
    if os.path.exists(merger):
        out = tmp_path / "merged"
        out.mkdir()
        subprocess.check_call([merger, "2", str(tmp_path) + "/", str(out) + "/"], stdout=subprocess.DEVNULL)
        io.merge_pileup(2, str(tmp_path), str(tmp_path))
        for n in ("merged_data.txt", "merged_labels.txt"):
            assert (tmp_path / n).read_text() == (out / n).read_text(), n


def test_binary_events_round_trip(tmp_path):
    """The binary loader gives the text loader's events (ids, coordinates, alpha, MC ids bit for bit)."""
    _unpack(tmp_path, "mixed", ("data.txt",))
    text_events = io.read_reference_events(str(tmp_path / "data.txt"))
    gen.write_binary_events(text_events, str(tmp_path / "events.bin"))
    bin_events = io.read_binary_events(str(tmp_path / "events.bin"))
    assert events_dump(bin_events) == events_dump(text_events) == _golden("mixed.events.dump")
    for a, b in zip(text_events, bin_events):
        assert np.array_equal(a.vertices.view(np.uint32), b.vertices.view(np.uint32))
        for la, lb in zip(a.layers, b.layers):
            assert np.array_equal(la.view(np.uint8), lb.view(np.uint8))


def run_counts(events):
    """Per run (every vertex of every event): cluster, tracklet and cell counts per layer and roads."""
    out = []
    for ev, iv, _ in runs_of(events):
        r = oracle.run_vertex(ev.layers, ev.vertices[iv])
        out.append(([len(x) for x in r["clusters"]], [len(x) for x in r["tracklets"]], [len(x) for x in r["cells"]], len(r["roads"])))
    return out


def test_memory_occupancy_matches_the_reference_benchmark(tmp_path):
    """MemoryOccupancy.txt of the reference's MEMORY_BENCHMARK build, from the oracle's counts: the
    coefficient reservations, push_back growth and capacities kept across vertices restated."""
    _unpack(tmp_path, "mixed", ("data.txt",))
    events = io.read_reference_events(str(tmp_path / "data.txt"))
    counts = run_counts(events)
    warmup = counts[: len(events[0].vertices)]
    assert io.memory_occupancy(warmup, counts) == _golden("mixed.MemoryOccupancy.txt")
