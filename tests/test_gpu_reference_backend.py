"""The reference's own tracker with the B200 backend behind its seam (oracle/_ref/ref_b200).

ref_b200 is the reference's sources (with the memory-safety and determinism patches P1-P5) plus
tracking-itsu_b200/host/reference_backend/TrackerB200.cxx, which supplies
TrackerTraits::computeLayerTracklets / computeLayerCells and the device clustering step of
PrimaryVertexContext::initialize through libitsu_b200.so; the reference's findCellsNeighbours,
findTracks, computeMontecarloLabels, clustersToTracks and IOUtils run unchanged on the host. The
reference harness drives it, so every list below is what the reference's own data structures
hold after each of its stages:
  dump    every vertex stage by stage (Tracker.cxx:253-259), every intermediate list
  report  main.cpp's run: clustersToTracks per event, then IOUtils::writeRoadsReport
  memory  main.cpp's MEMORY_BENCHMARK run (Tracker::clustersToTracksMemoryBenchmark)
Each must equal the reference CPU tracker's, byte for byte.
"""
import gzip
import os
import subprocess
import tempfile

import pytest

from helpers import CASES, GOLDEN, load_case, vertex_runs
from itsu import gen
from oracle import oracle

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not oracle.ref_available("b200"), reason="ref_b200 not built (oracle/build_ref.sh)"),
]

REPORT = os.path.join(GOLDEN, "report")


def _run(*args):
    return subprocess.run([oracle.ref_binary("b200"), *args], check=True, capture_output=True, text=True, timeout=600)


def _golden_text(name):
    with gzip.open(os.path.join(REPORT, name + ".gz"), "rt") as f:
        return f.read()


@pytest.mark.parametrize("case", CASES)
def test_reference_tracker_on_b200_matches_fixture(case, tmp_path):
    """The reference's stage loop on the B200 backend: sorted clusters, index tables, tracklets and
    their lookup tables, cells and levels, cells lookup, neighbour lists and labelled roads of every
    vertex equal the reference CPU tracker's fixture."""
    events, expected = load_case(case)
    txt = tmp_path / "events.txt"
    with gzip.open(os.path.join(GOLDEN, case + ".events.txt.gz"), "rt") as f:
        txt.write_text(f.read())
    _run("dump", str(txt), str(tmp_path / "out.bin"))
    got = oracle.parse_dump(str(tmp_path / "out.bin"))
    assert len(got) == len(expected) == len(vertex_runs(events))
    for k, (g, e) in enumerate(zip(got, expected)):
        assert oracle.diff(g, e) == [], "%s vertex %d" % (case, k)


def test_reference_tracker_on_b200_matches_cpu_tracker_on_pbpb():
    """Central Pb-Pb-like events (6000 tracks, 5% noise) and a pile-up frame of 5 collisions: the
    B200 backend against the reference CPU tracker (ref_cr) run beside it."""
    events = [gen.pbpb_event(1), gen.pileup_frame(9)]
    with tempfile.TemporaryDirectory() as d:
        want = oracle.run_reference(events, d, "cr")
        got = oracle.run_reference(events, d, "b200")
    assert len(got) == len(want) == 6
    for k, (g, e) in enumerate(zip(got, want)):
        assert oracle.diff(g, e) == [], "run %d" % k
    assert len(want[0]["roads"]) > 1000


def test_reference_main_on_b200_writes_the_reference_report(tmp_path):
    """main.cpp's run (clustersToTracks per event, then writeRoadsReport) on the B200 backend writes
    the reference CPU tracker's CorrectRoads / DuplicateRoads / FakeRoads files byte for byte."""
    (tmp_path / "data.txt").write_text(_golden_text("mixed.data.txt"))
    (tmp_path / "labels.txt").write_text(_golden_text("mixed.labels.txt"))
    _run("report", str(tmp_path / "data.txt"), str(tmp_path / "labels.txt"), str(tmp_path))
    for name in ("CorrectRoads.txt", "DuplicateRoads.txt", "FakeRoads.txt"):
        assert (tmp_path / name).read_text() == _golden_text("mixed." + name), name


def test_reference_memory_benchmark_on_b200(tmp_path):
    """Tracker::clustersToTracksMemoryBenchmark on the B200 backend: the host vectors the backend
    fills grow as the reference's, so MemoryOccupancy.txt is the reference's byte for byte."""
    (tmp_path / "data.txt").write_text(_golden_text("mixed.data.txt"))
    _run("memory", str(tmp_path / "data.txt"), str(tmp_path / "MemoryOccupancy.txt"))
    assert (tmp_path / "MemoryOccupancy.txt").read_text() == _golden_text("mixed.MemoryOccupancy.txt")
