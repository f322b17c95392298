"""The oracle (C restatement of the reference CPU path) against the reference itself.

Golden fixtures were produced by the patched reference tracker (tests/golden/make_golden.py);
when the reference build is present (oracle/_ref), fresh seeded events are compared too.
"""
import tempfile

import pytest

from helpers import CASES, beyond_z_event, load_case, vertex_runs
from itsu import gen
from oracle import oracle


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference_fixture(case):
    events, expected = load_case(case)
    runs = vertex_runs(events)
    assert len(runs) == len(expected)
    for (ev, iv), exp in zip(runs, expected):
        got = oracle.run_vertex(ev.layers, ev.vertices[iv])
        assert oracle.diff(got, exp) == [], case


def test_fixtures_cover_edge_cases():
    """The fixtures hold what they claim: empty layers, negative and 400 bins, phi bin 20
    windows, duplicated clusters, several vertices per event."""
    _, z = load_case("z_edges")
    assert any((c["bin"] < 0).any() for c in z[0]["clusters"])
    assert any((c["bin"] == 400).any() for c in z[0]["clusters"])
    events, e = load_case("empty_layers")
    assert [len(ev.layers[k]) for ev, k in zip(events, (0, 3, 6, 2))] == [0, 0, 0, 0]
    _, pb = load_case("phi_boundary")
    assert any((c["phi"] == gen.np.float32(2.0) * gen.np.float32(3.14159265359)).any() for c in pb[0]["clusters"])
    events, _ = load_case("pileup_small")
    assert len(events[0].vertices) == 3


needs_ref = pytest.mark.skipif(not oracle.ref_available("cr"), reason="reference build (oracle/_ref) not present")


@needs_ref
@pytest.mark.parametrize("seed", [101, 102])
def test_oracle_matches_reference_fresh_events(seed):
    events = [gen.pp_event(seed), gen.make_event(seed, 1500, pt_mean=0.6, noise=0.05), gen.pileup_frame(seed, 2, 300)]
    with tempfile.TemporaryDirectory() as d:
        expected = oracle.run_reference(events, d, "cr")
    for (ev, iv), exp in zip(vertex_runs(events), expected):
        assert oracle.diff(oracle.run_vertex(ev.layers, ev.vertices[iv]), exp) == []


@needs_ref
def test_oracle_matches_reference_at_full_size():
    """The sizes the GPU tests lean on the oracle for, against the reference binary directly: a
    central Pb-Pb-like event (6000 tracks, 5% noise), a pile-up frame of 5 collisions of 1500
    tracks with 10% noise (every vertex), and a layer with hundreds of clusters beyond its z
    range (negative z bins sorted apart from the index table)."""
    # the Pb-Pb events and the frame the GPU parity tests compare with the oracle
    events = [gen.pbpb_event(1), gen.pbpb_event(2), gen.pbpb_event(3), gen.pileup_frame(7), beyond_z_event(4244)]
    with tempfile.TemporaryDirectory() as d:
        expected = oracle.run_reference(events, d, "cr")
    runs = vertex_runs(events)
    assert len(runs) == len(expected) == 9
    for k, ((ev, iv), exp) in enumerate(zip(runs, expected)):
        assert oracle.diff(oracle.run_vertex(ev.layers, ev.vertices[iv]), exp) == [], k
    assert min(sum(len(t) for t in expected[k]["tracklets"]) for k in range(3)) > 200000  # central events indeed
    assert sum(int((c["bin"] < 0).sum()) for c in expected[-1]["clusters"]) > 1500
