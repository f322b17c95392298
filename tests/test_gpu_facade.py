"""The C++ facade (tracking-itsu_b200/host/itsu_ca.hpp: Tracker<true>, PrimaryVertexContext,
Event, IOUtils::loadEventData) run as the reference's driver program would, on the golden
fixtures' event files; every vertex's roads must equal the reference's."""
import gzip
import os
import subprocess
import tempfile

import numpy as np
import pytest

from helpers import GOLDEN, load_case
from itsu import capi

pytestmark = pytest.mark.gpu

MAIN = os.path.join(os.path.dirname(capi.LIB_PATH), "itsu_tracker_main")


@pytest.mark.parametrize("case", ["pp", "mid", "empty_layers", "z_edges", "pileup_small"])
def test_facade_driver_roads_match_reference(case):
    _, expected = load_case(case)
    with tempfile.TemporaryDirectory() as d:
        txt = os.path.join(d, "events.txt")
        with gzip.open(os.path.join(GOLDEN, case + ".events.txt.gz"), "rb") as f, open(txt, "wb") as o:
            o.write(f.read())
        out = os.path.join(d, "roads.bin")
        proc = subprocess.run([MAIN, txt, "--roads", out], capture_output=True, text=True, timeout=300)
        assert proc.returncode == 0, proc.stderr
        data = open(out, "rb").read()
    pos = 0
    for exp in expected:
        n = int(np.frombuffer(data, np.int32, 1, pos)[0])
        pos += 4
        roads = np.frombuffer(data, capi.ROAD_DTYPE, n, pos).copy()
        pos += 32 * n
        roads["pad"] = 0
        assert np.array_equal(roads.view(np.uint8), exp["roads"].view(np.uint8))
    assert pos == len(data)
