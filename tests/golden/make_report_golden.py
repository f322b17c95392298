"""Generates the road-report, loader and pile-up-merger fixtures under tests/golden/report/ from
the reference's own code.

Run in a checkout where oracle/build_ref.sh has built oracle/_ref/ref_cr and
oracle/_ref/merge_pileup (it needs the reference sources):  python tests/golden/make_report_golden.py
Cases (seeded synthetic events, written in the reference's text formats):
  mixed   a 120-track event, a dense 60-track jet (duplicate and fake roads) and a 3-vertex
          pile-up event of 120-track collisions: data.txt / labels.txt, the reference's road report
          ({Correct,Duplicate,Fake}Roads.txt: ref_cr report = main.cpp's benchmark data), the
          reference loaders' parse of both files (events.dump, labels.dump) and the MEMORY_BENCHMARK
          build's MemoryOccupancy.txt (ref_cr memory)
  merge   six 40-track events merged into frames of 3 by the reference's merger
          (merged_data.txt, merged_labels.txt)
Everything is stored gzip-compressed.
"""
from __future__ import annotations

import gzip
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tracking-itsu_b200"))

from itsu import gen  # noqa: E402
from oracle import oracle  # noqa: E402

OUT = os.path.join(HERE, "report")
REPORT_FILES = ("CorrectRoads.txt", "DuplicateRoads.txt", "FakeRoads.txt")


def mixed_events():
    return [gen.make_event(31, 120, noise=0.05), gen.jet_event(32, 60), gen.make_event(33, 120, noise=0.1, n_vertices=3)]


def merge_events():
    return [gen.make_event(40 + k, 40, noise=0.05) for k in range(6)]


def _gz(src: str, name: str) -> None:
    with open(src, "rb") as f, open(os.path.join(OUT, name + ".gz"), "wb") as raw:
        with gzip.GzipFile(filename="", mode="wb", compresslevel=9, fileobj=raw, mtime=0) as g:
            shutil.copyfileobj(f, g)


def main() -> None:
    ref, merger = oracle.ref_binary("cr"), os.path.join(oracle.REF_DIR, "merge_pileup")
    if not (os.path.exists(ref) and os.path.exists(merger)):
        raise SystemExit("build oracle/_ref first (oracle/build_ref.sh)")
    os.makedirs(OUT, exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        data, labels = os.path.join(tmp, "data.txt"), os.path.join(tmp, "labels.txt")
        events = mixed_events()
        gen.write_reference_events(events, data)
        gen.write_reference_labels(events, labels)
        oracle.run_reference_report(data, labels, tmp)
        subprocess.check_call([ref, "events", data, os.path.join(tmp, "events.dump")])
        subprocess.check_call([ref, "labels", labels, str(len(events)), os.path.join(tmp, "labels.dump")])
        subprocess.check_call([ref, "memory", data, os.path.join(tmp, "MemoryOccupancy.txt")])
        for name in ("data.txt", "labels.txt", "events.dump", "labels.dump", "MemoryOccupancy.txt") + REPORT_FILES:
            _gz(os.path.join(tmp, name), "mixed." + name)
    with tempfile.TemporaryDirectory() as tmp:
        events = merge_events()
        gen.write_reference_events(events, os.path.join(tmp, "data.txt"))
        gen.write_reference_labels(events, os.path.join(tmp, "labels.txt"))
        subprocess.check_call([merger, "3", tmp + "/", tmp + "/"], stdout=subprocess.DEVNULL)
        for name in ("data.txt", "labels.txt", "merged_data.txt", "merged_labels.txt"):
            _gz(os.path.join(tmp, name), "merge." + name)
    print("wrote", sorted(os.listdir(OUT)))


if __name__ == "__main__":
    main()
