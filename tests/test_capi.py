"""Host-side checks of the C ABI library: it loads, exports every entry point include/itsu.h
declares, and its records keep the reference layouts. No kernel runs here."""
import ctypes
import os
import re

import numpy as np
import pytest

from itsu import capi, gen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "itsu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(itsu_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_entry_point():
    lib = capi.load()
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(n for n, _, _ in capi.SIGNATURES) == names


def test_record_layouts_match_the_reference():
    assert gen.CLUSTER_DTYPE.itemsize == 36
    assert capi.TRACKLET_DTYPE.itemsize == 16
    assert capi.CELL_DTYPE.itemsize == 40
    assert capi.ROAD_DTYPE.itemsize == 32
    assert ctypes.sizeof(capi.Config) == 56
    assert ctypes.sizeof(capi.Batch) == 40
    assert ctypes.sizeof(capi.Counts) == 4 * (7 + 6 + 5 + 4 + 1)


def test_status_strings_and_version():
    lib = capi.load()
    assert b"sm_100a" in lib.itsu_version()
    assert lib.itsu_status_string(capi.OK) == b"ok"
    assert lib.itsu_status_string(capi.ERR_CAPACITY) == b"capacity exceeded"


def test_context_creation_fails_loudly_without_a_b200():
    import torch

    if torch.cuda.is_available():
        return  # covered by the GPU tests
    try:
        capi.Context()
    except capi.ItsuError as e:
        assert e.status == capi.ERR_CUDA
    else:
        raise AssertionError("a context was created without a GPU")


def test_reference_backend_is_built_against_the_library():
    """Where the reference was built (oracle/_ref), its tracker with the B200 backend behind its
    seam (ref_b200, tracking-itsu_b200/host/reference_backend/TrackerB200.cxx) is built too and
    resolves libitsu_b200.so from the tree (its GPU runs are in test_gpu_reference_backend.py)."""
    import subprocess

    from oracle import oracle

    if not oracle.ref_available("cr"):
        pytest.skip("reference build (oracle/_ref) not present")
    assert oracle.ref_available("b200")
    ldd = subprocess.run(["ldd", oracle.ref_binary("b200")], capture_output=True, text=True, check=True).stdout
    line = [l for l in ldd.splitlines() if "libitsu_b200.so" in l]
    assert line and "not found" not in line[0] and "tracking-itsu_b200/lib" in line[0]


def test_every_context_call_in_the_callers_exists():
    """Every method the tests, the bench and the package call on a context (`ctx.<name>`) is a
    method of capi.Context, so a wrapper cannot disappear from the binding while a GPU test, which
    only runs on a B200, still calls it."""
    import glob

    files = glob.glob(os.path.join(ROOT, "tests", "*.py")) + [os.path.join(ROOT, "bench.py")]
    files += glob.glob(os.path.join(ROOT, "tracking-itsu_b200", "itsu", "*.py"))
    instance_fields = {"lib", "h"}
    missing = set()
    for path in files:
        if os.path.basename(path) == "test_multirank_cpu.py":
            continue  # its ctx is a multiprocessing context
        for m in re.finditer(r"\bctx\w*\.([A-Za-z_]\w*)\b", open(path).read()):
            if m.group(1) not in instance_fields and not hasattr(capi.Context, m.group(1)):
                missing.add((os.path.basename(path), m.group(1)))
    assert not missing, sorted(missing)
