"""The device build of the correctly rounded atan2 (every cluster and tracklet azimuth) against the
host build of the same definition, bit for bit: random pairs over the detector's coordinate range,
tiny and huge magnitudes, random bit patterns, the inputs that take the double-double path, and
the special values."""
import ctypes

import numpy as np
import pytest

from itsu import capi
from oracle import oracle
from test_atan2f import SLOW_PATH

pytestmark = pytest.mark.gpu


def _host(y, x):
    out = np.empty(len(y), np.float32)
    oracle.lib().oracle_atan2f_n(y.ctypes.data, x.ctypes.data, out.ctypes.data, len(y))
    return out


def test_device_atan2f_equals_the_host_definition():
    import torch

    rng = np.random.default_rng(11)
    n = 1 << 21
    parts_y = [rng.uniform(-40, 40, n), rng.uniform(-1e-3, 1e-3, n // 4), rng.uniform(-1e30, 1e30, n // 8)]
    parts_x = [rng.uniform(-40, 40, n), rng.uniform(-40, 40, n // 4), rng.uniform(-1e-30, 1e-30, n // 8)]
    bits = rng.integers(0, 2**32, size=(n // 2, 2), dtype=np.uint64).astype(np.uint32)
    y = np.concatenate([p.astype(np.float32) for p in parts_y] + [bits[:, 0].view(np.float32)])
    x = np.concatenate([p.astype(np.float32) for p in parts_x] + [bits[:, 1].view(np.float32)])
    slow = np.array([[float.fromhex(a), float.fromhex(b)] for a, b in SLOW_PATH], np.float32)
    special = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1.0, -1.0], np.float32)
    sy, sx = np.meshgrid(special, special)
    y = np.concatenate([y, slow[:, 0], sy.ravel()])
    x = np.concatenate([x, slow[:, 1], sx.ravel()])
    dev = torch.device("cuda", 0)
    ty, tx = torch.from_numpy(y).to(dev), torch.from_numpy(x).to(dev)
    out = torch.empty_like(ty)
    ctx = capi.Context(device=0)
    try:
        ctx.atan2f_device(ty.data_ptr(), tx.data_ptr(), out.data_ptr(), len(y))
    finally:
        ctx.close()
    got = out.cpu().numpy()
    want = _host(y, x)
    nan = np.isnan(want)
    assert np.array_equal(np.isnan(got), nan)
    diff = np.flatnonzero(got[~nan].view(np.uint32) != want[~nan].view(np.uint32))
    assert len(diff) == 0, (len(diff), y[~nan][diff[:5]], x[~nan][diff[:5]])
