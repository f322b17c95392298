"""The correctly rounded atan2f shared by the device, the oracle and the reference harness."""
import math

import mpmath
import numpy as np
import pytest

from oracle import oracle

mpmath.mp.prec = 160


def _cr(y, x):
    """binary32 nearest to the exact atan2(y, x) (ties cannot occur for these arguments)."""
    ex = mpmath.atan2(mpmath.mpf(float(y)), mpmath.mpf(float(x)))
    f = np.float32(float(ex))
    cand = [np.nextafter(f, np.float32(-np.inf)), f, np.nextafter(f, np.float32(np.inf))]
    return min(cand, key=lambda c: abs(mpmath.mpf(float(c)) - ex))


def _bits(v):
    return np.array([v], np.float32).view(np.uint32)[0]


def test_special_values():
    f = oracle.lib().oracle_atan2f
    pi = np.float32(math.pi)
    cases = [
        ((0.0, 1.0), 0.0), ((-0.0, 1.0), -0.0), ((0.0, -1.0), pi), ((-0.0, -1.0), -pi),
        ((0.0, 0.0), 0.0), ((0.0, -0.0), pi), ((-0.0, -0.0), -pi),
        ((1.0, 0.0), np.float32(math.pi / 2)), ((-1.0, -0.0), -np.float32(math.pi / 2)),
        ((math.inf, math.inf), np.float32(math.pi / 4)), ((math.inf, -math.inf), np.float32(3 * math.pi / 4)),
        ((1.0, math.inf), 0.0), ((1.0, -math.inf), pi), ((-1.0, -math.inf), -pi), ((-math.inf, 5.0), -np.float32(math.pi / 2)),
    ]
    for (y, x), want in cases:
        assert _bits(f(y, x)) == _bits(np.float32(want)), (y, x)
    assert math.isnan(f(math.nan, 1.0)) and math.isnan(f(1.0, math.nan))


@pytest.mark.parametrize("seed", [0, 1])
def test_correctly_rounded_random(seed):
    f = oracle.lib().oracle_atan2f
    rng = np.random.default_rng(seed)
    ys = np.concatenate([rng.uniform(-40, 40, 3000), rng.uniform(-1e-3, 1e-3, 1000)]).astype(np.float32)
    xs = np.concatenate([rng.uniform(-40, 40, 3000), rng.uniform(-40, 40, 1000)]).astype(np.float32)
    bits = rng.integers(0, 2**32, size=(2000, 2), dtype=np.uint64).astype(np.uint32)
    by, bx = bits[:, 0].view(np.float32), bits[:, 1].view(np.float32)
    ok = np.isfinite(by) & np.isfinite(bx)
    ys = np.concatenate([ys, by[ok]])
    xs = np.concatenate([xs, bx[ok]])
    for y, x in zip(ys, xs):
        assert _bits(f(float(y), float(x))) == _bits(_cr(y, x)), (float(y).hex(), float(x).hex())


# Arguments whose fast binary64 result lies within 2^-44 of a rounding boundary, so they take
# the double-double path (found by scanning 2e7 random pairs in [-40, 40]^2).
SLOW_PATH = [
    ("-0x1.3bb97p+5", "-0x1.1c2278p+4"), ("-0x1.36017ap+2", "0x1.9a28aep+4"), ("-0x1.94730ep+2", "0x1.9388aap+0"),
    ("-0x1.7b94bp+1", "0x1.b0002p+3"), ("-0x1.6af8b6p+2", "0x1.19838cp+0"), ("0x1.5ebaep+2", "-0x1.354ccp-1"),
    ("-0x1.90dc68p+4", "0x1.34b1ccp+4"), ("0x1.8aad8ap+4", "0x1.4b7a68p+4"), ("0x1.0bde28p+2", "-0x1.32217p+4"),
    ("-0x1.88f02p+0", "0x1.a52738p+2"), ("0x1.7d0a08p+3", "0x1.ff3318p+0"), ("-0x1.f0fda2p+4", "-0x1.5d8cf2p+4"),
]


def test_slow_path_inputs_correctly_rounded():
    f = oracle.lib().oracle_atan2f
    for ys, xs in SLOW_PATH:
        y, x = np.float32(float.fromhex(ys)), np.float32(float.fromhex(xs))
        assert _bits(f(float(y), float(x))) == _bits(_cr(y, x)), (ys, xs)
