"""The device's one-compare form of the reference's wrap-around azimuth cut.

Tracker.cxx:93-100 (tracklets) and :161-166 (cells) test |delta_phi - TwoPi| < cut in binary32;
the kernels test delta_phi > W with W the largest binary32 value not above TwoPi - cut
(csrc/itsu_device.cuh kPhiWrapTracklet, kPhiWrapCell). Checked here: W itself, and that both
forms agree for every binary32 delta_phi in [Pi, TwoPi] and for a sample of those in [0, Pi)."""
import os
import re
from fractions import Fraction

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "tracking-itsu_b200", "csrc", "itsu_device.cuh")

PI = np.float32(3.14159265359)
TWO_PI = np.float32(2.0) * PI


def _constant(name):
    m = re.search(r"constexpr float %s = ([0-9a-fA-Fx.p+-]+)f;" % name, open(HEADER).read())
    assert m, name
    return np.float32(float.fromhex(m.group(1)))


@pytest.mark.parametrize("name, cut", [("kPhiWrapTracklet", np.float32(0.3)), ("kPhiWrapCell", np.float32(0.14))])
def test_wrap_threshold_is_the_exact_bound(name, cut):
    w = _constant(name)
    bound = Fraction(float(TWO_PI)) - Fraction(float(cut))
    assert Fraction(float(w)) <= bound < Fraction(float(np.nextafter(w, np.float32(np.inf))))


@pytest.mark.parametrize("name, cut", [("kPhiWrapTracklet", np.float32(0.3)), ("kPhiWrapCell", np.float32(0.14))])
def test_one_compare_form_equals_the_reference_cut(name, cut):
    w = _constant(name)
    lo, hi = int(PI.view(np.int32)), int(TWO_PI.view(np.int32))
    every = np.arange(lo, hi + 1, dtype=np.int32).view(np.float32)          # all of [Pi, TwoPi]
    sample = np.arange(0, lo, 101, dtype=np.int32).view(np.float32)        # a sample of [0, Pi)
    for d in (every, sample):
        reference = (d < cut) | (np.abs(d - TWO_PI) < cut)
        assert np.array_equal(reference, (d < cut) | (d > w))
