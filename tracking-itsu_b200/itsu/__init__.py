"""Python side of the B200 ITS CA track finder: the C ABI binding (capi) and the seeded event
generator (gen). The compute path is lib/libitsu_b200.so; this package only calls it."""
from . import gen  # noqa: F401
