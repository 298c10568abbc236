"""Shared input builders for the tests (seeded, smooth, periodic states)."""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
if os.path.join(HERE, "golden") not in sys.path:
    sys.path.insert(0, os.path.join(HERE, "golden"))

from make_golden import smooth_random_state  # noqa: E402


def smooth_state(nx, ny, dx, dy, seed, **kw):
    return smooth_random_state(nx, ny, dx, dy, seed, **kw)
