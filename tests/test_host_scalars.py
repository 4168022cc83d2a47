"""The scalar helpers of DigitalTwinSimulator.step_params (physics_engine._sqrt, _clip) give
exactly NumPy's results: np.sqrt and np.clip on the same scalars, including NaN, infinities,
signed zeros, bounds that cross, and NumPy scalars (which keep their dtype)."""
import math
import random

import numpy as np

from thruster_cx_code_b200.physics_engine import _clip, _sqrt


def _same(a, b):
    a, b = float(a), float(b)
    return (a == b and math.copysign(1.0, a) == math.copysign(1.0, b)) or (a != a and b != b)


def test_sqrt_matches_numpy():
    r = random.Random(1)
    vals = [0.0, -0.0, 1.0, 2.0, 1e-310, 5e-324, 1.7976931348623157e308, float("inf")]
    vals += [r.uniform(0.0, 1e6) * 10.0 ** r.randint(-300, 300) for _ in range(20000)]
    for v in vals:
        assert _same(_sqrt(v), np.sqrt(v)), v
    with np.errstate(invalid="ignore"):
        for v in (-1.0, float("nan"), -float("inf")):
            assert _same(_sqrt(v), np.sqrt(v)), v
    x32 = np.float32(2.0)
    assert _sqrt(x32).dtype == np.sqrt(x32).dtype == np.float32


def test_clip_matches_numpy():
    r = random.Random(2)
    for _ in range(20000):
        lo = r.randint(-50, 50)
        hi = lo + r.randint(-5, 60)  # sometimes lo > hi
        x = r.randint(-120, 120)
        assert _clip(x, lo, hi) == np.clip(x, lo, hi), (x, lo, hi)
    specials = [0.0, -0.0, 1.0, -1.0, 2.5, 1e-300, float("inf"), -float("inf"), float("nan")]
    for _ in range(20000):
        a, lo, hi = (r.choice(specials + [r.uniform(-5.0, 5.0)]) for _ in range(3))
        assert _same(_clip(a, lo, hi), np.clip(a, lo, hi)), (a, lo, hi)
