"""Statistical agreement of Monte Carlo results: independent chains (or runs) give independent estimates, whose spread
is the standard error of their mean. Two samplers agree when their means differ by less than 4 combined standard
errors (a false alarm in about 1 of 16,000 comparisons); no percentage slack is added."""

from __future__ import annotations

import math

import numpy as np


def mean_and_error(values) -> tuple[float, float]:
    v = np.asarray(values, dtype=np.float64)
    return float(v.mean()), float(v.std(ddof=1) / math.sqrt(len(v)))


def z_score(a, b=None, expected=None) -> float:
    """(mean(a) - mean(b)) / combined standard error, or (mean(a) - expected) / its standard error."""
    ma, ea = mean_and_error(a)
    if b is None:
        return (ma - expected) / ea
    mb, eb = mean_and_error(b)
    return (ma - mb) / math.hypot(ea, eb)


def assert_agree(a, b=None, expected=None, label="", limit=4.0):
    z = z_score(a, b, expected)
    ma, ea = mean_and_error(a)
    other = f"{expected}" if b is None else "%.6g +- %.2g" % mean_and_error(b)
    print(f"{label}: {ma:.6g} +- {ea:.2g} vs {other}: z = {z:+.2f}")
    assert abs(z) < limit, (label, ma, ea, other, z)
    return z
