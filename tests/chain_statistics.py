"""Statistical agreement of Monte Carlo results: independent chains (or runs) give independent estimates, whose spread
is the standard error of their mean. Two samplers agree when their means differ by less than the two-sided critical
value of Student's t at the false-alarm probability of a 4-sigma normal deviation (6.3e-5, about 1 in 16,000
comparisons), with the Welch-Satterthwaite degrees of freedom of the two estimated standard errors: with few runs the
errors themselves are uncertain and |z| < 4 would fail far more often than that. No percentage slack is added."""

from __future__ import annotations

import math

import numpy as np
from scipy import stats

FALSE_ALARM = 2.0 * stats.norm.sf(4.0)


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


def degrees_of_freedom(a, b=None) -> float:
    """n - 1 against an exact value; the Welch-Satterthwaite value for two samples."""
    na = len(a)
    if b is None:
        return float(na - 1)
    nb = len(b)
    va = np.var(a, ddof=1) / na
    vb = np.var(b, ddof=1) / nb
    if va + vb == 0.0:
        return float(na + nb - 2)
    return float((va + vb) ** 2 / (va ** 2 / (na - 1) + vb ** 2 / (nb - 1)))


def critical_value(df: float, false_alarm: float = FALSE_ALARM) -> float:
    return float(stats.t.isf(false_alarm / 2.0, df))


def assert_agree(a, b=None, expected=None, label="", false_alarm=FALSE_ALARM):
    z = z_score(a, b, expected)
    df = degrees_of_freedom(a, b)
    limit = critical_value(df, false_alarm)
    ma, ea = mean_and_error(a)
    other = f"{expected}" if b is None else "%.6g +- %.2g" % mean_and_error(b)
    print(f"{label}: {ma:.6g} +- {ea:.2g} vs {other}: z = {z:+.2f} (limit {limit:.2f} at {df:.0f} degrees of freedom)")
    assert abs(z) < limit, (label, ma, ea, other, z, limit)
    return z
