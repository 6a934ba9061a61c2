"""The glass-transition fits of a cooling scan (caps_gpu_fit_tg, host code in the engine library) against the
reference's own fit_bilinear and fit_two_ranges (core/src/mechanics.cpp:1218, 1310; oracle/_ref): the same points must
give the same Tg, slopes, bootstrap error and note, bit for bit. Needs no GPU."""
import math

import numpy as np
import pytest

from caps_b200 import fit_tg


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref is not built")
    return ref


def _same(a, b):
    assert a["ok"] == b["ok"] and a["note"] == b["note"], (a, b)
    for k in ("tg", "tg_err", "slope_low", "slope_high", "value_at_tg", "alpha_low", "alpha_high", "rss"):
        x, y = a[k], b[k]
        assert (math.isnan(x) and math.isnan(y)) or x == y, (k, x, y)


def _scan(seed, n=16, tg=370.0, noise=2e-4, descending=False):
    rng = np.random.default_rng(seed)
    T = np.linspace(200, 500, n)
    if descending:
        T = T[::-1]
    y = 0.95 + np.where(T < tg, 2.5e-4 * (T - tg), 6.5e-4 * (T - tg)) + rng.normal(0, noise, n)
    return T, y


@pytest.mark.parametrize("method", [0, 1])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_fit_matches_reference(method, seed):
    ref = _ref()
    T, y = _scan(seed, descending=seed == 2)
    a, b = fit_tg(T, y, method), ref.fit_tg(T, y, method)
    _same(a, b)
    assert a["ok"] and 330 < a["tg"] < 410


def test_fit_edge_cases_match_reference():
    ref = _ref()
    T, y = _scan(4, n=7)
    cases = [
        (T[:4], y[:4], 0, 0, 0),            # too few for the continuous fit
        (T[:3], y[:3], 1, 0, 0),            # too few for two ranges
        (T, y, 1, 400, 300),                # glassy range above the rubbery one
        (T, y, 1, 260, 420),                # two points per range: no error estimate (NaN)
        (T, 2.0 * T + 1, 1, 0, 0),          # parallel lines
        (T, 2.0 * T + 1, 0, 0, 0),          # one straight line: the slopes agree
        (T, np.where(T < 240, T, 240 + 3 * (T - 240)), 1, 0, 0),   # a kink outside the gap between the ranges
    ]
    for t, v, method, gmax, rmin in cases:
        _same(fit_tg(t, v, method, gmax, rmin), ref.fit_tg(t, v, method, gmax, rmin))


def test_fit_rejects_mismatched_lengths():
    with pytest.raises(ValueError):
        fit_tg([1, 2, 3], [1, 2], 0)
