"""The surrogate's error estimate (CPU): ``surrogate.control_variate_error``
on synthetic batch residuals whose spread is known."""

import numpy as np

from pyrite_b200.surrogate import control_variate_error


def _run(rng, B, sigma, stride, n_tile=4, n_bin=512, mean=0.0):
    r = mean + sigma[None] * rng.standard_normal((B,) + sigma.shape)
    return r.sum(0), (r * r).sum(0)


def test_estimate_tracks_the_true_error_of_the_correction():
    """Residuals with a known per-bin sigma (a smooth line profile): the
    estimate's three standard errors of the correction stride * sum_b r_b
    fall within 25 % of the true 3 * stride * sqrt(B) * sigma_max, and the
    correction's actual worst-bin deviation stays below the estimate in
    nearly every run (a calibrated gate)."""
    rng = np.random.default_rng(0)
    n_tile, n_bin, stride = 4, 512, 150
    x = np.arange(n_bin)
    prof = np.exp(-0.5 * ((x - 200) / 40.0) ** 2) + 0.05
    sigma = np.outer(np.linspace(0.5, 2.0, n_tile), prof) * 1e-3
    spectrum = np.full((n_tile, n_bin), 10.0)
    ratios, covered = [], 0
    trials = 200
    for _ in range(trials):
        B = 6
        rs, rq = _run(rng, B, sigma, stride)
        est = control_variate_error(rs, rq, B, stride, spectrum)
        true = 3.0 * stride * np.sqrt(B) * sigma.max(axis=1) / 10.0
        ratios.append(est / true)
        actual = np.max(np.abs(stride * rs), axis=1) / 10.0  # mean residual is zero here
        covered += int(np.all(actual <= est))
    ratios = np.array(ratios)
    assert 0.75 < np.median(ratios) < 1.25, np.median(ratios)
    assert covered >= 0.9 * trials, covered


def test_estimate_needs_two_batches_and_flags_a_poor_surrogate():
    rng = np.random.default_rng(1)
    sigma = np.full((2, 64), 1e-3)
    rs, rq = _run(rng, 1, sigma, 10)
    assert control_variate_error(rs, rq, 1, 10, np.ones((2, 64))) is None
    # 3 * 10 * sqrt(8) * 1e-5 = 0.085 % of the peak; the poor one 100 times that
    good = control_variate_error(*_run(rng, 8, 1e-2 * sigma, 10), 8, 10, np.ones((2, 64)))
    poor = control_variate_error(*_run(rng, 8, sigma, 10), 8, 10, np.ones((2, 64)))
    assert np.all(good < 0.01) and np.all(poor > 0.01)
    # a tile with an empty spectrum reports no error
    z = control_variate_error(*_run(rng, 4, sigma, 10), 4, 10, np.array([np.ones(64), np.zeros(64)]))
    assert z[1] == 0.0

