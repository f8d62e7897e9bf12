"""Host-side helpers of bench.py that need no GPU."""

import numpy as np

import bench


def test_spectrum_error_stats():
    ref = np.array([[1.0, 2.0, 4.0, 2.0], [0.5, 1.0, 1.0, 0.5]])
    got = ref.copy()
    got[0, 2] += 0.04   # 1 % of tile 0's peak
    got[1, 0] -= 0.005  # 0.5 % of tile 1's peak
    s = bench.spectrum_error_stats(got, ref)
    assert np.isclose(s["max_over_tiles"], 0.01)
    assert np.isclose(s["rms_over_tiles"], 0.04 / 2 / 4.0)  # sqrt(0.04^2 / 4) / 4
    tot = ref.sum(0)
    assert np.isclose(s["detector_total_max"], 0.04 / tot.max())
    assert np.isclose(s["detector_total_rms"], np.sqrt((0.04 ** 2 + 0.005 ** 2) / 4) / tot.max())
    z = bench.spectrum_error_stats(ref, ref)
    assert all(v == 0.0 for v in z.values())
    # an all-zero tile does not divide by zero
    ref2 = np.vstack([ref, np.zeros(4)])
    assert np.isfinite(list(bench.spectrum_error_stats(ref2, ref2).values())).all()


def test_sigma_stats():
    ref = np.array([[1.0, 2.0, 4.0, 1e-6]])
    sigma = np.array([[0.1, 0.1, 0.2, 1e-9]])
    got = ref + np.array([[0.05, 0.35, -0.2, 1.0]])  # 0.5, 3.5, 1.0 sigma; the last bin is below the floor
    s = bench.sigma_stats(got, ref, sigma)
    assert s["bins"] == 3 and np.isclose(s["max"], 3.5) and np.isclose(s["within_3_sigma"], 2 / 3)
