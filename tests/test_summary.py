"""The device tallies laid out as the reference's summary tables
(montecarlo/trajectory_summary.py:171-260): histogram rows with explicit
underflow and overflow (np.histogram bins in between), fate counts and
fractions of the sampled primaries, per-layer depth loss."""

import numpy as np


def test_tables_follow_the_reference_layout():
    from pyrite_b200.summary import tally_tables

    rng = np.random.default_rng(2)
    E = np.r_[rng.uniform(-5.0, 22000.0, 500), 0.0, 20000.0]  # with values on both outer edges
    edges = np.linspace(0.0, 20000.0, 65)
    # the device convention: under = v < lo, over = v > hi, hi itself in the last bin
    counts = np.r_[np.count_nonzero(E < edges[0]), np.histogram(E, edges)[0], np.count_nonzero(E > edges[-1])]
    th_edges = np.linspace(0.0, np.pi, 37)
    th = rng.uniform(0.0, np.pi, 300)
    th_counts = np.r_[0, np.histogram(th, th_edges)[0], 0]
    fates = np.array([10, 20, 30, 0, 1, 2])
    t = tally_tables(fates, counts, th_counts, [5.0, 7.0], E_lo=0.0, E_hi=20000.0, theta_lo=0.0,
                     theta_hi=np.pi, z_top=[0.0, 10.0], z_bot=[10.0, 30.0])
    ee = t["exit_energy"]
    assert list(ee.columns) == ["low_keV", "high_keV", "count"]
    assert ee["low_keV"].iloc[0] == -np.inf and ee["high_keV"].iloc[-1] == np.inf
    np.testing.assert_allclose(ee["low_keV"].iloc[1:-1], edges[:-1])
    np.testing.assert_allclose(ee["high_keV"].iloc[1:-1], edges[1:])
    assert ee["count"].sum() == E.size
    assert list(t["exit_angle"].columns) == ["low_rad", "high_rad", "count"]
    f = t["fates"].set_index("fate")
    assert f.loc["backscattered", "count"] == 20 and f.loc["transmitted", "count"] == 30
    assert f.loc["cutoff_stopped", "count"] == 10 and f.loc["unfinished", "count"] == 1
    assert abs(f["fraction"].sum() - 1.0) < 1e-12
    d = t["depth_loss"]
    assert list(d.columns) == ["layer", "depth_low_ang", "depth_high_ang", "continuous_loss_keV"]
    assert d["continuous_loss_keV"].tolist() == [5.0, 7.0]
