"""The benchmark scenes as case specs: the parameters each scene states
(energy, target, tilt, detector, grid, reflections) on the CPU."""

import numpy as np


def test_c1_hopg_20mev():
    from pyrite_b200 import configs

    s = configs.c1_hopg_20mev()
    assert s.beam.E0_keV == 20000.0
    assert s.stack.thickness == 1.0e6  # 100 um
    assert np.isclose(s.beam.tilt_polar_rad, np.deg2rad(45.0))
    assert s.surface_hkl == (0, 0, 1) and len(s.hkl_list) == 16  # (00l), |l| <= 8
    assert s.E_grid[0] == 1000.0 and s.E_grid[-1] == 40000.0 and np.allclose(np.diff(s.E_grid), 50.0)
    assert s.mosaic_nodes > 1 and s.mosaic_fwhm_rad > 0
    n = np.asarray(s.n_hats)
    assert n.shape == (1, 3) and np.allclose(np.linalg.norm(n, axis=1), 1.0)


def test_c2_si_50mev():
    from pyrite_b200 import configs

    s = configs.c2_si_50mev()
    assert s.beam.E0_keV == 50000.0
    assert s.stack.thickness == 5.0e6  # 500 um
    assert np.isclose(s.beam.tilt_polar_rad, np.deg2rad(10.0))
    assert s.surface_hkl == (2, 2, 0) and len(s.hkl_list) == 238  # diamond cubic, |g| < 8 / A
    assert s.E_grid.size == 2048 and s.E_grid[0] == 1000.0 and s.E_grid[-1] == 60000.0
    d = s.detector
    assert (d.nx, d.ny, d.width_mm, d.height_mm, d.distance_mm) == (64, 64, 20.0, 20.0, 1000.0)
    assert np.isclose(d.theta_obs_rad, np.deg2rad(20.0))
    n = np.asarray(s.n_hats)
    assert n.shape == (16, 3) and np.allclose(np.linalg.norm(n, axis=1), 1.0)
    # the 4x4 tiles span the 2 x 2 cm^2 plane at 1 m: ~1.1 deg across
    spread = np.degrees(np.arccos(np.clip(n @ n.mean(0) / np.linalg.norm(n.mean(0)), -1, 1))).max()
    assert 0.3 < spread < 1.0


def test_sweep_case_spec_matches_its_configuration():
    from pyrite_b200.sweep import c3_configs, case_spec

    for cfg in c3_configs()[:6]:
        s = case_spec(cfg)
        assert s.beam.E0_keV == cfg.E0_MeV * 1e3
        assert np.isclose(s.stack.thickness, cfg.thickness_um * 1e4)
        assert np.isclose(s.beam.tilt_polar_rad, np.deg2rad(cfg.tilt_deg))
        assert s.E_grid.size == 1024 and s.E_grid[0] == 1000.0 and s.E_grid[-1] == 60000.0
        assert s.crystal.name in ("silicon", "hopg")


def test_host_beam_entries_have_the_scene_spot_and_divergence():
    """oracle.beam_entries (the CPU baseline's entrance states) follows the
    50 MeV Si scene's Twiss beam: spot sigma 1 mm and divergence 0.2 mrad
    per plane (4,000 histories: within 5 %), on the tilted entrance face."""
    import oracle
    from pyrite_b200 import configs
    from pyrite_b200.api import _fill_beam
    from pyrite_b200.tables import beam_frame_basis

    spec = configs.c2_si_50mev(seed=3)
    beam = _fill_beam(None, spec.beam, spec.seed)
    pos, dirs, E = oracle.beam_entries(beam, 0, 4000, rng=1)
    assert np.all(pos[:, 2] == 0.0) and np.all(E == spec.beam.E0_keV)
    np.testing.assert_allclose(np.linalg.norm(dirs, axis=1), 1.0, rtol=1e-15)
    B = beam_frame_basis(np.asarray(spec.beam.beam_dir, float))
    xp, yp = dirs @ B[:, 0], dirs @ B[:, 1]
    assert abs(np.std(xp) / 0.2e-3 - 1.0) < 0.05 and abs(np.std(yp) / 0.2e-3 - 1.0) < 0.05
    # transverse offsets: the entry points seen along the beam (perpendicular plane)
    bd = np.asarray(spec.beam.beam_dir, float)
    perp = pos - np.outer(pos @ bd, bd)
    assert abs(np.std(perp @ B[:, 0]) / 1.0e7 - 1.0) < 0.05
    assert abs(np.std(perp @ B[:, 1]) / 1.0e7 - 1.0) < 0.05
