"""The five synthetic beam/crystal scenes of the benchmark suite as case specs.

Each builder returns a ``pipeline.CaseSpec`` with the scene's geometry, beam,
crystal, reflections, detector tiles and spectral grid. The atomic data
tables come from ``placeholder_data`` (the real Chantler/EPDL data are not
shipped with this package); see that module.
"""

from __future__ import annotations

import numpy as np

from . import placeholder_data as P
from .api import BeamSpec
from .detector import PlanarDetector, tiles_in_sample_frame
from .pipeline import CaseSpec
from .tables import HOPG, SILICON, LayerStack, diamond_hkls, tilted_geometry


def _twiss(E0_keV, sigma_mm, sigma_prime_rad):
    """Courant-Snyder waist (alpha = 0) with the given spot and divergence."""
    gamma = 1.0 + E0_keV / 510.99895
    bg = float(np.sqrt(gamma * gamma - 1.0))
    eps_geo = sigma_mm * sigma_prime_rad            # mm rad
    beta_m = sigma_mm / sigma_prime_rad * 1e-3     # mm/rad -> m
    eps_n = eps_geo * bg * 1e3                     # mm mrad
    return (eps_n, beta_m, 0.0)


def c1_hopg_20mev(seed=0):
    """20 MeV, 0.5 mm / 0.5 mrad, 100 um HOPG, (002) at 45 deg, 0.4 deg mosaic
    (Gaussian sigma), 1 cm^2 pixel at 1 m and 90 deg; 1-40 keV in 50 eV bins."""
    E0 = 20000.0
    tilt = np.deg2rad(45.0)
    beam_dir, n_hat = tilted_geometry(np.deg2rad(90.0), tilt)
    tw = _twiss(E0, 0.5, 0.5e-3)
    n_c = HOPG.n_atoms_per_ang3
    stack = LayerStack([(0.0, 1.0e6, [("C", n_c)])])
    E_grid = np.arange(1000.0, 40000.0 + 1e-6, 50.0)
    hkl = [(0, 0, l) for l in range(-8, 9) if l != 0]
    comp = [("C", n_c)]
    return CaseSpec(
        stack=stack, beam=BeamSpec(E0, beam_dir, tilt, 0.0, twiss_x=tw, twiss_y=tw), E_cut_keV=5.0,
        crystal=HOPG, hkl_list=hkl, n_hats=n_hat[None, :], E_grid=E_grid,
        line_tables=P.line_tables(HOPG, hkl, E_grid, comp), surface_hkl=(0, 0, 1),
        mosaic_fwhm_rad=np.deg2rad(0.4 * 2.3548200450309493), mosaic_nodes=3,
        brem_composition=comp, brem_mu=P.mu_total(comp, E_grid), seed=seed,
    )


def c2_si_50mev(seed=0, angular_shape=(4, 4), n_bins=2048):
    """50 MeV, 1 mm / 0.2 mrad, 500 um Si (220) at 10 deg, 64x64-pixel 2x2 cm^2
    detector at 20 deg and 1 m scored in angular tiles; 1-60 keV in 2048 bins."""
    E0 = 50000.0
    tilt = np.deg2rad(10.0)
    beam_dir, _ = tilted_geometry(np.deg2rad(20.0), tilt)
    det = PlanarDetector(np.deg2rad(20.0), 1000.0, 20.0, 20.0, 64, 64)
    _, n_hats, _ = tiles_in_sample_frame(det, angular_shape, tilt)
    tw = _twiss(E0, 1.0, 0.2e-3)
    n_si = SILICON.n_atoms_per_ang3
    stack = LayerStack([(0.0, 5.0e6, [("Si", n_si)])])
    E_grid = np.linspace(1000.0, 60000.0, n_bins)
    hkl = diamond_hkls(8.0)
    comp = [("Si", n_si)]
    return CaseSpec(
        stack=stack, beam=BeamSpec(E0, beam_dir, tilt, 0.0, twiss_x=tw, twiss_y=tw), E_cut_keV=5.0,
        crystal=SILICON, hkl_list=hkl, n_hats=n_hats, E_grid=E_grid,
        line_tables=P.line_tables(SILICON, hkl, E_grid, comp), surface_hkl=(2, 2, 0),
        brem_composition=comp, brem_mu=P.mu_total(comp, E_grid), seed=seed,
        detector=det, angular_shape=tuple(angular_shape),
    )


W_N_PER_ANG3 = 19.3 / 183.84 * 0.602214076  # amorphous W at 19.3 g/cm^3


def c5_stack_10mev(seed=0, angular_shape=(4, 4), n_bins=4096, si_g_max=8.0, detector_angles_deg=(20.0, 45.0, 90.0, 135.0)):
    """10 MeV, 0.5 mm / 0.5 mrad, normal incidence on a three-layer stack:
    20 um HOPG with (002) at 45 deg to the beam, 200 um Si with (220) at
    10 deg, 1 mm amorphous W (19.3 g/cm^3). Four 64x64-pixel 2x2 cm^2
    detectors at 1 m and 20/45/90/135 deg, each scored in angular tiles;
    1-80 keV in 4096 bins. Both crystals radiate PXR/CBS, every layer
    bremsstrahlung with its own composition, and C/Si/W their K and L lines,
    all escaping through the whole stack. The lattice tilts are crystal
    miscuts (the beam stays on the stack normal).

    One electron population is transported, at the 5 keV line cutoff; the
    reference transports bremsstrahlung and characteristic emitters again at
    1 keV with secondary electrons, which need EEDL tables this package does
    not ship."""
    from .detector import PlanarDetector, tiles_in_sample_frame
    from .pipeline import CharEmitter, Radiator

    E0 = 10000.0
    beam_dir, _ = tilted_geometry(np.deg2rad(detector_angles_deg[0]), 0.0)
    tw = _twiss(E0, 0.5, 0.5e-3)
    n_c, n_si, n_w = HOPG.n_atoms_per_ang3, SILICON.n_atoms_per_ang3, W_N_PER_ANG3
    comps = [[("C", n_c)], [("Si", n_si)], [("W", n_w)]]
    bounds = [(0.0, 2.0e5), (2.0e5, 2.2e6), (2.2e6, 1.22e7)]
    stack = LayerStack([(a, b, c) for (a, b), c in zip(bounds, comps)])
    E_grid = np.linspace(1000.0, 80000.0, n_bins)
    dets = [PlanarDetector(np.deg2rad(a), 1000.0, 20.0, 20.0, 64, 64) for a in detector_angles_deg]
    n_hats = np.concatenate([tiles_in_sample_frame(d, angular_shape, 0.0)[1] for d in dets])
    hopg_hkl = [(0, 0, l) for l in range(-8, 9) if l != 0]
    si_hkl = diamond_hkls(si_g_max)
    radiators = [
        Radiator(0, HOPG, hopg_hkl, P.line_tables(HOPG, hopg_hkl, E_grid, comps[0]), surface_hkl=(0, 0, 1),
                 recip_miscut_rad=(np.deg2rad(45.0), 0.0)),
        Radiator(1, SILICON, si_hkl, P.line_tables(SILICON, si_hkl, E_grid, comps[1]), surface_hkl=(2, 2, 0),
                 recip_miscut_rad=(np.deg2rad(10.0), 0.0)),
    ]
    emitters = []
    for k, (el, n) in enumerate([("C", n_c), ("Si", n_si), ("W", n_w)]):
        lines = P.characteristic_lines(el)
        mu_by_line = np.stack([P.mu_total(c, lines.line_E) for c in comps])
        emitters.append(CharEmitter(lines, n, mu_by_line, layer=k))
    return CaseSpec(
        stack=stack, beam=BeamSpec(E0, beam_dir, 0.0, 0.0, twiss_x=tw, twiss_y=tw), E_cut_keV=5.0,
        crystal=None, hkl_list=None, n_hats=n_hats, E_grid=E_grid, line_tables=None,
        radiators=radiators, escape_mu_tables=[P.exact_mu_table(c) for c in comps],
        brem_layers=comps, brem_mu_layer=np.stack([P.mu_total(c, E_grid) for c in comps]),
        char_emitters=emitters, seed=seed,
    )
