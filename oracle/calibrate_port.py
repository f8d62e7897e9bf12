"""Calibrate the CPU port against the reference's own CPU path (one core).

TEST INFRASTRUCTURE: a one-off measurement recipe, run in a container that
holds the reference tree ($PYRITE_REFERENCE_ROOT, else the path given with
--reference); it never runs on a GPU machine and nothing in pyrite_b200
imports it.

Both arms process the same histories of the 50 MeV Si scene (500 um Si,
(220) at 10 deg, 1 mm / 0.2 mrad Twiss beam, 16 tiles of the 2x2 cm^2
detector at 20 deg, 2048 bins 1-60 keV, the 238 reflections |g| < 8 1/A):

- reference: its per-electron Numba core (screened-Rutherford elastic,
  spliced stopping, uncoupled radiation, exact core), then
  ``mc_cxr_spectrum`` (bin-mean) and Bethe-Heitler ``mc_brem_spectrum`` on
  every tile, the line data injected at its seams (smooth synthetic
  tables, as the golden vectors do);
- port: this directory's C restatement (``oracle.transport`` exact core,
  ``cxr_lines`` + ``reduce_binmean``, ``brem_spectrum``) on the same entry
  states, tables from ``pyrite_b200.configs``.

Prints one JSON line: histories/s of each arm (after one warm-up history
each, so Numba's compilation is excluded) and their ratio.

    python oracle/calibrate_port.py [--histories 4] [--reference PATH]
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--histories", type=int, default=4)
    ap.add_argument("--reference", default=os.environ.get("PYRITE_REFERENCE_ROOT"))
    args = ap.parse_args()
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    os.environ["PYRITE_REFERENCE_ROOT"] = str(args.reference)
    import make_golden as mg  # imports the reference through oracle.ref_harness
    from pyrite.materials.crystal import CRYSTALS, reciprocal_g_vector
    from pyrite.montecarlo.spectrum import brem as ref_brem
    from pyrite.montecarlo.spectrum.cxr import _batched, _setup
    from pyrite.montecarlo.spectrum.cxr._spectrum import mc_cxr_spectrum
    from pyrite.montecarlo.transport import TransportLUTConfig, _simulate_trajectories
    from pyrite.montecarlo.transverse import TransverseDistribution, resolve_transverse_distribution
    from dataclasses import asdict

    import oracle
    from pyrite_b200 import configs
    from pyrite_b200.api import _fill_beam
    from pyrite_b200.tables import energy_bin_edges, line_keep_window, reflection_rows

    spec = configs.c2_si_50mev(seed=12345)
    st = spec.stack
    n = int(args.histories)
    beam = _fill_beam(None, spec.beam, spec.seed)
    E_grid = spec.E_grid
    n_dirs = spec.n_hats
    comp = spec.brem_composition

    # ---- reference arm ----
    info = CRYSTALS["silicon"]
    hkl = [tuple(h) for h in spec.hkl_list]
    g_mags = np.array([reciprocal_g_vector(h, info["lattice"])[1] for h in hkl])
    E_tab = mg.synthetic_E_tab(E_grid)
    tables = mg.synthetic_couplings(g_mags, E_tab)
    patches = [
        (_setup, "_line_tabulation_grid", lambda *a, **k: E_tab),
        (_setup, "_elemental_log_mu_table", lambda c, E: mg.synthetic_log_mu(c, E)),
        (_setup, "refractive_index", lambda cr, E, uh=True: (1.0 - mg.synthetic_delta(E)) + 0j),
        (_batched, "_reflection_tables", lambda *a, **k: tuple(np.array(t) for t in tables)),
    ]
    for m, name, f in patches:
        setattr(m, name, f)
    ref_brem._mu_total_inv_ang = lambda c, E: mg.synthetic_mu_total(c, np.asarray(E, dtype=float))

    en, beta_m, _alpha = spec.beam.twiss_x
    twiss = asdict(resolve_transverse_distribution(TransverseDistribution(en, beta_m), energy_keV=spec.beam.E0_keV))

    def reference(e_start, count):
        # the reference samples its own entries from the same Twiss beam
        out = _simulate_trajectories(
            E0_keV=spec.beam.E0_keV, Ne=count, thickness_ang=st.thickness, composition=comp, seed=spec.seed,
            elastic_model="sr", transport_core="per-electron", radiative_model="uncoupled",
            transport_lut_config=TransportLUTConfig(enabled=False), beam_dir=spec.beam.beam_dir,
            tilt_polar_rad=spec.beam.tilt_polar_rad, transverse_distribution=twiss, _electron_start=e_start)
        seg = {k: np.asarray(out[k]) for k in ("r_mid", "v_hat", "L_ang", "E_keV", "E_repr_keV", "elec_id")}
        seg["Ne"], seg["thickness_ang"] = count, st.thickness
        for d in range(n_dirs.shape[0]):
            mc_cxr_spectrum(seg, E_grid, crystal="silicon", hkl_list=hkl, B_ang2=float(info.get("B_ang2", 0.0)),
                            absorber_element="Si", n_hat=n_dirs[d], surface_hkl=spec.surface_hkl,
                            mosaic_fwhm_rad=None, mosaic_nodes=1, node_support_cutoff=None,
                            line_quadrature="bin-mean")
            ref_brem.mc_brem_spectrum(seg, E_grid, composition=comp, n_hat=n_dirs[d],
                                      cross_section_model="bethe-heitler")
        return int(np.size(out["L_ang"]))

    # ---- port arm (as bench.py's CPU baseline) ----
    lt = oracle.LayerTables(st.z_top, st.z_bot, st.n_el, st.Z, st.J, st.N, st.E_cross)
    rows = reflection_rows(spec.crystal, spec.hkl_list, n_dirs, surface_hkl=spec.surface_hkl)
    lo, hi = line_keep_window(E_grid)
    edges = energy_bin_edges(E_grid)
    lt_ = spec.line_tables

    def port(e_start, count):
        pos, dirs, E = oracle.beam_entries(beam, e_start, count, rng=oracle.RNG_PHILOX)
        out = oracle.transport(lt, pos, dirs, E, seed=spec.seed, E_cut=spec.E_cut_keV, rng=oracle.RNG_PHILOX,
                               e_start=e_start, cap=256)
        seg = dict(v_hat=out["v_hat"], E_keV=0.5 * (out["E_start"] + out["E_end"]), L_ang=out["L"],
                   r_mid=out["r_mid"], elec_id=out["elec_id"])
        for d in range(n_dirs.shape[0]):
            t = dict(G=rows.G, ES=rows.ES[d], EP=rows.EP[d], WM=rows.WM, row_table=rows.row_table,
                     E_tab=lt_.E_tab, chi_re=lt_.chi_re, chi_im=lt_.chi_im, u_re=lt_.u_re, u_im=lt_.u_im,
                     log_mu=lt_.log_mu, delta=lt_.delta, lo_keep=lo, hi_keep=hi)
            Er, aw, w, good = oracle.cxr_lines(t, n_dirs[d], st.thickness, seg, e_start + count)
            oracle.reduce_binmean(Er[good], aw[good], w[good], edges)
            oracle.brem_spectrum(seg, [14.0], [comp[0][1]], st.thickness, n_dirs[d], E_grid, spec.brem_mu, count)
        return int(out["L"].size)

    out = {}
    for name, fn in (("reference", reference), ("port", port)):
        fn(900, 1)  # warm-up: imports, Numba compilation, tables
        t0 = time.perf_counter()
        segs = fn(1000, n)
        dt = time.perf_counter() - t0
        out[name] = {"histories_per_s": n / dt, "seconds": dt, "segments": segs}
    out["ratio_port_over_reference"] = out["port"]["histories_per_s"] / out["reference"]["histories_per_s"]
    out["config"] = (f"{n} histories of the 50 MeV Si scene, 16 tiles, 2048 bins, 238 reflections, one core "
                     f"(NUMBA_NUM_THREADS={os.environ.get('NUMBA_NUM_THREADS')})")
    print(json.dumps(out))


if __name__ == "__main__":
    main()
