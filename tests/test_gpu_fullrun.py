"""Full-run statistical parity with the reference's CPU path.

The fixture ``fullrun_hopg20.npz`` (``make_golden.py --only fullrun``) holds
the reference's own run of the 20 MeV HOPG scene with its Twiss beam
(sigma 0.5 mm, 0.5 mrad; 100 um graphite, (002) at 45 deg, detector at 90
deg): 20,000 histories through its per-electron core (SplitMix64 stream,
transport LUT), then its PXR/CBS bin means (16 (00l) rows x 3 mosaic nodes on
injected tables), Bethe-Heitler continuum, exit-energy / exit-angle
histograms, fates and continuous depth loss, in 10 groups of 2,000 electrons.

This package runs the same scene on the GPU from its own Philox stream
(independent histories: 10 batches of 20,000) and every quantity must agree
bin by bin with the reference's within the combined statistical error,
sigma^2 = sigma_ref^2 + sigma_gpu^2, each sigma from its own batch means.
With 9 degrees of freedom per sigma the deviations follow a t distribution
(P(|t| > 3) = 1.5 %, P(|t| > 6) = 2e-4): over n bins at most 2 + 0.03 n
beyond 3 sigma (twice the expected count, plus two for histograms of a few
dozen bins) and none beyond 6 sigma.
"""

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _spec(d):
    from pyrite_b200 import LineTables
    from pyrite_b200.api import BeamSpec
    from pyrite_b200.pipeline import CaseSpec
    from pyrite_b200.tables import HOPG, LayerStack

    tw = (float(d["eps_n_mm_mrad"]), float(d["beta_m"]), 0.0)
    comp = [("C", float(d["n_C"]))]
    return CaseSpec(
        stack=LayerStack([(0.0, float(d["thickness"]), comp)]),
        beam=BeamSpec(float(d["E0_keV"]), np.asarray(d["beam_dir"]), np.deg2rad(float(d["tilt_deg"])), 0.0,
                      twiss_x=tw, twiss_y=tw),
        E_cut_keV=5.0, crystal=HOPG, hkl_list=[tuple(int(x) for x in h) for h in d["hkl"]],
        n_hats=np.asarray(d["n_hat"])[None, :], E_grid=np.asarray(d["E_grid"]),
        line_tables=LineTables(d["E_tab"], d["chi_re"], d["chi_im"], d["u_re"], d["u_im"], d["log_mu"],
                               d["delta"]),
        surface_hkl=(0, 0, 1), mosaic_fwhm_rad=float(d["mosaic_fwhm_rad"]), mosaic_nodes=3,
        brem_composition=comp, brem_mu=np.asarray(d["mu_grid"]), seed=20260,
    )


def _z(ref_groups, gpu_batches):
    """Per-bin deviation of the means in units of the combined sigma (bins
    where either run has a nonzero spread)."""
    r, g = np.asarray(ref_groups, float), np.asarray(gpu_batches, float)
    s2 = r.var(0, ddof=1) / r.shape[0] + g.var(0, ddof=1) / g.shape[0]
    m = s2 > 0
    return (g.mean(0)[m] - r.mean(0)[m]) / np.sqrt(s2[m]), int(m.sum())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_full_run_agrees_with_reference_within_3_sigma(precision, cuda_device):
    import torch

    from pyrite_b200.pipeline import ScoringCase

    d = golden("fullrun_hopg20")
    H, B = 20000, 10
    case = ScoringCase(_spec(d), precision=precision, rng="philox", lut=True, batch_histories=H,
                       device=cuda_device, exit_E_bins=int(d["E_edges"].size - 1),
                       exit_theta_bins=int(d["theta_edges"].size - 1))
    per = {k: [] for k in ("cxr", "brem", "exit_E", "exit_theta", "fates", "deposit")}
    for b in range(B):
        case.reset()
        case.run_batch(b * H, H)
        torch.cuda.synchronize()
        res = case.results()
        per["cxr"].append(res["cxr"][0])
        per["brem"].append(res["brem"][0])
        per["exit_E"].append(res["exit_E"] / H)
        per["exit_theta"].append(res["exit_theta"] / H)
        per["fates"].append(res["fates"][[1, 2, 3, 0]] / H)  # back, trans, side, cutoff
        per["deposit"].append(res["deposit_keV"])
        assert case.device_status() == 0
    Kr = int(d["groups"])
    per_ref = int(d["Ne"]) // Kr
    ref = {"cxr": d["cxr"], "brem": d["brem"], "exit_E": d["exit_E"] / per_ref,
           "exit_theta": d["exit_theta"] / per_ref, "fates": d["fates"] / per_ref,
           "deposit": d["depth_loss"].sum(axis=1, keepdims=True)}
    report = {}
    for k in ("cxr", "brem", "exit_E", "exit_theta", "deposit"):
        z, n = _z(ref[k], per[k])
        report[k] = (n, int(np.sum(np.abs(z) > 3.0)) if n else 0, float(np.max(np.abs(z))) if n else 0.0)
    for k, (n, beyond, zmax) in report.items():
        assert beyond <= 2 + 0.03 * n and zmax <= 6.0, (k, report)
    # Fates (back, trans, side, cutoff): nearly every electron is transmitted;
    # a few in 1e5 backscatter. Binomial errors of both runs, 4 sigma plus one
    # event of the reference's sample.
    p_ref, p_gpu = ref["fates"].mean(0), np.mean(per["fates"], axis=0)
    n_ref, n_gpu = Kr * per_ref, B * H
    p = 0.5 * (p_ref + p_gpu)
    se = np.sqrt(p * (1.0 - p) * (1.0 / n_ref + 1.0 / n_gpu))
    assert np.all(np.abs(p_gpu - p_ref) <= 4.0 * se + 1.0 / n_ref), (p_ref, p_gpu)
    # The spectra are not trivially empty.
    assert report["cxr"][0] > 100 and report["brem"][0] > 700
