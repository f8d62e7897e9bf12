"""Fused exit tallies (fates, exit-energy and exit-angle histograms with
under/overflow slots, per-layer deposit): against the reference's own summary
tables of the same histories (the FP64 replay of its SplitMix64 rows), and
against the same quantities recomputed on the host from the kernel's own
per-history outputs, with the reference's histogram convention
(trajectory_summary.py:147-260: np.histogram bins, explicit underflow and
overflow)."""

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu

_SYM = {6: "C", 8: "O", 14: "Si", 74: "W"}


def _layers_of(d):
    out = []
    for L in range(d["z_top"].size):
        n = int(d["n_el"][L])
        out.append((float(d["z_top"][L]), float(d["z_bot"][L]),
                    [(_SYM[int(z)], float(x)) for z, x in zip(d["Z"][L][:n], d["N"][L][:n])]))
    return out


def _slot(v, lo, hi, n):
    out = np.empty(v.shape, dtype=np.int64)
    under = ~(v >= lo)
    over = v > hi
    b = np.minimum(((v - lo) / (hi - lo) * n).astype(np.int64), n - 1) + 1
    out[:] = b
    out[over] = n + 1
    out[under] = 0
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tallies_match_per_history_outputs(precision, cuda_device):
    import ctypes as C

    from pyrite_b200 import _lib as L
    from pyrite_b200 import configs
    from pyrite_b200.pipeline import ScoringCase

    spec = configs.c1_hopg_20mev(seed=4)
    n = 4096
    case = ScoringCase(spec, precision=precision, batch_histories=n, device=cuda_device)
    code = torch.full((n,), -1, dtype=torch.int8, device=cuda_device)
    fE = torch.zeros(n, dtype=torch.float64, device=cuda_device)
    fdir = torch.zeros(n, 3, dtype=torch.float64, device=cuda_device)
    case.targs.exit_code, case.targs.final_E, case.targs.final_dir = code.data_ptr(), fE.data_ptr(), fdir.data_ptr()
    case.run_batch(0, n)
    torch.cuda.synchronize()
    assert case.device_status() == 0
    codes = code.cpu().numpy().astype(np.int64)
    assert codes.min() >= 0
    np.testing.assert_array_equal(case.fates.cpu().numpy(), np.bincount(codes, minlength=6))
    esc = np.isin(codes, (1, 2, 3))
    t = case.targs.tallies
    E = fE.cpu().numpy()[esc]
    want_E = np.bincount(_slot(E, t.E_lo, t.E_hi, t.n_E), minlength=t.n_E + 2)
    np.testing.assert_array_equal(case.exit_E.cpu().numpy(), want_E)
    th = np.arccos(np.clip(fdir.cpu().numpy()[esc, 2], -1.0, 1.0))
    want_th = np.bincount(_slot(th, t.theta_lo, t.theta_hi, t.n_theta), minlength=t.n_theta + 2)
    np.testing.assert_array_equal(case.exit_theta.cpu().numpy(), want_th)
    # Energy bookkeeping: what the histories lost in the slab is the deposit.
    lost = float(n * spec.beam.E0_keV - fE.cpu().numpy().sum())
    dep = float(case.deposit.sum().item())
    assert abs(dep - lost) <= 1e-6 * lost
    # the same tallies in the reference's summary-table layout
    from pyrite_b200.summary import case_tally_tables

    tab = case_tally_tables(case)
    assert int(tab["fates"]["count"].sum()) == n
    np.testing.assert_array_equal(tab["exit_energy"]["count"].to_numpy(), want_E)
    np.testing.assert_array_equal(tab["exit_angle"]["count"].to_numpy(), want_th)
    assert abs(float(tab["depth_loss"]["continuous_loss_keV"].sum()) - dep) <= 1e-9 * dep


@pytest.mark.parametrize("case", ["c20mev", "si50mev", "stack10mev", "si30kev", "sio2_300kev"])
def test_fused_tallies_equal_the_reference_summary(case, cuda_device):
    """The transport kernel's fused tallies of the FP64 exact core replaying
    the reference's SplitMix64 histories (same entrance states) equal the
    reference's own summary tables of its own rows (``_history_rows``,
    ``_histogram``, ``depth_loss_profile`` of trajectory_summary.py, run by
    make_golden.py): fates, exit-energy and exit-angle histograms with their
    under- and overflow bins count for count, continuous loss per layer to
    1e-12 (FP64 sums in another order)."""
    from pyrite_b200 import simulate_trajectories

    d = golden(f"transport_{case}")
    ref = golden(f"summary_{case}")
    n_E, n_th = int(ref["E_edges"].size - 1), int(ref["theta_edges"].size - 1)
    got = simulate_trajectories(float(d["E0_keV"]), int(d["Ne"]), layers=_layers_of(d),
                                E_cut_keV=float(d["E_cut_keV"]), seed=int(d["seed"]), device=cuda_device,
                                lut=False, rng="splitmix", precision="fp64",
                                entry=(d["initial_r"], d["initial_v"], d["initial_E"]), tallies=(n_E, n_th))
    assert got["device_status"] == 0
    np.testing.assert_array_equal(got["tally_fates"][[1, 2, 3, 0]], ref["fates"])
    np.testing.assert_array_equal(got["tally_exit_E"], ref["exit_E"])
    np.testing.assert_array_equal(got["tally_exit_theta"], ref["exit_theta"])
    np.testing.assert_allclose(got["tally_deposit_keV"], ref["deposit_per_layer"], rtol=1e-12)
