"""The layered-stack case through the device pipeline.

One batch of the 10 MeV HOPG / Si / W stack (two crystalline radiators, three
bremsstrahlung layers, C/Si/W characteristic emitters, four detectors) runs
through ``ScoringCase``; its spectra must equal the public per-layer scorers
(``mc_cxr_spectrum`` / ``mc_brem_spectrum`` / ``mc_characteristic_spectrum``
with layers and an emitting layer, each pinned to the reference's layered
spectra elsewhere) applied to the same batch's segment list.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stack_run():
    from pyrite_b200.configs import c5_stack_10mev
    from pyrite_b200.pipeline import ScoringCase

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    spec = c5_stack_10mev(angular_shape=(1, 2), n_bins=1024, si_g_max=4.0)
    # Electrons at 10 MeV take thousands of steps in the millimetre of W:
    # grow the segment buffer until one batch fits.
    per = 2048
    while True:
        case = ScoringCase(spec, precision="fp64", batch_histories=48, segs_per_history=per)
        case.run_batch(0, 48)
        torch.cuda.synchronize()
        if case.device_status() != 4 or per >= 1 << 15:
            break
        per *= 2
        del case
    assert case.device_status() == 0
    n = int(case.seg_count.item())
    assert 0 < n <= case.seg_capacity
    seg = dict(r_mid=case.seg_r[:n].cpu().numpy(), v_hat=case.seg_v[:n].cpu().numpy(),
               L_ang=case.seg_L[:n].cpu().numpy(), E_keV=case.seg_E[:n].cpu().numpy(),
               elec_id=case.seg_id[:n].cpu().numpy(), layer=case.seg_layer[:n].cpu().numpy(),
               Ne=48, thickness_ang=spec.stack.thickness)
    return spec, case, case.results(), seg


def test_every_layer_has_segments(stack_run):
    _spec, _case, res, seg = stack_run
    assert set(np.unique(seg["layer"])) == {0, 1, 2}
    assert res["fates"].sum() == 48


def test_stack_cxr_equals_per_layer_scorer(stack_run):
    import pyrite_b200 as pb

    spec, case, res, seg = stack_run
    layers = list(spec.stack.layers)
    total = np.zeros_like(res["cxr"])
    for r, rows in zip(spec.radiators, case._rows):
        total += pb.mc_cxr_spectrum(seg, spec.E_grid, r.crystal, None, tables=r.line_tables, n_hat=spec.n_hats,
                                    rows=rows, line_quadrature="bin-mean", precision="fp64",
                                    exact_widths=spec.exact_widths, layers=layers,
                                    mu_tables=spec.escape_mu_tables, emit_layer=r.layer)
    assert total.max() > 0
    assert np.max(np.abs(res["cxr"] - total)) <= 1e-9 * np.max(total)


def test_stack_brem_and_lines_equal_per_layer_scorers(stack_run):
    import pyrite_b200 as pb

    spec, _case, res, seg = stack_run
    layers = list(spec.stack.layers)
    brem = sum(pb.mc_brem_spectrum(seg, spec.E_grid, composition=c, n_hat=spec.n_hats, layers=layers,
                                   mu_layer=spec.brem_mu_layer, emit_layer=k, precision="fp64")
               for k, c in enumerate(spec.brem_layers))
    assert np.max(np.abs(res["brem"] - brem)) <= 1e-10 * np.max(brem)
    char = sum(pb.mc_characteristic_spectrum(seg, spec.E_grid, lines=em.lines, n_atoms_per_ang3=em.n_atoms_per_ang3,
                                             n_hat=spec.n_hats, mu_by_line=em.mu_by_line, layers=layers,
                                             emit_layer=em.layer, precision="fp64")
               for em in spec.char_emitters)
    assert char.max() > 0
    assert np.max(np.abs(res["characteristic"] - char)) <= 1e-10 * np.max(char)


def test_mixed_transport_through_the_stack_matches_fp64_step_counts():
    """The mixed-precision transport keeps FP64 positions: millimetres deep
    in the stack a float position cannot resolve the boundary nudge, and a
    particle crossing back out of the W layer would loop on the boundary
    until the step limit."""
    from pyrite_b200.configs import c5_stack_10mev
    from pyrite_b200.pipeline import ScoringCase

    spec = c5_stack_10mev(angular_shape=(1, 1), n_bins=256, si_g_max=4.0)
    per_hist = {}
    for prec in ("fp64", "mixed"):
        case = ScoringCase(spec, precision=prec, batch_histories=64, segs_per_history=1 << 15)
        case.run_batch(0, 64)
        torch.cuda.synchronize()
        assert case.device_status() == 0, (prec, case.device_status())
        per_hist[prec] = int(case.seg_count.item()) / 64
        assert int(case.fates.sum().item()) == 64
    ratio = per_hist["mixed"] / per_hist["fp64"]
    assert 0.8 < ratio < 1.25, per_hist
