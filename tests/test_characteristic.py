"""Characteristic lines: the oracle, the host line preparation and the CUDA kernel.

The goldens (``tests/golden/char_*.npz``) come from the reference's own
``mc_characteristic_spectrum`` with synthetic EEDL/EADL-like tables injected
through its module seams (see ``make_golden.py``): a Si slab at 50 MeV, the W
back layer of a C/Si/W stack at 10 MeV (escape through three absorbers), and
a C slab whose only line lies below the grid (tails only).
"""

import numpy as np
import pytest

import oracle.characteristic as OC
from conftest import golden

CASES = ("si50", "stack_w", "c20")


def _inputs(name):
    d = golden(f"char_{name}")
    tr = golden(f"transport_{d['transport']}")
    m = d["seg_mask"]
    seg = dict(r_mid=tr["r_mid"][m], v_hat=tr["v_hat"][m], L=tr["L_ang"][m], E_keV=tr["E_repr_keV"][m],
               elec_id=tr["elec_id"][m])
    layers = list(zip(d["layer_z_top"], d["layer_z_bot"])) if d["layer_z_top"].size else None
    return d, seg, layers


def _lines(d):
    from pyrite_b200 import CharacteristicLines

    offs = d["shell_offset"]
    n_shell = offs.size - 1
    return CharacteristicLines(
        shell_E=tuple(d["shell_E"][offs[i]:offs[i + 1]] for i in range(n_shell)),
        shell_sigma=tuple(d["shell_sigma"][offs[i]:offs[i + 1]] for i in range(n_shell)),
        line_E=d["line_E"], line_fwhm=d["line_fwhm"], response=d["response_all"])


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference(case):
    d, seg, layers = _inputs(case)
    y = OC.line_yields(seg, d["n_hat"], float(d["thickness"]), float(d["n_atoms"]), d["shell_E"], d["shell_sigma"],
                       d["shell_offset"], d["kept_response"], d["mu_by_line"], layers=layers, Ne=int(d["Ne"]))
    spec = OC.spectrum(y, d["profiles"], int(d["Ne"]))
    peak = np.max(np.abs(d["spec"]))
    assert peak > 0
    assert np.max(np.abs(spec - d["spec"])) <= 1e-13 * peak


@pytest.mark.parametrize("case", CASES)
def test_host_line_preparation_matches_reference(case):
    from pyrite_b200.api import prepare_characteristic_lines

    d, _seg, _layers = _inputs(case)
    kept, profiles = prepare_characteristic_lines(_lines(d), d["E_grid"])
    np.testing.assert_array_equal(profiles, d["profiles"])
    np.testing.assert_array_equal(np.asarray(_lines(d).response)[:, kept], d["kept_response"])


def test_cutoff_below_data_minimum_is_refused():
    from pyrite_b200.api import prepare_characteristic_lines

    d, _seg, _layers = _inputs("si50")
    with pytest.raises(ValueError):
        prepare_characteristic_lines(_lines(d), d["E_grid"], relaxation_cutoff_eV=10.0)


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-5)])
def test_kernel_matches_reference(case, precision, tol, cuda_device):
    from pyrite_b200 import mc_characteristic_spectrum

    d, seg, layers = _inputs(case)
    kept_mu_cols = d["mu_by_line"]
    lines = _lines(d)
    from pyrite_b200.api import prepare_characteristic_lines

    kept, _ = prepare_characteristic_lines(lines, d["E_grid"])
    mu_all = np.zeros((kept_mu_cols.shape[0], lines.line_E.size))
    mu_all[:, kept] = kept_mu_cols
    segments = dict(r_mid=seg["r_mid"], v_hat=seg["v_hat"], L_ang=seg["L"], E_repr_keV=seg["E_keV"],
                    elec_id=seg["elec_id"], Ne=int(d["Ne"]), thickness_ang=float(d["thickness"]))
    spec = mc_characteristic_spectrum(segments, d["E_grid"], lines=lines, n_atoms_per_ang3=float(d["n_atoms"]),
                                      n_hat=d["n_hat"], mu_by_line=mu_all, layers=layers, precision=precision,
                                      device=cuda_device)
    peak = np.max(np.abs(d["spec"]))
    assert np.max(np.abs(spec - d["spec"])) <= tol * peak
