"""CUDA Bethe-Heitler + Elwert scorer against the reference's spectra."""

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

SYM = {6.0: "C", 8.0: "O", 14.0: "Si", 74.0: "W"}


@pytest.mark.parametrize("case", ["c20", "sio2"])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 1e-6)])
def test_brem_matches_reference(case, precision, tol, cuda_device):
    """FP64 to 1e-13 of the peak (measured 1.5e-14: the same expression, the
    kernel's exp/log against numpy's); mixed to 1e-6 of the peak (measured
    3.5e-7: the float cross-section rewrite and transmission forms)."""
    from pyrite_b200 import mc_brem_spectrum

    d = golden(f"brem_{case}")
    tr = golden(f"transport_{d['transport']}")
    seg = dict(v_hat=tr["v_hat"], E_repr_keV=tr["E_repr_keV"], L_ang=tr["L_ang"], r_mid=tr["r_mid"],
               elec_id=tr["elec_id"], Ne=int(d["Ne"]), thickness_ang=float(d["thickness"]))
    comp = [(SYM[float(z)], float(n)) for z, n in zip(d["Z"], d["n_ang3"])]
    spec = mc_brem_spectrum(seg, d["E_grid"], composition=comp, n_hat=d["n_hat"], mu=d["mu_grid"],
                            precision=precision, device=cuda_device)
    peak = np.max(np.abs(d["spec"]))
    assert np.max(np.abs(spec - d["spec"])) <= tol * peak


def _c20_segments():
    d = golden("brem_c20")
    tr = golden(f"transport_{d['transport']}")
    seg = dict(v_hat=tr["v_hat"], E_repr_keV=tr["E_repr_keV"], L_ang=tr["L_ang"], r_mid=tr["r_mid"],
               elec_id=tr["elec_id"], Ne=int(d["Ne"]), thickness_ang=float(d["thickness"]))
    comp = [(SYM[float(z)], float(n)) for z, n in zip(d["Z"], d["n_ang3"])]
    return d, seg, comp


def _tile_directions(kind):
    from pyrite_b200 import configs

    tiles = configs.c2_si_50mev().n_hats  # 16 tiles, one exit face, rho = 0.13 %
    if kind == "tiles":
        return tiles
    if kind == "spread5pct":  # one exit face, rho ~ 5 %: order 7
        th = np.linspace(0.30, 0.55, 16)
        return np.stack([np.sin(th), np.zeros_like(th), np.cos(th)], axis=1)
    # both faces: the per-direction form
    n = tiles.copy()
    n[::2, 2] *= -1.0
    return n


@pytest.mark.parametrize("kind", ["tiles", "spread5pct", "both_faces"])
def test_mixed_brem_direction_forms_against_fp64(kind, cuda_device):
    """The mixed scorer's escape forms -- direction moments about the band
    centre (one exit face; order 3 for the detector tiles, order 7 for a 5 %
    spread) and the per-direction form (both faces) -- against the FP64
    scorer on the same segments and directions, per direction within 1e-4 of
    its peak (the float cross section and transmission carry ~1e-6; the
    moment truncation is below 3e-9)."""
    from pyrite_b200 import mc_brem_spectrum

    d, seg, comp = _c20_segments()
    n_hats = _tile_directions(kind)
    out = {}
    for prec in ("fp64", "mixed"):
        out[prec] = mc_brem_spectrum(seg, d["E_grid"], composition=comp, n_hat=n_hats, mu=d["mu_grid"],
                                     precision=prec, device=cuda_device)
    worst = 0.0
    for i in range(n_hats.shape[0]):
        peak = np.max(np.abs(out["fp64"][i]))
        assert peak > 0
        worst = max(worst, float(np.max(np.abs(out["mixed"][i] - out["fp64"][i])) / peak))
    assert worst <= 1e-4, worst
