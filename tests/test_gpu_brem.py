"""CUDA Bethe-Heitler + Elwert scorer against the reference's spectra."""

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

SYM = {6.0: "C", 8.0: "O", 14.0: "Si", 74.0: "W"}


@pytest.mark.parametrize("case", ["c20", "sio2"])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("mixed", 2e-3)])
def test_brem_matches_reference(case, precision, tol, cuda_device):
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
