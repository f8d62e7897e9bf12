"""Host-side table builders of pyrite_b200 against the reference's own tables."""

import numpy as np
import pytest

from conftest import CXR_CASES, LUT_CASES, golden
from pyrite_b200 import tables as T


def stack_of(d):
    sym = {6: "C", 8: "O", 14: "Si", 74: "W"}
    layers = []
    for L in range(d["z_top"].size):
        comp = [(sym[int(z)], float(n)) for z, n in zip(d["Z"][L][: d["n_el"][L]], d["N"][L][: d["n_el"][L]])]
        layers.append((float(d["z_top"][L]), float(d["z_bot"][L]), comp))
    return T.LayerStack(layers)


@pytest.mark.parametrize("case", ["c20mev", "stack10mev", "sio2_300kev"])
def test_layer_coefficients_match_reference(case):
    d = golden(f"transport_{case}")
    st = stack_of(d)
    np.testing.assert_array_equal(st.E_cross, d["E_cross"])
    np.testing.assert_array_equal(st.J, d["J"])


@pytest.mark.parametrize("case", LUT_CASES)
def test_transport_lut_matches_reference(case):
    d = golden(f"transport_lut_{case}")
    g = golden(f"transport_{case}")
    lut = T.build_transport_lut(stack_of(g), float(d["E_min_keV"]), float(d["E_max_keV"]))
    assert lut.n_energy == int(d["n_energy"])
    assert lut.log_E_min == float(d["log_E_min"])
    assert lut.inv_dlogE == float(d["inv_dlogE"])
    for name, ref in (("total_rate", "lut_total_rate"), ("dEds", "lut_dEds"), ("inv_beta", "lut_inv_beta"),
                      ("cdf", "lut_cdf"), ("alpha", "lut_alpha")):
        np.testing.assert_allclose(getattr(lut, name), d[ref], rtol=2e-15, atol=0, err_msg=name)


def test_lut_packing_is_aligned():
    g = golden("transport_stack10mev")
    lut = T.build_transport_lut(stack_of(g), 5.0, 1e4)
    for dtype in (np.float32, np.float64):
        buf, offs = lut.packed(dtype)
        assert buf.nbytes % 16 == 0
        for off in offs.values():
            assert (off * np.dtype(dtype).itemsize) % 16 == 0
        ne = lut.n_energy
        np.testing.assert_array_equal(buf[offs["inv_beta"]:offs["inv_beta"] + ne], lut.inv_beta.astype(dtype))


@pytest.mark.parametrize("case", CXR_CASES)
def test_reflection_rows_match_reference(case):
    d = golden(f"cxr_{case}")
    cr = T.CRYSTALS[str(d["crystal"])]
    mf = float(d["mosaic_fwhm_rad"])
    rows = T.reflection_rows(cr, [tuple(h) for h in d["hkl"]], d["n_hat"][None, :],
                             surface_hkl=tuple(int(v) for v in d["surface_hkl"]),
                             mosaic_fwhm_rad=None if np.isnan(mf) else mf,
                             mosaic_nodes=int(d["mosaic_nodes"]))
    np.testing.assert_allclose(rows.G, d["G"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(rows.ES[0], d["ES"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(rows.EP[0], d["EP"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(rows.WM, d["WM"], rtol=1e-14, atol=0)
    np.testing.assert_array_equal(rows.row_table, d["row_table"])
    np.testing.assert_allclose([cr.g_vector(h)[1] for h in d["hkl"]], d["g_mags"], rtol=1e-14)


def test_tilted_geometry_matches_transport_fixture():
    d = golden("transport_c20mev")
    bd, nh = T.tilted_geometry(np.deg2rad(90.0), np.deg2rad(45.0))
    np.testing.assert_allclose(bd, d["beam_dir"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(nh, d["n_hat"], rtol=0, atol=1e-15)


def test_bin_edges_and_keep_window():
    E = np.arange(1000.0, 40000.0 + 1e-6, 50.0)
    e = T.energy_bin_edges(E)
    assert e[0] == 975.0 and e[-1] == 40025.0 and e.size == E.size + 1
    lo, hi = T.line_keep_window(E)
    assert lo == 1000.0 - 0.2 * 39000.0 and hi == 40000.0 + 0.2 * 39000.0


def test_diamond_reflection_count():
    hkl = T.diamond_hkls(8.0)
    # every listed reflection is allowed and inside the sphere; the (220) set is present
    assert (2, 2, 0) in hkl and (1, 1, 1) in hkl and (2, 0, 0) not in hkl
    assert all(T.SILICON.g_vector(h)[1] < 8.0 for h in hkl)
