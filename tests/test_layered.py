"""Escape through a layered absorber (the 10 MeV C / Si / W stack).

The reference cuts each segment at the layer boundaries it crosses, takes the
per-layer escape paths of every linear piece and attenuates a line or a
photon energy by sum_k path_k mu_k (segment_escape.py:193-355); each layer
radiates bremsstrahlung with its own composition (runner/emission.py:155-172)
and each crystalline layer its own PXR/CBS lines (runner/case_driver.py:
742-770), all escaping through the whole stack. The fixture
``layered_stack10`` holds the reference's own spectra for that stack
(tests/golden/make_golden.py ``gen_layered``).

CPU: the oracle against those spectra, and the piece geometry on segments
that cross boundaries. GPU: ``pb_brem_score`` and ``pb_cxr_score`` with
layers against the reference and the oracle, through the C ABI.
"""

import numpy as np
import pytest
import torch

import oracle
from conftest import golden

NE_FIELDS = ("r_mid", "v_hat", "L_ang", "E_keV", "elec_id", "layer")


def stack():
    g = golden("layered_stack10")
    tr = golden("transport_stack10mev")
    mus = [(g[f"mu_knot_{k}"], g[f"mu_value_{k}"], g[f"mu_slope_{k}"]) for k in range(g["z_top"].size)]
    return g, tr, mus


def layer_segments(tr, L, Ne):
    """Segments emitted in layer L by the first Ne histories, energies at the
    propagator's representative point (brem.py:997-1001, cxr/_setup.py)."""
    keep = (tr["layer"] == L) & (tr["elec_id"] < Ne)
    seg = {k: tr[k][keep] for k in NE_FIELDS}
    seg["E_keV"] = tr["E_repr_keV"][keep]
    return seg


def cxr_tables(g, L):
    E_grid = g["cxr_E_grid"]
    pad = 0.2 * (E_grid[-1] - E_grid[0])
    t = {k: g[f"cxr_{k}_{L}"] for k in ("G", "ES", "EP", "WM", "row_table", "chi_re", "chi_im", "u_re", "u_im",
                                        "log_mu")}
    t.update(E_tab=g["cxr_E_tab"], delta=g["cxr_delta"], lo_keep=E_grid[0] - pad, hi_keep=E_grid[-1] + pad)
    return t


def test_oracle_layered_brem_matches_reference():
    g, tr, mus = stack()
    ly = oracle.LayerEscape(g["z_top"], g["z_bot"], mus)
    Ne = int(g["Ne"])
    for L in range(g["z_top"].size):
        seg = layer_segments(tr, L, Ne)
        s = oracle.brem_spectrum_layered(seg, g[f"brem_Z_{L}"], g[f"brem_n_{L}"], ly, g["n_hat"],
                                         g["brem_E_grid"], g["brem_mu_layer"], Ne)
        ref = g[f"brem_spec_{L}"]
        assert ref.max() > 0
        np.testing.assert_allclose(s, ref, rtol=1e-12, atol=1e-14 * ref.max())


@pytest.mark.parametrize("L", [0, 1])
def test_oracle_layered_cxr_matches_reference(L):
    g, tr, mus = stack()
    ly = oracle.LayerEscape(g["z_top"], g["z_bot"], mus)
    Ne = int(g["Ne"])
    seg = layer_segments(tr, L, Ne)
    E_res, aw, w, good = oracle.cxr_lines(cxr_tables(g, L), g["n_hat"], g["thickness"], seg, Ne, layers=ly)
    assert good.any()
    node = oracle.reduce_node(E_res[good], aw[good], w[good], g["cxr_E_grid"]) / Ne
    ref = g[f"cxr_spec_node_{L}"]
    assert np.max(np.abs(node - ref)) <= 1e-9 * np.max(np.abs(ref))
    edges = oracle.energy_bin_edges(g["cxr_E_grid"])
    binm = oracle.reduce_binmean(E_res[good], aw[good], w[good], edges) / Ne
    ref = g[f"cxr_spec_binmean_{L}"]
    assert np.max(np.abs(binm - ref)) <= 1e-8 * np.max(np.abs(ref))


def test_oracle_layer_escape_differs_from_single_slab():
    """The stack's escape is not the single slab's: the W backing absorbs."""
    g, tr, mus = stack()
    ly = oracle.LayerEscape(g["z_top"], g["z_bot"], mus)
    Ne = int(g["Ne"])
    seg = layer_segments(tr, 1, Ne)
    lay = oracle.brem_spectrum_layered(seg, g["brem_Z_1"], g["brem_n_1"], ly, g["n_hat"], g["brem_E_grid"],
                                       g["brem_mu_layer"], Ne)
    slab = oracle.brem_spectrum(seg, g["brem_Z_1"], g["brem_n_1"], g["thickness"], g["n_hat"], g["brem_E_grid"],
                                g["brem_mu_layer"][1], Ne)
    assert np.max(np.abs(lay - slab)) > 1e-3 * np.max(slab)


def crossing_segments(z_top, z_bot, n=64, seed=3):
    """Segments that cross 0, 1, 2 or 3 layer boundaries, some exactly ending
    on one, in both directions."""
    rng = np.random.default_rng(seed)
    T = z_bot[-1]
    z0 = rng.uniform(0.0, T, n)
    z1 = rng.uniform(0.0, T, n)
    z1[:8] = z_top[1]                      # ends on a boundary
    z1[8:12] = z0[8:12]                    # horizontal
    vx = rng.normal(size=n)
    vy = rng.normal(size=n)
    dz = z1 - z0
    lat = np.abs(dz) * rng.uniform(0.0, 2.0, n) + 1.0
    L = np.sqrt(dz * dz + lat * lat)
    v = np.stack([vx / np.hypot(vx, vy) * lat / L, vy / np.hypot(vx, vy) * lat / L, dz / L], axis=1)
    r = np.stack([np.zeros(n), np.zeros(n), 0.5 * (z0 + z1)], axis=1)
    return dict(r_mid=r, v_hat=v, L_ang=L, E_keV=rng.uniform(30.0, 9000.0, n),
                elec_id=np.arange(n, dtype=np.int64), layer=np.zeros(n, dtype=np.int32))


def test_oracle_pieces_cover_crossing_segments():
    g, _tr, mus = stack()
    ly = oracle.LayerEscape(g["z_top"], g["z_bot"], mus)
    seg = crossing_segments(g["z_top"], g["z_bot"])
    for i in range(seg["L_ang"].size):
        half = 0.5 * seg["L_ang"][i] * seg["v_hat"][i, 2]
        z = seg["r_mid"][i, 2]
        for n_z in (-0.6, 0.3):
            f, p0, p1 = ly.pieces(z - half, z + half, n_z)
            assert abs(f.sum() - 1.0) < 1e-12
            assert np.all(p0 >= 0) and np.all(p1 >= 0)
            # the path is continuous from one piece to the next
            np.testing.assert_allclose(p1[:-1], p0[1:], rtol=1e-9, atol=1e-6)


def test_api_rejects_gapped_layers():
    from pyrite_b200.api import _escape_layers

    with pytest.raises(ValueError):
        _escape_layers([(0.0, 10.0, []), (11.0, 20.0, [])])
    with pytest.raises(ValueError):
        _escape_layers([(0.0, 1.0, [])] * 5)
    z_top, z_bot = _escape_layers([(0.0, 10.0, []), (10.0, 20.0, [])])
    assert list(z_top) == [0.0, 10.0] and list(z_bot) == [10.0, 20.0]


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
def _layers_list(g):
    return [(float(a), float(b), []) for a, b in zip(g["z_top"], g["z_bot"])]


def _brem_composition(g, L):
    from pyrite_b200.tables import ELEMENTS

    by_z = {int(v[0]): el for el, v in ELEMENTS.items()}
    return [(by_z[int(z)], float(n)) for z, n in zip(g[f"brem_Z_{L}"], g[f"brem_n_{L}"])]


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("mixed", 2e-3)])
def test_layered_brem_kernel_matches_reference(precision, tol):
    import pyrite_b200 as pb

    g, tr, _mus = stack()
    Ne = int(g["Ne"])
    seg = {k: tr[k] for k in NE_FIELDS}
    seg.update(E_repr_keV=tr["E_repr_keV"], Ne=Ne, thickness_ang=float(g["thickness"]))
    for L in range(g["z_top"].size):
        s = pb.mc_brem_spectrum(seg, g["brem_E_grid"], composition=_brem_composition(g, L), n_hat=g["n_hat"],
                                layers=_layers_list(g), mu_layer=g["brem_mu_layer"], emit_layer=L,
                                precision=precision)
        ref = g[f"brem_spec_{L}"]
        assert np.max(np.abs(s - ref)) <= tol * np.max(ref), (L, np.max(np.abs(s - ref)) / np.max(ref))


def _cxr_call(g, tr, L, mus, quadrature, precision, return_pairs=False):
    import pyrite_b200 as pb
    from pyrite_b200.api import LineTables
    from pyrite_b200.tables import ReflectionRows

    Ne = int(g["Ne"])
    seg = {k: tr[k] for k in NE_FIELDS}
    seg.update(E_repr_keV=tr["E_repr_keV"], Ne=Ne, thickness_ang=float(g["thickness"]))
    rows = ReflectionRows(G=g[f"cxr_G_{L}"], ES=g[f"cxr_ES_{L}"][None], EP=g[f"cxr_EP_{L}"][None],
                          WM=g[f"cxr_WM_{L}"], row_table=g[f"cxr_row_table_{L}"])
    tables = LineTables(E_tab=g["cxr_E_tab"], chi_re=g[f"cxr_chi_re_{L}"], chi_im=g[f"cxr_chi_im_{L}"],
                        u_re=g[f"cxr_u_re_{L}"], u_im=g[f"cxr_u_im_{L}"], log_mu=g[f"cxr_log_mu_{L}"],
                        delta=g["cxr_delta"])
    return pb.mc_cxr_spectrum(seg, g["cxr_E_grid"], "silicon", None, tables=tables, n_hat=g["n_hat"], rows=rows,
                              line_quadrature=quadrature, precision=precision, layers=_layers_list(g),
                              mu_tables=mus, emit_layer=L, return_pairs=return_pairs)


@pytest.mark.gpu
@pytest.mark.parametrize("L", [0, 1])
def test_layered_cxr_kernel_matches_reference(L):
    g, tr, mus = stack()
    node = _cxr_call(g, tr, L, mus, "node", "fp64")
    ref = g[f"cxr_spec_node_{L}"]
    assert np.max(np.abs(node - ref)) <= 1e-8 * np.max(np.abs(ref))
    binm = _cxr_call(g, tr, L, mus, "bin-mean", "fp64")
    ref = g[f"cxr_spec_binmean_{L}"]
    assert np.max(np.abs(binm - ref)) <= 1e-8 * np.max(np.abs(ref))
    mixed = _cxr_call(g, tr, L, mus, "bin-mean", "mixed")
    assert np.max(np.abs(mixed - ref)) <= 1e-2 * np.max(np.abs(ref))


@pytest.mark.gpu
def test_layered_kernels_match_oracle_on_crossing_segments():
    """Segments that cross up to three boundaries (the general piece split)."""
    import pyrite_b200 as pb

    g, _tr, mus = stack()
    ly = oracle.LayerEscape(g["z_top"], g["z_bot"], mus)
    seg = crossing_segments(g["z_top"], g["z_bot"])
    n = seg["L_ang"].size
    n_hats = np.array([[0.3, 0.1, -0.95], [0.2, -0.3, 0.93]])
    n_hats /= np.linalg.norm(n_hats, axis=1, keepdims=True)
    full = dict(seg, Ne=n, thickness_ang=float(g["thickness"]))
    comp = _brem_composition(g, 2)
    s = pb.mc_brem_spectrum(full, g["brem_E_grid"], composition=comp, n_hat=n_hats, layers=_layers_list(g),
                            mu_layer=g["brem_mu_layer"], precision="fp64")
    for d in range(2):
        ref = oracle.brem_spectrum_layered(seg, g["brem_Z_2"], g["brem_n_2"], ly, n_hats[d], g["brem_E_grid"],
                                           g["brem_mu_layer"], n)
        assert np.max(np.abs(s[d] - ref)) <= 1e-11 * np.max(ref)
    # CXR: per-pair weights of the Si rows against the oracle's chain
    tables = cxr_tables(g, 1)
    E_res, aw, w, good = oracle.cxr_lines(tables, g["n_hat"], g["thickness"], seg, n, layers=ly)
    from pyrite_b200.api import LineTables
    from pyrite_b200.tables import ReflectionRows

    rows = ReflectionRows(G=g["cxr_G_1"], ES=g["cxr_ES_1"][None], EP=g["cxr_EP_1"][None], WM=g["cxr_WM_1"],
                          row_table=g["cxr_row_table_1"])
    lt = LineTables(E_tab=g["cxr_E_tab"], chi_re=g["cxr_chi_re_1"], chi_im=g["cxr_chi_im_1"], u_re=g["cxr_u_re_1"],
                    u_im=g["cxr_u_im_1"], log_mu=g["cxr_log_mu_1"], delta=g["cxr_delta"])
    _s, pairs = pb.mc_cxr_spectrum(full, g["cxr_E_grid"], "silicon", None, tables=lt, n_hat=g["n_hat"], rows=rows,
                                   line_quadrature="node", precision="fp64", layers=_layers_list(g),
                                   mu_tables=mus, return_pairs=True)
    pe, pa, pw, pg = pairs[0]
    assert np.array_equal(pg.astype(bool), good)
    np.testing.assert_allclose(pw[good], w[good], rtol=1e-9)
    torch.cuda.synchronize()


def test_stack_case_spec_builds():
    from pyrite_b200.configs import c5_stack_10mev
    from pyrite_b200.tables import HOPG, reflection_rows

    spec = c5_stack_10mev(angular_shape=(1, 1), n_bins=512, si_g_max=4.0)
    assert spec.n_hats.shape == (4, 3)
    assert spec.stack.n_layers == 3 and spec.stack.thickness == 1.22e7
    assert [r.layer for r in spec.radiators] == [0, 1]
    assert spec.brem_mu_layer.shape == (3, 512) and len(spec.escape_mu_tables) == 3
    assert [e.layer for e in spec.char_emitters] == [0, 1, 2]
    # the HOPG (002) normal sits 45 deg from the stack normal (the beam axis)
    rows = reflection_rows(HOPG, [(0, 0, 2)], spec.n_hats[:1], surface_hkl=(0, 0, 1),
                           recip_miscut_rad=spec.radiators[0].recip_miscut_rad)
    g = rows.G[0] / np.linalg.norm(rows.G[0])
    assert abs(np.degrees(np.arccos(g[2])) - 45.0) < 1e-9


def test_uniform_training_segments_cover_the_input_domain():
    """The surrogate's domain-wide training segments: energies log-uniform
    over 5-100 MeV, directions within 5 mrad of the beam, whole segments
    inside the slab, lengths from the given pool."""
    from pyrite_b200.configs import c2_si_50mev
    from pyrite_b200.surrogate import uniform_segments

    spec = c2_si_50mev(angular_shape=(1, 1))
    pool = np.array([10.0, 1.0e3, 5.0e4])
    seg = uniform_segments(spec, 4000, 7, "cpu", pool)
    E = seg["E"].numpy()
    assert E.min() >= 5e3 and E.max() <= 1e5
    assert np.mean(E < np.sqrt(5e3 * 1e5)) == pytest.approx(0.5, abs=0.05)  # log-uniform median
    v = seg["v"].numpy()
    d0 = np.asarray(spec.beam.beam_dir) / np.linalg.norm(spec.beam.beam_dir)
    ang = np.arccos(np.clip(v @ d0, -1, 1))
    assert ang.max() <= 5e-3 * np.sqrt(2) + 1e-9
    L, z = seg["L"].numpy(), seg["r"].numpy()[:, 2]
    assert set(np.unique(L)) <= set(pool)
    half = 0.5 * L * np.abs(v[:, 2])
    assert np.all(z - half >= 0) and np.all(z + half <= spec.stack.thickness)
