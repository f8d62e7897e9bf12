"""The CPU oracle against golden vectors produced by the reference itself.

Transport rows (exact and LUT cores) must be bit-identical; the CXR chain,
its reductions and Bethe-Heitler agree to FP64 rounding. The fixtures and the
script that made them live in tests/golden/.
"""

import numpy as np
import pytest

import oracle
from conftest import CXR_CASES, LUT_CASES, TRANSPORT_CASES, golden

ROW_MAP = [
    ("r_mid", "r_mid"), ("v_hat", "v_hat"), ("L_ang", "L"), ("E_keV", "E_start"),
    ("E_end_keV", "E_end"), ("t_ang", "t_start"), ("t_end_ang", "t_end"), ("elec_id", "elec_id"),
    ("layer", "layer"), ("flight_id", "flight"), ("event_kind", "event"),
]


def exact_layers(d):
    return oracle.LayerTables(d["z_top"], d["z_bot"], d["n_el"], d["Z"], d["J"], d["N"], d["E_cross"])


def test_splitmix64_known_answers():
    d = golden("rng")
    for x, y in zip(d["splitmix_in"], d["splitmix_out"]):
        assert oracle.splitmix64(int(x)) == int(y)


def test_stream_keys_and_uniforms():
    d = golden("rng")
    assert [oracle.stream_key(7, e) for e in range(64)] == [int(k) for k in d["stream_keys_seed7"]]
    assert [oracle.stream_key(7, 100 + e) for e in range(16)] == [
        int(k) for k in d["stream_keys_seed7_start100"]
    ]
    for elec, c, key, u in zip(d["uniform_elec"], d["uniform_counter"], d["uniform_key"], d["uniform_value"]):
        assert oracle.stream_key(3, int(elec)) == int(key)
        assert oracle.stream_uniform(int(key), int(c)) == float(u)


def test_philox_published_zero_vector():
    d = golden("rng")
    assert oracle.philox4x32_10([0, 0, 0, 0], [0, 0]) == [int(w) for w in d["philox_zero_words"]]
    w = [int(x) for x in d["philox_zero_words"]]
    expected = [((w[i] >> 5) * 2**26 + (w[i + 1] >> 6)) / 2**53 for i in (0, 2)]
    assert [oracle.philox_uniform(0, 0), oracle.philox_uniform(0, 1)] == expected


def test_physics_leaves():
    d = golden("physics_leaves")
    for name in ("C", "Si", "W", "SiO2"):
        n = d[f"{name}_Z"].size
        lt = oracle.LayerTables([0.0], [1.0], [n], d[f"{name}_Z"][None], d[f"{name}_J"][None],
                                d[f"{name}_n"][None], d[f"{name}_E_cross"][None])
        got = np.array([lt.dEds(0, e) for e in d["E_keV"]])
        np.testing.assert_array_equal(got, d[f"{name}_dEds"])


@pytest.mark.parametrize("case", TRANSPORT_CASES)
def test_exact_core_bitwise(case):
    d = golden(f"transport_{case}")
    out = oracle.transport(exact_layers(d), d["initial_r"], d["initial_v"], d["initial_E"],
                           seed=int(d["seed"]), E_cut=float(d["E_cut_keV"]))
    for ref_key, key in ROW_MAP:
        np.testing.assert_array_equal(out[key], d[ref_key], err_msg=f"{case}:{ref_key}")
    counts = [int(np.sum(out["exit_code"] == c)) for c in (1, 2, 3, 0, 4)]
    assert counts == [int(v) for v in d["counts"][:5]]


@pytest.mark.parametrize("case", LUT_CASES)
def test_lut_core_bitwise(case):
    d = golden(f"transport_lut_{case}")
    g = golden(f"transport_{case}")
    lt = oracle.LutTables(g["z_top"], g["z_bot"], d["lut_n_el"], d["log_E_min"], d["inv_dlogE"],
                          d["lut_total_rate"], d["lut_dEds"], d["lut_inv_beta"], d["lut_cdf"], d["lut_alpha"])
    out = oracle.transport(lt, d["initial_r"], d["initial_v"], d["initial_E"], seed=int(g["seed"]),
                           E_cut=float(g["E_cut_keV"]))
    for ref_key, key in ROW_MAP:
        np.testing.assert_array_equal(out[key], d[ref_key], err_msg=f"{case}:{ref_key}")


def cxr_inputs(name):
    d = golden(f"cxr_{name}")
    tr = golden(f"transport_{d['transport']}")
    seg = dict(v_hat=tr["v_hat"], E_keV=tr["E_repr_keV"], L_ang=tr["L_ang"], r_mid=tr["r_mid"],
               elec_id=tr["elec_id"])
    E_grid = d["E_grid"]
    pad = 0.2 * (E_grid[-1] - E_grid[0])
    tables = {k: d[k] for k in ("G", "ES", "EP", "WM", "row_table", "E_tab", "chi_re", "chi_im",
                                "u_re", "u_im", "log_mu", "delta")}
    tables["lo_keep"] = E_grid[0] - pad
    tables["hi_keep"] = E_grid[-1] + pad
    return d, seg, tables


@pytest.mark.parametrize("case", CXR_CASES)
def test_cxr_chain_node_and_binmean(case):
    d, seg, tables = cxr_inputs(case)
    Ne = int(d["Ne"])
    E_res, aw, w, good = oracle.cxr_lines(tables, d["n_hat"], d["thickness"], seg, Ne)
    assert good.any()
    node = oracle.reduce_node(E_res[good], aw[good], w[good], d["E_grid"]) / Ne
    peak = np.max(np.abs(d["spec_node"]))
    assert np.max(np.abs(node - d["spec_node"])) <= 1e-9 * peak
    edges = oracle.energy_bin_edges(d["E_grid"])
    binm = oracle.reduce_binmean(E_res[good], aw[good], w[good], edges) / Ne
    peak = np.max(np.abs(d["spec_binmean"]))
    # The reference's own bin-mean route is a Fourier evaluation accurate to ~1e-10.
    assert np.max(np.abs(binm - d["spec_binmean"])) <= 1e-8 * peak


@pytest.mark.parametrize("case", ["c20", "sio2"])
def test_brem_bethe_heitler(case):
    d = golden(f"brem_{case}")
    tr = golden(f"transport_{d['transport']}")
    seg = dict(v_hat=tr["v_hat"], E_keV=tr["E_repr_keV"], L_ang=tr["L_ang"], r_mid=tr["r_mid"],
               elec_id=tr["elec_id"])
    s = oracle.brem_spectrum(seg, d["Z"], d["n_ang3"], d["thickness"], d["n_hat"], d["E_grid"],
                             d["mu_grid"], int(d["Ne"]))
    np.testing.assert_allclose(s, d["spec"], rtol=1e-12, atol=1e-14 * np.max(d["spec"]))


def test_cxr_leaves():
    d = golden("cxr_leaves")
    keys = ["h", "gamma", "vdg", "k_dot_v", "k_dot_g", "g2", "k2", "v_dot_e", "g_dot_e", "k_dot_e"]
    for i in range(d["qlf_h"].size):
        p, c = oracle.quantum_line_factors(*[d["qlf_" + k][i] for k in keys])
        assert p == d["qlf_pxr"][i] and c == d["qlf_cbs"][i]
    np.testing.assert_allclose(oracle.sincsq_tail(d["tail_x"]), d["tail"], rtol=0, atol=1e-15)
    edges = d["bm_edges"]
    for a, e, ref in zip(d["bm_a"], d["bm_E"], d["bm_mass"]):
        m = oracle.reduce_binmean([e], [a], [1.0], edges) * np.diff(edges)
        np.testing.assert_allclose(m, ref, rtol=0, atol=1e-14 * np.max(d["bm_mass"]))
    mt = [oracle.mean_transmission(a, b) for a, b in zip(d["mt_t0"], d["mt_t1"])]
    np.testing.assert_allclose(mt, d["mt"], rtol=1e-15, atol=0)


def test_philox_oracle_transport_is_deterministic_and_differs_from_splitmix():
    d = golden("transport_c20mev")
    lt = exact_layers(d)
    a = oracle.transport(lt, d["initial_r"], d["initial_v"], d["initial_E"], seed=0, E_cut=5.0,
                         rng=oracle.RNG_PHILOX)
    b = oracle.transport(lt, d["initial_r"], d["initial_v"], d["initial_E"], seed=0, E_cut=5.0,
                         rng=oracle.RNG_PHILOX)
    np.testing.assert_array_equal(a["L"], b["L"])
    assert not np.array_equal(a["L"][:10], d["L_ang"][:10])
