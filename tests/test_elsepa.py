"""ELSEPA tabulated elastic scattering (the reference's default elastic
model, transport/scattering.py:330-640 with cores.py:425-440, 1120-1190),
pinned with synthetic tables passed through the reference's own
``elastic_tables`` argument (make_golden.py --only elsepa): the host packer
against the reference's packed group, the oracle's sampler leaves and
per-electron histories against the reference's bit for bit (CPU), and the
device's FP64 exact core replaying those histories (GPU)."""

import numpy as np
import pytest

import oracle
from conftest import golden

CASES = ("si30kev", "sio2_300kev", "c20mev")
ROW_MAP = [
    ("r_mid", "r_mid"), ("v_hat", "v_hat"), ("L_ang", "L"), ("E_keV", "E_start"),
    ("E_end_keV", "E_end"), ("t_ang", "t_start"), ("t_end_ang", "t_end"), ("elec_id", "elec_id"),
    ("layer", "layer"), ("flight_id", "flight"), ("event_kind", "event"),
]
GROUP = ("start", "length", "logE", "log_rate", "cdf", "pdf", "mu", "guide")


def raw_tables(d, t):
    """The synthetic ``elastic_tables`` a fixture was made from."""
    out = []
    for L in range(t["z_top"].size):
        layer = []
        for k in range(int(t["n_el"][L])):
            layer.append(dict(energy_eV=d[f"raw_{L}_{k}_energy_eV"], total_elastic_cm2=d[f"raw_{L}_{k}_total_elastic_cm2"],
                              mu=d["el_mu"], dcs_cm2_sr=d[f"raw_{L}_{k}_dcs_cm2_sr"]))
        out.append(layer)
    return out


def oracle_group(d):
    return oracle.ElsepaTables(*(d[f"el_{k}"] for k in GROUP))


def stack_of(t):
    from pyrite_b200.tables import LayerStack

    sym = {6: "C", 8: "O", 14: "Si", 74: "W"}
    layers = []
    for L in range(t["z_top"].size):
        n = int(t["n_el"][L])
        layers.append((float(t["z_top"][L]), float(t["z_bot"][L]),
                       [(sym[int(z)], float(x)) for z, x in zip(t["Z"][L][:n], t["N"][L][:n])]))
    return LayerStack(layers)


@pytest.mark.parametrize("case", CASES)
def test_packer_equals_the_reference_group(case):
    """``tables.pack_elsepa`` of the raw tables gives the reference's packed
    group: densities, CDFs, log rates and guide tables bit for bit."""
    from pyrite_b200.tables import pack_elsepa

    d, t = golden(f"elsepa_{case}"), golden(f"transport_{case}")
    g = pack_elsepa(stack_of(t), raw_tables(d, t))
    for k in GROUP:
        ref = d[f"el_{k}"]
        got = getattr(g, k)
        if k in ("start", "length"):
            ref = np.where(d["el_has"], ref, 0)
        np.testing.assert_array_equal(got, ref, err_msg=k)


def test_guide_window_gives_the_full_bisection_panel():
    """For every row and 4,000 seeded xi (cell edges included) the guided
    panel equals a bisection over the whole row: the oracle's sampled mu is
    the reference's, and a guide with 2 cells samples the same cosines."""
    from pyrite_b200.tables import elsepa_guide

    d = golden("elsepa_sio2_300kev")
    g = oracle_group(d)
    coarse = oracle.ElsepaTables(d["el_start"], d["el_length"], d["el_logE"], d["el_log_rate"], d["el_cdf"],
                                 d["el_pdf"], d["el_mu"], elsepa_guide(d["el_cdf"], 2))
    rng = np.random.default_rng(3)
    xs = np.concatenate([rng.uniform(0, 1, 4000), np.arange(1025) / 1024.0])
    Es = np.exp(rng.uniform(np.log(2.0), np.log(9e4), xs.size))
    for L, k in ((0, 0), (0, 1)):
        for E, xi in zip(Es[::7], xs[::7]):
            assert g.cos_theta(L, k, E, xi) == coarse.cos_theta(L, k, E, xi)


@pytest.mark.parametrize("case", CASES)
def test_oracle_sampler_leaves_equal_the_reference(case):
    """Rates and polar cosines of every element at 64 seeded (E, xi),
    table ends and a clamp below the table included: equal bit for bit."""
    d = golden(f"elsepa_{case}")
    g = oracle_group(d)
    for L in range(d["leaf_rate"].shape[0]):
        for k in range(d["leaf_rate"].shape[1]):
            if not d["el_has"][L, k]:
                continue
            for j in range(d["leaf_E"].size):
                assert g.rate(L, k, d["leaf_E"][j]) == d["leaf_rate"][L, k, j]
                assert g.cos_theta(L, k, d["leaf_E"][j], d["leaf_xi"][j]) == d["leaf_cos"][L, k, j]


@pytest.mark.parametrize("case", CASES)
def test_oracle_elsepa_transport_replays_the_reference(case):
    """The oracle's exact per-electron core with ELSEPA tables replays the
    reference's own ELSEPA histories (SplitMix64, same entrance states) bit
    for bit, and ELSEPA changes the histories against the analytic model."""
    d, t = golden(f"elsepa_{case}"), golden(f"transport_{case}")
    lt = oracle.LayerTables(t["z_top"], t["z_bot"], t["n_el"], t["Z"], t["J"], t["N"], t["E_cross"])
    lt.use_elsepa(oracle_group(d))
    out = oracle.transport(lt, d["initial_r"], d["initial_v"], d["initial_E"], seed=int(d["seed"]),
                           E_cut=float(d["E_cut_keV"]), cap=4096)
    for ref_key, got_key in ROW_MAP:
        np.testing.assert_array_equal(out[got_key], d[ref_key], err_msg=ref_key)
    assert d["L_ang"].size != t["L_ang"].size or not np.array_equal(d["L_ang"], t["L_ang"])


def test_api_refuses_what_the_reference_refuses():
    """No tables, an energy outside the tables, a foreign mu grid -- all
    refused on the host before any device work."""
    from pyrite_b200 import simulate_trajectories
    from pyrite_b200.tables import LayerStack, pack_elsepa

    d, t = golden("elsepa_si30kev"), golden("transport_si30kev")
    slab = [(0.0, 5e4, [("Si", 0.04996)])]
    with pytest.raises(ValueError, match="needs elastic_tables"):
        simulate_trajectories(30.0, 4, layers=slab, elastic_model="elsepa")
    raw = raw_tables(d, t)
    with pytest.raises(ValueError, match="within the ELSEPA table"):
        simulate_trajectories(2.0e5, 4, layers=slab, elastic_model="elsepa", elastic_tables=raw)
    with pytest.raises(ValueError, match="elastic_model must be"):
        simulate_trajectories(30.0, 4, layers=slab, elastic_model="mott")
    other = dict(raw[0][0], mu=raw[0][0]["mu"] * 0.5)
    with pytest.raises(ValueError, match="one mu grid"):
        pack_elsepa(LayerStack([(0.0, 5e4, [("Si", 0.02), ("O", 0.04)])]), [[raw[0][0], other]])


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_gpu_elsepa_fp64_replays_reference(case, cuda_device):
    """The device's FP64 exact core with the reference's packed ELSEPA
    tables and SplitMix64 streams: every history has the reference's rows
    within 1e-10 (the first rows of all of them), as the analytic core."""
    from pyrite_b200 import simulate_trajectories
    from pyrite_b200.tables import ElsepaGroup
    from test_gpu_transport import history_agreement, layers_of

    d, t = golden(f"elsepa_{case}"), golden(f"transport_{case}")
    group = ElsepaGroup(*(d[f"el_{k}"] for k in GROUP))
    got = simulate_trajectories(float(d["E0_keV"]), int(d["Ne"]), layers=layers_of(t), E_cut_keV=float(d["E_cut_keV"]),
                                seed=int(d["seed"]), device=cuda_device, elastic_model="elsepa",
                                elastic_tables=group, entry=(d["initial_r"], d["initial_v"], d["initial_E"]))
    assert got["device_status"] == 0
    frac, first = history_agreement(d, got)
    assert first
    assert frac == 1.0, frac
    assert got["L_ang"].size == d["L_ang"].size


@pytest.mark.gpu
def test_gpu_elsepa_mixed_and_philox_statistics(cuda_device):
    """Mixed precision with Philox and the same tables: exit fates within
    binomial scatter of the FP64 run, mean rows per history within 5 %."""
    from pyrite_b200 import simulate_trajectories
    from pyrite_b200.tables import ElsepaGroup
    from test_gpu_transport import layers_of

    d, t = golden("elsepa_si30kev"), golden("transport_si30kev")
    group = ElsepaGroup(*(d[f"el_{k}"] for k in GROUP))
    kw = dict(E0_keV=30.0, Ne=4000, layers=layers_of(t), E_cut_keV=5.0, seed=9, rng="philox",
              device=cuda_device, elastic_model="elsepa", elastic_tables=group, tallies=(16, 16))
    a = simulate_trajectories(precision="fp64", **kw)
    b = simulate_trajectories(precision="mixed", **kw)
    for r in (a, b):
        assert r["device_status"] == 0
    fa, fb = a["tally_fates"].astype(float), b["tally_fates"].astype(float)
    n = fa.sum()
    p = (fa + fb) / (2 * n)
    assert np.all(np.abs(fa - fb) <= 5.0 * np.sqrt(2 * n * p * (1 - p)) + 2), (fa, fb)
    assert abs(a["seg_count"].mean() / b["seg_count"].mean() - 1.0) < 0.05
