"""Urban energy-loss straggling (the reference's transport/straggling.py),
on the CPU: the oracle's restatement against the reference's own sampler
outputs and its straggled per-electron histories (make_golden.py --only
straggling), bit for bit, and the model's closure identity <dE> = C s."""

import numpy as np
import pytest

import oracle
from conftest import golden

ROW_MAP = [
    ("r_mid", "r_mid"), ("v_hat", "v_hat"), ("L_ang", "L"), ("E_keV", "E_start"),
    ("E_end_keV", "E_end"), ("t_ang", "t_start"), ("t_end_ang", "t_end"), ("elec_id", "elec_id"),
    ("layer", "layer"), ("flight_id", "flight"), ("event_kind", "event"),
]
CASES = ("c20mev", "si30kev", "sio2_300kev")


def test_urban_sampler_leaves_equal_the_reference():
    """Per element: the spliced stopping C, one sampled loss with its draw
    counter, and the analytic mean and variance, on 96 seeded (element,
    energy, path, key) points from 0.5 keV to 50 MeV -- equal bit for bit."""
    d = golden("straggling_leaves")
    for i in range(d["Z"].size):
        C = -oracle.dEds_element(d["J"][i], d["k"][i], d["coeff"][i], d["E_cross"][i], d["E"][i])
        assert C == d["C"][i]
        dE, ctr = oracle.urban_sample_element(d["Z"][i], d["J"][i], C, d["E"][i], d["s"][i], int(d["key"][i]))
        assert dE == d["dE"][i] and ctr == int(d["counter"][i]), i
        m, v = oracle.urban_moments_element(d["Z"][i], d["J"][i], C, d["E"][i], d["s"][i])
        assert m == d["mean"][i] and v == d["var"][i]


def test_urban_closure_mean_is_the_stopping_power():
    """The model's defining identity: mean loss = C s for every element,
    energy and path (straggling.py:93-101), to FP64 rounding."""
    d = golden("straggling_leaves")
    for i in range(d["Z"].size):
        m, _ = oracle.urban_moments_element(d["Z"][i], d["J"][i], d["C"][i], d["E"][i], d["s"][i])
        assert m == pytest.approx(d["C"][i] * d["s"][i], rel=1e-12)


def test_urban_sampled_mean_and_variance():
    """4,000 seeded draws of a 10 um flight of a 300 keV electron in Si: the
    sample mean and variance within 4 standard errors of the analytic ones."""
    Z, J, k, N = 14.0, 0.173, 0.731 + 0.0688 * np.log10(14.0), 0.04994
    coeff = N / 0.602214076 * Z
    E, s = 300.0, 1.0e5
    C = -oracle.dEds_element(J, k, coeff, 1.0e9, E)
    m, v = oracle.urban_moments_element(Z, J, C, E, s)
    x = np.array([oracle.urban_sample_element(Z, J, C, E, s, 1000 + i)[0] for i in range(4000)])
    assert abs(x.mean() - m) < 4.0 * np.sqrt(v / x.size)
    assert abs(x.var() - v) < 4.0 * v * np.sqrt(2.0 / x.size) * 3.0  # heavy-tailed: loose


@pytest.mark.parametrize("case", CASES)
def test_oracle_straggled_transport_replays_the_reference(case):
    """The oracle's exact core with straggling replays the reference's own
    straggled per-electron histories (SplitMix64, same entrance states) bit
    for bit."""
    d = golden(f"straggling_{case}")
    t = golden(f"transport_{case}")
    lt = oracle.LayerTables(t["z_top"], t["z_bot"], t["n_el"], t["Z"], t["J"], t["N"], t["E_cross"])
    out = oracle.transport(lt, d["initial_r"], d["initial_v"], d["initial_E"], seed=int(d["seed"]),
                           E_cut=float(d["E_cut_keV"]), straggling=True, cap=4096)
    for ref_key, got_key in ROW_MAP:
        np.testing.assert_array_equal(out[got_key], d[ref_key], err_msg=ref_key)
    # straggling changes the histories (not the plain core's rows)
    assert not np.array_equal(d["E_end_keV"][:50], t["E_end_keV"][:50])
