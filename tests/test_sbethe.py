"""SBETHE table stopping (transport/stopping.py:11-103, cores.py:581-604 and
720-780), pinned with synthetic per-layer tables passed through the
reference's own ``stopping_tables`` argument (make_golden.py --only sbethe):
the host packer against the reference's packed tables, the oracle's
interpolation and per-electron histories (plain and straggled) against the
reference's bit for bit (CPU), and the device's FP64 exact core replaying
those histories (GPU)."""

import numpy as np
import pytest

import oracle
from conftest import golden

CASES = ("si30kev", "sio2_300kev", "c20mev", "sio2_300kev_straggled")
ROW_MAP = [
    ("r_mid", "r_mid"), ("v_hat", "v_hat"), ("L_ang", "L"), ("E_keV", "E_start"),
    ("E_end_keV", "E_end"), ("t_ang", "t_start"), ("t_end_ang", "t_end"), ("elec_id", "elec_id"),
    ("layer", "layer"), ("flight_id", "flight"), ("event_kind", "event"),
]


def _pair(case):
    return golden(f"sbethe_{case}"), golden(f"transport_{case.replace('_straggled', '')}")


def _raw(d, n_layers):
    return [dict(stopping_energy_eV=d[f"raw_{L}_stopping_energy_eV"],
                 stopping_eV_per_angstrom=d[f"raw_{L}_stopping_eV_per_angstrom"]) for L in range(n_layers)]


def _oracle_layers(d, t):
    lt = oracle.LayerTables(t["z_top"], t["z_bot"], t["n_el"], t["Z"], t["J"], t["N"], t["E_cross"])
    return lt.use_sbethe(d["sb_count"], d["sb_logE"], d["sb_logS"])


@pytest.mark.parametrize("case", CASES)
def test_packer_equals_the_reference_tables(case):
    from test_elsepa import stack_of

    from pyrite_b200.tables import pack_stopping

    d, t = _pair(case)
    g = pack_stopping(stack_of(t), _raw(d, t["z_top"].size))
    np.testing.assert_array_equal(g.count, d["sb_count"])
    np.testing.assert_array_equal(g.logE, d["sb_logE"])
    np.testing.assert_array_equal(g.logS, d["sb_logS"])


@pytest.mark.parametrize("case", CASES)
def test_oracle_stopping_and_histories_equal_the_reference(case):
    """The interpolated stopping on 97 energies from below the table's first
    node to 2 GeV (both clamps), and the per-electron histories -- with
    straggling, whose Urban means the table rescales -- bit for bit."""
    d, t = _pair(case)
    lt = _oracle_layers(d, t)
    for L in range(d["leaf_S"].shape[0]):
        for j, E in enumerate(d["leaf_E"]):
            assert lt.sbethe_dEds(L, E) == d["leaf_S"][L, j]
    out = oracle.transport(lt, d["initial_r"], d["initial_v"], d["initial_E"], seed=int(d["seed"]),
                           E_cut=float(d["E_cut_keV"]), straggling=bool(d["straggling"]), cap=4096)
    for ref_key, got_key in ROW_MAP:
        np.testing.assert_array_equal(out[got_key], d[ref_key], err_msg=ref_key)


def test_api_refuses_out_of_range_and_malformed_tables():
    from pyrite_b200 import simulate_trajectories
    from pyrite_b200.tables import LayerStack, pack_stopping

    d, t = _pair("si30kev")
    slab = [(0.0, 5e4, [("Si", 0.04996)])]
    raw = _raw(d, 1)
    with pytest.raises(ValueError, match="within the SBETHE table"):
        simulate_trajectories(30.0, 4, layers=slab, E_cut_keV=0.5, stopping_tables=raw)
    with pytest.raises(ValueError, match="one SBETHE table per layer"):
        pack_stopping(LayerStack(slab), raw + raw)
    bad = dict(raw[0], stopping_eV_per_angstrom=-raw[0]["stopping_eV_per_angstrom"])
    with pytest.raises(ValueError, match="strictly positive"):
        pack_stopping(LayerStack(slab), [bad])


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_gpu_sbethe_fp64_replays_reference(case, cuda_device):
    """The device's FP64 exact core with the reference's packed SBETHE tables
    and SplitMix64 streams: every first row, and every history row for row
    within 1e-10 (straggled: at least 90 %, as the Urban replay)."""
    from test_gpu_transport import history_agreement, layers_of

    from pyrite_b200 import simulate_trajectories
    from pyrite_b200.tables import StoppingTables

    d, t = _pair(case)
    stop = StoppingTables(d["sb_count"], d["sb_logE"], d["sb_logS"])
    got = simulate_trajectories(float(d["E0_keV"]), int(d["Ne"]), layers=layers_of(t),
                                E_cut_keV=float(d["E_cut_keV"]), seed=int(d["seed"]), device=cuda_device,
                                stopping_tables=stop, straggling=bool(d["straggling"]),
                                entry=(d["initial_r"], d["initial_v"], d["initial_E"]))
    assert got["device_status"] == 0
    frac, first = history_agreement(d, got)
    assert first
    assert frac >= (0.9 if d["straggling"] else 1.0), frac


@pytest.mark.gpu
def test_gpu_sbethe_with_elsepa_and_mixed(cuda_device):
    """Both tables at once on the mixed Philox core: the mean rows per history
    and the fates agree with the FP64 core statistically."""
    from test_elsepa import GROUP
    from test_gpu_transport import layers_of

    from pyrite_b200 import simulate_trajectories
    from pyrite_b200.tables import ElsepaGroup, StoppingTables

    d, t = _pair("si30kev")
    e = golden("elsepa_si30kev")
    kw = dict(E0_keV=30.0, Ne=4000, layers=layers_of(t), E_cut_keV=5.0, seed=19, rng="philox", device=cuda_device,
              elastic_model="elsepa", elastic_tables=ElsepaGroup(*(e[f"el_{k}"] for k in GROUP)),
              stopping_tables=StoppingTables(d["sb_count"], d["sb_logE"], d["sb_logS"]), tallies=(16, 16))
    a = simulate_trajectories(precision="fp64", **kw)
    b = simulate_trajectories(precision="mixed", **kw)
    assert a["device_status"] == 0 and b["device_status"] == 0
    fa, fb = a["tally_fates"].astype(float), b["tally_fates"].astype(float)
    p = (fa + fb) / (2 * fa.sum())
    assert np.all(np.abs(fa - fb) <= 5.0 * np.sqrt(2 * fa.sum() * p * (1 - p)) + 2), (fa, fb)
    assert abs(a["seg_count"].mean() / b["seg_count"].mean() - 1.0) < 0.05
