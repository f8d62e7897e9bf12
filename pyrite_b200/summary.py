"""The device tallies as the reference's tidy summary tables.

The reference reduces a trajectory capture to fixed-bin tables
(``montecarlo/trajectory_summary.py:180-260``: ``exit_energy`` and
``exit_angle`` with explicit underflow and overflow rows, ``fates`` with
counts and fractions of the sampled primaries, ``depth_loss`` per layer and
depth bin). The transport kernel accumulates the same quantities on the
device while it runs (``pb_tallies``), without writing the trajectory rows;
``tally_tables`` lays them out in the reference's columns so code that reads
those tables reads these. The depth-loss table has one depth bin per layer
(the layer's bounds), the resolution the device tally keeps.
"""

from __future__ import annotations

import numpy as np

# exit codes of the transport (transport/cores.py:88-93) -> the reference's fate names
FATE_NAMES = {0: "cutoff_stopped", 1: "backscattered", 2: "transmitted", 3: "side_exited",
              4: "unfinished", 5: "missed"}


def _hist_frame(counts, edges, unit):
    import pandas as pd

    edges = np.asarray(edges, dtype=float)
    counts = np.asarray(counts, dtype=np.int64)
    if counts.size != edges.size + 1:
        raise ValueError("a histogram with under/overflow has len(edges) + 1 counts")
    return pd.DataFrame({
        f"low_{unit}": np.r_[-np.inf, edges[:-1], edges[-1]],
        f"high_{unit}": np.r_[edges[0], edges[1:], np.inf],
        "count": counts,
    })


def tally_tables(fates, exit_E, exit_theta, deposit_keV, *, E_lo, E_hi, theta_lo, theta_hi, z_top, z_bot):
    """Tidy tables of one run's device tallies.

    ``fates`` counts per exit code (6), ``exit_E`` / ``exit_theta`` the
    escaped primaries' histograms with an underflow slot first and an
    overflow slot last (n + 2), ``deposit_keV`` the energy lost per layer
    (total over the run), ``z_top`` / ``z_bot`` the layer bounds [Angstrom].
    """
    import pandas as pd

    fates = np.asarray(fates, dtype=np.int64)
    total = int(fates.sum())
    fate_rows = [(FATE_NAMES[c], int(fates[c]), (int(fates[c]) / total) if total else 0.0)
                 for c in (1, 2, 3, 0, 4, 5)]
    exit_E = np.asarray(exit_E, dtype=np.int64)
    exit_theta = np.asarray(exit_theta, dtype=np.int64)
    e_edges = np.linspace(float(E_lo), float(E_hi), exit_E.size - 1)
    a_edges = np.linspace(float(theta_lo), float(theta_hi), exit_theta.size - 1)
    z_top = np.atleast_1d(np.asarray(z_top, dtype=float))
    z_bot = np.atleast_1d(np.asarray(z_bot, dtype=float))
    dep = np.atleast_1d(np.asarray(deposit_keV, dtype=float))
    return {
        "exit_energy": _hist_frame(exit_E, e_edges, "keV"),
        "exit_angle": _hist_frame(exit_theta, a_edges, "rad"),
        "fates": pd.DataFrame(fate_rows, columns=["fate", "count", "fraction"]),
        "depth_loss": pd.DataFrame({"layer": np.arange(dep.size), "depth_low_ang": z_top[:dep.size],
                                    "depth_high_ang": z_bot[:dep.size], "continuous_loss_keV": dep}),
    }


def case_tally_tables(case):
    """``tally_tables`` of a ``pipeline.ScoringCase`` (totals over its batches)."""
    t = case.targs.tallies
    st = case.spec.stack
    return tally_tables(case.fates.cpu().numpy(), case.exit_E.cpu().numpy(), case.exit_theta.cpu().numpy(),
                        case.deposit.cpu().numpy(), E_lo=t.E_lo, E_hi=t.E_hi, theta_lo=t.theta_lo,
                        theta_hi=t.theta_hi, z_top=[l[0] for l in st.layers], z_bot=[l[1] for l in st.layers])
