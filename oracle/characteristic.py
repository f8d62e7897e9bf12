"""Oracle (test infrastructure): characteristic-line scoring in numpy, FP64.

A restatement of the reference's CPU route of ``mc_characteristic_spectrum``
(``pyrite/montecarlo/spectrum/characteristic.py:1033-1230``) for injected
tables: shell cross sections interpolated at each segment's energy
(``_interpolate_shell_cross_sections``, ``:760-801``), the shell-to-line
response and per-layer line attenuation (``_accumulate_line_yields``,
``:837-900``), segment-mean escape transmission
(``pyrite/montecarlo/spectrum/segment_escape.py:191-330``), and exactly
bin-integrated Lorentzian profiles (``_lorentzian_bin_weights``, ``:649-680``;
edges ``_energy_bin_edges_and_widths``, ``:621-646``). Only tests, the smoke
check and the benchmark's CPU baseline use it; it is pinned against
``tests/golden/char_*.npz``, which the reference itself produced.
"""

from __future__ import annotations

import numpy as np


def bin_edges_and_widths(E_grid_eV):
    """Midpoint edges, reflected outer half-widths, low edge clamped at 0 (``:621-646``)."""
    g = np.asarray(E_grid_eV, dtype=float)
    edges = np.empty(g.size + 1)
    edges[1:-1] = 0.5 * (g[:-1] + g[1:])
    edges[0] = max(0.0, g[0] - 0.5 * (g[1] - g[0]))
    edges[-1] = g[-1] + 0.5 * (g[-1] - g[-2])
    return edges, np.diff(edges)


def lorentzian_profile(edges, line_E, fwhm):
    """Per-eV density of one line on the bins: arctan CDF differences / pi / width (``:649-680``)."""
    gamma = 0.5 * float(fwhm)
    w = (np.arctan((edges[1:] - line_E) / gamma) - np.arctan((edges[:-1] - line_E) / gamma)) / np.pi
    return np.maximum(w, 0.0) / np.diff(edges)


def shell_sigma(E_keV, shell_E, shell_sigma_cm2, offsets):
    """(rows, n_shell) masked linear interpolation of each shell table at 1e3 E (``:760-801``)."""
    q = np.asarray(E_keV, dtype=float) * 1.0e3
    cols = []
    for s in range(offsets.size - 1):
        e = shell_E[offsets[s]:offsets[s + 1]]
        v = shell_sigma_cm2[offsets[s]:offsets[s + 1]]
        inside = (q >= e[0]) & (q <= e[-1])
        cols.append(np.where(inside, np.interp(q, e, v), 0.0))
    return np.stack(cols, axis=1)


def _cut_at_zero(a, b):
    den = a - b
    f = a / np.where(den == 0.0, 1.0, den)
    return np.where((f > 0.0) & (f < 1.0), f, 1.0)


def _paths_at(z, n_z, thickness, layers):
    inv = 1.0 / max(abs(n_z), 1.0e-12)
    if layers is None:
        depth = np.clip(z, 0.0, thickness)
        return (depth * inv if n_z < 0 else (thickness - depth) * inv)[:, None]
    out = []
    for z_top, z_bot in layers:
        if n_z < 0:
            dz = np.maximum(np.minimum(z, z_bot) - z_top, 0.0)
        else:
            dz = np.maximum(z_bot - np.maximum(z, z_top), 0.0)
        out.append(dz * inv)
    return np.stack(out, axis=1)


def escape_pieces(r_mid, v_hat, L, n_hat, thickness, layers=None):
    """(owner, fraction, path_start, path_end) of every linear piece (``segment_escape.py:191-268``)."""
    r0 = r_mid - 0.5 * L[:, None] * v_hat
    r1 = r_mid + 0.5 * L[:, None] * v_hat
    n_z = float(n_hat[2])
    n = r_mid.shape[0]
    if layers is None:
        return (np.arange(n), np.ones(n), _paths_at(r0[:, 2], n_z, thickness, None),
                _paths_at(r1[:, 2], n_z, thickness, None))
    cuts = [np.zeros(n), np.ones(n)]
    for z_top, _z_bot in layers[1:]:
        cuts.append(_cut_at_zero(r0[:, 2] - z_top, r1[:, 2] - z_top))
    ordered = np.sort(np.stack(cuts, axis=1), axis=1)
    frac_all = ordered[:, 1:] - ordered[:, :-1]
    owner, part = np.nonzero(frac_all > 1.0e-12)
    fraction = frac_all[owner, part]
    dz = r1[owner, 2] - r0[owner, 2]
    left = ordered[owner, part]
    width = ordered[owner, part + 1] - left
    zq = r0[owner, 2] + (left + 0.25 * width) * dz
    z3 = r0[owner, 2] + (left + 0.75 * width) * dz
    q = _paths_at(zq, n_z, thickness, layers)
    t = _paths_at(z3, n_z, thickness, layers)
    return owner, fraction, np.maximum(1.5 * q - 0.5 * t, 0.0), np.maximum(1.5 * t - 0.5 * q, 0.0)


def mean_transmission(t0, t1):
    lo = np.minimum(t0, t1)
    d = np.abs(t1 - t0)
    safe = np.where(d > 1.0e-4, d, 1.0)
    ratio = np.where(d > 1.0e-4, -np.expm1(-safe) / safe, 1.0 - 0.5 * d + d * d / 6.0)
    return np.exp(-lo) * ratio


def line_yields(seg, n_hat, thickness, n_atoms, shell_E, shell_sigma_cm2, offsets, response, mu_by_line,
                layers=None, Ne=None):
    """Segment-summed yield of every line (``characteristic.py:837-900``)."""
    sel = np.ones(seg["L"].size, bool) if Ne is None else seg["elec_id"] < Ne
    r_mid, v_hat, L, E = seg["r_mid"][sel], seg["v_hat"][sel], seg["L"][sel], seg["E_keV"][sel]
    owner, fraction, p0, p1 = escape_pieces(r_mid, v_hat, L, n_hat, thickness, layers)
    Lp = L[owner] * fraction
    sig = shell_sigma(E[owner], shell_E, shell_sigma_cm2, offsets) @ response
    path_cm = n_atoms * 1.0e24 * (Lp * 1.0e-8)
    tr = mean_transmission(p0 @ mu_by_line, p1 @ mu_by_line)
    return np.sum(path_cm[:, None] * sig * tr, axis=0)


def spectrum(yields, profiles, Ne):
    """Photons/eV/sr/electron: sum of yield x profile, / (4 pi Ne) (``characteristic.py:1219-1230``)."""
    return (np.asarray(yields) @ np.asarray(profiles)) / (4.0 * np.pi) / int(Ne)
