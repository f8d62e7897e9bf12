"""Oracle (test infrastructure): coherent (field-sum) CXR reduction in numpy, FP64.

A restatement of the reference's flat coherent reduction of per-row line
records (``pyrite/montecarlo/spectrum/cxr/_batched_finalize.py:209-243``):
for every row (one reflection x mosaic orientation) and output energy E,

    F_pol(E) = sum_j c_pol,j  F_j(E)  exp(i phi_j(E)),        pol = sigma, pi
    phi_j(E) = phase_slope_j E - g_phase_j - L_esc,j delta_omega(E)
    spec(E) += row_weight * (|F_sigma(E)|^2 + |F_pi(E)|^2)

with the complex formation factor of an absorbed line piece
(``cxr/_formation.py:84-130``): ``v = a_vac (E - E_vac) - half_dL
delta_omega(E)``, ``w2 = q^2 + v^2``, and

    Re F = (v apb sin v - q bma cos v) / (2 w2),
    Im F = -(v bma cos v + q apb sin v) / (2 w2),

or its second-order series below ``w2 < 1e-6`` (``FORMATION_SERIES_W2``).
The route divides the summed spectrum by the electron count
(``cxr/_spectrum.py:285-318``). Only tests, the smoke check and the
benchmark's CPU baseline use this; it is pinned against
``tests/golden/coherent_*.npz``, which the reference itself produced.
"""

from __future__ import annotations

import numpy as np

FIELDS = ("E_vac", "a_vac", "phase_slope", "g_phase", "cs_re", "cs_im", "cp_re", "cp_im",
          "L_esc", "half_dL", "apb", "bma", "q")
FORMATION_SERIES_W2 = 1.0e-6


def formation_factor(v, apb, bma, q):
    """Complex ``exp(-tau_c/2) sinh(w)/w``, ``w = i v - q`` (``_formation.py:84-110``)."""
    w2 = q * q + v * v
    series = w2 < FORMATION_SERIES_W2
    safe = np.where(series, 1.0, 2.0 * w2)
    sv, cv = np.sin(v), np.cos(v)
    half = 0.5 * apb
    re = np.where(series, half * (1.0 - q * q / 3.0 - v * v / 6.0), (v * apb * sv - q * bma * cv) / safe)
    im = np.where(series, -half * q * v / 3.0, -(v * bma * cv + q * apb * sv) / safe)
    return re + 1j * im


def row_field(rec, lo, hi, E, delta_omega, chunk=2048):
    """``(F_sigma(E), F_pi(E))`` of the lines ``lo:hi`` of ``rec`` (field dict)."""
    f_s = np.zeros(E.size, dtype=np.complex128)
    f_p = np.zeros(E.size, dtype=np.complex128)
    for j0 in range(lo, hi, chunk):
        sl = slice(j0, min(j0 + chunk, hi))
        phi = (rec["phase_slope"][sl, None] * E[None, :] - rec["g_phase"][sl, None]
               - rec["L_esc"][sl, None] * delta_omega[None, :])
        v = rec["a_vac"][sl, None] * (E[None, :] - rec["E_vac"][sl, None]) - rec["half_dL"][sl, None] * delta_omega[None, :]
        SP = formation_factor(v, rec["apb"][sl, None], rec["bma"][sl, None], rec["q"][sl, None]) * np.exp(1j * phi)
        f_s += (rec["cs_re"][sl] + 1j * rec["cs_im"][sl]) @ SP
        f_p += (rec["cp_re"][sl] + 1j * rec["cp_im"][sl]) @ SP
    return f_s, f_p


def coherent_spectrum(rec, row_count, row_weight, E, delta_omega, Ne=1):
    """Flat coherent reduction of every row, summed over rows, divided by ``Ne``.

    ``rec`` maps ``FIELDS`` to line arrays laid out row after row;
    ``row_count[r]`` lines belong to row ``r``, whose intensity is weighted by
    ``row_weight[r]`` (the mosaic node weight). Rows add incoherently.
    """
    E = np.asarray(E, dtype=np.float64)
    delta_omega = np.asarray(delta_omega, dtype=np.float64)
    rec = {k: np.asarray(rec[k], dtype=np.float64) for k in FIELDS}
    spec = np.zeros(E.size)
    off = np.concatenate([[0], np.cumsum(np.asarray(row_count, dtype=np.int64))])
    for r in range(len(row_count)):
        if off[r + 1] == off[r]:
            continue
        f_s, f_p = row_field(rec, int(off[r]), int(off[r + 1]), E, delta_omega)
        spec += (np.abs(f_s) ** 2 + np.abs(f_p) ** 2) * float(row_weight[r])
    return spec / Ne


def decoherence_factor(A_pop, xy0_pop, g_vec, omega):
    """Row factor F(E) = |<exp(i (omega A_e - g_perp . xy0_e))>_e|^2 over the
    sampled population, A_e = t0_e - n_perp . xy0_e (``cxr/_per_hkl.py:121-160``,
    ``cxr/_setup.py:745-760``)."""
    A_pop = np.asarray(A_pop, dtype=np.float64)
    B = np.asarray(xy0_pop, dtype=np.float64) @ np.asarray(g_vec, dtype=np.float64)[:2]
    chi = np.exp(1j * (np.asarray(omega)[None, :] * A_pop[:, None] - B[:, None])).sum(axis=0) / A_pop.size
    return chi.real ** 2 + chi.imag ** 2


def grouped_row(rec, lo, hi, elec_id, E, delta_omega):
    """sum_e (|F_sigma,e|^2 + |F_pi,e|^2): each electron's lines of the row
    summed as a field, squared, then summed over electrons
    (``cxr/_per_hkl.py:457-500``)."""
    total = np.zeros(E.size)
    eid = np.asarray(elec_id[lo:hi])
    for e in np.unique(eid):
        idx = lo + np.flatnonzero(eid == e)
        sub = {k: rec[k][idx] for k in FIELDS}
        f_s, f_p = row_field(sub, 0, idx.size, E, delta_omega)
        total += np.abs(f_s) ** 2 + np.abs(f_p) ** 2
    return total


def coherent_spectrum_decoherent(rec, elec_id, row_count, row_weight, G, A_pop, xy0_pop, E, delta_omega, omega,
                                 Ne):
    """The sampled-bunch blend per row, (1 - F) grouped + F flat, weighted and
    summed over rows, divided by ``Ne`` (``cxr/_batched_finalize.py:163-243``,
    ``spectrum/coherent_population.py:83-96`` without a physical population).
    Records are offset-free (``cxr/_setup.py:637-642``)."""
    E = np.asarray(E, dtype=np.float64)
    delta_omega = np.asarray(delta_omega, dtype=np.float64)
    rec = {k: np.asarray(rec[k], dtype=np.float64) for k in FIELDS}
    spec = np.zeros(E.size)
    off = np.concatenate([[0], np.cumsum(np.asarray(row_count, dtype=np.int64))])
    for r in range(len(row_count)):
        lo, hi = int(off[r]), int(off[r + 1])
        if hi == lo:
            continue
        F = decoherence_factor(A_pop, xy0_pop, G[r], omega)
        f_s, f_p = row_field(rec, lo, hi, E, delta_omega)
        flat = np.abs(f_s) ** 2 + np.abs(f_p) ** 2
        grouped = grouped_row(rec, lo, hi, elec_id, E, delta_omega)
        spec += ((1.0 - F) * grouped + F * flat) * float(row_weight[r])
    return spec / Ne


def rows_from_pairs(pairs, good, n_g):
    """Per-row record layout of the reference's block loop (cxr/_batched.py:640-660
    flattens g-major and keeps ``good``): row r holds its good pairs in
    segment order. ``pairs`` maps FIELDS to segment-major [n_seg*n_g] arrays.
    Returns ``(records, row_count)``."""
    good = np.asarray(good, dtype=bool).reshape(-1, n_g)
    keep_t = good.T.reshape(-1)
    rec = {k: np.asarray(pairs[k]).reshape(-1, n_g).T.reshape(-1)[keep_t] for k in FIELDS}
    return rec, good.sum(axis=0).astype(np.int64)


def load_golden(path):
    """``(records, row_count, row_weight, E, delta_omega, Ne, spec)`` of a coherent fixture."""
    z = np.load(path)
    rec = {k: z[k] for k in FIELDS}
    return rec, z["row_count"], z["row_weight"], z["E_grid"], z["delta_omega"], int(z["Ne"]), z["spec"]
