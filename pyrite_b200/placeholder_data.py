"""Stand-in atomic data for the CXR and bremsstrahlung tables.

The reference reads Waasmaier-Kirfel f0 and Chantler f'/f'' through xraydb
(src/pyrite/materials/atomic.py:1-20) and EPDL attenuation
(materials/photon_cross_sections.py:74). Neither dataset ships with this
package, so the tables that the hot path consumes are produced here from
smooth placeholder form factors with the right structure and magnitude:

* f0(s) = Z (0.6 exp(-b s^2) + 0.4 exp(-b s^2 / 4)), b = 8 / (1 + 0.05 Z),
  s = g / (4 pi) [1/Angstrom];
* f'(E) = -0.02 Z 1000/(E + 1000);  f''(E) = 0.5 Z (Z/30) (1000/(E + 200))^2;
* mu_el(E) = 2 r_e lambda n_el f''(E) (optical theorem).

The formulas that turn form factors into couplings are the reference's:
chi_g = -r_e lambda^2 S(g) / (pi V) with Debye-Waller exp(-B s^2)
(materials/crystal.py:302-431), U_g/m = 4 pi e^2 sum (Z - f0) e^{i g.R} e^{-W}
/ (g^2 V m c^2) (crystal.py:547-603), both in the emission convention
conj(chi(-hkl)), U(hkl) (crystal.py:730-761), and delta = 1 - Re sqrt(1 + chi_0)
(crystal.py:432-510). Spectra computed from these tables are therefore
non-physical in absolute value; the arithmetic on the hot path is unchanged
when real tables are supplied through ``api.LineTables``.
"""

from __future__ import annotations

import numpy as np

from .api import LineTables
from .tables import ELEMENTS, Crystal, line_keep_window

R_E_ANG = 2.8179403e-5
HC_EV_ANG = 12398.4198
E2_EV_ANG = 14.399645
M_E_EV = 510998.95


def f0(element: str, s):
    z = ELEMENTS[element][0]
    s = np.asarray(s, dtype=float)
    b = 8.0 / (1.0 + 0.05 * z)
    return z * (0.6 * np.exp(-b * s * s) + 0.4 * np.exp(-0.25 * b * s * s))


def f1(element: str, E):
    z = ELEMENTS[element][0]
    return -0.02 * z * (1.0e3 / (np.asarray(E, dtype=float) + 1.0e3))


def f2(element: str, E):
    z = ELEMENTS[element][0]
    return 0.5 * z * (z / 30.0) * (1.0e3 / (np.asarray(E, dtype=float) + 2.0e2)) ** 2


def tabulation_grid(E_grid, n=700):
    """Geometric tabulation mesh over the line keep window, floored at 1 eV."""
    lo, hi = line_keep_window(E_grid)
    return np.geomspace(max(lo, 1.0), hi, n)


def line_tables(crystal: Crystal, hkl_list, E_grid, absorber=None, n_tab=700) -> LineTables:
    """Coupling, attenuation and refraction tables on the tabulation mesh."""
    E = tabulation_grid(E_grid, n_tab)
    lam = HC_EV_ANG / E
    V = crystal.volume
    chi_scale = -R_E_ANG * lam**2 / (np.pi * V)
    u_scale = 4.0 * np.pi * E2_EV_ANG / V / M_E_EV
    n_hkl = len(hkl_list)
    chi_re = np.empty((n_hkl, E.size))
    chi_im = np.empty((n_hkl, E.size))
    u_re = np.empty((n_hkl, E.size))
    u_im = np.empty((n_hkl, E.size))
    for i, hkl in enumerate(hkl_list):
        _, g = crystal.g_vector(hkl)
        s = g / (4.0 * np.pi)
        dwf = np.exp(-crystal.B_ang2 * s * s)
        S = np.zeros(E.size, dtype=complex)
        a = 0.0 + 0.0j
        for el, R in crystal.basis:
            # emission convention: conj(chi(-hkl)) = chi(hkl) with f'' negated
            ph = np.exp(1j * 2.0 * np.pi * np.dot(hkl, R))
            S += (f0(el, s) + f1(el, E) - 1j * f2(el, E)) * ph
            a += (ELEMENTS[el][0] - f0(el, s)) * ph
        chi = chi_scale * S * dwf
        chi_re[i], chi_im[i] = chi.real, chi.imag
        u = u_scale * a * dwf / (g * g)
        u_re[i], u_im[i] = u.real, u.imag
    S0 = np.zeros(E.size, dtype=complex)
    for el, _R in crystal.basis:
        S0 += ELEMENTS[el][0] + f1(el, E) + 1j * f2(el, E)
    chi0 = -R_E_ANG * lam**2 / (np.pi * V) * S0
    delta = 1.0 - np.sqrt(1.0 + chi0).real
    comp = absorber if absorber is not None else _crystal_composition(crystal)
    log_mu = np.stack([np.log(mu_element(el, n, E)) for el, n in comp], axis=0)
    return LineTables(E, chi_re, chi_im, u_re, u_im, log_mu, delta)


def _crystal_composition(crystal: Crystal):
    counts = {}
    for el, _ in crystal.basis:
        counts[el] = counts.get(el, 0) + 1
    return [(el, c / crystal.volume) for el, c in counts.items()]


def mu_element(element: str, n_per_ang3: float, E):
    """Placeholder photo-absorption coefficient [1/Angstrom]."""
    lam = HC_EV_ANG / np.asarray(E, dtype=float)
    return 2.0 * R_E_ANG * lam * n_per_ang3 * f2(element, E)


def mu_total(composition, E):
    return sum(mu_element(el, n, E) for el, n in composition)


def exact_mu_table(composition, knots=None):
    """mu(E) of a composition as the piecewise-linear (knots, values, slopes)
    tables of the layered escape (cxr/_escape_mu.py:41-57), on a geometric
    knot set."""
    kn = np.geomspace(200.0, 3.0e5, 600) if knots is None else np.asarray(knots, dtype=float)
    val = mu_total(composition, kn)
    slope = np.empty_like(val)
    slope[:-1] = np.diff(val) / np.diff(kn)
    slope[-1] = slope[-2]
    return kn, val, slope


# Edge and line energies [eV] (standard X-ray data) with placeholder widths;
# ionisation cross sections and cascade responses are smooth stand-ins for the
# EEDL/EADL-derived tables the reference reads (characteristic.py:111-160).
_CHAR_DATA = {
    "C": dict(shells=[284.2], lines=[(277.0, 0.5)], resp=[[0.0026]]),
    "Si": dict(shells=[1839.0, 149.7], lines=[(1739.98, 0.5), (1835.94, 0.6)],
               resp=[[0.045, 0.002], [0.0, 0.0]]),
    "W": dict(
        shells=[69525.0, 12100.0, 11544.0, 10207.0],
        lines=[(59318.2, 43.0), (57981.7, 44.0), (67244.3, 45.0), (8397.6, 6.5), (9672.4, 7.0),
               (9961.5, 7.5), (11285.9, 9.0)],
        resp=[[0.52, 0.30, 0.12, 0.11, 0.04, 0.02, 0.0],
              [0.0, 0.0, 0.0, 0.05, 0.02, 0.01, 0.08],
              [0.0, 0.0, 0.0, 0.0, 0.21, 0.0, 0.06],
              [0.0, 0.0, 0.0, 0.22, 0.0, 0.05, 0.0]],
    ),
}


def characteristic_lines(element: str):
    """Placeholder ``CharacteristicLines`` of C, Si or W (K and L lines)."""
    from .api import CharacteristicLines

    d = _CHAR_DATA[element]
    Z = ELEMENTS[element][0]
    grids, sigmas = [], []
    for i, Eb in enumerate(d["shells"]):
        E = np.geomspace(Eb, 1.0e9, 80)
        u = E / Eb
        sig = 2.0e-20 * (Eb / 1000.0) ** -2 * (1.0 + 0.5 * i) * np.log(u) / (u + 1.0) * (Z / 14.0) ** 0.2
        sig[0] = 0.0
        grids.append(E)
        sigmas.append(sig)
    return CharacteristicLines(
        shell_E=tuple(grids), shell_sigma=tuple(sigmas),
        line_E=np.array([e for e, _ in d["lines"]]), line_fwhm=np.array([w for _, w in d["lines"]]),
        response=np.array(d["resp"], dtype=float), recommended_cutoff_eV=50.0,
    )
