"""Placeholder ``xraydb`` for importing the reference in a container without it.

Test infrastructure only. The real package (pinned 4.6.1 by the reference's
lock file) ships tabulated Waasmaier-Kirfel f0 and Chantler f'/f'' data that
are not available offline. These smooth stand-ins let the reference's modules
import and run; every number derived from them is non-physical. Parity tests
never rely on them: the data seams the hot path reads (chi/U tables, mu,
refractive decrement) are injected explicitly by the golden-vector generator.
"""

import numpy as np

__version__ = "4.6.1-placeholder"

_SYMBOLS = [
    "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si", "P", "S",
    "Cl", "Ar", "K", "Ca", "Sc", "Ti", "V", "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga",
    "Ge", "As", "Se", "Br", "Kr", "Rb", "Sr", "Y", "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd",
    "Ag", "Cd", "In", "Sn", "Sb", "Te", "I", "Xe", "Cs", "Ba", "La", "Ce", "Pr", "Nd", "Pm",
    "Sm", "Eu", "Gd", "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu", "Hf", "Ta", "W", "Re", "Os",
    "Ir", "Pt", "Au", "Hg", "Tl", "Pb", "Bi", "Po", "At", "Rn", "Fr", "Ra", "Ac", "Th", "Pa",
    "U",
]
_Z = {s: i + 1 for i, s in enumerate(_SYMBOLS)}


def atomic_number(element):
    if isinstance(element, (int, np.integer)):
        return int(element)
    return _Z[str(element).strip().capitalize()]


def atomic_symbol(z):
    return _SYMBOLS[int(z) - 1]


def f0(element, s):
    """Two-Gaussian screened form factor with f0(0) = Z (placeholder)."""
    z = atomic_number(element)
    s = np.atleast_1d(np.asarray(s, dtype=float))
    b1 = 8.0 / (1.0 + 0.05 * z)
    return z * (0.6 * np.exp(-b1 * s * s) + 0.4 * np.exp(-0.25 * b1 * s * s))


def chantler_energies(element):
    return np.geomspace(10.0, 9.0e5, 600)


def f1_chantler(element, energy):
    e = np.asarray(energy, dtype=float)
    z = atomic_number(element)
    return -0.02 * z * (1.0e3 / (e + 1.0e3))


def f2_chantler(element, energy):
    e = np.asarray(energy, dtype=float)
    z = atomic_number(element)
    return 0.5 * z * (z / 30.0) * (1.0e3 / (e + 2.0e2)) ** 2


class _Edge:
    def __init__(self, energy, fyield=0.5, jump_ratio=10.0):
        self.energy = energy
        self.fyield = fyield
        self.jump_ratio = jump_ratio


def xray_edges(element):
    z = atomic_number(element)
    return {"K": _Edge(13.6 * z * z * 0.9), "L3": _Edge(3.4 * z * z * 0.25)}


def xray_edge(element, edge):
    return xray_edges(element).get(edge)


def xray_lines(element, *args, **kwargs):
    return {}


def core_width(element, edge=None):
    return 1.0


def get_xraydb():
    raise RuntimeError("placeholder xraydb has no database")
