"""Host-side tables of the transport and scoring hot path (NumPy, FP64).

Everything here runs once per case on the host and produces the flat arrays
the CUDA kernels read: per-layer element coefficients for the exact physics,
the uniform-log-energy transport LUT, entrance-beam geometry, crystal
reflection rows (reciprocal vectors, orientation, mosaic quadrature,
polarisation pairs) and the bin edges of the spectral axes. Each function
cites the reference function it reproduces (paths relative to the PyRITE
v0.36.2 tree).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# ---------------------------------------------------------------------------
# Element data: Z, standard atomic weight A (CIAAW 2024) and mean excitation
# energy J (PDG atomic and nuclear properties), the same public constants the
# reference tabulates in src/pyrite/materials/_transport_data.py:11-55.
# ---------------------------------------------------------------------------
ELEMENTS = {
    "H": (1, 1.008, 0.0218),
    "C": (6, 12.011, 0.078),
    "N": (7, 14.007, 0.082),
    "O": (8, 15.999, 0.095),
    "Al": (13, 26.982, 0.166),
    "Si": (14, 28.085, 0.173),
    "Cu": (29, 63.546, 0.322),
    "Ge": (32, 72.630, 0.350),
    "Mo": (42, 95.95, 0.424),
    "W": (74, 183.84, 0.727),
    "Au": (79, 196.966569, 0.79),
}

MC2_KEV = 510.99895
LN2 = 0.6931471805599453
BS_PREFACTOR = 1.535e-6
HBARC_EV_ANG = 1973.269804
M_E_EV = 510998.95


def _dEds_joy_luo(Z, A, J, rho, E):
    """Joy-Luo stopping [keV/Angstrom], negative (transport/stopping.py:131-135)."""
    k = 0.731 + 0.0688 * np.log10(Z)
    return -7.85e-4 * rho * Z / (A * E) * np.log(1.166 * (E + k * J) / J)


def _dEds_bethe_bs(Z, A, J, rho, E):
    """Berger-Seltzer collision stopping [keV/Angstrom] (stopping.py:216-227)."""
    tau = E / MC2_KEV
    gamma = 1.0 + tau
    beta_sq = 1.0 - 1.0 / (gamma * gamma)
    f_minus = 1.0 - beta_sq + (tau * tau / 8.0 - (2.0 * tau + 1.0) * LN2) / (gamma * gamma)
    I_rel = J / MC2_KEV
    log_term = np.log(tau * tau * (tau + 2.0) / (2.0 * I_rel * I_rel))
    return -BS_PREFACTOR * rho * Z / (A * beta_sq) * (log_term + f_minus)


_CROSSOVER = {}


def crossover_keV(symbol: str) -> float:
    """Per-element Joy-Luo / Berger-Seltzer crossover by bisection
    (stopping.py:271-302): 200 halvings of [2 J, 300] keV."""
    if symbol in _CROSSOVER:
        return _CROSSOVER[symbol]
    Z, A, J = (float(v) for v in ELEMENTS[symbol])

    def diff(E):
        return _dEds_joy_luo(Z, A, J, 1.0, E) - _dEds_bethe_bs(Z, A, J, 1.0, E)

    lo, hi = 2.0 * J, 300.0
    if diff(lo) * diff(hi) > 0.0:
        raise ValueError(f"no Joy-Luo/Berger-Seltzer crossover for {symbol}")
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if diff(lo) * diff(mid) <= 0.0:
            hi = mid
        else:
            lo = mid
    _CROSSOVER[symbol] = 0.5 * (lo + hi)
    return _CROSSOVER[symbol]


# ---------------------------------------------------------------------------
# Layer stack (transport/layer_tables.py:52-114, batching.py:33-105)
# ---------------------------------------------------------------------------
@dataclass
class LayerStack:
    """``[(z_top, z_bot, [(element, n_per_Ang3), ...]), ...]`` and its padded rows."""

    layers: list
    z_top: np.ndarray = field(init=False)
    z_bot: np.ndarray = field(init=False)
    n_el: np.ndarray = field(init=False)
    Z: np.ndarray = field(init=False)
    A: np.ndarray = field(init=False)
    J: np.ndarray = field(init=False)
    N: np.ndarray = field(init=False)
    k: np.ndarray = field(init=False)
    coeff: np.ndarray = field(init=False)
    E_cross: np.ndarray = field(init=False)
    sr_rate_numer: np.ndarray = field(init=False)
    sr_joy_numer: np.ndarray = field(init=False)

    def __post_init__(self):
        if not self.layers:
            raise ValueError("a layer stack needs at least one layer")
        n_layers = len(self.layers)
        if n_layers > 8:
            raise ValueError("at most 8 layers")
        max_el = max(len(l[2]) for l in self.layers)
        if max_el > 8:
            raise ValueError("at most 8 elements per layer")
        prev = None
        for z0, z1, comp in self.layers:
            if not z1 > z0 or (prev is not None and z0 != prev):
                raise ValueError("layers must be contiguous with z_bot > z_top")
            if not comp:
                raise ValueError("every layer needs a composition")
            prev = z1
        if self.layers[0][0] != 0.0:
            raise ValueError("the stack must start at z = 0")
        shape = (n_layers, max_el)
        self.z_top = np.array([l[0] for l in self.layers], dtype=np.float64)
        self.z_bot = np.array([l[1] for l in self.layers], dtype=np.float64)
        self.n_el = np.array([len(l[2]) for l in self.layers], dtype=np.int32)
        for name in ("Z", "A", "J", "N", "k", "coeff", "E_cross", "sr_rate_numer", "sr_joy_numer"):
            setattr(self, name, np.zeros(shape))
        for L, (_z0, _z1, comp) in enumerate(self.layers):
            for i, (el, n_i) in enumerate(comp):
                if el not in ELEMENTS:
                    raise ValueError(f"no transport data for element {el!r}")
                Z, A, J = ELEMENTS[el]
                Z = float(Z)
                self.Z[L, i], self.A[L, i], self.J[L, i], self.N[L, i] = Z, A, J, n_i
                self.k[L, i] = 0.731 + 0.0688 * np.log10(Z)
                self.coeff[L, i] = (n_i / 0.602214076) * Z
                self.E_cross[L, i] = crossover_keV(el)
                n_cm3 = n_i * 1e24
                self.sr_rate_numer[L, i] = 5.21e-21 * Z * Z * np.float64(4.0) * np.float64(np.pi) * n_cm3
                self.sr_joy_numer[L, i] = np.float64(3.4e-3) * Z ** np.float64(0.67)

    @property
    def n_layers(self) -> int:
        return len(self.layers)

    @property
    def max_el(self) -> int:
        return int(self.Z.shape[1])

    @property
    def thickness(self) -> float:
        return float(self.z_bot[-1])

    def dEds(self, L: int, E):
        """Spliced stopping [keV/Angstrom] of layer L (stopping.py:384-410)."""
        E = np.asarray(E, dtype=np.float64)
        tau = E / MC2_KEV
        gamma = 1.0 + tau
        beta_sq = 1.0 - 1.0 / (gamma * gamma)
        f_minus = 1.0 - beta_sq + (tau * tau / 8.0 - (2.0 * tau + 1.0) * LN2) / (gamma * gamma)
        jl = np.zeros_like(E)
        bs = np.zeros_like(E)
        for i in range(int(self.n_el[L])):
            J, coeff = self.J[L, i], self.coeff[L, i]
            use_bs = E >= self.E_cross[L, i]
            I_rel = J / MC2_KEV
            jl = jl + np.where(use_bs, 0.0, coeff * np.log(1.166 * (E + self.k[L, i] * J) / J))
            bs = bs + np.where(
                use_bs, coeff * (np.log(tau * tau * (tau + 2.0) / (2.0 * I_rel * I_rel)) + f_minus), 0.0
            )
        return -7.85e-4 / E * jl - BS_PREFACTOR / beta_sq * bs


# ---------------------------------------------------------------------------
# ELSEPA tabulated elastic scattering (transport/scattering.py:330-490).
# ---------------------------------------------------------------------------
ELSEPA_GUIDE_CELLS = 1024  # a power of two: xi * cells and the cell bounds j / cells are exact


@dataclass
class ElsepaGroup:
    """Packed ELSEPA tables in the reference's layout (``pack_elsepa_tables``):
    ``start``/``length`` [n_layers, max_el] energy rows of every element slot,
    the flat rows' ``logE`` (ln eV) and ``log_rate`` (ln of n sigma in 1/cm),
    ``pdf``/``cdf`` [rows, n_mu] on the shared ``mu`` grid, ``guide``
    [rows, cells + 1]."""

    start: np.ndarray
    length: np.ndarray
    logE: np.ndarray
    log_rate: np.ndarray
    cdf: np.ndarray
    pdf: np.ndarray
    mu: np.ndarray
    guide: np.ndarray


def elsepa_density(mu, dcs):
    """Angular densities p(mu) of DCS rows, mu = (1 - cos theta) / 2, each row
    normalised by its trapezoid integral, and the CDFs (exact integrals of the
    piecewise-linear densities, last node 1): scattering.py:330-356."""
    mu = np.asarray(mu, dtype=np.float64)
    dcs = np.atleast_2d(np.asarray(dcs, dtype=np.float64))
    panel = 0.5 * (dcs[:, :-1] + dcs[:, 1:]) * np.diff(mu)
    total = panel.sum(axis=1)
    if not np.all(np.isfinite(total)) or np.any(total <= 0.0):
        raise ValueError("every ELSEPA DCS row needs a positive finite integral")
    cdf = np.zeros_like(dcs)
    cdf[:, 1:] = np.cumsum(panel, axis=1) / total[:, None]
    cdf[:, -1] = 1.0
    return dcs / total[:, None], cdf


def elsepa_guide(cdf, cells=ELSEPA_GUIDE_CELLS):
    """Guide table of each CDF row (scattering.py:366-396): entry j is the last
    panel k <= n_mu - 2 with cdf[k] <= j / cells, so the panel of any xi in
    cell j lies between entries j and j + 1 and a bisection there finds the
    same panel as one over the whole row."""
    cdf = np.atleast_2d(np.asarray(cdf, dtype=np.float64))
    if cells < 1 or cells & (cells - 1):
        raise ValueError("the guide cell count must be a positive power of two")
    n_mu = cdf.shape[1]
    head = cdf[:, : n_mu - 1]
    if np.any(np.diff(head, axis=1) < 0.0):
        raise ValueError("ELSEPA CDF rows must be nondecreasing")
    edges = np.arange(cells + 1, dtype=np.float64) / cells
    guide = np.stack([np.searchsorted(row, edges, side="right") - 1 for row in head]).astype(np.int32)
    np.clip(guide, 0, n_mu - 2, out=guide)
    guide[:, 0] = 0
    guide[:, -1] = n_mu - 2
    return guide


def pack_elsepa(stack: "LayerStack", elastic_tables, cells=ELSEPA_GUIDE_CELLS) -> ElsepaGroup:
    """Pack ``elastic_tables`` (one list per layer of one mapping per element,
    in composition order, with ``energy_eV``, ``total_elastic_cm2``, ``mu``,
    ``dcs_cm2_sr`` on one shared mu grid: the reference's ``elastic_tables``
    argument) for the transport kernel (scattering.py:398-490)."""
    if len(elastic_tables) != stack.n_layers:
        raise ValueError("elastic_tables needs one entry per layer")
    start = np.zeros((stack.n_layers, stack.max_el), dtype=np.int64)
    length = np.zeros_like(start)
    logE, log_rate, pdf, cdf = [], [], [], []
    mu_ref = None
    row = 0
    for L, layer in enumerate(elastic_tables):
        if len(layer) != int(stack.n_el[L]):
            raise ValueError(f"elastic_tables layer {L} needs one table per element")
        for k, t in enumerate(layer):
            E = np.asarray(t["energy_eV"], dtype=np.float64)
            sigma = np.asarray(t["total_elastic_cm2"], dtype=np.float64)
            mu = np.asarray(t["mu"], dtype=np.float64)
            if mu_ref is None:
                mu_ref = mu
            elif not np.array_equal(mu, mu_ref):
                raise ValueError("every ELSEPA table must share one mu grid")
            if E.size < 2 or np.any(np.diff(E) <= 0.0) or np.any(sigma <= 0.0):
                raise ValueError("ELSEPA tables need >= 2 increasing energies and positive cross sections")
            p, c = elsepa_density(mu, t["dcs_cm2_sr"])
            start[L, k], length[L, k] = row, E.size
            logE.append(np.log(E))
            log_rate.append(np.log(float(stack.N[L, k]) * 1e24 * sigma))
            pdf.append(p)
            cdf.append(c)
            row += E.size
    cdf = np.vstack(cdf)
    return ElsepaGroup(start, length, np.concatenate(logE), np.concatenate(log_rate), cdf, np.vstack(pdf),
                       np.ascontiguousarray(mu_ref), elsepa_guide(cdf, cells))


def check_elsepa_range(group: ElsepaGroup, stack: "LayerStack", E_min_keV: float, E_max_keV: float):
    """Refuse a transport energy range outside any element's table: the
    tables are never extrapolated (scattering.py:493-505)."""
    for L in range(stack.n_layers):
        for k in range(int(stack.n_el[L])):
            s, n = int(group.start[L, k]), int(group.length[L, k])
            lo, hi = np.exp(group.logE[s]) / 1e3, np.exp(group.logE[s + n - 1]) / 1e3
            if E_min_keV < lo * (1 - 1e-12) or E_max_keV > hi * (1 + 1e-12):
                raise ValueError(f"transport energy range must be within the ELSEPA table [{lo:g}, {hi:g}] keV")


# ---------------------------------------------------------------------------
# SBETHE table stopping (transport/stopping.py:11-83).
# ---------------------------------------------------------------------------
@dataclass
class StoppingTables:
    """Per-layer SBETHE collision stopping, padded: layer L's first
    ``count[L]`` entries of ``logE[L]`` / ``logS[L]`` hold ln(E / keV) and
    ln(S / (keV/Angstrom))."""

    count: np.ndarray
    logE: np.ndarray
    logS: np.ndarray


def pack_stopping(stack: "LayerStack", stopping_tables) -> StoppingTables:
    """One table per layer, each a mapping with ``stopping_energy_eV`` and
    ``stopping_eV_per_angstrom`` (the reference's ``stopping_tables``
    argument) or an already prepared ``(logE, logS)`` pair: validated,
    converted to keV and keV/Angstrom, log-transformed and padded."""
    if len(stopping_tables) != stack.n_layers:
        raise ValueError("stopping_tables needs one SBETHE table per layer")
    rows = []
    for t in stopping_tables:
        if not isinstance(t, dict) and len(t) == 2 and np.asarray(t[0]).ndim == 1:
            rows.append((np.asarray(t[0], dtype=np.float64), np.asarray(t[1], dtype=np.float64)))
            continue
        E = np.asarray(t["stopping_energy_eV"], dtype=np.float64) * 1.0e-3
        S = np.asarray(t["stopping_eV_per_angstrom"], dtype=np.float64) * 1.0e-3
        if E.ndim != 1 or S.shape != E.shape or E.size < 2 or not np.all(np.diff(E) > 0.0):
            raise ValueError("an SBETHE table needs matching vectors on a strictly increasing energy grid")
        if not (np.all(np.isfinite(E)) and np.all(np.isfinite(S))) or np.any(E <= 0.0) or np.any(S <= 0.0):
            raise ValueError("SBETHE table values must be finite and strictly positive")
        rows.append((np.log(E), np.log(S)))
    count = np.array([r[0].size for r in rows], dtype=np.int32)
    width = int(count.max())
    logE = np.zeros((stack.n_layers, width))
    logS = np.zeros((stack.n_layers, width))
    for L, (e, v) in enumerate(rows):
        logE[L, : e.size] = e
        logS[L, : v.size] = v
    return StoppingTables(count, logE, logS)


def check_stopping_range(t: StoppingTables, E_min_keV: float, E_max_keV: float):
    """Refuse a transport energy range outside any layer's table
    (host_pass.py:598-608: node ends widened by one ulp, no extrapolation)."""
    for L in range(t.count.size):
        lo = float(np.nextafter(np.exp(t.logE[L, 0]), -np.inf))
        hi = float(np.nextafter(np.exp(t.logE[L, t.count[L] - 1]), np.inf))
        if E_min_keV < lo or E_max_keV > hi:
            raise ValueError(f"transport energy range must be within the SBETHE table [{lo:g}, {hi:g}] keV")


# ---------------------------------------------------------------------------
# Transport LUT (transport/lut.py:64-283): uniform in log kinetic energy.
# ---------------------------------------------------------------------------
@dataclass
class TransportLUT:
    log_E_min: float
    inv_dlogE: float
    n_energy: int
    n_el: np.ndarray
    total_rate: np.ndarray  # (L, ne)
    dEds: np.ndarray        # (L, ne)
    inv_beta: np.ndarray    # (ne,)
    cdf: np.ndarray         # (L, max_el, ne)
    alpha: np.ndarray       # (L, max_el, ne)
    E_min_keV: float
    E_max_keV: float

    def packed(self, dtype) -> tuple[np.ndarray, dict]:
        """One contiguous buffer, every block padded to 16 bytes (pb_lut layout)."""
        dtype = np.dtype(dtype)
        per = 16 // dtype.itemsize
        blocks = [
            ("total_rate", self.total_rate.reshape(-1)),
            ("dEds", self.dEds.reshape(-1)),
            ("inv_beta", self.inv_beta.reshape(-1)),
            ("cdf", self.cdf.reshape(-1)),
            ("alpha", self.alpha.reshape(-1)),
        ]
        offsets = {}
        parts = []
        off = 0
        for name, arr in blocks:
            offsets[name] = off
            n = arr.size
            pad = (-n) % per
            parts.append(arr.astype(dtype))
            if pad:
                parts.append(np.zeros(pad, dtype=dtype))
            off += n + pad
        return np.concatenate(parts), offsets


def build_transport_lut(stack: LayerStack, E_min_keV: float, E_max_keV: float,
                        intervals_per_decade: int = 1024, min_points: int = 256,
                        max_points: int = 16384) -> TransportLUT:
    """The reference's transport LUT for SR elastic and spliced stopping
    (lut.py:283-437 grid; lut.py:140-209 nodes)."""
    E_min_keV = float(E_min_keV)
    E_max_keV = float(E_max_keV)
    if not (np.isfinite(E_min_keV) and np.isfinite(E_max_keV)) or E_min_keV <= 0.0:
        raise ValueError("transport LUT energy bounds must be finite and positive")
    if E_max_keV <= E_min_keV:
        E_max_keV = float(np.nextafter(E_min_keV, np.inf))
    min_points = max(2, int(min_points))
    max_points = max(min_points, int(max_points))
    log_E_min = float(np.log(E_min_keV))
    log_E_max = float(np.log(E_max_keV))
    log_span = log_E_max - log_E_min
    decades = log_span / np.log(10.0)
    requested = int(np.ceil(decades * float(intervals_per_decade))) + 1
    n_energy = min(max_points, max(min_points, requested))
    min_dlog = 8.0 * float(np.finfo(np.float32).eps)
    if log_span / (n_energy - 1) < min_dlog:
        n_energy = max(2, int(log_span / min_dlog) + 1)
    inv_dlogE = np.float64((n_energy - 1) / log_span)
    logE_grid = np.linspace(log_E_min, log_E_max, n_energy, dtype=np.float64)
    E = np.exp(logE_grid)
    E[0] = E_min_keV
    E[-1] = E_max_keV
    n_layers, max_el = stack.n_layers, stack.max_el
    total_rate = np.empty((n_layers, n_energy))
    dEds = np.empty((n_layers, n_energy))
    cdf = np.ones((n_layers, max_el, n_energy))
    alpha = np.zeros((n_layers, max_el, n_energy))
    g = 1.0 + E / MC2_KEV
    beta = np.sqrt(1.0 - 1.0 / (g * g))
    inv_beta = 1.0 / beta
    rel = (E + 511.0) / (E + 1024.0)
    rel2 = rel * rel
    for L in range(n_layers):
        n = int(stack.n_el[L])
        rates = np.empty((n, n_energy))
        dEds[L] = _spliced_elementwise(stack, L, E)
        for i in range(n):
            sj = float(stack.sr_joy_numer[L, i])
            a = sj / E
            rates[i] = float(stack.sr_rate_numer[L, i]) / (E * E) / (a * (1.0 + a)) * rel2
            alpha[L, i] = sj / E
        layer_total = rates.sum(axis=0)
        total_rate[L] = layer_total
        layer_cdf = np.cumsum(rates, axis=0) / layer_total[None, :]
        layer_cdf[-1, :] = 1.0
        cdf[L, :n, :] = layer_cdf
    return TransportLUT(np.float64(log_E_min), inv_dlogE, n_energy, stack.n_el.copy(), total_rate,
                        dEds, inv_beta, cdf, alpha, E_min_keV, E_max_keV)


def _spliced_elementwise(stack: LayerStack, L: int, E: np.ndarray) -> np.ndarray:
    """``_dEds_spliced_compound`` node by node, in its scalar order (stopping.py:328-335)."""
    out = np.empty_like(E)
    n = int(stack.n_el[L])
    J = stack.J[L, :n]
    k = stack.k[L, :n]
    coeff = stack.coeff[L, :n]
    Ec = stack.E_cross[L, :n]
    for j, e in enumerate(E):
        tau = e / MC2_KEV
        gamma = 1.0 + tau
        beta_sq = 1.0 - 1.0 / (gamma * gamma)
        f_minus = 1.0 - beta_sq + (tau * tau / 8.0 - (2.0 * tau + 1.0) * LN2) / (gamma * gamma)
        jl = 0.0
        bs = 0.0
        for i in range(n):
            if e < Ec[i]:
                jl += coeff[i] * np.log(1.166 * (e + k[i] * J[i]) / J[i])
            else:
                I_rel = J[i] / MC2_KEV
                bs += coeff[i] * (np.log(tau * tau * (tau + 2.0) / (2.0 * I_rel * I_rel)) + f_minus - 0.0)
        out[j] = -7.85e-4 / e * jl - BS_PREFACTOR / beta_sq * bs
    return out


# ---------------------------------------------------------------------------
# Geometry: rotations, tilt, beam entry (materials/crystal.py:894-917,
# montecarlo/geometry.py:263-420,532-700)
# ---------------------------------------------------------------------------
def _cross3(u, v):
    return np.array([u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]])


def rotation_between(u_hat, t_hat):
    """Minimal rotation with R @ u_hat = t_hat (crystal.py:894-917)."""
    u_hat = np.asarray(u_hat, dtype=float)
    t_hat = np.asarray(t_hat, dtype=float)
    c = float(np.dot(u_hat, t_hat))
    axis = _cross3(u_hat, t_hat)
    s = np.linalg.norm(axis)
    if s < 1e-12:
        if c > 0:
            return np.eye(3)
        tmp = np.array([1.0, 0.0, 0.0]) if abs(u_hat[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
        axis = _cross3(u_hat, tmp)
        axis /= np.linalg.norm(axis)
        K = np.array([[0.0, -axis[2], axis[1]], [axis[2], 0.0, -axis[0]], [-axis[1], axis[0], 0.0]])
        return np.eye(3) + 2.0 * K @ K
    axis = axis / s
    K = np.array([[0.0, -axis[2], axis[1]], [axis[2], 0.0, -axis[0]], [-axis[1], axis[0], 0.0]])
    return np.eye(3) + s * K + (1.0 - c) * (K @ K)


def tilted_geometry(theta_obs_rad, tilt_polar_rad, tilt_azim_rad=0.0):
    """Sample-frame (beam_dir, n_hat) of a tilted slab (geometry.py:263-307)."""
    st, ct = np.sin(tilt_polar_rad), np.cos(tilt_polar_rad)
    normal_lab = np.array([st * np.cos(tilt_azim_rad), st * np.sin(tilt_azim_rad), ct])
    R = rotation_between(np.array([0.0, 0.0, 1.0]), normal_lab)
    beam_dir = R.T @ np.array([0.0, 0.0, 1.0])
    n_hat = R.T @ np.array([np.sin(theta_obs_rad), 0.0, np.cos(theta_obs_rad)])
    return beam_dir, n_hat


def sample_to_lab(tilt_polar_rad, tilt_azim_rad=0.0):
    """R with v_lab = R v_sample (geometry.py:310-328)."""
    st, ct = np.sin(tilt_polar_rad), np.cos(tilt_polar_rad)
    normal_lab = np.array([st * np.cos(tilt_azim_rad), st * np.sin(tilt_azim_rad), ct])
    return rotation_between(np.array([0.0, 0.0, 1.0]), normal_lab)


def beam_entry_basis(tilt_polar_rad, tilt_azim_rad=0.0):
    """Sample-frame lab spot axes and beam axis (geometry.py:393-410)."""
    if not tilt_polar_rad:
        eye = np.eye(3)
        return eye[:, 0], eye[:, 1], eye[:, 2]
    Rt = sample_to_lab(tilt_polar_rad, tilt_azim_rad).T
    return Rt[:, 0], Rt[:, 1], Rt[:, 2]


def _small_tilt_R(dx_rad, dy_rad):
    """Rodrigues tilt of the slab normal by (dx, dy, 0) (geometry.py:572-584)."""
    ang = float(np.hypot(dx_rad, dy_rad))
    if ang < 1e-15:
        return np.eye(3)
    kx, ky = dx_rad / ang, dy_rad / ang
    K = np.array([[0.0, 0.0, ky], [0.0, 0.0, -kx], [-ky, kx, 0.0]])
    return np.eye(3) + np.sin(ang) * K + (1.0 - np.cos(ang)) * (K @ K)


def beam_frame_basis(beam_dir):
    """Lab axes carried onto the beam frame (geometry.py:587-609)."""
    d = np.asarray(beam_dir, dtype=float)
    d = d / np.linalg.norm(d)
    sin_theta = float(np.hypot(d[0], d[1]))
    if sin_theta < 1e-15:
        return np.eye(3)
    theta = float(np.arctan2(sin_theta, d[2]))
    return _small_tilt_R(-d[1] * theta / sin_theta, d[0] * theta / sin_theta)


def child_stream_root(seed: int, n_children: int, index: int) -> int:
    """Root of the ``SeedSequence(seed).spawn(n)[index]`` namespace (kinematics.py:249-259)."""
    child = np.random.SeedSequence(seed).spawn(n_children)[index]
    return int(child.generate_state(1, np.uint64)[0])


def mosaic_quadrature(fwhm_rad, nodes):
    """Gauss-Hermite product quadrature of the mosaic tilt (geometry.py:612-643)."""
    if not fwhm_rad or nodes is None or nodes <= 1:
        return None
    x, w = np.polynomial.hermite.hermgauss(int(nodes))
    sigma = float(fwhm_rad) / 2.3548200450309493
    tilt = np.sqrt(2.0) * sigma * x
    wt = w / np.sqrt(np.pi)
    return [(_small_tilt_R(tilt[j], tilt[k]), float(wt[j] * wt[k]))
            for j in range(len(tilt)) for k in range(len(tilt))]


# ---------------------------------------------------------------------------
# Crystals: lattice, reciprocal vectors, orientation (crystal.py:63-162,919-961)
# ---------------------------------------------------------------------------
@dataclass(frozen=True)
class Crystal:
    name: str
    a: float
    b: float
    c: float
    alpha: float
    beta: float
    gamma: float
    basis: tuple  # ((element, (x, y, z)), ...)
    B_ang2: float = 0.0

    def direct_vectors(self):
        """'general' lattice construction (crystal.py:101-113)."""
        al, be, ga = (np.radians(v) for v in (self.alpha, self.beta, self.gamma))
        a1 = np.array([self.a, 0.0, 0.0])
        a2 = np.array([self.b * np.cos(ga), self.b * np.sin(ga), 0.0])
        cx = self.c * np.cos(be)
        cy = self.c * (np.cos(al) - np.cos(be) * np.cos(ga)) / np.sin(ga)
        cz = np.sqrt(max(self.c**2 - cx**2 - cy**2, 0.0))
        return a1, a2, np.array([cx, cy, cz])

    def reciprocal_basis(self):
        a1, a2, a3 = self.direct_vectors()
        V = np.dot(a1, _cross3(a2, a3))
        return 2.0 * np.pi * np.array([_cross3(a2, a3), _cross3(a3, a1), _cross3(a1, a2)]) / V

    @property
    def volume(self) -> float:
        a1, a2, a3 = self.direct_vectors()
        return float(abs(np.dot(a1, _cross3(a2, a3))))

    def g_vector(self, hkl):
        g = np.asarray(hkl, dtype=float) @ self.reciprocal_basis()
        return g, float(np.linalg.norm(g))

    def orientation(self, surface_hkl=None, beam_uvw=None, azimuth_rad=0.0, recip_miscut_rad=None):
        """Rotation of every reciprocal vector (crystal.py:919-963): the cut
        direction onto +z, a roll about +z, then an optional miscut
        (polar, azimuth) tilting the lattice away from the slab normal."""
        if beam_uvw is not None and surface_hkl is not None:
            raise ValueError("beam_uvw and surface_hkl are mutually exclusive")
        R = None
        if beam_uvw is not None:
            a1, a2, a3 = self.direct_vectors()
            u, v, w = np.asarray(beam_uvw, dtype=float)
            axis = u * a1 + v * a2 + w * a3
            R = rotation_between(axis / np.linalg.norm(axis), np.array([0.0, 0.0, 1.0]))
        elif surface_hkl is not None:
            axis, norm = self.g_vector(surface_hkl)
            R = rotation_between(axis / norm, np.array([0.0, 0.0, 1.0]))
        if azimuth_rad:
            ca, sa = np.cos(azimuth_rad), np.sin(azimuth_rad)
            Rz = np.array([[ca, -sa, 0.0], [sa, ca, 0.0], [0.0, 0.0, 1.0]])
            R = Rz if R is None else Rz @ R
        if recip_miscut_rad is not None:
            mp, ma = recip_miscut_rad
            if mp:
                st, ct = np.sin(mp), np.cos(mp)
                R_m = rotation_between(np.array([0.0, 0.0, 1.0]), np.array([st * np.cos(ma), st * np.sin(ma), ct]))
                R = R_m if R is None else R_m @ R
        return R

    @property
    def n_atoms_per_ang3(self) -> float:
        return len(self.basis) / self.volume


# Cells of the reference catalog's P1 CIFs (src/pyrite/data/cifs/silicon.cif,
# hopg.cif): silicon diamond cubic a = 5.4309 A with B = 0.4632 A^2 at 293 K;
# HOPG graphite 2H a = 2.461 A, c = 6.711 A, gamma = 120 deg, B = 1.30 A^2
# for (00l). Basis sites are the standard ones of the two structures.
SILICON = Crystal(
    "silicon", 5.4309, 5.4309, 5.4309, 90.0, 90.0, 90.0,
    tuple(("Si", p) for p in [
        (0.0, 0.0, 0.0), (0.25, 0.25, 0.25), (0.0, 0.5, 0.5), (0.25, 0.75, 0.75),
        (0.5, 0.0, 0.5), (0.75, 0.25, 0.75), (0.5, 0.5, 0.0), (0.75, 0.75, 0.25),
    ]),
    B_ang2=0.4632,
)
HOPG = Crystal(
    "hopg", 2.461, 2.461, 6.711, 90.0, 90.0, 120.0,
    tuple(("C", p) for p in [
        (0.0, 0.0, 0.0), (1.0 / 3.0, 2.0 / 3.0, 0.0), (0.0, 0.0, 0.5), (2.0 / 3.0, 1.0 / 3.0, 0.5),
    ]),
    B_ang2=1.30,
)
CRYSTALS = {"silicon": SILICON, "hopg": HOPG}


def polarization_pairs(k_hat, g_rows):
    """sigma/pi polarisation per reflection row (cxr/_polarization.py:20-38,
    cxr/_kernels.py:1135-1144)."""
    g_rows = np.asarray(g_rows, dtype=float).reshape(-1, 3)
    k_hat = np.asarray(k_hat, dtype=float)
    n_plane = np.cross(k_hat[None, :], g_rows)
    npl = np.sqrt(np.array([row.dot(row) for row in n_plane]))
    degenerate = npl < 1e-12
    npl[degenerate] = 1.0
    e_s = n_plane / npl[:, None]
    e_p = np.cross(e_s, k_hat[None, :])
    epl = np.sqrt(np.array([row.dot(row) for row in e_p]))
    epl[degenerate] = 1.0
    e_p /= epl[:, None]
    for i in np.flatnonzero(degenerate):
        n_pl = np.cross(k_hat, np.array([0.0, 1.0, 0.0]))
        e_s[i] = n_pl / np.linalg.norm(n_pl)
        p = np.cross(e_s[i], k_hat)
        e_p[i] = p / np.linalg.norm(p)
    return e_s, e_p


@dataclass
class ReflectionRows:
    """Reflection x orientation rows of one direction set (cxr/_batched.py:232-331)."""

    G: np.ndarray          # (n_g, 3)
    ES: np.ndarray         # (n_dir, n_g, 3)
    EP: np.ndarray         # (n_dir, n_g, 3)
    WM: np.ndarray         # (n_g,)
    row_table: np.ndarray  # (n_g,)


def reflection_rows(crystal: Crystal, hkl_list, n_hats, *, surface_hkl=None, beam_uvw=None,
                    azimuth_rad=0.0, mosaic_fwhm_rad=None, mosaic_nodes=1, recip_miscut_rad=None) -> ReflectionRows:
    """One row per (reflection, mosaic orientation); polarisations per direction."""
    R_orient = crystal.orientation(surface_hkl, beam_uvw, azimuth_rad, recip_miscut_rad)
    quad = mosaic_quadrature(mosaic_fwhm_rad, mosaic_nodes)
    orients = ((None, 1.0),) if quad is None else quad
    g_rows, wm_rows, table_rows = [], [], []
    for i_hkl, hkl in enumerate(hkl_list):
        g_vec, _ = crystal.g_vector(hkl)
        if R_orient is not None:
            g_vec = R_orient @ g_vec
        for R_m, wm in orients:
            g_rows.append(g_vec if R_m is None else R_m @ g_vec)
            wm_rows.append(wm)
            table_rows.append(i_hkl)
    G = np.array(g_rows, dtype=float).reshape(-1, 3)
    n_hats = np.atleast_2d(np.asarray(n_hats, dtype=float))
    ES = np.empty((n_hats.shape[0], G.shape[0], 3))
    EP = np.empty_like(ES)
    for d, nh in enumerate(n_hats):
        ES[d], EP[d] = polarization_pairs(nh / np.linalg.norm(nh), G)
    return ReflectionRows(G, ES, EP, np.array(wm_rows, dtype=float), np.array(table_rows, dtype=np.int32))


def diamond_hkls(g_max: float, crystal: Crystal = SILICON):
    """Diamond-cubic allowed reflections with |g| < g_max (all odd, or all
    even with h + k + l = 0 mod 4): the nonzero independent-atom set."""
    hmax = int(np.ceil(g_max * crystal.a / (2.0 * np.pi))) + 1
    out = []
    r = range(-hmax, hmax + 1)
    for h in r:
        for k in r:
            for l in r:
                if (h, k, l) == (0, 0, 0):
                    continue
                odd = h % 2 and k % 2 and l % 2
                even = h % 2 == 0 and k % 2 == 0 and l % 2 == 0 and (h + k + l) % 4 == 0
                if (odd or even) and crystal.g_vector((h, k, l))[1] < g_max:
                    out.append((h, k, l))
    return out


def geometric_grid(E_tab, rtol=1e-9):
    """(log E_0, log step) when E_tab is geometric to ``rtol`` of a step, else (0, 0)."""
    E = np.asarray(E_tab, dtype=float)
    if E.size < 3 or np.any(E <= 0) or np.any(np.diff(E) <= 0):
        return 0.0, 0.0
    lg = np.log(E)
    step = (lg[-1] - lg[0]) / (E.size - 1)
    pred = lg[0] + step * np.arange(E.size)
    if np.max(np.abs(pred - lg)) <= rtol * step:
        return float(lg[0]), float(step)
    return 0.0, 0.0


def energy_bin_edges(E_grid):
    """Bin edges of the bin-mean routes (spectrum/characteristic.py:621-646)."""
    grid = np.asarray(E_grid, dtype=float)
    if grid.ndim != 1 or grid.size < 2 or np.any(np.diff(grid) <= 0.0):
        raise ValueError("energy bin centres must be a strictly increasing vector of >= 2")
    edges = np.empty(grid.size + 1)
    edges[1:-1] = 0.5 * (grid[:-1] + grid[1:])
    edges[0] = max(0.0, grid[0] - 0.5 * (grid[1] - grid[0]))
    edges[-1] = grid[-1] + 0.5 * (grid[-1] - grid[-2])
    return edges


def line_keep_window(E_grid):
    """Resonance window of the lines a grid scores (cxr/_kernels.py:110-127)."""
    e_lo, e_hi = float(E_grid[0]), float(E_grid[-1])
    pad = 0.2 * (e_hi - e_lo)
    return e_lo - pad, e_hi + pad
