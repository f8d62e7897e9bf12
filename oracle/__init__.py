"""CPU ORACLE -- test infrastructure, never the product.

A C restatement (``oracle/csrc``) of the reference's (PyRITE v0.36.2) transport
and emission-scoring arithmetic, plus this thin ctypes wrapper. Only the tests,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline use it, as the
checker or as the timed CPU reference; ``pyrite_b200`` never imports it.

Parity status: pinned against golden vectors produced by running the reference
itself (``tests/golden/make_golden.py`` through ``oracle.ref_harness``):
transport rows bit for bit, the CXR line chain and its reductions and the
Bethe-Heitler spectrum to FP64 rounding.
"""

from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"

RNG_SPLITMIX = 0
RNG_PHILOX = 1

_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.is_file():
            build()
        _lib = C.CDLL(str(LIB_PATH))
        _declare(_lib)
    return _lib


_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)
_I32 = C.POINTER(C.c_int)
_I16 = C.POINTER(C.c_int16)
_I8 = C.POINTER(C.c_int8)
_U8 = C.POINTER(C.c_uint8)


class _Elsepa(C.Structure):
    _fields_ = [
        ("n_mu", C.c_int),
        ("cells", C.c_int),
        ("start", C.POINTER(C.c_int64)),
        ("length", C.POINTER(C.c_int64)),
        ("logE", _D),
        ("log_rate", _D),
        ("cdf", _D),
        ("pdf", _D),
        ("mu", _D),
        ("guide", C.POINTER(C.c_int32)),
    ]


class _Layers(C.Structure):
    _fields_ = [
        ("n_layers", C.c_int),
        ("max_el", C.c_int),
        ("z_top", _D),
        ("z_bot", _D),
        ("n_el", _I32),
        ("J", _D),
        ("k", _D),
        ("coeff", _D),
        ("E_cross", _D),
        ("sr_rate_numer", _D),
        ("sr_joy_numer", _D),
        ("Z", _D),
        ("straggling", C.c_int),
        ("elsepa", C.POINTER(_Elsepa)),
        ("sb_width", C.c_int),
        ("sb_count", C.POINTER(C.c_int32)),
        ("sb_logE", _D),
        ("sb_logS", _D),
    ]


class _Rows(C.Structure):
    _fields_ = [
        ("r_mid", _D),
        ("v_hat", _D),
        ("L", _D),
        ("E_start", _D),
        ("E_end", _D),
        ("t_start", _D),
        ("t_end", _D),
        ("elec_id", _I64),
        ("layer", _I16),
        ("flight", _I64),
        ("event", _I8),
    ]


class _Lut(C.Structure):
    _fields_ = [
        ("n_layers", C.c_int),
        ("max_el", C.c_int),
        ("n_energy", C.c_int),
        ("log_E_min", C.c_double),
        ("inv_dlogE", C.c_double),
        ("z_top", _D),
        ("z_bot", _D),
        ("n_el", _I32),
        ("total_rate", _D),
        ("dEds", _D),
        ("inv_beta", _D),
        ("cdf", _D),
        ("alpha", _D),
    ]


class _CxrTables(C.Structure):
    _fields_ = [
        ("n_g", C.c_int),
        ("G", _D),
        ("ES", _D),
        ("EP", _D),
        ("WM", _D),
        ("row_table", _I32),
        ("n_tab", C.c_int),
        ("E_tab", _D),
        ("chi_re", _D),
        ("chi_im", _D),
        ("u_re", _D),
        ("u_im", _D),
        ("n_mu", C.c_int),
        ("log_mu", _D),
        ("delta", _D),
        ("lo_keep", C.c_double),
        ("hi_keep", C.c_double),
    ]


class _LayerEscape(C.Structure):
    _fields_ = [
        ("n_layer", C.c_int), ("z_top", _D), ("z_bot", _D), ("mu_off", _I32),
        ("mu_knot", _D), ("mu_value", _D), ("mu_slope", _D),
    ]


class _CxrGeom(C.Structure):
    _fields_ = [("n_hat", C.c_double * 3), ("thickness", C.c_double), ("layers", C.POINTER(_LayerEscape))]


class LayerEscape:
    """A planar layered absorber for the oracle: bounds [z_top, z_bot) per
    layer and, for the CXR chain, each layer's piecewise-linear mu(E) as
    (knots, values, slopes) (cxr/_escape_mu.py:41-57)."""

    def __init__(self, z_top, z_bot, mu_tables=None):
        self.z_top = _f64(z_top)
        self.z_bot = _f64(z_bot)
        n = int(self.z_top.size)
        if mu_tables is None:
            mu_tables = [(np.array([1.0]), np.zeros(1), np.zeros(1))] * n
        self.mu_off = np.ascontiguousarray(np.cumsum([0] + [len(k) for k, _v, _s in mu_tables]), dtype=np.int32)
        self.mu_knot = _f64(np.concatenate([k for k, _v, _s in mu_tables]))
        self.mu_value = _f64(np.concatenate([v for _k, v, _s in mu_tables]))
        self.mu_slope = _f64(np.concatenate([sl for _k, _v, sl in mu_tables]))
        self.c = _LayerEscape(n, _p(self.z_top, _D), _p(self.z_bot, _D), _p(self.mu_off, _I32),
                              _p(self.mu_knot, _D), _p(self.mu_value, _D), _p(self.mu_slope, _D))

    def pieces(self, z0, z1, n_z):
        """(fraction[P], path0[P, K], path1[P, K]) of one segment."""
        K = int(self.z_top.size)
        f = np.zeros(8)
        p0 = np.zeros(64)
        p1 = np.zeros(64)
        P = lib().or_layer_pieces(float(z0), float(z1), C.byref(self.c), float(n_z), _p(f, _D), _p(p0, _D),
                                  _p(p1, _D))
        return f[:P].copy(), p0[:P * K].reshape(P, K).copy(), p1[:P * K].reshape(P, K).copy()


def _declare(L):
    L.or_splitmix64.restype = C.c_uint64
    L.or_splitmix64.argtypes = [C.c_uint64]
    L.or_stream_key.restype = C.c_uint64
    L.or_stream_key.argtypes = [C.c_uint64, C.c_uint64]
    L.or_stream_uniform.restype = C.c_double
    L.or_stream_uniform.argtypes = [C.c_uint64, C.c_uint64]
    L.or_dEds_element.restype = C.c_double
    L.or_dEds_element.argtypes = [C.c_double] * 5
    L.or_urban_sample_element.restype = C.c_double
    L.or_urban_sample_element.argtypes = [C.c_double] * 5 + [C.c_uint64, C.POINTER(C.c_uint64)]
    L.or_urban_moments_element.restype = None
    L.or_urban_moments_element.argtypes = [C.c_double] * 5 + [C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.or_philox_uniform.restype = C.c_double
    L.or_philox_uniform.argtypes = [C.c_uint64, C.c_uint64]
    L.or_philox4x32_10.restype = None
    L.or_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    L.or_dEds_spliced.restype = C.c_double
    L.or_dEds_spliced.argtypes = [C.POINTER(_Layers), C.c_int, C.c_double]
    L.or_sbethe_dEds.restype = C.c_double
    L.or_sbethe_dEds.argtypes = [C.POINTER(_Layers), C.c_int, C.c_double]
    L.or_elsepa_rate.restype = C.c_double
    L.or_elsepa_rate.argtypes = [C.POINTER(_Elsepa), C.c_int64, C.c_int64, C.c_double]
    L.or_elsepa_cos_theta.restype = C.c_double
    L.or_elsepa_cos_theta.argtypes = [C.POINTER(_Elsepa), C.c_int64, C.c_int64, C.c_double, C.c_double]
    L.or_sr_rate.restype = C.c_double
    L.or_sr_rate.argtypes = [C.c_double, C.c_double, C.c_double]
    L.or_transport.restype = None
    L.or_transport.argtypes = [
        C.POINTER(_Layers), C.c_int, C.c_uint64, C.c_int64, C.c_int64, C.c_double, C.c_int64,
        C.c_int64, _D, _D, _D, _D, C.POINTER(_Rows), _I64, _I8, C.c_int,
    ]
    L.or_transport_lut.restype = None
    L.or_transport_lut.argtypes = [
        C.POINTER(_Lut), C.c_int, C.c_uint64, C.c_int64, C.c_int64, C.c_double, C.c_int64,
        C.c_int64, _D, _D, _D, _D, C.POINTER(_Rows), _I64, _I8,
    ]
    L.or_cxr_lines.restype = None
    L.or_cxr_lines.argtypes = [
        C.POINTER(_CxrTables), C.POINTER(_CxrGeom), C.c_int64, _D, _D, _D, _D, _I64, C.c_int64,
        _D, _D, _D, _U8, C.c_int,
    ]
    L.or_cxr_coherent_records.restype = None
    L.or_cxr_coherent_records.argtypes = [
        C.POINTER(_CxrTables), C.POINTER(_CxrGeom), C.c_int64, _D, _D, _D, _D, _D, _I64, C.c_int64,
        C.POINTER(_D), _U8,
    ]
    L.or_reduce_node.restype = None
    L.or_reduce_node.argtypes = [C.c_int64, _D, _D, _D, C.c_int64, _D, _D, C.c_int]
    L.or_reduce_binmean.restype = None
    L.or_reduce_binmean.argtypes = [C.c_int64, _D, _D, _D, C.c_int64, _D, _D, C.c_int]
    L.or_sincsq_tail.restype = C.c_double
    L.or_sincsq_tail.argtypes = [C.c_double]
    L.or_mean_transmission.restype = C.c_double
    L.or_mean_transmission.argtypes = [C.c_double, C.c_double]
    L.or_quantum_line_factors.restype = None
    L.or_quantum_line_factors.argtypes = [C.c_double] * 10 + [_D, _D]
    L.or_layer_pieces.restype = C.c_int
    L.or_layer_pieces.argtypes = [C.c_double, C.c_double, C.POINTER(_LayerEscape), C.c_double, _D, _D, _D]
    L.or_brem_spectrum_layered.restype = None
    L.or_brem_spectrum_layered.argtypes = [
        C.c_int64, _D, _D, _D, _D, C.c_int, _D, _D, C.POINTER(_LayerEscape), _D, C.c_int64, _D, _D, _D,
        C.c_int,
    ]
    L.or_brem_spectrum.restype = None
    L.or_brem_spectrum.argtypes = [
        C.c_int64, _D, _D, _D, _D, C.c_int, _D, _D, C.c_double, _D, C.c_int64, _D, _D, _D,
        C.c_int,
    ]


def _p(a, ctype):
    return a.ctypes.data_as(ctype)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ---------------------------------------------------------------------------
# RNG
# ---------------------------------------------------------------------------
def splitmix64(x: int) -> int:
    return int(lib().or_splitmix64(C.c_uint64(int(x))))


def stream_key(seed: int, elec: int) -> int:
    return int(lib().or_stream_key(C.c_uint64(int(seed) % 2**64), C.c_uint64(int(elec))))


def stream_uniform(key: int, counter: int) -> float:
    return float(lib().or_stream_uniform(C.c_uint64(int(key)), C.c_uint64(int(counter))))


def philox_uniform(key: int, draw: int) -> float:
    return float(lib().or_philox_uniform(C.c_uint64(int(key)), C.c_uint64(int(draw))))


def philox4x32_10(ctr, key):
    c = (C.c_uint32 * 4)(*[int(v) for v in ctr])
    k = (C.c_uint32 * 2)(*[int(v) for v in key])
    lib().or_philox4x32_10(c, k)
    return [int(v) for v in c]


def dEds_element(J, k, coeff, E_cross, E):
    """One element's spliced stopping power [keV/Angstrom] (negative)."""
    return float(lib().or_dEds_element(J, k, coeff, E_cross, E))


def urban_sample_element(Z, J, C_keV_per_ang, E, s, key, counter=0):
    """One element's Urban loss over ``s`` [keV] and the next counter."""
    c = C.c_uint64(int(counter))
    dE = float(lib().or_urban_sample_element(Z, J, C_keV_per_ang, E, s, C.c_uint64(int(key) % 2**64),
                                              C.byref(c)))
    return dE, int(c.value)


def urban_moments_element(Z, J, C_keV_per_ang, E, s):
    """Analytic (mean, variance) of one element's Urban loss [keV, keV^2]."""
    m, v = C.c_double(), C.c_double()
    lib().or_urban_moments_element(Z, J, C_keV_per_ang, E, s, C.byref(m), C.byref(v))
    return m.value, v.value


def beam_entries(beam, e_start: int, n: int, rng: int = 1):
    """Entrance states (pos [n,3], dir [n,3], E [n]) of histories
    [e_start, e_start + n) of a Gaussian-spot or Twiss beam, drawn from the
    counter-addressed entry stream as the reference samples them:
    normals z_c = ndtri(u_c) of open uniforms of the stream keyed
    (beam.root, history) (src/pyrite/montecarlo/transport/kinematics.py:270-311;
    ``rng`` 1 = Philox4x32-10 with a 52-bit open uniform, 0 = SplitMix64);
    Twiss phase space x = sqrt(eps beta) z0, x' = sqrt(eps / beta)(z1 - alpha z0)
    (src/pyrite/montecarlo/transverse.py:177-186); offsets projected onto the
    tilted entrance face (src/pyrite/montecarlo/geometry.py:374-390); direction
    (x', y', 1) in the beam frame, normalised
    (src/pyrite/montecarlo/transport/beam_entry.py:347-359).
    ``beam`` carries the pb_beam fields (mode 1 spot / 2 Twiss, root,
    twiss_x/y = (eps [mm rad], beta [mm/rad], alpha), sigma_x/y_ang, tilted,
    e_x, e_y, beam_dir, basis (row-major 3x3), E0_keV)."""
    from scipy.special import ndtri

    twiss = int(beam.mode) == 2
    nz = 4 if twiss else 2
    z = np.empty((n, nz))
    for i in range(n):
        key = stream_key(int(beam.root), e_start + i)
        for c in range(nz):
            if rng == 1:
                w = philox_uniform(key, c)
                u = (np.floor(w * 4503599627370496.0) + 0.5) * (1.0 / 4503599627370496.0)
            else:
                z64 = splitmix64((key + 0x9E3779B97F4A7C15 * (c + 1)) % 2**64)
                u = ((z64 >> 12) + 0.5) * (1.0 / 4503599627370496.0)
            z[i, c] = ndtri(u)
    bd = np.array(beam.beam_dir[:], float)
    if twiss:
        ex, bx, ax = beam.twiss_x[:]
        ey, by, ay = beam.twiss_y[:]
        u_off = np.sqrt(ex * bx) * z[:, 0] * 1.0e7
        xp = np.sqrt(ex / bx) * (z[:, 1] - ax * z[:, 0])
        v_off = np.sqrt(ey * by) * z[:, 2] * 1.0e7
        yp = np.sqrt(ey / by) * (z[:, 3] - ay * z[:, 2])
    else:
        u_off, v_off = z[:, 0] * beam.sigma_x_ang, z[:, 1] * beam.sigma_y_ang
        xp = yp = np.zeros(n)
    e_x, e_y = np.array(beam.e_x[:], float), np.array(beam.e_y[:], float)
    pos = np.zeros((n, 3))
    if beam.tilted:
        s_star = -(u_off * e_x[2] + v_off * e_y[2]) / bd[2]
        pos[:, 0] = (u_off * e_x[0] + v_off * e_y[0]) + s_star * bd[0]
        pos[:, 1] = (u_off * e_x[1] + v_off * e_y[1]) + s_star * bd[1]
    else:
        pos[:, 0], pos[:, 1] = u_off, v_off
    if twiss:
        B = np.array(beam.basis[:], float).reshape(3, 3)
        d = (xp[:, None] * B[:, 0][None, :] + yp[:, None] * B[:, 1][None, :]) + bd[None, :]
        nrm = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
        dirs = d / nrm[:, None]
    else:
        dirs = np.tile(bd, (n, 1))
    return pos, dirs, np.full(n, float(beam.E0_keV))


# ---------------------------------------------------------------------------
# Layer tables (src/pyrite/montecarlo/transport/layer_tables.py:52-114)
# ---------------------------------------------------------------------------
class LayerTables:
    """Per-layer element coefficients, as ``build_layer_tables`` hoists them."""

    def __init__(self, z_top, z_bot, n_el, Z, J, N, E_cross):
        self.z_top = _f64(z_top)
        self.z_bot = _f64(z_bot)
        self.n_el = np.ascontiguousarray(n_el, dtype=np.int32)
        Z = _f64(Z)
        self.Z = Z
        self.J = _f64(J)
        N = _f64(N)
        safe_Z = np.where(Z > 0, Z, 1.0)
        self.k = np.where(Z > 0, 0.731 + 0.0688 * np.log10(safe_Z), 0.0)
        self.coeff = (N / 0.602214076) * Z
        self.E_cross = _f64(E_cross)
        self.sr_rate_numer = 5.21e-21 * Z * Z * np.float64(4.0) * np.float64(np.pi) * (N * 1e24)
        self.sr_joy_numer = np.where(Z > 0, np.float64(3.4e-3) * safe_Z ** np.float64(0.67), 0.0)
        for name in ("k", "coeff", "sr_rate_numer", "sr_joy_numer"):
            setattr(self, name, _f64(getattr(self, name)))
        self.struct = _Layers(
            len(self.z_top), Z.shape[1], _p(self.z_top, _D), _p(self.z_bot, _D),
            _p(self.n_el, _I32), _p(self.J, _D), _p(self.k, _D), _p(self.coeff, _D),
            _p(self.E_cross, _D), _p(self.sr_rate_numer, _D), _p(self.sr_joy_numer, _D),
            _p(self.Z, _D), 0, None, 0, None, None, None,
        )
        self.elsepa = None
        self.sbethe = None

    def use_elsepa(self, tables: "ElsepaTables | None"):
        """Sample elastic events from ELSEPA tables (None: screened Rutherford)."""
        self.elsepa = tables
        self.struct.elsepa = C.pointer(tables.struct) if tables is not None else None
        return self

    def use_sbethe(self, count, logE, logS):
        """Continuous stopping from SBETHE tables, packed as
        ``pack_sbethe_stopping_tables`` returns them (None: spliced)."""
        if count is None:
            self.sbethe = None
            self.struct.sb_count, self.struct.sb_logE, self.struct.sb_logS, self.struct.sb_width = None, None, None, 0
            return self
        self.sbethe = (np.ascontiguousarray(count, dtype=np.int32), _f64(logE), _f64(logS))
        c, e, v = self.sbethe
        self.struct.sb_width = int(e.shape[1])
        self.struct.sb_count = c.ctypes.data_as(C.POINTER(C.c_int32))
        self.struct.sb_logE, self.struct.sb_logS = _p(e, _D), _p(v, _D)
        return self

    def sbethe_dEds(self, L, E):
        return float(lib().or_sbethe_dEds(C.byref(self.struct), int(L), float(E)))

    def dEds(self, L, E):
        return float(lib().or_dEds_spliced(C.byref(self.struct), int(L), float(E)))


class ElsepaTables:
    """A packed ELSEPA group in the layout of ``pack_elsepa_tables``
    (``scattering.py:398-490``): ``start``/``length`` [n_layers, max_el], the
    flat ``logE``/``log_rate`` rows, ``cdf``/``pdf`` [rows, n_mu], ``mu``
    [n_mu] and ``guide`` [rows, cells + 1]."""

    def __init__(self, start, length, logE, log_rate, cdf, pdf, mu, guide):
        self.start = np.ascontiguousarray(start, dtype=np.int64)
        self.length = np.ascontiguousarray(length, dtype=np.int64)
        self.logE, self.log_rate = _f64(logE), _f64(log_rate)
        self.cdf, self.pdf, self.mu = _f64(cdf), _f64(pdf), _f64(mu)
        self.guide = np.ascontiguousarray(guide, dtype=np.int32)
        self.struct = _Elsepa(
            int(self.mu.size), int(self.guide.shape[1] - 1), self.start.ctypes.data_as(C.POINTER(C.c_int64)),
            self.length.ctypes.data_as(C.POINTER(C.c_int64)), _p(self.logE, _D), _p(self.log_rate, _D),
            _p(self.cdf, _D), _p(self.pdf, _D), _p(self.mu, _D), self.guide.ctypes.data_as(C.POINTER(C.c_int32)),
        )

    def slot(self, L, k):
        return int(self.start[L, k]), int(self.length[L, k])

    def rate(self, L, k, E_keV):
        """Macroscopic elastic rate [1/cm] of element ``k`` of layer ``L``."""
        return float(lib().or_elsepa_rate(C.byref(self.struct), *self.slot(L, k), float(E_keV)))

    def cos_theta(self, L, k, E_keV, xi):
        """Polar deflection cosine for the uniform ``xi``."""
        return float(lib().or_elsepa_cos_theta(C.byref(self.struct), *self.slot(L, k), float(E_keV), float(xi)))


class LutTables:
    """A transport LUT as ``build_transport_energy_lut`` returns it (lut.py:283-437)."""

    def __init__(self, z_top, z_bot, n_el, log_E_min, inv_dlogE, total_rate, dEds, inv_beta, cdf,
                 alpha):
        self.z_top, self.z_bot = _f64(z_top), _f64(z_bot)
        self.n_el = np.ascontiguousarray(n_el, dtype=np.int32)
        self.total_rate, self.dEds = _f64(total_rate), _f64(dEds)
        self.inv_beta, self.cdf, self.alpha = _f64(inv_beta), _f64(cdf), _f64(alpha)
        n_layers, max_el, n_energy = self.cdf.shape
        self.struct = _Lut(
            n_layers, max_el, n_energy, float(log_E_min), float(inv_dlogE), _p(self.z_top, _D),
            _p(self.z_bot, _D), _p(self.n_el, _I32), _p(self.total_rate, _D), _p(self.dEds, _D),
            _p(self.inv_beta, _D), _p(self.cdf, _D), _p(self.alpha, _D),
        )


def transport(layers, pos, direction, E, *, seed, E_cut, rng=RNG_SPLITMIX,
              e_start=0, max_steps=400_000, cap=4096, keep_rows=True, clock=None, straggling=False):
    """Per-electron transport of ``len(E)`` histories; returns a dict of rows and finals.

    ``layers`` is a :class:`LayerTables` (the exact analytic core) or a
    :class:`LutTables` (the reference's default LUT core). ``straggling``:
    Urban energy-loss straggling per flight (exact core).
    """
    if straggling and isinstance(layers, LutTables):
        raise ValueError("the oracle's LUT core has no straggling")
    if isinstance(layers, LayerTables):
        layers.struct.straggling = 1 if straggling else 0
    n = int(np.asarray(E).size)
    pos = _f64(pos).reshape(n, 3).copy()
    direction = _f64(direction).reshape(n, 3).copy()
    E = _f64(E).copy()
    clock = np.zeros(n) if clock is None else _f64(clock).copy()
    seg_count = np.zeros(n, dtype=np.int64)
    exit_code = np.zeros(n, dtype=np.int8)
    rows = None
    holders = None
    if keep_rows:
        m = n * cap
        holders = dict(
            r_mid=np.zeros((m, 3)), v_hat=np.zeros((m, 3)), L=np.zeros(m), E_start=np.zeros(m),
            E_end=np.zeros(m), t_start=np.zeros(m), t_end=np.zeros(m),
            elec_id=np.zeros(m, dtype=np.int64), layer=np.zeros(m, dtype=np.int16),
            flight=np.zeros(m, dtype=np.int64), event=np.zeros(m, dtype=np.int8),
        )
        h = holders
        rows = _Rows(
            _p(h["r_mid"], _D), _p(h["v_hat"], _D), _p(h["L"], _D), _p(h["E_start"], _D),
            _p(h["E_end"], _D), _p(h["t_start"], _D), _p(h["t_end"], _D), _p(h["elec_id"], _I64),
            _p(h["layer"], _I16), _p(h["flight"], _I64), _p(h["event"], _I8),
        )
    args = (
        C.byref(layers.struct), int(rng), C.c_uint64(int(seed) % 2**64), int(e_start), n,
        float(E_cut), int(max_steps), int(cap), _p(pos, _D), _p(direction, _D), _p(E, _D),
        _p(clock, _D), C.byref(rows) if rows is not None else None, _p(seg_count, _I64),
        _p(exit_code, _I8),
    )
    if isinstance(layers, LutTables):
        lib().or_transport_lut(*args)
    else:
        lib().or_transport(*args, 1)
    out = dict(pos=pos, dir=direction, E=E, clock=clock, seg_count=seg_count, exit_code=exit_code)
    if holders is not None:
        stored = np.minimum(seg_count, cap)
        mask = (np.arange(cap)[None, :] < stored[:, None]).reshape(-1)
        for k, v in holders.items():
            out[k] = v[mask]
    return out


# ---------------------------------------------------------------------------
# CXR line chain and reductions
# ---------------------------------------------------------------------------
def cxr_lines(tables: dict, n_hat, thickness, seg: dict, Ne, layers: LayerEscape | None = None):
    """Line (E_res, a_width, weight, good) per (segment, row), segment-major.
    ``layers``: a layered absorber (escape pieces with each layer's exact mu)."""
    G = _f64(tables["G"])
    ES, EP, WM = _f64(tables["ES"]), _f64(tables["EP"]), _f64(tables["WM"])
    row_table = np.ascontiguousarray(tables["row_table"], dtype=np.int32)
    E_tab = _f64(tables["E_tab"])
    chi_re, chi_im = _f64(tables["chi_re"]), _f64(tables["chi_im"])
    u_re, u_im = _f64(tables["u_re"]), _f64(tables["u_im"])
    log_mu = _f64(np.atleast_2d(tables["log_mu"]))
    delta = _f64(tables["delta"])
    t = _CxrTables(
        int(G.shape[0]), _p(G, _D), _p(ES, _D), _p(EP, _D), _p(WM, _D), _p(row_table, _I32),
        int(E_tab.size), _p(E_tab, _D), _p(chi_re, _D), _p(chi_im, _D), _p(u_re, _D),
        _p(u_im, _D), int(log_mu.shape[0]), _p(log_mu, _D), _p(delta, _D),
        float(tables["lo_keep"]), float(tables["hi_keep"]),
    )
    geo = _CxrGeom((C.c_double * 3)(*[float(v) for v in n_hat]), float(thickness),
                   C.pointer(layers.c) if layers is not None else None)
    v_hat = _f64(seg["v_hat"])
    E = _f64(seg["E_keV"])
    L = _f64(seg["L_ang"])
    r = _f64(seg["r_mid"])
    eid = np.ascontiguousarray(seg["elec_id"], dtype=np.int64)
    n = int(E.size)
    m = n * int(G.shape[0])
    E_res = np.empty(m)
    aw = np.empty(m)
    w = np.empty(m)
    good = np.empty(m, dtype=np.uint8)
    lib().or_cxr_lines(
        C.byref(t), C.byref(geo), n, _p(v_hat, _D), _p(E, _D), _p(L, _D), _p(r, _D),
        _p(eid, _I64), int(Ne), _p(E_res, _D), _p(aw, _D), _p(w, _D), _p(good, _U8), 1,
    )
    return E_res, aw, w, good.astype(bool)


def cxr_coherent_records(tables: dict, n_hat, thickness, seg: dict, Ne):
    """Coherent route line records per (segment, row), segment-major, single
    slab: ``({field: [n_seg*n_g]}, good)`` with the fields of
    ``oracle.coherent.FIELDS``; ``seg`` may carry ``t_ang`` (start ages)."""
    from .coherent import FIELDS

    G = _f64(tables["G"])
    ES, EP, WM = _f64(tables["ES"]), _f64(tables["EP"]), _f64(tables["WM"])
    row_table = np.ascontiguousarray(tables["row_table"], dtype=np.int32)
    E_tab = _f64(tables["E_tab"])
    chi_re, chi_im = _f64(tables["chi_re"]), _f64(tables["chi_im"])
    u_re, u_im = _f64(tables["u_re"]), _f64(tables["u_im"])
    log_mu = _f64(np.atleast_2d(tables["log_mu"]))
    delta = _f64(tables["delta"])
    t = _CxrTables(
        int(G.shape[0]), _p(G, _D), _p(ES, _D), _p(EP, _D), _p(WM, _D), _p(row_table, _I32),
        int(E_tab.size), _p(E_tab, _D), _p(chi_re, _D), _p(chi_im, _D), _p(u_re, _D),
        _p(u_im, _D), int(log_mu.shape[0]), _p(log_mu, _D), _p(delta, _D),
        float(tables["lo_keep"]), float(tables["hi_keep"]),
    )
    geo = _CxrGeom((C.c_double * 3)(*[float(v) for v in n_hat]), float(thickness), None)
    v_hat, E, L, r = (_f64(seg[k]) for k in ("v_hat", "E_keV", "L_ang", "r_mid"))
    t_ang = _f64(seg["t_ang"]) if seg.get("t_ang") is not None else None
    eid = np.ascontiguousarray(seg["elec_id"], dtype=np.int64)
    n = int(E.size)
    m = n * int(G.shape[0])
    out = {k: np.empty(m) for k in FIELDS}
    ptrs = (_D * len(FIELDS))(*[_p(out[k], _D) for k in FIELDS])
    good = np.empty(m, dtype=np.uint8)
    lib().or_cxr_coherent_records(
        C.byref(t), C.byref(geo), n, _p(v_hat, _D), _p(E, _D), _p(L, _D), _p(r, _D),
        None if t_ang is None else _p(t_ang, _D), _p(eid, _I64), int(Ne), ptrs, _p(good, _U8),
    )
    return out, good.astype(bool)


def reduce_node(E_res, a_width, weight, E_grid):
    E_res, a_width, weight, E_grid = (_f64(x) for x in (E_res, a_width, weight, E_grid))
    spec = np.zeros(E_grid.size)
    lib().or_reduce_node(E_res.size, _p(E_res, _D), _p(a_width, _D), _p(weight, _D), E_grid.size,
                         _p(E_grid, _D), _p(spec, _D), 1)
    return spec


def reduce_binmean(E_res, a_width, weight, edges):
    E_res, a_width, weight, edges = (_f64(x) for x in (E_res, a_width, weight, edges))
    spec = np.zeros(edges.size - 1)
    lib().or_reduce_binmean(E_res.size, _p(E_res, _D), _p(a_width, _D), _p(weight, _D),
                            edges.size - 1, _p(edges, _D), _p(spec, _D), 1)
    return spec


def sincsq_tail(x):
    return np.array([lib().or_sincsq_tail(float(v)) for v in np.ravel(x)]).reshape(np.shape(x))


def mean_transmission(t0, t1):
    return float(lib().or_mean_transmission(float(t0), float(t1)))


def quantum_line_factors(h, gamma, vdg, k_dot_v, k_dot_g, g2, k2, v_dot_e, g_dot_e, k_dot_e):
    a, b = C.c_double(), C.c_double()
    lib().or_quantum_line_factors(
        *[float(v) for v in (h, gamma, vdg, k_dot_v, k_dot_g, g2, k2, v_dot_e, g_dot_e, k_dot_e)],
        C.byref(a), C.byref(b),
    )
    return a.value, b.value


def energy_bin_edges(E_grid):
    """Bin edges of the bin-mean routes (spectrum/characteristic.py:621-646)."""
    grid = np.asarray(E_grid, dtype=float)
    edges = np.empty(grid.size + 1)
    edges[1:-1] = 0.5 * (grid[:-1] + grid[1:])
    edges[0] = max(0.0, grid[0] - 0.5 * (grid[1] - grid[0]))
    edges[-1] = grid[-1] + 0.5 * (grid[-1] - grid[-2])
    return edges


def brem_spectrum(seg: dict, Z, n_ang3, thickness, n_hat, E_grid, mu_grid, Ne):
    """BH + Elwert track-length spectrum [photons/eV/sr/electron] (brem.py:829-1239)."""
    E = _f64(seg["E_keV"])
    L = _f64(seg["L_ang"])
    r = _f64(seg["r_mid"])
    v = _f64(seg["v_hat"])
    Z = _f64(Z)
    n_ang3 = _f64(n_ang3)
    nh = _f64(n_hat)
    E_grid = _f64(E_grid)
    mu_grid = _f64(mu_grid)
    spec = np.zeros(E_grid.size)
    lib().or_brem_spectrum(E.size, _p(E, _D), _p(L, _D), _p(r, _D), _p(v, _D), int(Z.size),
                           _p(Z, _D), _p(n_ang3, _D), float(thickness), _p(nh, _D), E_grid.size,
                           _p(E_grid, _D), _p(mu_grid, _D), _p(spec, _D), 1)
    return spec / (4.0 * np.pi) / Ne


def brem_spectrum_layered(seg: dict, Z, n_ang3, layers: LayerEscape, n_hat, E_grid, mu_layer, Ne):
    """Layered BH + Elwert spectrum of the given segments (one emitting
    layer's composition Z/n_ang3; brem.py:978-1005,1195-1239)."""
    E = _f64(seg["E_keV"])
    L = _f64(seg["L_ang"])
    r = _f64(seg["r_mid"])
    v = _f64(seg["v_hat"])
    Z = _f64(Z)
    n_ang3 = _f64(n_ang3)
    nh = _f64(n_hat)
    E_grid = _f64(E_grid)
    mu_layer = _f64(np.atleast_2d(mu_layer))
    spec = np.zeros(E_grid.size)
    lib().or_brem_spectrum_layered(E.size, _p(E, _D), _p(L, _D), _p(r, _D), _p(v, _D), int(Z.size), _p(Z, _D),
                                   _p(n_ang3, _D), C.byref(layers.c), _p(nh, _D), E_grid.size, _p(E_grid, _D),
                                   _p(mu_layer, _D), _p(spec, _D), 1)
    return spec / (4.0 * np.pi) / Ne
