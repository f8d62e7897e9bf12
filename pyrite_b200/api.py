"""Python host API mirroring the reference's calls on the hot path.

``simulate_trajectories`` stands where ``_simulate_trajectories`` with a
per-electron core sits (src/pyrite/montecarlo/transport/api.py:19),
``mc_cxr_spectrum`` where the incoherent CXR scorer sits
(spectrum/cxr/_spectrum.py:25) and ``mc_brem_spectrum`` where the
Bethe-Heitler scorer sits (spectrum/brem.py:829); argument names, units and
outputs follow the reference. Device memory and streams come from PyTorch;
every computation runs in ``libpyrite_b200.so`` through its C ABI.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from .tables import (
    CRYSTALS,
    ElsepaGroup,
    LayerStack,
    StoppingTables,
    check_elsepa_range,
    check_stopping_range,
    pack_elsepa,
    pack_stopping,
    beam_entry_basis,
    beam_frame_basis,
    build_transport_lut,
    child_stream_root,
    energy_bin_edges,
    geometric_grid,
    line_keep_window,
    reflection_rows,
)

EXIT_NAMES = ("n_cutoff_stopped", "n_backscattered", "n_transmitted", "n_side_exited",
              "n_step_limited", "n_missed")


def _device(device=None) -> torch.device:
    if device is None:
        if not torch.cuda.is_available():
            raise L.PyriteB200Error("pyrite_b200 needs a CUDA device; none is visible")
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device(device)


class _Holder:
    """Keeps device tensors alive while the C structures point at them."""

    def __init__(self, device):
        self.device = device
        self.keep = []
        self.inputs = []  # device tensors filled from host data (the call's inputs)

    def f64(self, a) -> torch.Tensor:
        t = torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64) if not torch.is_tensor(a) else a)
        t = t.to(self.device, torch.float64).contiguous()
        self.keep.append(t)
        self.inputs.append(t)
        return t

    def typed(self, a, dtype) -> torch.Tensor:
        t = a if torch.is_tensor(a) else torch.as_tensor(np.ascontiguousarray(a))
        t = t.to(self.device, dtype).contiguous()
        self.keep.append(t)
        self.inputs.append(t)
        return t

    def zeros(self, shape, dtype) -> torch.Tensor:
        t = torch.zeros(shape, dtype=dtype, device=self.device)
        self.keep.append(t)
        return t

    def empty(self, shape, dtype) -> torch.Tensor:
        t = torch.empty(shape, dtype=dtype, device=self.device)
        self.keep.append(t)
        return t


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


def _stream_ptr(stream) -> int | None:
    if stream is None:
        stream = torch.cuda.current_stream()
    return stream.cuda_stream


# ---------------------------------------------------------------------------
# Transport
# ---------------------------------------------------------------------------
@dataclass
class BeamSpec:
    """Entrance beam: mono-energetic, optional Gaussian spot or Twiss phase space."""

    E0_keV: float
    beam_dir: np.ndarray | None = None
    tilt_polar_rad: float = 0.0
    tilt_azim_rad: float = 0.0
    beam_fwhm_mm: float | None = None
    beam_fwhm_y_mm: float | None = None
    # (normalized emittance [mm mrad], beta [m], alpha) per plane, as the
    # reference's TransverseDistribution (transverse.py:96-114).
    twiss_x: tuple | None = None
    twiss_y: tuple | None = None


def _fill_layers(h: _Holder, stack: LayerStack) -> L.PbLayers:
    s = L.PbLayers()
    s.n_layers, s.max_el = stack.n_layers, stack.max_el
    s.z_top, s.z_bot = _ptr(h.f64(stack.z_top)), _ptr(h.f64(stack.z_bot))
    s.n_el = _ptr(h.typed(stack.n_el, torch.int32))
    for name in ("J", "k", "coeff", "E_cross", "sr_rate_numer", "sr_joy_numer"):
        setattr(s, name, _ptr(h.f64(getattr(stack, name))))
    return s


def _fill_lut(h: _Holder, lut, precision) -> L.PbLut:
    dtype = np.float32 if precision == L.PB_MIXED else np.float64
    buf, offs = lut.packed(dtype)
    t = h.typed(torch.from_numpy(buf), torch.float32 if dtype == np.float32 else torch.float64)
    s = L.PbLut()
    s.n_energy = lut.n_energy
    s.elem_bytes = np.dtype(dtype).itemsize
    s.log_E_min = float(lut.log_E_min)
    s.inv_dlogE = float(lut.inv_dlogE)
    s.base = _ptr(t)
    s.total_bytes = buf.nbytes
    s.off_total_rate, s.off_dEds = offs["total_rate"], offs["dEds"]
    s.off_inv_beta, s.off_cdf, s.off_alpha = offs["inv_beta"], offs["cdf"], offs["alpha"]
    return s


def _fill_beam(h: _Holder, beam: BeamSpec | None, seed: int, entry=None) -> L.PbBeam:
    b = L.PbBeam()
    if entry is not None:
        pos0, dir0, E0 = entry
        b.mode = L.PB_BEAM_EXPLICIT
        b.pos0, b.dir0, b.E0 = _ptr(h.f64(pos0)), _ptr(h.f64(dir0)), _ptr(h.f64(E0))
        return b
    bd = np.array([0.0, 0.0, 1.0]) if beam.beam_dir is None else np.asarray(beam.beam_dir, float)
    bd = bd / np.linalg.norm(bd)
    b.E0_keV = float(beam.E0_keV)
    b.beam_dir[:] = list(bd)
    e_x, e_y, _ = beam_entry_basis(beam.tilt_polar_rad, beam.tilt_azim_rad)
    b.e_x[:] = list(e_x)
    b.e_y[:] = list(e_y)
    b.tilted = 1 if beam.tilt_polar_rad else 0
    basis = beam_frame_basis(bd)
    b.basis[:] = list(basis.reshape(-1))
    if beam.twiss_x is not None:
        # transverse.py:96-153: geometric emittance from the normalised one.
        gamma_rel = 1.0 + beam.E0_keV / 510.99895
        bg = float(np.sqrt(gamma_rel**2 - 1.0))
        ty = beam.twiss_y if beam.twiss_y is not None else beam.twiss_x
        for dst, (en, beta_m, alpha) in ((b.twiss_x, beam.twiss_x), (b.twiss_y, ty)):
            dst[0] = en * 1e-3 / bg
            dst[1] = beta_m * 1e3
            dst[2] = alpha
        b.mode = L.PB_BEAM_TWISS
        b.root = child_stream_root(seed, 5, 4)
    elif beam.beam_fwhm_mm or beam.beam_fwhm_y_mm:
        f2s = 1.0 / (2.0 * np.sqrt(2.0 * np.log(2.0)))
        fy = beam.beam_fwhm_mm if beam.beam_fwhm_y_mm is None else beam.beam_fwhm_y_mm
        b.sigma_x_ang = float(beam.beam_fwhm_mm or 0.0) * 1.0e7 * f2s
        b.sigma_y_ang = float(fy or 0.0) * 1.0e7 * f2s
        b.mode = L.PB_BEAM_SPOT
        b.root = child_stream_root(seed, 2, 1)
    else:
        b.mode = L.PB_BEAM_SPOT
        b.sigma_x_ang = b.sigma_y_ang = 0.0
        b.root = child_stream_root(seed, 2, 1)
    return b


_RNG = {"splitmix": L.PB_RNG_SPLITMIX, "philox": L.PB_RNG_PHILOX}
_PREC = {"fp64": L.PB_FP64, "mixed": L.PB_MIXED}


def _fill_elsepa(h: "_Holder", g: ElsepaGroup) -> "L.PbElsepa":
    t = L.PbElsepa()
    t.n_mu, t.cells = int(g.mu.size), int(g.guide.shape[1] - 1)
    t.start = _ptr(h.typed(np.asarray(g.start, dtype=np.int64).reshape(-1), torch.int64))
    t.length = _ptr(h.typed(np.asarray(g.length, dtype=np.int64).reshape(-1), torch.int64))
    t.logE, t.log_rate = _ptr(h.f64(g.logE)), _ptr(h.f64(g.log_rate))
    t.cdf, t.pdf, t.mu = _ptr(h.f64(g.cdf)), _ptr(h.f64(g.pdf)), _ptr(h.f64(g.mu))
    t.guide = _ptr(h.typed(np.asarray(g.guide, dtype=np.int32), torch.int32))
    return t


def simulate_trajectories(E0_keV, Ne, thickness_ang=None, element=None, n_atoms_per_ang3=None,
                          E_cut_keV=5.0, seed=0, max_steps=400_000, beam_dir=None,
                          composition=None, layers=None, beam_fwhm_mm=None, beam_fwhm_y_mm=None,
                          tilt_polar_rad=0.0, tilt_azim_rad=0.0, transverse_distribution=None,
                          *, lut=True, rng="splitmix", precision="fp64", entry=None, cap=None,
                          device=None, stream=None, block_threads=0, tallies=None, straggling=False,
                          elastic_model="sr", elastic_tables=None, stopping_tables=None):
    """Transport ``Ne`` electrons into a slab or layer stack; returns segment rows.

    Same contract as the reference's per-electron cores: rows of history i
    in order, true ``seg_count``, exit counts, entrance snapshot. ``lut`` picks
    the reference's default LUT core or its exact analytic core; ``rng`` the
    reference's SplitMix64 counter stream (draw-for-draw compatible) or
    Philox4x32-10; ``precision`` "fp64" or "mixed". ``entry`` replaces the
    sampled entrance state with explicit (pos, dir, E) arrays. ``straggling``
    samples each flight's loss from the Urban model (the reference's
    ``straggling=True``, transport/straggling.py) instead of the
    deterministic midpoint loss.

    ``elastic_model="elsepa"`` samples elastic events from tabulated ELSEPA
    cross sections and angular distributions (the reference's default model,
    scattering.py:330-640): ``elastic_tables`` is either the reference's
    ``elastic_tables`` argument (one list per layer of one mapping per
    element with ``energy_eV``, ``total_elastic_cm2``, ``mu``,
    ``dcs_cm2_sr``) or an already packed ``tables.ElsepaGroup``. As in the
    reference the exact core runs (``lut`` is ignored) and energies outside
    the tables are refused. ``"sr"`` (the default here, since the production
    ELSEPA tables are not shipped) is the analytic screened-Rutherford model.
    ``stopping_tables`` (one SBETHE table per layer, the reference's argument
    of that name) replaces the spliced analytic stopping by the tables'
    log-log interpolation (stopping.py:11-103; exact core, range checked).

    ``tallies=(n_E, n_theta)`` also returns the kernel's fused summary
    tallies, the reference's summary tables (trajectory_summary.py:147-260)
    without materialising rows for them: ``tally_fates`` (counts by exit
    code), ``tally_exit_E`` (escaped primaries' exit energy on n_E bins over
    [0, E0] with under- and overflow) and ``tally_exit_theta`` (exit polar
    angle on n_theta bins over [0, pi]), ``tally_deposit_keV`` (continuous
    loss per layer, summed over the histories).
    """
    lib = L.load()
    if layers is None:
        comp = composition if composition is not None else [(element, n_atoms_per_ang3)]
        layers = [(0.0, float(thickness_ang), list(comp))]
    stack = LayerStack([(float(a), float(b), list(c)) for a, b, c in layers])
    group = None
    if elastic_model == "elsepa":
        if elastic_tables is None:
            raise ValueError("elastic_model='elsepa' needs elastic_tables (the production tables are not shipped)")
        group = elastic_tables if isinstance(elastic_tables, ElsepaGroup) else pack_elsepa(stack, elastic_tables)
        E_hi = float(E0_keV) if entry is None else float(np.max(entry[2]))
        check_elsepa_range(group, stack, float(E_cut_keV), E_hi)
        lut = False  # the exact core, as the reference bypasses its LUT for tabulated elastic scattering
    elif elastic_model != "sr":
        raise ValueError(f"elastic_model must be 'sr' or 'elsepa', not {elastic_model!r}")
    stop = None
    if stopping_tables is not None:
        stop = stopping_tables if isinstance(stopping_tables, StoppingTables) else pack_stopping(stack, stopping_tables)
        E_hi = float(E0_keV) if entry is None else float(np.max(entry[2]))
        check_stopping_range(stop, float(E_cut_keV), E_hi)
        lut = False  # table stopping runs on the exact core
    dev = _device(device)
    h = _Holder(dev)
    a = L.PbTransportArgs()
    a.rng = _RNG[rng]
    a.precision = _PREC[precision]
    a.use_lut = 1 if lut else 0
    a.block_threads = int(block_threads)
    a.seed = int(seed) % 2**64
    a.e_start = 0
    a.n = int(Ne)
    a.E_cut_keV = float(E_cut_keV)
    a.max_steps = int(max_steps)
    a.layers = _fill_layers(h, stack)
    if straggling:
        a.straggling, a.Z = 1, _ptr(h.f64(stack.Z))
    if group is not None:
        a.elastic_model = L.PB_ELASTIC_ELSEPA
        a.elsepa = _fill_elsepa(h, group)
    if stop is not None:
        a.stopping.width = int(stop.logE.shape[1])
        a.stopping.count = _ptr(h.typed(np.asarray(stop.count, dtype=np.int32), torch.int32))
        a.stopping.logE, a.stopping.logS = _ptr(h.f64(stop.logE)), _ptr(h.f64(stop.logS))
    if lut:
        E_hi = float(E0_keV) if entry is None else float(np.max(entry[2]))
        a.lut = _fill_lut(h, build_transport_lut(stack, E_cut_keV, E_hi), a.precision)
    if transverse_distribution is not None:
        tx = transverse_distribution["x"]
        ty = transverse_distribution.get("y", tx)
    else:
        tx = ty = None
    beam = BeamSpec(E0_keV, beam_dir, tilt_polar_rad, tilt_azim_rad, beam_fwhm_mm, beam_fwhm_y_mm, tx, ty)
    a.beam = _fill_beam(h, beam, int(seed), entry)
    cap = int(cap) if cap is not None else 512
    n = int(Ne)
    m = n * cap
    rows = dict(
        r_mid=h.empty((m, 3), torch.float64), v_hat=h.empty((m, 3), torch.float64),
        L_ang=h.empty(m, torch.float64), E_keV=h.empty(m, torch.float64),
        E_end_keV=h.empty(m, torch.float64), t_ang=h.empty(m, torch.float64),
        t_end_ang=h.empty(m, torch.float64), elec_id=h.empty(m, torch.int64),
        layer=h.empty(m, torch.int16), flight_id=h.empty(m, torch.int64),
        event_kind=h.empty(m, torch.int8),
    )
    a.cap = cap
    r = L.PbRows()
    r.r_mid, r.v_hat, r.L = _ptr(rows["r_mid"]), _ptr(rows["v_hat"]), _ptr(rows["L_ang"])
    r.E_start, r.E_end = _ptr(rows["E_keV"]), _ptr(rows["E_end_keV"])
    r.t_start, r.t_end = _ptr(rows["t_ang"]), _ptr(rows["t_end_ang"])
    r.elec_id, r.layer = _ptr(rows["elec_id"]), _ptr(rows["layer"])
    r.flight, r.event = _ptr(rows["flight_id"]), _ptr(rows["event_kind"])
    a.rows = r
    seg_count = h.zeros(n, torch.int64)
    exit_code = h.zeros(n, torch.int8)
    final_E = h.zeros(n, torch.float64)
    a.seg_count, a.exit_code, a.final_E = _ptr(seg_count), _ptr(exit_code), _ptr(final_E)
    wc = h.zeros(1, torch.int64)
    status = h.zeros(1, torch.int32)
    a.work_counter, a.status = _ptr(wc), _ptr(status)
    tal_t = None
    if tallies is not None:
        n_tE, n_tth = (int(x) for x in tallies)
        tal_t = dict(fates=h.zeros(6, torch.int64), exit_E=h.zeros(n_tE + 2, torch.int64),
                     exit_theta=h.zeros(n_tth + 2, torch.int64), deposit=h.zeros(stack.n_layers, torch.float64))
        tal = L.PbTallies()
        tal.fates, tal.exit_E, tal.exit_theta = (_ptr(tal_t[k]) for k in ("fates", "exit_E", "exit_theta"))
        tal.n_E, tal.E_lo, tal.E_hi = n_tE, 0.0, float(E0_keV)
        tal.n_theta, tal.theta_lo, tal.theta_hi = n_tth, 0.0, float(np.pi)
        tal.deposit = _ptr(tal_t["deposit"])
        a.tallies = tal
    L.check(lib.pb_transport(C.byref(a), _stream_ptr(stream)), "pb_transport")
    torch.cuda.synchronize(dev)
    st = int(status.item())
    counts = seg_count.cpu().numpy()
    if int(counts.max(initial=0)) > cap:
        # Exact replay at the measured capacity (batching.py:545-558).
        return simulate_trajectories(
            E0_keV, Ne, thickness_ang, element, n_atoms_per_ang3, E_cut_keV, seed, max_steps,
            beam_dir, composition, layers, beam_fwhm_mm, beam_fwhm_y_mm, tilt_polar_rad,
            tilt_azim_rad, transverse_distribution, lut=lut, rng=rng, precision=precision,
            entry=entry, cap=int(counts.max()), device=device, stream=stream,
            block_threads=block_threads, tallies=tallies, straggling=straggling)
    mask = (np.arange(cap)[None, :] < counts[:, None]).reshape(-1)
    idx = torch.from_numpy(np.flatnonzero(mask)).to(dev)
    out = {k: v.index_select(0, idx).cpu().numpy() for k, v in rows.items()}
    out["E_repr_keV"] = 0.5 * (out["E_keV"] + out["E_end_keV"])
    out["E_start_keV"] = out["E_keV"]
    codes = exit_code.cpu().numpy()
    for code, name in enumerate(EXIT_NAMES):
        out[name] = int(np.count_nonzero(codes == code))
    out["n_missed"] = 0
    out["Ne"] = int(Ne)
    out["thickness_ang"] = stack.thickness
    out["n_layers"] = stack.n_layers
    out["seg_count"] = counts
    out["exit_code"] = codes
    out["final_E_keV"] = final_E.cpu().numpy()
    out["device_status"] = st
    if tal_t is not None:
        for k, v in tal_t.items():
            out[f"tally_{k}" if k != "deposit" else "tally_deposit_keV"] = v.cpu().numpy()
    return out


TRANSPORT_MAX_STEPS = 400_000  # per-history step ceiling (runner/step_budget.py:8-10)


class TransportStepLimitError(L.PyriteB200Error):
    """Some histories reached the step budget at the ceiling."""


def retry_step_budget(simulate, *args, initial_max_steps=TRANSPORT_MAX_STEPS, ceiling=TRANSPORT_MAX_STEPS,
                      **kwargs):
    """Run ``simulate`` (``simulate_trajectories`` or a function with its
    result keys) from ``initial_max_steps``, doubling the budget while any
    history ends step-limited, up to ``ceiling``, where the step limit raises
    ``TransportStepLimitError`` (runner/step_budget.py:33-53). Trajectories
    depend on the seed alone, so a rerun at a doubled budget is exactly the
    run that budget gives from the start."""
    if not 1 <= int(initial_max_steps) <= int(ceiling):
        raise ValueError(f"initial_max_steps must be in [1, {ceiling}]")
    max_steps = int(initial_max_steps)
    while True:
        out = simulate(*args, max_steps=max_steps, **kwargs)
        if int(out.get("n_step_limited", 0)) == 0:
            return out
        if max_steps >= ceiling:
            raise TransportStepLimitError(
                f"{out['n_step_limited']} histories reached the step budget of {max_steps}")
        max_steps = min(2 * max_steps, int(ceiling))


# ---------------------------------------------------------------------------
# Emission scoring
# ---------------------------------------------------------------------------
@dataclass
class LineTables:
    """Data the line scorer reads at each resonance (the reference's data
    seams cxr/_setup.py:962-999 and cxr/_kernels.py:1225-1249): a tabulation
    grid, chi_g and U_g/m per reflection, log(mu) per absorber element and the
    refractive decrement delta = 1 - Re n."""

    E_tab: np.ndarray
    chi_re: np.ndarray
    chi_im: np.ndarray
    u_re: np.ndarray
    u_im: np.ndarray
    log_mu: np.ndarray
    delta: np.ndarray


def _segments_on_device(h: _Holder, segments: dict):
    E_field = "E_repr_keV" if segments.get("E_repr_keV") is not None else "E_keV"
    out = {}
    for key, src in (("r_mid", "r_mid"), ("v_hat", "v_hat"), ("L", "L_ang"), ("E", E_field)):
        v = segments[src]
        out[key] = h.f64(v) if not torch.is_tensor(v) else h.typed(v, torch.float64)
    eid = segments["elec_id"]
    out["elec_id"] = h.typed(eid if torch.is_tensor(eid) else np.asarray(eid, dtype=np.int64), torch.int64)
    out["n"] = int(out["L"].numel())
    return out


MAX_ESCAPE_LAYERS = 4


def _escape_layers(layers):
    """(z_top, z_bot) of a layered absorber given as the reference's
    ``layers`` list of (z_top, z_bot, composition); contiguous, in depth
    order, at most MAX_ESCAPE_LAYERS."""
    z_top = np.array([float(l[0]) for l in layers])
    z_bot = np.array([float(l[1]) for l in layers])
    if not 1 <= z_top.size <= MAX_ESCAPE_LAYERS:
        raise ValueError(f"layered escape supports 1..{MAX_ESCAPE_LAYERS} layers, got {z_top.size}")
    if np.any(z_bot <= z_top) or np.any(np.abs(z_bot[:-1] - z_top[1:]) > 1e-9 * np.maximum(1.0, np.abs(z_bot[:-1]))):
        raise ValueError("layers must be contiguous [z_top, z_bot) intervals in depth order")
    return z_top, z_bot


def _seg_layer(h: _Holder, segments: dict, emit_layer):
    if emit_layer is None:
        return None
    lay = segments["layer"]
    return h.typed(lay if torch.is_tensor(lay) else np.asarray(lay, dtype=np.int32), torch.int32)


def _fill_tables(h: _Holder, rows, tables: LineTables, lo_keep, hi_keep, d_index=None):
    t = L.PbCxrTables()
    t.n_g = int(rows.G.shape[0])
    t.G = _ptr(h.f64(rows.G))
    t.WM = _ptr(h.f64(rows.WM))
    t.row_table = _ptr(h.typed(rows.row_table, torch.int32))
    t.n_tab = int(np.asarray(tables.E_tab).size)
    t.E_tab = _ptr(h.f64(tables.E_tab))
    for name in ("chi_re", "chi_im", "u_re", "u_im"):
        setattr(t, name, _ptr(h.f64(getattr(tables, name))))
    lm = np.atleast_2d(np.asarray(tables.log_mu, dtype=np.float64))
    t.n_mu = int(lm.shape[0])
    t.log_mu = _ptr(h.f64(lm))
    t.delta = _ptr(h.f64(tables.delta))
    t.lo_keep, t.hi_keep = float(lo_keep), float(hi_keep)
    t.tab_log0, t.tab_log_step = geometric_grid(tables.E_tab)
    t.delta_tail_absmax = _ptr(h.f64(np.maximum.accumulate(np.abs(np.asarray(tables.delta, float))[::-1])[::-1]))
    return t


def mc_cxr_spectrum(segments, E_grid_eV, crystal, hkl_list, *, tables: LineTables, n_hat,
                    surface_hkl=None, beam_uvw=None, azimuth_rad=0.0, mosaic_fwhm_rad=None,
                    mosaic_nodes=1, line_quadrature="node", precision="fp64", exact_widths=None,
                    rows=None, return_pairs=False, layers=None, mu_tables=None, emit_layer=None,
                    device=None, stream=None):
    """Per-electron incoherent PXR + CBS density [photons/eV/sr/electron].

    ``n_hat`` is one direction (3,) or several (n_dir, 3); the result is then
    (n_dir, n_E). ``exact_widths`` (bin-mean) keeps exact bin integrals within
    that many sinc widths of each line and the far envelope beyond; None is
    exact everywhere.

    ``layers`` (the reference's list of (z_top, z_bot, composition)) makes the
    escape run through a layered absorber, with ``mu_tables`` one
    (knots [eV], values, slopes [per eV]) piecewise-linear attenuation per
    layer (cxr/_escape_mu.py:41-57); ``emit_layer`` keeps only the segments
    of that layer (``segments["layer"]``) radiating, as the reference scores
    each crystalline layer of a stack (runner/case_driver.py:742-770).
    """
    dev = _device(device)
    lib = L.load()
    h = _Holder(dev)
    cr = CRYSTALS[crystal] if isinstance(crystal, str) else crystal
    n_hats = np.atleast_2d(np.asarray(n_hat, dtype=float))
    n_hats = n_hats / np.linalg.norm(n_hats, axis=1, keepdims=True)
    single = np.asarray(n_hat).ndim == 1
    if rows is None:
        rows = reflection_rows(cr, hkl_list, n_hats, surface_hkl=surface_hkl, beam_uvw=beam_uvw,
                               azimuth_rad=azimuth_rad, mosaic_fwhm_rad=mosaic_fwhm_rad,
                               mosaic_nodes=mosaic_nodes)
    seg = _segments_on_device(h, segments)
    E_grid = np.asarray(E_grid_eV, dtype=np.float64)
    lo_keep, hi_keep = line_keep_window(E_grid)
    n_dir = n_hats.shape[0]
    n_E = int(E_grid.size)
    quad = L.PB_QUAD_BINMEAN if line_quadrature == "bin-mean" else L.PB_QUAD_NODE
    spec = h.zeros((n_dir, n_E), torch.float64)
    status = h.zeros(1, torch.int32)
    n_g = int(rows.G.shape[0])
    pairs = None
    out = np.zeros((n_dir, n_E))
    pair_out = []
    for d in range(n_dir):
        a = L.PbCxrArgs()
        a.precision = _PREC[precision]
        a.quadrature = quad
        a.n_dir = 1
        a.n_hat = _ptr(h.f64(n_hats[d]))
        a.thickness = float(segments["thickness_ang"])
        a.Ne = int(segments["Ne"])
        a.n_seg = seg["n"]
        a.r_mid, a.v_hat, a.L = _ptr(seg["r_mid"]), _ptr(seg["v_hat"]), _ptr(seg["L"])
        a.E_keV, a.elec_id = _ptr(seg["E"]), _ptr(seg["elec_id"])
        t = _fill_tables(h, rows, tables, lo_keep, hi_keep)
        t.ES = _ptr(h.f64(rows.ES[d]))
        t.EP = _ptr(h.f64(rows.EP[d]))
        a.tables = t
        if layers is not None:
            z_top, z_bot = _escape_layers(layers)
            if mu_tables is None or len(mu_tables) != z_top.size:
                raise ValueError("a layered absorber needs one mu table per layer")
            a.n_layer = int(z_top.size)
            a.z_top, a.z_bot = _ptr(h.f64(z_top)), _ptr(h.f64(z_bot))
            a.mu_off = _ptr(h.typed(np.cumsum([0] + [len(k) for k, _v, _s in mu_tables]).astype(np.int32), torch.int32))
            a.mu_knot = _ptr(h.f64(np.concatenate([np.asarray(k, float) for k, _v, _s in mu_tables])))
            a.mu_value = _ptr(h.f64(np.concatenate([np.asarray(v, float) for _k, v, _s in mu_tables])))
            a.mu_slope = _ptr(h.f64(np.concatenate([np.asarray(sl, float) for _k, _v, sl in mu_tables])))
        sl_t = _seg_layer(h, segments, emit_layer)
        if sl_t is not None:
            a.seg_layer, a.emit_layer = _ptr(sl_t), int(emit_layer)
        a.n_E = n_E
        a.E_grid = _ptr(h.f64(E_grid))
        spec_d = h.zeros(n_E, torch.float64)
        a.spec = _ptr(spec_d)
        a.status = _ptr(status)
        if quad == L.PB_QUAD_BINMEAN:
            edges = energy_bin_edges(E_grid)
            a.edges = _ptr(h.f64(edges))
            w = np.diff(edges)
            uniform = np.allclose(w, w[0], rtol=1e-9, atol=0.0)
            if exact_widths is not None and exact_widths > 0 and uniform:
                a.exact_widths = float(exact_widths)
                pad = int(np.ceil(max(edges[0] - lo_keep, hi_keep - edges[-1]) / w[0])) + 2
                a.far_pad = pad
                a.far_moments = _ptr(h.zeros((n_E + 2 * pad) * 3, torch.float64))
            else:
                a.exact_widths = 0.0
                a.far_pad = -1
        else:
            cap = max(1, seg["n"] * n_g)
            a.line_capacity = cap
            a.line_count = _ptr(h.zeros(1, torch.int64))
            a.line_E, a.line_a = _ptr(h.empty(cap, torch.float64)), _ptr(h.empty(cap, torch.float64))
            a.line_w = _ptr(h.empty(cap, torch.float64))
            a.line_dir = _ptr(h.zeros(cap, torch.int32))
        if return_pairs:
            m = seg["n"] * n_g
            pe, pa, pw = (h.empty(m, torch.float64) for _ in range(3))
            pg = h.zeros(m, torch.uint8)
            a.pair_E, a.pair_a, a.pair_w, a.pair_good = _ptr(pe), _ptr(pa), _ptr(pw), _ptr(pg)
            pair_out.append((pe, pa, pw, pg))
        L.check(lib.pb_cxr_score(C.byref(a), _stream_ptr(stream)), "pb_cxr_score")
        torch.cuda.synchronize(dev)
        out[d] = spec_d.cpu().numpy()
    out /= int(segments["Ne"])
    result = out[0] if single else out
    if return_pairs:
        pairs = [tuple(x.cpu().numpy() for x in p) for p in pair_out]
        return result, pairs
    return result


def mc_brem_spectrum(segments, E_grid_eV, *, composition, n_hat, mu=None, precision="fp64",
                     layers=None, mu_layer=None, emit_layer=None, device=None, stream=None, depth_nodes=True):
    """Bethe-Heitler + Elwert continuum density [photons/eV/sr/electron].

    ``mu`` is the absorber's total attenuation [1/Angstrom] on ``E_grid_eV``
    (the reference reads EPDL, brem.py:961-963; the tables are an input here).
    ``layers`` (the reference's list of (z_top, z_bot, composition)) with
    ``mu_layer`` [n_layer, n_E] makes the escape run through a layered
    absorber (brem.py:978-1005); ``composition`` is then the emitting layer's
    and ``emit_layer`` keeps only that layer's segments radiating
    (runner/emission.py:155-172).

    ``depth_nodes`` (mixed precision, single slab, one or two elements) lets
    the scorer take the segments of the batch's top electron-energy window
    in the depth-node form; False keeps the per-(segment, energy) form for
    every segment.
    """
    from .tables import ELEMENTS

    dev = _device(device)
    lib = L.load()
    h = _Holder(dev)
    seg = _segments_on_device(h, segments)
    n_hats = np.atleast_2d(np.asarray(n_hat, dtype=float))
    n_hats = n_hats / np.linalg.norm(n_hats, axis=1, keepdims=True)
    single = np.asarray(n_hat).ndim == 1
    E_grid = np.asarray(E_grid_eV, dtype=np.float64)
    n_dir, n_E = n_hats.shape[0], int(E_grid.size)
    a = L.PbBremArgs()
    a.precision = _PREC[precision]
    a.n_dir = n_dir
    a.n_hat = _ptr(h.f64(n_hats))
    a.thickness = float(segments["thickness_ang"])
    a.Ne = int(segments["Ne"])
    a.n_seg = seg["n"]
    a.r_mid, a.v_hat, a.L = _ptr(seg["r_mid"]), _ptr(seg["v_hat"]), _ptr(seg["L"])
    a.E_keV, a.elec_id = _ptr(seg["E"]), _ptr(seg["elec_id"])
    a.n_el = len(composition)
    a.Z = _ptr(h.f64([float(ELEMENTS[el][0]) for el, _ in composition]))
    a.n_ang3 = _ptr(h.f64([float(n) for _, n in composition]))
    a.n_E = n_E
    a.E_grid = _ptr(h.f64(E_grid))
    if layers is None:
        if mu is None:
            raise ValueError("a single slab needs mu")
        a.mu = _ptr(h.f64(mu))
    else:
        z_top, z_bot = _escape_layers(layers)
        ml = np.atleast_2d(np.asarray(mu_layer, dtype=np.float64))
        if ml.shape != (z_top.size, n_E):
            raise ValueError(f"mu_layer must be [{z_top.size}, {n_E}]")
        a.n_layer = int(z_top.size)
        a.z_top, a.z_bot = _ptr(h.f64(z_top)), _ptr(h.f64(z_bot))
        a.mu_layer = _ptr(h.f64(ml))
    sl_t = _seg_layer(h, segments, emit_layer)
    if sl_t is not None:
        a.seg_layer, a.emit_layer = _ptr(sl_t), int(emit_layer)
    spec = h.zeros((n_dir, n_E), torch.float64)
    a.spec = _ptr(spec)
    a.status = _ptr(h.zeros(1, torch.int32))
    if depth_nodes:
        nb = C.c_int64(0)
        L.check(lib.pb_brem_work_size(C.byref(a), C.byref(nb)), "pb_brem_work_size")
        if nb.value > 0:
            a.work, a.work_bytes = _ptr(h.empty(int(nb.value), torch.uint8)), int(nb.value)
    L.check(lib.pb_brem_score(C.byref(a), _stream_ptr(stream)), "pb_brem_score")
    torch.cuda.synchronize(dev)
    out = spec.cpu().numpy() / (4.0 * np.pi) / int(segments["Ne"])
    return out[0] if single else out


# ---------------------------------------------------------------------------
# Characteristic lines (pyrite/montecarlo/spectrum/characteristic.py:1033)
# ---------------------------------------------------------------------------
CHARACTERISTIC_TRANSPORT_FLOOR_KEV = 1.0


@dataclass
class CharacteristicLines:
    """Line data of one emitting element, as the reference derives it from
    EEDL/EADL/xraydb (``characteristic.py:111-160``): per-shell ionisation
    tables (projectile energy [eV] ascending, cross section [cm^2]), line
    energies and natural FWHMs [eV], and ``response[shell, line]``, the
    photons of each line per primary vacancy in each shell after the cascade.
    """

    shell_E: tuple
    shell_sigma: tuple
    line_E: np.ndarray
    line_fwhm: np.ndarray
    response: np.ndarray
    recommended_cutoff_eV: float = 50.0


def characteristic_bin_edges(E_grid_eV):
    """Edges and widths of the characteristic bins (``characteristic.py:621-646``):
    midpoints inside, reflected half-widths outside, the low edge clamped at 0."""
    g = np.asarray(E_grid_eV, dtype=float)
    if g.ndim != 1 or g.size < 2 or not np.all(np.isfinite(g)) or np.any(np.diff(g) <= 0.0):
        raise ValueError("characteristic energy-bin centres must be >= 2 finite, strictly increasing values")
    edges = np.empty(g.size + 1)
    edges[1:-1] = 0.5 * (g[:-1] + g[1:])
    edges[0] = max(0.0, g[0] - 0.5 * (g[1] - g[0]))
    edges[-1] = g[-1] + 0.5 * (g[-1] - g[-2])
    return edges, np.diff(edges)


def lorentzian_bin_weights(edges_eV, line_energy_eV, fwhm_eV):
    """Exact in-window bin masses of a Lorentzian normalised on all energies
    (``characteristic.py:649-680``); the tail outside the window is not
    redistributed."""
    if not (np.isfinite(fwhm_eV) and fwhm_eV > 0.0 and np.isfinite(line_energy_eV) and line_energy_eV > 0.0):
        raise ValueError("line energy and FWHM must be finite and positive")
    gamma = 0.5 * float(fwhm_eV)
    e = np.asarray(edges_eV, dtype=float)
    w = (np.arctan((e[1:] - line_energy_eV) / gamma) - np.arctan((e[:-1] - line_energy_eV) / gamma)) / np.pi
    w = np.maximum(w, 0.0)
    if not np.all(np.isfinite(w)):
        raise ValueError("Lorentzian line has no finite mass on the requested energy grid")
    return w


def prepare_characteristic_lines(lines: CharacteristicLines, E_grid_eV, relaxation_cutoff_eV=None):
    """Kept line indices and their per-eV profiles ``[n_kept, n_bin]``
    (``_prepare_lines``, ``characteristic.py:935-990``): lines above the
    relaxation cutoff, fed by some shell, with mass on the grid."""
    cutoff = lines.recommended_cutoff_eV if relaxation_cutoff_eV is None else float(relaxation_cutoff_eV)
    if cutoff < lines.recommended_cutoff_eV:
        raise ValueError(f"relaxation_cutoff_eV={cutoff:g} is below the data's minimum "
                         f"{lines.recommended_cutoff_eV:g} eV")
    edges, widths = characteristic_bin_edges(E_grid_eV)
    response = np.asarray(lines.response, dtype=float)
    kept, profiles = [], []
    for j, (E, fwhm) in enumerate(zip(lines.line_E, lines.line_fwhm)):
        if E <= cutoff or not np.any(response[:, j] > 0.0):
            continue
        w = lorentzian_bin_weights(edges, float(E), float(fwhm))
        if not np.any(w > 0.0):
            continue
        kept.append(j)
        profiles.append(w / widths)
    return np.asarray(kept, dtype=np.int64), (np.stack(profiles) if profiles else np.zeros((0, widths.size)))


def mc_characteristic_spectrum(segments, E_grid_eV, *, lines: CharacteristicLines, n_atoms_per_ang3, n_hat,
                               mu_by_line, layers=None, relaxation_cutoff_eV=None, E_cut_keV=None,
                               precision="fp64", emit_layer=None, device=None, stream=None,
                               return_yields=False):
    """Characteristic X-ray density [photons/eV/sr/electron] of one emitting element.

    ``mu_by_line[k, j]`` is the attenuation [1/Angstrom] of absorber layer k
    (one row for the single slab) at line j's energy (the reference reads
    EPDL, ``characteristic.py:975-985``); ``layers`` is the absorber stack as
    ``(z_top, z_bot)`` bounds in Angstrom, or None for the slab of
    ``segments["thickness_ang"]``. Segments are expected above the 1 keV
    transport floor already (a transport cutoff >= 1 keV makes the
    reference's clipping the identity). ``emit_layer`` keeps only the
    segments of that layer (``segments["layer"]``) emitting.
    """
    if E_cut_keV is not None and float(E_cut_keV) < CHARACTERISTIC_TRANSPORT_FLOOR_KEV:
        raise ValueError("characteristic scoring requires E_cut_keV >= 1 keV")
    kept, profiles = prepare_characteristic_lines(lines, E_grid_eV, relaxation_cutoff_eV)
    n_hats = np.atleast_2d(np.asarray(n_hat, dtype=float))
    n_hats = n_hats / np.linalg.norm(n_hats, axis=1, keepdims=True)
    single = np.asarray(n_hat).ndim == 1
    n_dir, n_E = n_hats.shape[0], profiles.shape[1]
    Ne = int(segments["Ne"])
    if kept.size == 0:
        out = np.zeros((n_dir, n_E))
        return out[0] if single else out
    dev = _device(device)
    lib = L.load()
    h = _Holder(dev)
    seg = _segments_on_device(h, segments)
    mu = np.atleast_2d(np.asarray(mu_by_line, dtype=float))[:, kept]
    n_layer = 0 if layers is None else len(layers)
    if mu.shape[0] != max(n_layer, 1):
        raise ValueError("mu_by_line needs one row per absorber layer (one for the slab)")
    offs = np.cumsum([0] + [int(np.size(e)) for e in lines.shell_E]).astype(np.int64)
    a = L.PbCharArgs()
    a.precision = _PREC[precision]
    a.n_dir = n_dir
    a.n_hat = _ptr(h.f64(n_hats))
    a.thickness = float(segments.get("thickness_ang", 0.0) or 0.0)
    a.n_layer = n_layer
    if n_layer:
        a.z_top = _ptr(h.f64([float(l[0]) for l in layers]))
        a.z_bot = _ptr(h.f64([float(l[1]) for l in layers]))
    a.Ne = Ne
    a.n_seg = seg["n"]
    a.r_mid, a.v_hat, a.L = _ptr(seg["r_mid"]), _ptr(seg["v_hat"]), _ptr(seg["L"])
    a.E_keV, a.elec_id = _ptr(seg["E"]), _ptr(seg["elec_id"])
    a.n_atoms = float(n_atoms_per_ang3)
    a.n_shell = len(lines.shell_E)
    a.shell_E = _ptr(h.f64(np.concatenate([np.asarray(e, float) for e in lines.shell_E])))
    a.shell_sigma = _ptr(h.f64(np.concatenate([np.asarray(v, float) for v in lines.shell_sigma])))
    a.shell_offset = _ptr(h.typed(offs, torch.int64))
    a.n_line = int(kept.size)
    a.response = _ptr(h.f64(np.asarray(lines.response, float)[:, kept]))
    a.mu = _ptr(h.f64(mu))
    yields = h.zeros((n_dir, int(kept.size)), torch.float64)
    a.line_yield = _ptr(yields)
    a.status = _ptr(h.zeros(1, torch.int32))
    sl_t = _seg_layer(h, segments, emit_layer)
    if sl_t is not None:
        a.seg_layer, a.emit_layer = _ptr(sl_t), int(emit_layer)
    s = _stream_ptr(stream)
    L.check(lib.pb_char_yields(C.byref(a), s), "pb_char_yields")
    spec = h.zeros((n_dir, n_E), torch.float64)
    L.check(lib.pb_char_spectrum(n_dir, int(kept.size), n_E, _ptr(yields), _ptr(h.f64(profiles)), _ptr(spec), s),
            "pb_char_spectrum")
    torch.cuda.synchronize(dev)
    out = spec.cpu().numpy() / (4.0 * np.pi) / Ne
    out = out[0] if single else out
    if return_yields:
        y = yields.cpu().numpy()
        return out, (y[0] if single else y), kept
    return out
