"""Device-resident transport + scoring pipeline: one case, many history batches.

``ScoringCase`` builds every table of a case once in device memory and then
runs batches of histories with no host synchronisation inside a batch:

    pb_transport  (persistent kernel, compact segment list + exit tallies)
      -> pb_cxr_score  (PXR + CBS lines of every segment x reflection x
                        detector tile, bin means deposited on chip)
      -> pb_brem_score (Bethe-Heitler continuum, every tile)

The segment list lives in HBM between the kernels; its length is read on the
device (``n_seg_device``), so the host only sizes the buffer. Spectra and
tallies accumulate across batches and are additive over history ranges, so a
run is resumable by summing completed ranges (the reference's streamed
block scoring, src/pyrite/montecarlo/runner/streamed_scoring.py:105-441).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from .api import BeamSpec, LineTables, _fill_beam, _fill_layers, _fill_lut, _Holder, _ptr
from .tables import (
    ELEMENTS,
    Crystal,
    LayerStack,
    build_transport_lut,
    energy_bin_edges,
    geometric_grid,
    line_keep_window,
    reflection_rows,
)

_PREC = {"fp64": L.PB_FP64, "mixed": L.PB_MIXED}
_RNG = {"splitmix": L.PB_RNG_SPLITMIX, "philox": L.PB_RNG_PHILOX}


@dataclass
class Radiator:
    """A crystalline layer of a stack and its PXR/CBS reflections; the layer's
    segments radiate its lines, which escape through the whole stack
    (runner/case_driver.py:742-770)."""

    layer: int
    crystal: Crystal
    hkl_list: list
    line_tables: LineTables
    surface_hkl: tuple | None = None
    recip_miscut_rad: tuple | None = None
    mosaic_fwhm_rad: float | None = None
    mosaic_nodes: int = 1


@dataclass
class CharEmitter:
    """One element's characteristic lines, emitted by the segments of its
    layer (``layer`` None: every segment) and escaping through the stack;
    ``mu_by_line[k, j]`` the attenuation of layer k at line j
    (characteristic.py:975-985)."""

    lines: object                 # api.CharacteristicLines
    n_atoms_per_ang3: float
    mu_by_line: np.ndarray
    layer: int | None = None


@dataclass
class CaseSpec:
    """One beam/crystal scene: a single crystal slab, or a layered stack with
    per-layer radiators, bremsstrahlung compositions and characteristic
    emitters (``radiators`` / ``brem_layers`` / ``char_emitters``)."""

    stack: LayerStack
    beam: BeamSpec
    E_cut_keV: float
    crystal: Crystal
    hkl_list: list
    n_hats: np.ndarray             # (n_dir, 3) sample-frame detector directions
    E_grid: np.ndarray             # spectral nodes [eV]
    line_tables: LineTables
    surface_hkl: tuple | None = None
    mosaic_fwhm_rad: float | None = None
    mosaic_nodes: int = 1
    brem_composition: list | None = None
    brem_mu: np.ndarray | None = None  # [1/Angstrom] on E_grid
    exact_widths: float = 64.0
    seed: int = 0
    # Detector plane and angular tiling behind n_hats (the surrogate's pixel
    # coordinates); None when the directions were given directly.
    detector: object | None = None
    angular_shape: tuple | None = None
    # Layered stack (the reference's layer_radiators / abs_layers cases): the
    # CXR escape runs through every layer with its exact mu(E) table
    # (knots, values, slopes per layer), each layer radiates bremsstrahlung
    # with its own composition and mu_layer [n_layer, n_E].
    radiators: list | None = None
    escape_mu_tables: list | None = None
    brem_layers: list | None = None
    brem_mu_layer: np.ndarray | None = None
    char_emitters: list | None = None
    # Urban energy-loss straggling per flight (transport/straggling.py).
    straggling: bool = False


class ScoringCase:
    def __init__(self, spec: CaseSpec, *, precision="mixed", rng="philox", lut=True,
                 batch_histories=1 << 17, segs_per_history=48, device=None,
                 exit_E_bins=64, exit_theta_bins=36, max_steps=400_000):
        self.spec = spec
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.lib = L.load()
        self.h = h = _Holder(self.device)
        self.precision = _PREC[precision]
        self.batch = int(batch_histories)
        st = spec.stack
        # ---- transport arguments (fixed across batches except e_start/n) ----
        a = L.PbTransportArgs()
        a.rng = _RNG[rng]
        a.precision = self.precision
        a.use_lut = 1 if lut else 0
        a.seed = int(spec.seed) % 2**64
        a.E_cut_keV = float(spec.E_cut_keV)
        a.max_steps = int(max_steps)
        a.layers = _fill_layers(h, st)
        if spec.straggling:
            a.straggling, a.Z = 1, _ptr(h.f64(st.Z))
        if lut:
            a.lut = _fill_lut(h, build_transport_lut(st, spec.E_cut_keV, spec.beam.E0_keV), self.precision)
        a.beam = _fill_beam(h, spec.beam, int(spec.seed))
        cap = int(self.batch * segs_per_history)
        self.seg_capacity = cap
        self.seg_count = h.zeros(1, torch.int64)
        seg = L.PbSegments()
        seg.capacity = cap
        seg.count = _ptr(self.seg_count)
        self.seg_r = h.empty((cap, 3), torch.float64)
        self.seg_v = h.empty((cap, 3), torch.float64)
        self.seg_L = h.empty(cap, torch.float64)
        self.seg_E = h.empty(cap, torch.float64)
        self.seg_id = h.empty(cap, torch.int64)
        self.seg_layer = h.empty(cap, torch.int32)
        seg.r_mid, seg.v_hat, seg.L = _ptr(self.seg_r), _ptr(self.seg_v), _ptr(self.seg_L)
        seg.E_repr, seg.elec_id, seg.layer = _ptr(self.seg_E), _ptr(self.seg_id), _ptr(self.seg_layer)
        a.seg = seg
        tal = L.PbTallies()
        self.fates = h.zeros(6, torch.int64)
        self.exit_E = h.zeros(exit_E_bins + 2, torch.int64)
        self.exit_theta = h.zeros(exit_theta_bins + 2, torch.int64)
        self.deposit = h.zeros(st.n_layers, torch.float64)
        tal.fates, tal.exit_E, tal.exit_theta = _ptr(self.fates), _ptr(self.exit_E), _ptr(self.exit_theta)
        tal.n_E, tal.E_lo, tal.E_hi = exit_E_bins, 0.0, float(spec.beam.E0_keV)
        tal.n_theta, tal.theta_lo, tal.theta_hi = exit_theta_bins, 0.0, float(np.pi)
        tal.deposit = _ptr(self.deposit)
        a.tallies = tal
        self.work = h.zeros(1, torch.int64)
        self.status = h.zeros(1, torch.int32)
        a.work_counter, a.status = _ptr(self.work), _ptr(self.status)
        self.targs = a
        # ---- CXR scorer (one argument set per radiator) ----
        n_hats = np.atleast_2d(np.asarray(spec.n_hats, dtype=float))
        self.n_dir = n_hats.shape[0]
        E_grid = np.asarray(spec.E_grid, dtype=np.float64)
        self.n_E = int(E_grid.size)
        self._n_hat_dev = h.f64(n_hats)
        self._E_grid_dev = h.f64(E_grid)
        self.spec_cxr = h.zeros((self.n_dir, self.n_E), torch.float64)
        self.far = None
        self.layered = spec.radiators is not None
        if self.layered:
            z_top = np.array([l[0] for l in st.layers], dtype=float)
            z_bot = np.array([l[1] for l in st.layers], dtype=float)
            self._z_top, self._z_bot = h.f64(z_top), h.f64(z_bot)
            mt = spec.escape_mu_tables
            if mt is None or len(mt) != st.n_layers:
                raise ValueError("a stack needs one escape mu table per layer")
            self._mu_off = h.typed(np.cumsum([0] + [len(k) for k, _v, _s in mt]).astype(np.int32), torch.int32)
            self._mu_knot = h.f64(np.concatenate([np.asarray(k, float) for k, _v, _s in mt]))
            self._mu_value = h.f64(np.concatenate([np.asarray(v, float) for _k, v, _s in mt]))
            self._mu_slope = h.f64(np.concatenate([np.asarray(sl, float) for _k, _v, sl in mt]))
            radiators = list(spec.radiators)
        else:
            radiators = [Radiator(-1, spec.crystal, spec.hkl_list, spec.line_tables, spec.surface_hkl, None,
                                  spec.mosaic_fwhm_rad, spec.mosaic_nodes)]
        self.cargs_all = [self._cxr_args(r, n_hats, E_grid, cap) for r in radiators]
        self.cargs = self.cargs_all[0]
        self.rows = self._rows[0]
        # ---- brem scorer (one argument set per emitting layer) ----
        self.bargs = None
        self.bargs_all = []
        self.brem_work = []  # depth-node workspaces of the mixed single-slab brem scorer
        brem_sets = []
        if spec.brem_layers:
            brem_sets = [(k, comp) for k, comp in enumerate(spec.brem_layers) if comp]
        elif spec.brem_composition:
            brem_sets = [(None, spec.brem_composition)]
        if brem_sets:
            self.spec_brem = h.zeros((self.n_dir, self.n_E), torch.float64)
            mu_layer = None
            if spec.brem_layers:
                mu_layer = h.f64(np.asarray(spec.brem_mu_layer, dtype=np.float64).reshape(st.n_layers, self.n_E))
                if st.n_layers > 4:
                    raise ValueError("layered bremsstrahlung supports up to 4 layers")
            for k, comp in brem_sets:
                b = L.PbBremArgs()
                b.precision = self.precision
                b.n_dir = self.n_dir
                b.n_hat = _ptr(self._n_hat_dev)
                b.thickness = st.thickness
                b.Ne = 1 << 62
                b.n_seg = cap
                b.r_mid, b.v_hat, b.L = _ptr(self.seg_r), _ptr(self.seg_v), _ptr(self.seg_L)
                b.E_keV, b.elec_id = _ptr(self.seg_E), _ptr(self.seg_id)
                b.n_seg_device = _ptr(self.seg_count)
                b.n_el = len(comp)
                b.Z = _ptr(h.f64([float(ELEMENTS[el][0]) for el, _ in comp]))
                b.n_ang3 = _ptr(h.f64([float(n) for _, n in comp]))
                b.n_E = self.n_E
                b.E_grid = _ptr(self._E_grid_dev)
                if mu_layer is None:
                    b.mu = _ptr(h.f64(spec.brem_mu))
                else:
                    b.n_layer = st.n_layers
                    b.z_top, b.z_bot = _ptr(self._z_top), _ptr(self._z_bot)
                    b.mu_layer = _ptr(mu_layer)
                    b.seg_layer, b.emit_layer = _ptr(self.seg_layer), int(k)
                b.spec = _ptr(self.spec_brem)
                b.status = _ptr(self.status)
                # workspace of the depth-node form (mixed single slab; 0 bytes elsewhere)
                nb = C.c_int64(0)
                L.check(self.lib.pb_brem_work_size(C.byref(b), C.byref(nb)), "pb_brem_work_size")
                if nb.value > 0:
                    wk = h.empty(int(nb.value), torch.uint8)
                    b.work, b.work_bytes = _ptr(wk), int(nb.value)
                    self.brem_work.append(wk)
                self.bargs_all.append(b)
            self.bargs = self.bargs_all[0]
        # ---- characteristic lines (one argument set per emitter) ----
        self.chargs_all = []
        self.char_yields = []
        self.char_profiles = []
        if spec.char_emitters:
            from .api import prepare_characteristic_lines

            self.spec_char = h.zeros((self.n_dir, self.n_E), torch.float64)
            layered = st.n_layers > 1
            for em in spec.char_emitters:
                kept, profiles = prepare_characteristic_lines(em.lines, E_grid)
                if kept.size == 0:
                    continue
                ch = L.PbCharArgs()
                ch.precision = self.precision
                ch.n_dir = self.n_dir
                ch.n_hat = _ptr(self._n_hat_dev)
                ch.thickness = st.thickness
                mu = np.atleast_2d(np.asarray(em.mu_by_line, dtype=float))[:, kept]
                if layered:
                    ch.n_layer = st.n_layers
                    ch.z_top = _ptr(h.f64([l[0] for l in st.layers]))
                    ch.z_bot = _ptr(h.f64([l[1] for l in st.layers]))
                ch.Ne = 1 << 62
                ch.n_seg = cap
                ch.r_mid, ch.v_hat, ch.L = _ptr(self.seg_r), _ptr(self.seg_v), _ptr(self.seg_L)
                ch.E_keV, ch.elec_id = _ptr(self.seg_E), _ptr(self.seg_id)
                ch.n_seg_device = _ptr(self.seg_count)
                ch.n_atoms = float(em.n_atoms_per_ang3)
                ch.n_shell = len(em.lines.shell_E)
                offs = np.cumsum([0] + [int(np.size(e)) for e in em.lines.shell_E]).astype(np.int64)
                ch.shell_E = _ptr(h.f64(np.concatenate([np.asarray(e, float) for e in em.lines.shell_E])))
                ch.shell_sigma = _ptr(h.f64(np.concatenate([np.asarray(v, float) for v in em.lines.shell_sigma])))
                ch.shell_offset = _ptr(h.typed(offs, torch.int64))
                ch.n_line = int(kept.size)
                ch.response = _ptr(h.f64(np.asarray(em.lines.response, float)[:, kept]))
                ch.mu = _ptr(h.f64(mu))
                y = h.zeros((self.n_dir, int(kept.size)), torch.float64)
                ch.line_yield = _ptr(y)
                ch.status = _ptr(self.status)
                if em.layer is not None:
                    ch.seg_layer, ch.emit_layer = _ptr(self.seg_layer), int(em.layer)
                self.chargs_all.append(ch)
                self.char_yields.append(y)
                self.char_profiles.append(h.f64(profiles))
        self.histories = 0

    def _cxr_args(self, rad: Radiator, n_hats, E_grid, cap, spec_out=None):
        """pb_cxr_args of one radiator over the case's segment buffer; with
        ``spec_out`` a separate argument set for the directions ``n_hats``
        (a subset of the case's) writing into ``spec_out`` [len(n_hats), n_E]
        with a far-field workspace of its own."""
        h, spec, st = self.h, self.spec, self.spec.stack
        rows = reflection_rows(rad.crystal, rad.hkl_list, n_hats, surface_hkl=rad.surface_hkl,
                               mosaic_fwhm_rad=rad.mosaic_fwhm_rad, mosaic_nodes=rad.mosaic_nodes,
                               recip_miscut_rad=rad.recip_miscut_rad)
        if spec_out is None:
            self._rows = getattr(self, "_rows", []) + [rows]
        n_dir = int(np.atleast_2d(n_hats).shape[0])
        lo_keep, hi_keep = line_keep_window(E_grid)
        edges = energy_bin_edges(E_grid)
        c = L.PbCxrArgs()
        c.precision = self.precision
        c.quadrature = L.PB_QUAD_BINMEAN
        c.n_dir = n_dir
        c.n_hat = _ptr(self._n_hat_dev) if spec_out is None else _ptr(h.f64(np.atleast_2d(n_hats)))
        c.thickness = st.thickness
        # Every streamed history radiates (elec_id < Ne for all of them).
        c.Ne = 1 << 62
        c.n_seg = cap
        c.r_mid, c.v_hat, c.L = _ptr(self.seg_r), _ptr(self.seg_v), _ptr(self.seg_L)
        c.E_keV, c.elec_id = _ptr(self.seg_E), _ptr(self.seg_id)
        c.n_seg_device = _ptr(self.seg_count)
        t = L.PbCxrTables()
        lt = rad.line_tables
        t.n_g = int(rows.G.shape[0])
        t.G, t.WM = _ptr(h.f64(rows.G)), _ptr(h.f64(rows.WM))
        t.ES, t.EP = _ptr(h.f64(rows.ES)), _ptr(h.f64(rows.EP))
        t.row_table = _ptr(h.typed(rows.row_table, torch.int32))
        t.n_tab = int(np.asarray(lt.E_tab).size)
        t.E_tab = _ptr(h.f64(lt.E_tab))
        for name in ("chi_re", "chi_im", "u_re", "u_im"):
            setattr(t, name, _ptr(h.f64(getattr(lt, name))))
        lm = np.atleast_2d(np.asarray(lt.log_mu, dtype=np.float64))
        t.n_mu, t.log_mu = int(lm.shape[0]), _ptr(h.f64(lm))
        t.delta = _ptr(h.f64(lt.delta))
        t.lo_keep, t.hi_keep = lo_keep, hi_keep
        t.tab_log0, t.tab_log_step = geometric_grid(lt.E_tab)
        t.delta_tail_absmax = _ptr(h.f64(np.maximum.accumulate(np.abs(np.asarray(lt.delta, float))[::-1])[::-1]))
        c.tables = t
        c.n_E = self.n_E
        c.E_grid = _ptr(self._E_grid_dev)
        c.edges = _ptr(h.f64(edges))
        w = np.diff(edges)
        uniform = np.allclose(w, w[0], rtol=1e-9, atol=0.0)
        if spec.exact_widths and spec.exact_widths > 0 and uniform:
            pad = int(np.ceil(max(edges[0] - lo_keep, hi_keep - edges[-1]) / w[0])) + 2
            c.exact_widths, c.far_pad = float(spec.exact_widths), pad
            if spec_out is not None:
                c.far_moments = _ptr(h.zeros(n_dir * (self.n_E + 2 * pad) * 3, torch.float64))
            else:
                if self.far is None:  # shared by the radiators: each call clears it
                    self.far = h.zeros(self.n_dir * (self.n_E + 2 * pad) * 3, torch.float64)
                c.far_moments = _ptr(self.far)
        else:
            c.exact_widths, c.far_pad = 0.0, -1
        c.spec = _ptr(self.spec_cxr if spec_out is None else spec_out)
        c.status = _ptr(self.status)
        if self.layered:
            c.n_layer = st.n_layers
            c.z_top, c.z_bot = _ptr(self._z_top), _ptr(self._z_bot)
            c.mu_off, c.mu_knot = _ptr(self._mu_off), _ptr(self._mu_knot)
            c.mu_value, c.mu_slope = _ptr(self._mu_value), _ptr(self._mu_slope)
            c.seg_layer, c.emit_layer = _ptr(self.seg_layer), int(rad.layer)
        return c

    # -- one batch ---------------------------------------------------------
    def use_surrogate(self, models, exact_stride=20, tol=0.01, probe_batches=4, sample_exact_widths=None):
        """Score PXR+CBS with an ensemble of trained surrogates plus an exact
        control variate, instead of the exact reflection sum on every segment.

        Per batch: one ``pb_mlp_infer`` launch per model over all segments
        (length-weighted last-layer sums per direction; the linear output
        layers are applied at readout), and, on the segments of every
        ``exact_stride``-th history (``pb_segments_sample``), the exact
        mixed-precision scorer and the surrogate again. The estimate
            S = S_sur(all) + stride (S_exact(sample) - S_sur(sample))
        is unbiased for the exact spectrum whatever the surrogate's error; the
        surrogate only has to make the sampled difference small. The result
        lives on the coarse grid of the surrogate (``surrogate_spectrum``;
        ``surrogate_spectrum_fine`` on the case's bins).
        ``exact_stride=0`` uses the surrogate alone.

        Error gate and fallback: after ``probe_batches`` batches (counted from
        the last ``reset``) the error of the estimate is estimated per tile
        from the batch-to-batch scatter of the sub-sample residuals
        (``surrogate.control_variate_error``: three standard errors, worst
        bin, relative to the tile's peak). Tiles above ``tol`` are scored by
        the exact mixed scorer from then on, and the batches already run are
        replayed (transport again from the same counter-based streams, no
        tallies) so that those tiles' spectra cover the whole run exactly.
        The decision stands across ``reset``. ``surrogate_report`` gives the
        estimate, the fallback tiles and the run's audit: the surrogate alone
        against the exact sum on the run's sub-sample (histories the training
        never saw).

        ``sample_exact_widths`` narrows the sub-sample scorer's exact bin-mean
        window (first-zero widths each side; None keeps the case's, the
        reference's 64). Beyond the window a line's bins take the far-field
        envelope through the moments, which omits only the sinc^2
        oscillation averaged over a bin: on the 50 MeV Si scene the spectrum
        with 2 widths differs from the one with 64 by 8e-7 of the tile peak
        (4 widths: 7e-7, 16 widths: 4e-7), against the estimator's per-mille
        sampling noise, and the sub-sample's scorer takes 40 % of the time.
        The estimate is then unbiased for that scorer's spectrum."""
        from .detector import tile_uv

        if self.spec.detector is None or self.spec.angular_shape is None:
            raise ValueError("the surrogate needs the case's detector tiling")
        if len(self.cargs_all) != 1 or self.layered:
            raise ValueError("the surrogate covers a single-crystal slab; a stack scores its layers exactly")
        n_bins = models[0].n_bins
        if self.n_E % n_bins != 0:
            raise ValueError("the case's bins must split evenly into the surrogate's coarse bins")
        tiles = {int(m.n_tiles) for m in models}
        if len(tiles) != 1 or {m.n_bins for m in models} != {n_bins}:
            raise ValueError("an ensemble needs one form and one coarse grid")
        self.sur_factored = tiles.pop() > 1
        if self.sur_factored and models[0].n_tiles != self.n_dir:
            raise ValueError("a tile-factored surrogate needs one head per direction of the case")
        self.surrogates = list(models)
        self.sur_stride = int(exact_stride)
        dev, h = self.device, self.h
        if self.sur_factored:
            # one feature direction: the tile heads are applied at readout
            self.sur_uv = torch.zeros(1, 2, dtype=torch.float32, device=dev)
        else:
            self.sur_uv = torch.as_tensor(tile_uv(self.spec.detector, self.spec.angular_shape),
                                          dtype=torch.float32, device=dev)
        n_feat_dir = int(self.sur_uv.shape[0])

        def infer_set(seg, cap, count):
            hs = [torch.zeros(n_feat_dir, 256, device=dev, dtype=torch.float64) for _ in self.surrogates]
            ls = [torch.zeros(n_feat_dir, device=dev, dtype=torch.float64) for _ in self.surrogates]
            args = [m.infer_args(self.spec, seg, cap, self.sur_uv, a, b, n_seg_device=count, status=self.status)
                    for m, a, b in zip(self.surrogates, hs, ls)]
            return hs, ls, args

        seg_all = {"r": self.seg_r, "v": self.seg_v, "L": self.seg_L, "E": self.seg_E, "id": self.seg_id}
        self.sur_hsum, self.sur_lsum, self.sur_args = infer_set(seg_all, self.seg_capacity, self.seg_count)
        self.sur_args_s = []
        if self.sur_stride > 0:
            cap_s = self.seg_capacity // self.sur_stride * 2 + 4096
            self.smp = {"r": h.empty((cap_s, 3), torch.float64), "v": h.empty((cap_s, 3), torch.float64),
                        "L": h.empty(cap_s, torch.float64), "E": h.empty(cap_s, torch.float64),
                        "id": h.empty(cap_s, torch.int64), "count": h.zeros(1, torch.int64)}
            src = L.PbSegments()
            src.capacity, src.count = self.seg_capacity, _ptr(self.seg_count)
            src.r_mid, src.v_hat, src.L = _ptr(self.seg_r), _ptr(self.seg_v), _ptr(self.seg_L)
            src.E_repr, src.elec_id = _ptr(self.seg_E), _ptr(self.seg_id)
            dst = L.PbSegments()
            dst.capacity, dst.count = cap_s, _ptr(self.smp["count"])
            dst.r_mid, dst.v_hat, dst.L = _ptr(self.smp["r"]), _ptr(self.smp["v"]), _ptr(self.smp["L"])
            dst.E_repr, dst.elec_id = _ptr(self.smp["E"]), _ptr(self.smp["id"])
            self.smp_src, self.smp_dst = src, dst
            cs = L.PbCxrArgs.from_buffer_copy(self.cargs)
            if sample_exact_widths is not None and cs.exact_widths > 0.0:
                cs.exact_widths = float(sample_exact_widths)
            cs.n_seg = cap_s
            cs.r_mid, cs.v_hat, cs.L = _ptr(self.smp["r"]), _ptr(self.smp["v"]), _ptr(self.smp["L"])
            cs.E_keV, cs.elec_id = _ptr(self.smp["E"]), _ptr(self.smp["id"])
            cs.n_seg_device = _ptr(self.smp["count"])
            self.spec_sample = h.zeros((self.n_dir, self.n_E), torch.float64)
            cs.spec = _ptr(self.spec_sample)
            self.cargs_s = cs
            self.sur_hsum_s, self.sur_lsum_s, self.sur_args_s = infer_set(self.smp, cap_s, self.smp["count"])
        n_out = self.surrogates[0].n_bins
        self.sur_tol = float(tol)
        self.sur_probe = max(2, int(probe_batches))
        self.sur_checked = False
        self.sur_estimate = None
        self.sur_fallback = np.zeros(self.n_dir, dtype=bool)
        self._fb_args = None
        self._fb_spec = None
        self._sur_res_prev = torch.zeros(self.n_dir, n_out, device=dev, dtype=torch.float64)
        self._sur_res_sq = torch.zeros_like(self._sur_res_prev)
        self._run_batches = []

    def _head(self, hsums, lsums):
        """The surrogate spectrum [n_dir, n_bins] from the summed last-layer
        activations: per direction (pairwise form), or every tile's head on
        the one shared sum (tile-factored form)."""
        n_feat_dir = int(self.sur_uv.shape[0])
        out = torch.zeros(n_feat_dir, self.surrogates[0].n_out, device=self.device, dtype=torch.float64)
        k = len(self.surrogates)
        for m, hs, ls in zip(self.surrogates, hsums, lsums):
            L.check(self.lib.pb_mlp_head(n_feat_dir, m.n_out, m.W5r.data_ptr(), m.p["b5"].data_ptr(),
                                         hs.data_ptr(), ls.data_ptr(), float(m.t_scale) / k, out.data_ptr(),
                                         torch.cuda.current_stream().cuda_stream), "pb_mlp_head")
        return out.view(self.n_dir, self.surrogates[0].n_bins)

    def coarse(self, spec_fine):
        """Mean of each run of n_E / n_bins fine bins: the surrogate's coarse bins."""
        n_bins = self.surrogates[0].n_bins
        return spec_fine.view(spec_fine.shape[0], n_bins, -1).mean(-1)

    def surrogate_spectrum(self):
        """Surrogate (+ exact control variate) spectrum [n_dir, n_coarse] so far,
        per history, in the exact scorer's units; fallback tiles carry the
        exact scorer's spectrum."""
        s = self._cv_coarse()
        if self._fb_args is not None:
            s[self._fb_index] = self.coarse(self._fb_spec)
        return s.cpu().numpy() / max(self.histories, 1)

    def _cv_coarse(self):
        s = self._head(self.sur_hsum, self.sur_lsum)
        if self.sur_stride > 0:
            s += self.sur_stride * (self.coarse(self.spec_sample) - self._head(self.sur_hsum_s, self.sur_lsum_s))
        return s

    def surrogate_check(self):
        """Estimate the control variate's error per tile now and move the
        tiles above the tolerance to the exact scorer (replaying the batches
        run since the last reset). Returns the per-tile estimate."""
        from .surrogate import control_variate_error

        B = len(self._run_batches)
        est = control_variate_error(self._sur_res_prev.cpu().numpy(), self._sur_res_sq.cpu().numpy(), B,
                                    self.sur_stride, self._cv_coarse().cpu().numpy())
        if est is None:
            return None
        self.sur_estimate = est
        self.sur_checked = True
        new = (est > self.sur_tol) & ~self.sur_fallback
        if np.any(new):
            self._enable_fallback(self.sur_fallback | new)
        return est

    def _enable_fallback(self, flagged):
        """Exact scoring of the tiles ``flagged`` on every segment from now
        on, after replaying this run's batches for them."""
        idx = np.flatnonzero(flagged)
        n_hats = np.atleast_2d(np.asarray(self.spec.n_hats, dtype=float))[idx]
        rad = Radiator(-1, self.spec.crystal, self.spec.hkl_list, self.spec.line_tables, self.spec.surface_hkl,
                       None, self.spec.mosaic_fwhm_rad, self.spec.mosaic_nodes)
        self._fb_spec = self.h.zeros((idx.size, self.n_E), torch.float64)
        self._fb_args = self._cxr_args(rad, n_hats, np.asarray(self.spec.E_grid, dtype=np.float64),
                                       self.seg_capacity, spec_out=self._fb_spec)
        self._fb_index = torch.as_tensor(idx, device=self.device)
        self.sur_fallback = np.asarray(flagged, dtype=bool).copy()
        # Replay: the same histories transported again (counter-based
        # streams give the same segments), tallies into scratch buffers.
        ta = L.PbTransportArgs.from_buffer_copy(self.targs)
        scratch = L.PbTallies.from_buffer_copy(self.targs.tallies)
        self._replay_tallies = [self.h.zeros(tuple(t.shape), t.dtype) for t in (self.fates, self.exit_E,
                                                                                self.exit_theta, self.deposit)]
        scratch.fates, scratch.exit_E, scratch.exit_theta, scratch.deposit = (_ptr(t) for t in self._replay_tallies)
        ta.tallies = scratch
        s = torch.cuda.current_stream(self.device).cuda_stream
        for e_start, n in self._run_batches:
            self.seg_count.zero_()
            ta.e_start, ta.n = int(e_start), int(n)
            L.check(self.lib.pb_transport(C.byref(ta), s), "pb_transport")
            L.check(self.lib.pb_cxr_score(C.byref(self._fb_args), s), "pb_cxr_score")

    def surrogate_report(self) -> dict:
        """The run's error estimate per tile, the tiles on the exact
        fallback, and the audit: the surrogate alone against the exact sum on
        the run's sub-sample, max |difference| over bins relative to each
        tile's peak."""
        ex = self.coarse(self.spec_sample).cpu().numpy() if self.sur_stride > 0 else None
        audit = None
        if ex is not None and self.histories > 0:
            su = self._head(self.sur_hsum_s, self.sur_lsum_s).cpu().numpy()
            peak = np.max(np.abs(ex), axis=1)
            audit = (np.max(np.abs(su - ex), axis=1) / np.where(peak > 0, peak, np.inf)).tolist()
        return {"tolerance": self.sur_tol, "probe_batches": self.sur_probe, "checked": self.sur_checked,
                "estimate_per_tile": None if self.sur_estimate is None else self.sur_estimate.tolist(),
                "fallback_tiles": np.flatnonzero(self.sur_fallback).tolist(),
                "audit_surrogate_alone_per_tile": audit}

    def surrogate_spectrum_fine(self):
        """Surrogate (+ exact control variate) spectrum on the case's own bins
        [n_dir, n_E] so far, per history: each coarse surrogate value spread
        over its fine bins (U), corrected by the exact sub-sample at full
        resolution,
            S = U(S_sur(all)) + stride (S_exact(sample) - U(S_sur(sample))),
        unbiased for the exact fine-bin spectrum whatever U is. Inside a coarse
        bin its noise is the exact sub-sample's: a segment's lines are much
        narrower than a fine bin, which no smooth U follows, so the fine-bin
        error falls as 1 / sqrt(histories). (Shaping each coarse total by the
        sub-sample's own fine proportions instead was measured no better: the
        proportions carry the same sampling noise.)"""
        rep = self.n_E // self.surrogates[0].n_bins
        s = self._head(self.sur_hsum, self.sur_lsum).repeat_interleave(rep, dim=1)
        if self.sur_stride > 0:
            s += self.sur_stride * (self.spec_sample
                                    - self._head(self.sur_hsum_s, self.sur_lsum_s).repeat_interleave(rep, dim=1))
        if self._fb_args is not None:
            s[self._fb_index] = self._fb_spec
        return s.cpu().numpy() / max(self.histories, 1)

    def run_batch(self, e_start: int, n: int, stream=None, events=None):
        """Transport histories [e_start, e_start + n) and score them. Stream ordered."""
        if n > self.batch:
            raise ValueError("batch larger than the case's segment buffer was sized for")
        s = (stream or torch.cuda.current_stream()).cuda_stream
        a = self.targs
        a.e_start, a.n = int(e_start), int(n)
        if events is None and not getattr(self, "surrogates", None):
            # the whole exact pass in one C call: transport, then every scorer
            p = L.PbTransportScoreArgs()
            p.transport = a
            p.n_cxr, p.n_brem, p.n_char = len(self.cargs_all), len(self.bargs_all), len(self.chargs_all)
            keep = ((L.PbCxrArgs * max(p.n_cxr, 1))(*self.cargs_all), (L.PbBremArgs * max(p.n_brem, 1))(*self.bargs_all),
                    (L.PbCharArgs * max(p.n_char, 1))(*self.chargs_all))
            p.cxr, p.brem, p.chars = (C.cast(k, C.POINTER(t)) for k, t in
                                      zip(keep, (L.PbCxrArgs, L.PbBremArgs, L.PbCharArgs)))
            L.check(self.lib.pb_transport_score(C.byref(p), s), "pb_transport_score")
            self.histories += int(n)
            return
        self.seg_count.zero_()
        if events is not None:
            events[0].record()
        L.check(self.lib.pb_transport(C.byref(a), s), "pb_transport")
        if events is not None:
            events[1].record()
        if getattr(self, "surrogates", None):
            if self.sur_stride > 0:
                L.check(self.lib.pb_segments_sample(C.byref(self.smp_src), self.sur_stride, C.byref(self.smp_dst),
                                                    _ptr(self.status), s), "pb_segments_sample")
                L.check(self.lib.pb_cxr_score(C.byref(self.cargs_s), s), "pb_cxr_score")
            if events is not None and len(events) > 4:
                events[4].record()  # exact sub-sample done; the surrogate follows
            for sa in self.sur_args + self.sur_args_s:
                L.check(self.lib.pb_mlp_infer(C.byref(sa), s), "pb_mlp_infer")
            if self.sur_stride > 0:
                # this batch's sub-sample residual r_b = cumulative - previous
                cur = self.coarse(self.spec_sample) - self._head(self.sur_hsum_s, self.sur_lsum_s)
                r = cur - self._sur_res_prev
                self._sur_res_sq.add_(r * r)
                self._sur_res_prev.copy_(cur)
            if self._fb_args is not None:
                L.check(self.lib.pb_cxr_score(C.byref(self._fb_args), s), "pb_cxr_score")
        else:
            for ca in self.cargs_all:
                L.check(self.lib.pb_cxr_score(C.byref(ca), s), "pb_cxr_score")
        if events is not None:
            events[2].record()
        for ba in self.bargs_all:
            L.check(self.lib.pb_brem_score(C.byref(ba), s), "pb_brem_score")
        for ch in self.chargs_all:
            L.check(self.lib.pb_char_yields(C.byref(ch), s), "pb_char_yields")
        if events is not None:
            events[3].record()
        self.histories += int(n)
        if getattr(self, "surrogates", None):
            self._run_batches.append((int(e_start), int(n)))
            if not self.sur_checked and self.sur_stride > 0 and len(self._run_batches) >= self.sur_probe:
                self.surrogate_check()

    def kernel_launches_per_batch(self) -> int:
        """This library's kernels launched per batch (transport 1, CXR 2 with
        the far-field finalize; brem: FP64 one per 16 directions, mixed two per
        16 directions plus the depth-node form's five where it has a
        workspace)."""
        if getattr(self, "surrogates", None):
            n = 1 + len(self.surrogates) * (2 if self.sur_stride > 0 else 1)
            if self.sur_stride > 0:
                n += 1 + 1 + (1 if self.cargs.exact_widths > 0 else 0)
                n += len(self.surrogates)  # pb_mlp_head of the sub-sample residual
            if self._fb_args is not None:
                n += 1 + (1 if self._fb_args.exact_widths > 0 else 0)
        else:
            n = 1 + sum(1 + (1 if ca.exact_widths > 0 else 0) for ca in self.cargs_all)
        per_group = 2 if self.precision == L.PB_MIXED else 1
        n += len(self.bargs_all) * per_group * ((self.n_dir + 15) // 16) + 5 * len(self.brem_work)
        n += len(self.chargs_all)
        return n

    def brem_node_state(self) -> list:
        """Launch state of the depth-node bremsstrahlung form after the last
        batch, per workspace: whether it scored the batch (``ok``), how many
        radiating segments it left to the per-(segment, energy) form
        (``left_out``), its depth cells and its electron-energy window [keV]
        (the header ``BremNodeHdr`` at the start of the workspace)."""
        out = []
        for wk in self.brem_work:
            raw = wk[:88].cpu().numpy()
            u64 = raw[:24].view(np.uint64)
            u32 = raw[24:40].view(np.uint32)
            f64 = raw[40:88].view(np.float64)
            out.append({"ok": bool(u32[0]), "left_out": int(u64[2]), "faces": int(u32[1]),
                        "n_cells": int(u32[2]), "T_lo_keV": float(f64[0]), "T_hi_keV": float(f64[1])})
        return out

    def device_status(self) -> int:
        return int(self.status.item())

    def results(self) -> dict:
        """Normalised spectra [photons/eV/sr/electron] and tallies so far."""
        Ne = max(self.histories, 1)
        sur = getattr(self, "surrogates", None)
        out = {
            # with the surrogate: its control-variate estimate on the case's bins
            "cxr": self.surrogate_spectrum_fine() if sur else self.spec_cxr.cpu().numpy() / Ne,
            "fates": self.fates.cpu().numpy(),
            "exit_E": self.exit_E.cpu().numpy(),
            "exit_theta": self.exit_theta.cpu().numpy(),
            "deposit_keV": self.deposit.cpu().numpy() / Ne,
            "segments_last_batch": int(self.seg_count.item()),
        }
        if self.bargs is not None:
            out["brem"] = self.spec_brem.cpu().numpy() / (4.0 * np.pi) / Ne
        if self.chargs_all:
            out["characteristic"] = self.characteristic_spectrum().cpu().numpy() / (4.0 * np.pi) / Ne
        return out

    def characteristic_spectrum(self):
        """Line yields so far spread on the bins (pb_char_spectrum), summed
        over emitters, un-normalised [n_dir, n_E]."""
        self.spec_char.zero_()
        s = torch.cuda.current_stream(self.device).cuda_stream
        for y, prof in zip(self.char_yields, self.char_profiles):
            L.check(self.lib.pb_char_spectrum(self.n_dir, int(y.shape[1]), self.n_E, _ptr(y), _ptr(prof),
                                              _ptr(self.spec_char), s), "pb_char_spectrum")
        return self.spec_char

    def device_results(self) -> dict:
        """The device-resident accumulators (un-normalised), for a cross-rank sum."""
        out = {"cxr": self.spec_cxr, "fates": self.fates, "exit_E": self.exit_E,
               "exit_theta": self.exit_theta, "deposit": self.deposit}
        if self.bargs is not None:
            out["brem"] = self.spec_brem
        for i, y in enumerate(self.char_yields):
            out[f"char_yield_{i}"] = y
        return out

    def reset(self):
        for t in (self.spec_cxr, self.fates, self.exit_E, self.exit_theta, self.deposit):
            t.zero_()
        for t in (getattr(self, "sur_hsum", []) + getattr(self, "sur_lsum", []) + getattr(self, "sur_hsum_s", [])
                  + getattr(self, "sur_lsum_s", [])):
            t.zero_()
        if getattr(self, "spec_sample", None) is not None:
            self.spec_sample.zero_()
        if getattr(self, "surrogates", None):
            self._sur_res_prev.zero_()
            self._sur_res_sq.zero_()
            self._run_batches = []
            if self._fb_spec is not None:
                self._fb_spec.zero_()
        if self.bargs is not None:
            self.spec_brem.zero_()
        for y in self.char_yields:
            y.zero_()
        self.histories = 0


def simulate_case_host(spec: CaseSpec, histories_per_step: int, *, steps: int = 1, warmup: int = 1,
                       precision="mixed", rng="philox", e_start: int = 0, device=None, surrogates=None,
                       exact_stride=50, tol=0.01, probe_batches=None, sample_exact_widths=None) -> dict:
    """End-to-end run through host buffers: every step copies the case's input
    tables from pinned host memory to the device, runs one batch, and reads
    the spectra and tallies back to pinned host memory -- one copy each way
    through a pinned staging buffer (``pb_copy_segments`` scatters and gathers
    the case's tensors on the device), double-buffered on two copy streams so
    that the next step's inputs and this step's results cross the host link
    while the GPU computes. Returns the rate, the bytes moved per step and the
    last step's read-back. With ``surrogates`` the PXR+CBS part is the
    surrogate with its exact sub-sample; the per-direction accumulators read
    back each step are the ones its readout needs. The surrogate's error
    probe runs on the warm-up batches (``probe_batches`` defaults to the
    warm-up count, at least two)."""
    case = ScoringCase(spec, precision=precision, rng=rng, batch_histories=histories_per_step,
                       device=device)
    if surrogates:
        probe = max(2, int(warmup)) if probe_batches is None else int(probe_batches)
        case.use_surrogate(surrogates, exact_stride=exact_stride, tol=tol, probe_batches=probe,
                           sample_exact_widths=sample_exact_widths)
    ins = list(case.h.inputs)
    if surrogates:
        outs = case.sur_hsum + case.sur_lsum + case.sur_hsum_s + case.sur_lsum_s
        outs += [case.spec_sample] if case.sur_stride > 0 else []
        outs += [case.fates, case.exit_E, case.exit_theta, case.deposit]
    else:
        outs = [case.spec_cxr, case.fates, case.exit_E, case.exit_theta, case.deposit]
    if case.bargs is not None:
        outs.append(case.spec_brem)
    outs += case.char_yields
    h2d = sum(t.numel() * t.element_size() for t in ins)
    d2h = sum(t.numel() * t.element_size() for t in outs)

    # One pinned host staging buffer per direction, 16-byte aligned slots: a
    # step crosses the host link in one copy each way, and pb_copy_segments
    # moves the slots to and from the case's tensors on the device. The device
    # staging buffers are double-buffered, so the next step's inputs cross on
    # a copy stream while this step computes, and its results leave on another.
    def layout(tensors):
        offs, o = [], 0
        for t in tensors:
            offs.append(o)
            o += (t.numel() * t.element_size() + 15) & ~15
        return offs, max(o, 16)

    in_offs, in_total = layout(ins)
    out_offs, out_total = layout(outs)
    dev = case.device
    stage_h = torch.empty(in_total, dtype=torch.uint8).pin_memory()
    for t, off in zip(ins, in_offs):
        nb = t.numel() * t.element_size()
        stage_h[off:off + nb].copy_(t.detach().reshape(-1).view(torch.uint8).cpu())
    stage_d = [torch.empty(in_total, dtype=torch.uint8, device=dev) for _ in range(2)]
    ostage_d = [torch.empty(out_total, dtype=torch.uint8, device=dev) for _ in range(2)]
    ostage_h = [torch.empty(out_total, dtype=torch.uint8).pin_memory() for _ in range(2)]

    def descriptors(triples):
        rows = []
        for src, dst, nb in triples:  # pieces of at most 256 KB spread a large table over blocks
            for o in range(0, nb, 1 << 18):
                rows += [src + o, dst + o, min(1 << 18, nb - o)]
        return torch.tensor(rows, dtype=torch.int64, device=dev).reshape(-1, 3)

    d_in = [descriptors([(stage_d[k].data_ptr() + off, t.data_ptr(), t.numel() * t.element_size())
                         for t, off in zip(ins, in_offs)]) for k in range(2)]
    d_out = [descriptors([(t.data_ptr(), ostage_d[k].data_ptr() + off, t.numel() * t.element_size())
                          for t, off in zip(outs, out_offs)]) for k in range(2)]
    lib = case.lib
    main = torch.cuda.current_stream(dev)
    up, down = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    ev = {name: [torch.cuda.Event() for _ in range(2)] for name in ("h2d", "used", "out", "d2h")}
    for k in range(2):
        ev["used"][k].record(main)
        ev["d2h"][k].record(main)

    def step(i):
        k = i & 1
        up.wait_event(ev["used"][k])  # the scatter two steps back has read this buffer
        with torch.cuda.stream(up):
            stage_d[k].copy_(stage_h, non_blocking=True)
        ev["h2d"][k].record(up)
        main.wait_event(ev["h2d"][k])
        L.check(lib.pb_copy_segments(int(d_in[k].shape[0]), d_in[k].data_ptr(), main.cuda_stream),
                "pb_copy_segments")
        ev["used"][k].record(main)
        case.run_batch(e_start + i * histories_per_step, histories_per_step, stream=main)
        main.wait_event(ev["d2h"][k])  # the read-back two steps back has left this buffer
        L.check(lib.pb_copy_segments(int(d_out[k].shape[0]), d_out[k].data_ptr(), main.cuda_stream),
                "pb_copy_segments")
        ev["out"][k].record(main)
        down.wait_event(ev["out"][k])
        with torch.cuda.stream(down):
            ostage_h[k].copy_(ostage_d[k], non_blocking=True)
        ev["d2h"][k].record(down)

    for i in range(warmup):
        step(i)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(main)
    up.wait_event(t0)
    for i in range(steps):
        step(warmup + i)
    for k in range(2):
        main.wait_event(ev["d2h"][k])
    t1.record(main)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / steps
    last = ostage_h[(warmup + steps - 1) & 1]
    result = []
    for t, off in zip(outs, out_offs):
        nb = t.numel() * t.element_size()
        result.append(last[off:off + nb].view(t.dtype).reshape(t.shape).numpy().copy())
    return {"histories_per_s": histories_per_step / (ms / 1e3), "ms_per_step": ms,
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "result": result}
