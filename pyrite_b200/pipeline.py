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
class CaseSpec:
    """One beam/crystal scene."""

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
        # ---- CXR scorer ----
        n_hats = np.atleast_2d(np.asarray(spec.n_hats, dtype=float))
        self.n_dir = n_hats.shape[0]
        rows = reflection_rows(spec.crystal, spec.hkl_list, n_hats, surface_hkl=spec.surface_hkl,
                               mosaic_fwhm_rad=spec.mosaic_fwhm_rad, mosaic_nodes=spec.mosaic_nodes)
        self.rows = rows
        E_grid = np.asarray(spec.E_grid, dtype=np.float64)
        self.n_E = int(E_grid.size)
        lo_keep, hi_keep = line_keep_window(E_grid)
        edges = energy_bin_edges(E_grid)
        c = L.PbCxrArgs()
        c.precision = self.precision
        c.quadrature = L.PB_QUAD_BINMEAN
        c.n_dir = self.n_dir
        c.n_hat = _ptr(h.f64(n_hats))
        c.thickness = st.thickness
        # Every streamed history radiates (elec_id < Ne for all of them).
        c.Ne = 1 << 62
        c.n_seg = cap
        c.r_mid, c.v_hat, c.L = _ptr(self.seg_r), _ptr(self.seg_v), _ptr(self.seg_L)
        c.E_keV, c.elec_id = _ptr(self.seg_E), _ptr(self.seg_id)
        c.n_seg_device = _ptr(self.seg_count)
        t = L.PbCxrTables()
        lt = spec.line_tables
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
        c.E_grid = _ptr(h.f64(E_grid))
        c.edges = _ptr(h.f64(edges))
        w = np.diff(edges)
        uniform = np.allclose(w, w[0], rtol=1e-9, atol=0.0)
        if spec.exact_widths and spec.exact_widths > 0 and uniform:
            pad = int(np.ceil(max(edges[0] - lo_keep, hi_keep - edges[-1]) / w[0])) + 2
            c.exact_widths, c.far_pad = float(spec.exact_widths), pad
            self.far = h.zeros(self.n_dir * (self.n_E + 2 * pad) * 3, torch.float64)
            c.far_moments = _ptr(self.far)
        else:
            c.exact_widths, c.far_pad = 0.0, -1
        self.spec_cxr = h.zeros((self.n_dir, self.n_E), torch.float64)
        c.spec = _ptr(self.spec_cxr)
        c.status = _ptr(self.status)
        self.cargs = c
        # ---- brem scorer ----
        self.bargs = None
        if spec.brem_composition:
            b = L.PbBremArgs()
            b.precision = self.precision
            b.n_dir = self.n_dir
            b.n_hat = c.n_hat
            b.thickness = st.thickness
            b.Ne = c.Ne
            b.n_seg = cap
            b.r_mid, b.v_hat, b.L, b.E_keV, b.elec_id = c.r_mid, c.v_hat, c.L, c.E_keV, c.elec_id
            b.n_seg_device = c.n_seg_device
            b.n_el = len(spec.brem_composition)
            b.Z = _ptr(h.f64([float(ELEMENTS[el][0]) for el, _ in spec.brem_composition]))
            b.n_ang3 = _ptr(h.f64([float(n) for _, n in spec.brem_composition]))
            b.n_E = self.n_E
            b.E_grid = c.E_grid
            b.mu = _ptr(h.f64(spec.brem_mu))
            self.spec_brem = h.zeros((self.n_dir, self.n_E), torch.float64)
            b.spec = _ptr(self.spec_brem)
            b.status = c.status
            self.bargs = b
        self.histories = 0

    # -- one batch ---------------------------------------------------------
    def use_surrogate(self, models, exact_stride=20):
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
        lives on the coarse grid of the surrogate (``surrogate_spectrum``).
        ``exact_stride=0`` uses the surrogate alone."""
        from .detector import tile_uv

        if self.spec.detector is None or self.spec.angular_shape is None:
            raise ValueError("the surrogate needs the case's detector tiling")
        n_out = models[0].n_out
        if self.n_E % n_out != 0:
            raise ValueError("the case's bins must split evenly into the surrogate's coarse bins")
        self.surrogates = list(models)
        self.sur_stride = int(exact_stride)
        dev, h = self.device, self.h
        self.sur_uv = torch.as_tensor(tile_uv(self.spec.detector, self.spec.angular_shape), dtype=torch.float32,
                                      device=dev)

        def infer_set(seg, cap, count):
            hs = [torch.zeros(self.n_dir, 256, device=dev, dtype=torch.float64) for _ in self.surrogates]
            ls = [torch.zeros(self.n_dir, device=dev, dtype=torch.float64) for _ in self.surrogates]
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
            cs.n_seg = cap_s
            cs.r_mid, cs.v_hat, cs.L = _ptr(self.smp["r"]), _ptr(self.smp["v"]), _ptr(self.smp["L"])
            cs.E_keV, cs.elec_id = _ptr(self.smp["E"]), _ptr(self.smp["id"])
            cs.n_seg_device = _ptr(self.smp["count"])
            self.spec_sample = h.zeros((self.n_dir, self.n_E), torch.float64)
            cs.spec = _ptr(self.spec_sample)
            self.cargs_s = cs
            self.sur_hsum_s, self.sur_lsum_s, self.sur_args_s = infer_set(self.smp, cap_s, self.smp["count"])

    def _head(self, hsums, lsums):
        out = torch.zeros(self.n_dir, self.surrogates[0].n_out, device=self.device, dtype=torch.float64)
        k = len(self.surrogates)
        for m, hs, ls in zip(self.surrogates, hsums, lsums):
            L.check(self.lib.pb_mlp_head(self.n_dir, m.n_out, m.W5r.data_ptr(), m.p["b5"].data_ptr(),
                                         hs.data_ptr(), ls.data_ptr(), float(m.t_scale) / k, out.data_ptr(),
                                         torch.cuda.current_stream().cuda_stream), "pb_mlp_head")
        return out

    def coarse(self, spec_fine):
        """Mean of each run of n_E / n_out fine bins: the surrogate's coarse bins."""
        n_out = self.surrogates[0].n_out
        return spec_fine.view(spec_fine.shape[0], n_out, -1).mean(-1)

    def surrogate_spectrum(self):
        """Surrogate (+ exact control variate) spectrum [n_dir, n_coarse] so far,
        per history, in the exact scorer's units."""
        s = self._head(self.sur_hsum, self.sur_lsum)
        if self.sur_stride > 0:
            s += self.sur_stride * (self.coarse(self.spec_sample) - self._head(self.sur_hsum_s, self.sur_lsum_s))
        return s.cpu().numpy() / max(self.histories, 1)

    def run_batch(self, e_start: int, n: int, stream=None, events=None):
        """Transport histories [e_start, e_start + n) and score them. Stream ordered."""
        if n > self.batch:
            raise ValueError("batch larger than the case's segment buffer was sized for")
        s = (stream or torch.cuda.current_stream()).cuda_stream
        self.seg_count.zero_()
        a = self.targs
        a.e_start, a.n = int(e_start), int(n)
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
        else:
            L.check(self.lib.pb_cxr_score(C.byref(self.cargs), s), "pb_cxr_score")
        if events is not None:
            events[2].record()
        if self.bargs is not None:
            L.check(self.lib.pb_brem_score(C.byref(self.bargs), s), "pb_brem_score")
        if events is not None:
            events[3].record()
        self.histories += int(n)

    def kernel_launches_per_batch(self) -> int:
        """This library's kernels launched per batch (transport 1, CXR 2 with
        the far-field finalize, brem one per 16 directions)."""
        if getattr(self, "surrogates", None):
            n = 1 + len(self.surrogates) * (2 if self.sur_stride > 0 else 1)
            if self.sur_stride > 0:
                n += 1 + 1 + (1 if self.cargs.exact_widths > 0 else 0)
        else:
            n = 1 + 1 + (1 if self.cargs.exact_widths > 0 else 0)
        if self.bargs is not None:
            n += (self.n_dir + 15) // 16
        return n

    def device_status(self) -> int:
        return int(self.status.item())

    def results(self) -> dict:
        """Normalised spectra [photons/eV/sr/electron] and tallies so far."""
        Ne = max(self.histories, 1)
        out = {
            "cxr": self.spec_cxr.cpu().numpy() / Ne,
            "fates": self.fates.cpu().numpy(),
            "exit_E": self.exit_E.cpu().numpy(),
            "exit_theta": self.exit_theta.cpu().numpy(),
            "deposit_keV": self.deposit.cpu().numpy() / Ne,
            "segments_last_batch": int(self.seg_count.item()),
        }
        if self.bargs is not None:
            out["brem"] = self.spec_brem.cpu().numpy() / (4.0 * np.pi) / Ne
        return out

    def device_results(self) -> dict:
        """The device-resident accumulators (un-normalised), for a cross-rank sum."""
        out = {"cxr": self.spec_cxr, "fates": self.fates, "exit_E": self.exit_E,
               "exit_theta": self.exit_theta, "deposit": self.deposit}
        if self.bargs is not None:
            out["brem"] = self.spec_brem
        return out

    def reset(self):
        for t in (self.spec_cxr, self.fates, self.exit_E, self.exit_theta, self.deposit):
            t.zero_()
        for t in (getattr(self, "sur_hsum", []) + getattr(self, "sur_lsum", []) + getattr(self, "sur_hsum_s", [])
                  + getattr(self, "sur_lsum_s", [])):
            t.zero_()
        if getattr(self, "spec_sample", None) is not None:
            self.spec_sample.zero_()
        if self.bargs is not None:
            self.spec_brem.zero_()
        self.histories = 0


def simulate_case_host(spec: CaseSpec, histories_per_step: int, *, steps: int = 1, warmup: int = 1,
                       precision="mixed", rng="philox", e_start: int = 0, device=None, surrogates=None,
                       exact_stride=50) -> dict:
    """End-to-end run through host buffers: every step copies the case's input
    tables from pinned host memory to the device, runs one batch, and reads
    the spectra and tallies back to pinned host memory. Returns the rate and
    the bytes moved per step. With ``surrogates`` the PXR+CBS part is the
    surrogate with its exact sub-sample; the per-direction accumulators read
    back each step are the ones its readout needs."""
    case = ScoringCase(spec, precision=precision, rng=rng, batch_histories=histories_per_step,
                       device=device)
    if surrogates:
        case.use_surrogate(surrogates, exact_stride=exact_stride)
    pairs = [(t.cpu().pin_memory(), t) for t in case.h.inputs]
    if surrogates:
        outs = case.sur_hsum + case.sur_lsum + case.sur_hsum_s + case.sur_lsum_s
        outs += [case.spec_sample] if case.sur_stride > 0 else []
        outs += [case.fates, case.exit_E, case.exit_theta, case.deposit]
    else:
        outs = [case.spec_cxr, case.fates, case.exit_E, case.exit_theta, case.deposit]
    if case.bargs is not None:
        outs.append(case.spec_brem)
    host_out = [torch.empty_like(t, device="cpu").pin_memory() for t in outs]
    h2d = sum(h.numel() * h.element_size() for h, _ in pairs)
    d2h = sum(t.numel() * t.element_size() for t in outs)

    def step(i):
        for hsrc, dst in pairs:
            dst.copy_(hsrc, non_blocking=True)
        case.run_batch(e_start + i * histories_per_step, histories_per_step)
        for src, hdst in zip(outs, host_out):
            hdst.copy_(src, non_blocking=True)

    for i in range(warmup):
        step(i)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for i in range(steps):
        step(warmup + i)
    t1.record()
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / steps
    return {"histories_per_s": histories_per_step / (ms / 1e3), "ms_per_step": ms,
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "result": [h.numpy().copy() for h in host_out]}
