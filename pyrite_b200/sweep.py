"""Batched design sweep: many small cases autotuned and replayed as one CUDA graph.

A sweep is a list of independent cases (crystal, tilt, thickness, beam
energy, history count), as the reference runs design studies
(``pyrite/montecarlo/runner/case_driver.py:1025`` once per case). Each case
keeps its own device-resident tables and segment buffer (``ScoringCase``);
its histories are split into batches of the largest size its buffer holds,
and the autotuner picks each case's transport block shape by timing one
full batch per option. Cases run concurrently on several streams, assigned
largest-first to the least-loaded stream, so a small case (a thin slab, a
few thousand histories) does not leave most of the GPU idle. The whole
sweep -- every batch of every case: transport, PXR+CBS lines,
bremsstrahlung and tallies, on every stream -- is captured once into a CUDA
graph (a fork/join of the streams) and launched with a single replay.
Histories are keyed by (case seed, history index), so the graph, the eager
loop, any batch split and any stream assignment give the same histories.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import placeholder_data as P
from .api import BeamSpec
from .detector import PlanarDetector, tiles_in_sample_frame
from .pipeline import CaseSpec, ScoringCase
from .tables import HOPG, SILICON, LayerStack, diamond_hkls, tilted_geometry


@dataclass(frozen=True)
class SweepConfig:
    crystal: str          # "Si" or "HOPG"
    tilt_deg: float
    thickness_um: float
    E0_MeV: float
    histories: int
    seed: int = 0


def c3_configs(n=256, seed=1, histories_scale=1.0):
    """The design sweep's configurations: tilt U(0, 20 deg), thickness
    logU(10, 1000 um), Si or HOPG, beam energy logU(5, 100 MeV), histories
    logU(1e4, 1e6) (times ``histories_scale``)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        out.append(SweepConfig(
            crystal="Si" if rng.uniform() < 0.5 else "HOPG",
            tilt_deg=float(rng.uniform(0.0, 20.0)),
            thickness_um=float(np.exp(rng.uniform(np.log(10.0), np.log(1000.0)))),
            E0_MeV=float(np.exp(rng.uniform(np.log(5.0), np.log(100.0)))),
            histories=max(1, int(round(histories_scale * np.exp(rng.uniform(np.log(1e4), np.log(1e6)))))),
            seed=seed * 100003 + i,
        ))
    return out


def case_spec(cfg: SweepConfig, n_bins=1024, theta_obs_deg=20.0):
    """CaseSpec of one sweep point: 1 mm / 0.2 mrad beam, detector centre at
    ``theta_obs_deg`` and 1 m, ``n_bins`` bins over 1-60 keV."""
    E0 = cfg.E0_MeV * 1e3
    tilt = np.deg2rad(cfg.tilt_deg)
    beam_dir, _ = tilted_geometry(np.deg2rad(theta_obs_deg), tilt)
    det = PlanarDetector(np.deg2rad(theta_obs_deg), 1000.0, 20.0, 20.0, 64, 64)
    _, n_hats, _ = tiles_in_sample_frame(det, (1, 1), tilt)
    gamma = 1.0 + E0 / 510.99895
    bg = float(np.sqrt(gamma * gamma - 1.0))
    tw = (1.0 * 0.2e-3 * bg * 1e3, 1.0 / 0.2e-3 * 1e-3, 0.0)
    cr = SILICON if cfg.crystal == "Si" else HOPG
    sym = "Si" if cfg.crystal == "Si" else "C"
    n_at = cr.n_atoms_per_ang3
    stack = LayerStack([(0.0, cfg.thickness_um * 1e4, [(sym, n_at)])])
    E_grid = np.linspace(1000.0, 60000.0, n_bins)
    if cfg.crystal == "Si":
        hkl, surface = diamond_hkls(8.0), (2, 2, 0)
    else:
        hkl, surface = [(0, 0, l) for l in range(-8, 9) if l != 0], (0, 0, 1)
    comp = [(sym, n_at)]
    return CaseSpec(
        stack=stack, beam=BeamSpec(E0, beam_dir, tilt, 0.0, twiss_x=tw, twiss_y=tw), E_cut_keV=5.0,
        crystal=cr, hkl_list=hkl, n_hats=n_hats, E_grid=E_grid,
        line_tables=P.line_tables(cr, hkl, E_grid, comp), surface_hkl=surface,
        brem_composition=comp, brem_mu=P.mu_total(comp, E_grid), seed=cfg.seed,
        detector=det, angular_shape=(1, 1),
    )


def assign_streams(work, n_streams):
    """Longest-processing-time assignment: items in decreasing ``work``, each
    to the stream with the least work so far (ties to the lowest index).
    Returns the stream index of every item."""
    n_streams = max(1, int(n_streams))
    load = [0.0] * n_streams
    out = [0] * len(work)
    for i in sorted(range(len(work)), key=lambda i: -work[i]):
        s = min(range(n_streams), key=lambda k: load[k])
        out[i] = s
        load[s] += work[i]
    return out


def L_check(case):
    """Transport one trial batch of ``case`` (transport only) and wait."""
    import ctypes as C

    from . import _lib as L

    L.check(case.lib.pb_transport(C.byref(case.targs), torch.cuda.current_stream().cuda_stream), "pb_transport")
    torch.cuda.synchronize(case.device)


class DesignSweep:
    """Cases of a sweep on one GPU, with per-case autotuned batches and a
    single-graph replay of the whole sweep."""

    SEG_BYTES = 76  # segment list row: r_mid, v_hat, L, E (FP64), elec_id (i64), layer (i32)

    def __init__(self, configs, *, precision="mixed", device=None, batch_options=(4096, 16384),
                 thread_options=(128, 256), n_bins=1024, segment_budget_bytes=256 << 20, streams=1):
        self.configs = list(configs)
        self.device = torch.device(device or "cuda")
        self.batch_options = tuple(sorted(batch_options))
        self.thread_options = tuple(thread_options)
        self.precision = precision
        self.n_bins = n_bins
        self.budget = int(segment_budget_bytes)
        self.specs = [case_spec(cfg, n_bins=n_bins) for cfg in self.configs]
        self.cases = [self._calibrated_case(i) for i in range(len(self.configs))]
        self.plan = [(c.batch, 0) for c in self.cases]
        self.graph = None
        self.tuning = []
        self.set_streams(streams)

    def set_streams(self, n):
        """Assign the cases to ``n`` streams, largest expected work first to
        the least-loaded stream (work ~ histories x segments per history)."""
        self.n_streams = max(1, int(n))
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(self.n_streams)]
        work = [cfg.histories * c.seg_capacity / max(c.batch, 1) for cfg, c in zip(self.configs, self.cases)]
        self.assign = assign_streams(work, self.n_streams)

    def _case(self, i, segs_per_history):
        cap_hist = min(max(self.batch_options), self.configs[i].histories,
                       max(1, self.budget // (self.SEG_BYTES * segs_per_history)))
        return ScoringCase(self.specs[i], precision=self.precision, rng="philox", lut=True,
                           batch_histories=cap_hist, segs_per_history=segs_per_history, device=self.device)

    def _calibrated_case(self, i, trial=128, e_start=1 << 41):
        """Size the case's segment buffer from a trial transport: the mean
        segments per history (thin or high-energy slabs need few, thick
        low-energy ones thousands) with margin, within the memory budget."""
        probe = self._case(i, 64)
        n = min(trial, probe.batch)
        probe.seg_count.zero_()
        t = probe.targs
        t.e_start, t.n = int(e_start), int(n)
        L_check(probe)
        mean = int(probe.seg_count.item()) / n
        segs = int(np.ceil(1.5 * mean + 16))
        del probe
        return self._case(i, segs)

    def autotune(self, trial_histories=None, e_start=1 << 40):
        """Pick the transport block threads per case from one timed batch per
        option at the case's own batch size (histories outside the sweep's
        own range; accumulators reset). Batches stay at the largest size the
        case's buffer holds: a smaller batch only adds launches. A trial
        smaller than a full batch (``trial_histories``) under-fills the GPU
        and times nothing useful, so it is capped below at the batch size
        unless the case has fewer histories."""
        self.tuning = []
        for i, (cfg, case) in enumerate(zip(self.configs, self.cases)):
            b = min(case.batch, cfg.histories)
            n = b if trial_histories is None else min(b, max(int(trial_histories), b))
            best = None
            for t in self.thread_options:
                case.targs.block_threads = t
                ev0 = torch.cuda.Event(enable_timing=True)
                ev1 = torch.cuda.Event(enable_timing=True)
                ev0.record()
                case.run_batch(e_start, n)
                ev1.record()
                torch.cuda.synchronize(self.device)
                per_hist = ev0.elapsed_time(ev1) / n
                if best is None or per_hist < best[0]:
                    best = (per_hist, t)
            case.reset()
            case.targs.block_threads = best[1]
            self.plan[i] = (case.batch, best[1])
            self.tuning.append({"case": i, "batch": case.batch, "block_threads": best[1],
                                "us_per_history": 1e3 * best[0]})
        return self.tuning

    def _launch_all(self):
        """Every batch of every case, each case on its assigned stream, the
        streams forked from and joined back to the current one."""
        main = torch.cuda.current_stream(self.device)
        for st in self.streams:
            st.wait_stream(main)
        for i, (cfg, case, (b, t)) in enumerate(zip(self.configs, self.cases, self.plan)):
            st = self.streams[self.assign[i]]
            case.targs.block_threads = t
            with torch.cuda.stream(st):
                for e in range(0, cfg.histories, b):
                    case.run_batch(e, min(b, cfg.histories - e), stream=st)
        for st in self.streams:
            main.wait_stream(st)

    def capture(self):
        """Record every batch of every case into one CUDA graph."""
        for case in self.cases:
            case.reset()
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        stream = torch.cuda.Stream(device=self.device)
        stream.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(stream):
            g.capture_begin()
            self._launch_all()
            g.capture_end()
        torch.cuda.current_stream(self.device).wait_stream(stream)
        self.graph = g
        for case in self.cases:  # capture did not execute anything
            case.histories = 0
        return g

    def run(self, use_graph=True):
        """Run the sweep once; returns (per-case results, seconds on the device)."""
        for case in self.cases:
            case.reset()
        torch.cuda.synchronize(self.device)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record()
        if use_graph:
            if self.graph is None:
                raise RuntimeError("capture() first")
            self.graph.replay()
            for cfg, case in zip(self.configs, self.cases):
                case.histories = cfg.histories
        else:
            self._launch_all()
        ev1.record()
        torch.cuda.synchronize(self.device)
        seconds = ev0.elapsed_time(ev1) / 1e3
        results = []
        for case in self.cases:
            if case.device_status() != 0:
                raise RuntimeError(f"sweep case reported device status {case.device_status()}")
            results.append(case.results())
        return results, seconds

    @property
    def total_histories(self):
        return sum(c.histories for c in self.configs)

    def launches(self):
        return sum(math.ceil(cfg.histories / b) * case.kernel_launches_per_batch()
                   for cfg, case, (b, _) in zip(self.configs, self.cases, self.plan))
