"""Benchmark: e- histories/s of the transport + radiation-scoring hot path on B200.

Workload (one "step"): a batch of histories of the 50 MeV Si scene (500 um
Si, (220) cut at a 10 deg tilt, 1 mm / 0.2 mrad beam, 2x2 cm^2 64x64-pixel
detector at 20 deg and 1 m scored in 4x4 angular tiles, 1-60 keV in 2048
bins) through transport -> PXR+CBS lines of every segment x 238 Si
reflections (|g| < 8 1/A) x 16 tiles -> bin means, plus the Bethe-Heitler
continuum on every tile, plus exit tallies. ``value`` is the mixed-precision
(FP32 flight/lines, FP64 energy bookkeeping and tallies) rate with device
resident inputs; ``fp64`` beside it is the plain all-FP64 path on the same
work. ``e2e`` runs the same batches through the public host API, copying the
case tables from pinned host memory each step and reading the spectra back.

``--impl reference`` times the CPU oracle (the C restatement of the
reference's algorithm) on the host cores, one process per core over disjoint
history blocks, on a bounded sample of the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "e- histories/s on 1 B200: surrogate+mixed vs plain FP64, at <=1% spectrum error"
UNIT = "histories/s"
ALG_FLOPS_PAIR = 300.0   # FP32 census of one (segment, reflection, tile) line: kinematics, amplitudes, escape
ALG_FLOPS_ITEM = 80.0    # FP32 flops of one (line, bin) item of the bin-mean deposit
# Surrogate: one (segment, tile) pair through the hidden layers, 2 (6*256 + 3*256*256); the linear
# output layer is applied once per tile to the length-weighted sums, not per pair.
ALG_FLOPS_INFER = 2.0 * (6 * 256 + 3 * 256 * 256)
# Bethe-Heitler + Elwert per (segment, energy), all the tiles of one exit face at once (direction
# moments, order 2 for this detector's spread), on the path this scene takes (one element, each
# 256-segment chunk within a narrow energy range): the cross section is a cubic in the electron
# energy (3 FMA), the escape at the band centre one exponential (its exponent carries the segment
# factor) and the thin-segment series, then three moment updates -- 36 FP32 flops (FMA = 2) and
# 1 SFU operation per pair where the warp's segment is optically thin (x = mu f_c e2 <= 0.1 for
# all its 64 energies), 3 more flops and a second exponential elsewhere; plus seven exact
# cross-section evaluations (3 SFU each) per energy and chunk for the fit (0.08 per pair). The
# thin share is counted from the last batch's segments (brem_thin_fraction); the tiles are rebuilt
# from the moments once per launch.
ALG_FLOPS_BREM_THIN, ALG_FLOPS_BREM_THICK = 36.0, 39.0
BREM_FIT_SFU_PER_PAIR = 7 * 3 / 256.0
SFU_OPS_PER_SM_CLOCK = 16.0  # MUFU lanes per SM per cycle
# DRAM bytes (read + write) per history of the three scorers, from one ncu
# capture each of a 2,048-history batch of this workload (profiles/*_si50_2048hist.md);
# a kernel's traffic grows with its segments, so a full launch is this x histories.
DRAM_BYTES_PER_HISTORY = {"cxr_kernel": 6.868736e6 / 2048, "brem_kernel": 5.239552e6 / 2048,
                          "mlp_infer_kernel": 5.484032e6 / 2048}
BENCH_SEED = 12345  # seed of the 50 MeV Si scene in every arm
MEASURED_BF16_SUSTAINED = float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["bf16_tflops_sustained"]) \
    if (ROOT / "MEASURED_PEAKS.json").exists() else 1400.0
MEASURED_HBM_GBS = float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"]) \
    if (ROOT / "MEASURED_PEAKS.json").exists() else 6650.0
# cxr_kernel<float> on the control variate's sub-sample (4 exact widths, ~14,560 segments, L2-resident):
# DRAM bytes (read + write) per sampled segment from the one-pass ncu capture of the bench's own
# sub-sample launches (profiles/cxr_kernel_subsample_si50_65536hist.md): 2.80-2.98 MB per launch.
DRAM_BYTES_PER_SUBSAMPLE_SEGMENT = 2.9e6 / 14560
# Depth-node bremsstrahlung: the segment fields its passes read per segment (electron energy,
# length, z of the midpoint, v_z, electron id: 5 x 8 B); nothing per (segment, energy).
NODE_BYTES_PER_SEGMENT = 40.0


def spectrum_error_stats(got, ref):
    """Max and RMS error of per-tile spectra ``got`` against ``ref`` (both
    [tiles][bins]), each tile relative to its own peak, and of the
    tile-summed detector spectrum relative to its peak."""
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    peak = np.max(np.abs(ref), axis=1)
    peak = np.where(peak > 0, peak, np.inf)
    d = got - ref
    tot_ref, tot_d = ref.sum(0), d.sum(0)
    tot_peak = float(np.max(np.abs(tot_ref))) or float("inf")
    return {"max_over_tiles": float(np.max(np.max(np.abs(d), axis=1) / peak)),
            "rms_over_tiles": float(np.max(np.sqrt(np.mean(d * d, axis=1)) / peak)),
            "detector_total_max": float(np.max(np.abs(tot_d)) / tot_peak),
            "detector_total_rms": float(np.sqrt(np.mean(tot_d * tot_d)) / tot_peak)}


def sigma_stats(got, ref, sigma, floor=1e-3):
    """|got - ref| in units of the reference's own statistical error (sigma
    of its batch means), over the bins where the reference is above
    ``floor`` of its tile's peak: the largest ratio and the fraction of those
    bins within 3 sigma."""
    got, ref, sigma = (np.asarray(x, dtype=np.float64) for x in (got, ref, sigma))
    peak = np.max(np.abs(ref), axis=1, keepdims=True)
    m = (np.abs(ref) > floor * peak) & (sigma > 0)
    if not np.any(m):
        return {"max": None, "within_3_sigma": None, "bins": 0}
    z = np.abs(got - ref)[m] / sigma[m]
    return {"max": float(z.max()), "within_3_sigma": float(np.mean(z <= 3.0)), "bins": int(m.sum())}


def brem_thin_fraction(case, spec, n_seg, torch):
    """Share of the (segment, energy) pairs that brem_moment_packed_kernel scores on its
    thin-segment path: the segment's depth extent e2 in the slab is at most 0.1 / (mu f_c) for
    the largest attenuation mu of the 64 energies a warp holds (f_c the centre path factor of
    the tiles). Counted on the device from the last batch's segments."""
    z = case.seg_r.reshape(-1)[:3 * n_seg].view(-1, 3)[:, 2]
    vz = case.seg_v.reshape(-1)[:3 * n_seg].view(-1, 3)[:, 2]
    half = 0.5 * case.seg_L.reshape(-1)[:n_seg]
    T = float(case.bargs.thickness)
    e2 = ((z + half * vz).clamp(0.0, T) - (z - half * vz).clamp(0.0, T)).abs()
    f = 1.0 / np.maximum(np.abs(np.asarray(spec.n_hats)[:case.n_dir, 2]), 1e-12)
    f_c = 0.5 * (f.min() + f.max())
    mu = np.asarray(spec.brem_mu, dtype=np.float64)
    n_E = mu.size
    thin = 0.0
    for g0 in range(0, n_E, 64):
        m = mu[g0:g0 + 64].max() * f_c
        lim = 0.1 / m if m > 0 else np.inf
        thin += (mu[g0:g0 + 64].size) * float((e2 <= lim).sum().item())
    return thin / max(1.0, float(n_seg) * n_E)


def workload_config(args, n_dir, n_g, n_bins):
    return {
        "workload": "50 MeV e- on 500 um Si (220) at 10 deg; 238 reflections |g|<8/A; "
                    "4x4 angular tiles of a 64x64 px detector at 20 deg; 2048 bins 1-60 keV; "
                    "PXR+CBS bin-mean + Bethe-Heitler + exit tallies",
        "histories_per_step": args.histories,
        "reflection_rows": n_g,
        "directions": n_dir,
        "bins": n_bins,
        "precision": "mixed (FP32 flight/lines, FP64 energy/tallies)",
        "rng": "philox4x32-10",
        "transport": "LUT core in shared memory",
        "l2": "segment list (~64 B x 33 segments x histories) > 126 MB L2 every step",
        "data": "synthetic beam; placeholder atomic tables (Chantler/EPDL absent)",
    }


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"pb_clocks_{os.getpid()}.csv"

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.5)  # nvidia-smi's start-up, so samples cover the whole region
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        med = float(np.median(sm)) if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU reference arm: the oracle on the host cores
# ---------------------------------------------------------------------------
def _cpu_worker(payload):
    import oracle
    from pyrite_b200 import configs

    from pyrite_b200.api import _fill_beam

    e_start, n, directions = payload
    spec = configs.c2_si_50mev(seed=BENCH_SEED)
    st = spec.stack
    lt = oracle.LayerTables(st.z_top, st.z_bot, st.n_el, st.Z, st.J, st.N, st.E_cross)
    # Entrance states of these histories from the scene's Twiss beam, drawn
    # from the same Philox entry stream as the device (oracle.beam_entries).
    pos, dirs, E = oracle.beam_entries(_fill_beam(None, spec.beam, spec.seed), e_start, n, rng=oracle.RNG_PHILOX)
    out = oracle.transport(lt, pos, dirs, E, seed=spec.seed, E_cut=spec.E_cut_keV, rng=oracle.RNG_PHILOX,
                           e_start=e_start, cap=256)
    from pyrite_b200.tables import energy_bin_edges, line_keep_window, reflection_rows

    seg = dict(v_hat=out["v_hat"], E_keV=0.5 * (out["E_start"] + out["E_end"]), L_ang=out["L"],
               r_mid=out["r_mid"], elec_id=out["elec_id"])
    rows = reflection_rows(spec.crystal, spec.hkl_list, spec.n_hats[:directions], surface_hkl=spec.surface_hkl)
    lo, hi = line_keep_window(spec.E_grid)
    edges = energy_bin_edges(spec.E_grid)
    lt_ = spec.line_tables
    for d in range(directions):
        tables = dict(G=rows.G, ES=rows.ES[d], EP=rows.EP[d], WM=rows.WM, row_table=rows.row_table,
                      E_tab=lt_.E_tab, chi_re=lt_.chi_re, chi_im=lt_.chi_im, u_re=lt_.u_re, u_im=lt_.u_im,
                      log_mu=lt_.log_mu, delta=lt_.delta, lo_keep=lo, hi_keep=hi)
        Er, aw, w, good = oracle.cxr_lines(tables, spec.n_hats[d], st.thickness, seg, e_start + n)
        oracle.reduce_binmean(Er[good], aw[good], w[good], edges)
        oracle.brem_spectrum(seg, [14.0], [spec.brem_composition[0][1]], st.thickness, spec.n_hats[d],
                             spec.E_grid, spec.brem_mu, n)
    return n


def run_cpu_reference(args):
    """Time the oracle port on every host core; returns (histories/s, cores, sample text)."""
    import multiprocessing as mp

    cores = os.cpu_count() or 1
    per = max(1, args.cpu_per_process)
    n_dir = 16
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        pool.map(_cpu_worker, [(i, 1, 1) for i in range(cores)])  # warm (imports, tables)
        t0 = time.perf_counter()
        done = sum(pool.map(_cpu_worker, [(1000 + i * per, per, n_dir) for i in range(cores)]))
        dt = time.perf_counter() - t0
    sample = (f"{done} histories of the same scene and beam ({per} per process x {cores} processes; "
              f"Twiss entrance states from the device's Philox entry stream), exact SR transport + "
              f"PXR/CBS bin means + Bethe-Heitler on all {n_dir} tiles")
    return done / dt, cores, sample


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def time_pipeline(case, args, rank, world, torch, dist, n_steps, n_warm):
    stream = torch.cuda.current_stream()
    base = rank * (n_steps + n_warm) * args.histories
    for i in range(n_warm):
        case.run_batch(base + i * args.histories, args.histories)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    n_ev = 5 if getattr(case, "surrogates", None) else 4
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(n_ev)] for _ in range(n_steps)]
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    for i in range(n_steps):
        case.run_batch(base + (n_warm + i) * args.histories, args.histories, events=ev[i])
    stop.record(stream)
    torch.cuda.synchronize()
    total_ms = start.elapsed_time(stop)
    t_tr = np.mean([e[0].elapsed_time(e[1]) for e in ev])
    t_cxr = np.mean([e[1].elapsed_time(e[2]) for e in ev])
    t_brem = np.mean([e[2].elapsed_time(e[3]) for e in ev])
    if n_ev == 5:
        # surrogate arm: split the PXR+CBS part into exact sub-sample and surrogate
        case.t_split = (float(np.mean([e[1].elapsed_time(e[4]) for e in ev])),
                        float(np.mean([e[4].elapsed_time(e[2]) for e in ev])))
    if dist is not None:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    return total_ms, t_tr, t_cxr, t_brem


def run_stack(args, torch):
    """The layered stack: 10 MeV on 20 um HOPG / 200 um Si / 1 mm W, four
    detectors (20/45/90/135 deg) in 4x4 angular tiles each, 4096 bins 1-80 keV;
    per batch transport, PXR+CBS of both crystal layers, per-layer brem,
    C/Si/W characteristic lines and tallies, in mixed precision and in FP64."""
    from pyrite_b200.configs import c5_stack_10mev
    from pyrite_b200.pipeline import ScoringCase

    torch.cuda.set_device(0)
    spec = c5_stack_10mev()
    H = 256
    out = {}
    for prec in ("mixed", "fp64"):
        per = 4096
        while True:  # size the segment buffer from a trial batch
            case = ScoringCase(spec, precision=prec, batch_histories=H, segs_per_history=per)
            case.run_batch(1 << 40, H)
            torch.cuda.synchronize()
            if case.device_status() != 4 or per >= 1 << 15:
                break
            per *= 2
            del case
        case.reset()
        for w in range(args.warmup):
            case.run_batch((1 << 40) + (w + 1) * H, H)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for i in range(args.steps):
            case.run_batch(i * H, H)
        ev1.record()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / args.steps
        res = case.results()
        out[prec] = {"histories_per_s": H / (ms / 1e3), "ms_per_batch": ms, "device_status": case.device_status(),
                     "segments_per_history": float(case.seg_count.item()) / H,
                     "launches_per_batch": case.kernel_launches_per_batch(),
                     "cxr_integral": float(res["cxr"].sum()), "brem_integral": float(res["brem"].sum()),
                     "characteristic_integral": float(res["characteristic"].sum())}
        del case
    line = {"metric": "stacked case histories/s (10 MeV HOPG/Si/W, 4 detectors x 16 tiles, 4096 bins)",
            "value": out["mixed"]["histories_per_s"], "unit": "histories/s", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f32+f64", "data": "synthetic", "histories_per_batch": H, "steps": args.steps,
            "mixed": out["mixed"], "fp64": out["fp64"],
            "speedup_mixed_vs_fp64": out["mixed"]["histories_per_s"] / out["fp64"]["histories_per_s"]}
    print(json.dumps(line), flush=True)


def run_sweep(args, torch):
    """The design sweep: 256 configurations (seed 1; tilt, thickness, Si/HOPG,
    energy, histories), each case scored exactly in mixed precision (PXR+CBS
    bin means on 1024 bins, Bethe-Heitler, exit tallies). Timed twice on the
    same histories: every case's batches launched one after another with the
    default plan (largest batch, default transport block) on one stream, and
    the whole sweep autotuned per case, spread over concurrent streams and
    replayed as one CUDA graph."""
    from pyrite_b200.sweep import DesignSweep, c3_configs

    torch.cuda.set_device(0)
    configs = c3_configs(n=256, seed=1, histories_scale=args.sweep_scale)
    t0 = time.perf_counter()
    sw = DesignSweep(configs, device="cuda")
    t_build = time.perf_counter() - t0
    # warm every case once (module load, tables) outside both timings
    for case in sw.cases:
        case.run_batch(1 << 40, min(256, case.batch))
        case.reset()
    torch.cuda.synchronize()
    plain, t_plain = sw.run(use_graph=False)
    t0 = time.perf_counter()
    sw.autotune()
    sw.set_streams(args.sweep_streams)
    t_tune = time.perf_counter() - t0
    tuned_eager, t_tuned = sw.run(use_graph=False)
    sw.capture()
    sw.run(use_graph=True)  # warm replay
    graph, t_graph = sw.run(use_graph=True)
    n_hist = sw.total_histories
    worst = 0.0
    for a, b in zip(plain, graph):
        for k in ("cxr", "brem"):
            peak = float(np.max(np.abs(a[k])))
            if peak > 0:
                worst = max(worst, float(np.max(np.abs(a[k] - b[k]))) / peak)
    line = {
        "metric": "design sweep histories/s (256 configurations, one graph replay)", "value": n_hist / t_graph,
        "unit": "histories/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": "256 configs from seed 1: tilt U(0,20) deg, thickness logU(10,1000) um, Si or HOPG, "
                               "E0 logU(5,100) MeV, histories logU(1e4,1e6) x %g; 1024 bins 1-60 keV; "
                               "PXR+CBS bin-mean + Bethe-Heitler + exit tallies" % args.sweep_scale,
                   "histories": n_hist},
        "sequential_plain": {"value": n_hist / t_plain, "seconds": t_plain},
        "autotuned_eager": {"value": n_hist / t_tuned, "seconds": t_tuned},
        "graph": {"seconds": t_graph, "launches_in_graph": sw.launches(), "streams": sw.n_streams},
        "speedup_vs_sequential_plain": t_plain / t_graph,
        "max_spectrum_difference_vs_plain": worst,
        "setup_s": {"build": t_build, "autotune": t_tune},
    }
    print(json.dumps(line), flush=True)


# Issued thread-instructions per (line, energy) pair of coh_field_kernel, from its ncu
# capture (profiles/coh_field_kernel_8rows_1M_lines_2048E.md); with 4 warp issue slots per SM
# per cycle this sets the kernel's issue ceiling in pairs/s.
COH_INSTR_PER_PAIR = 65.5


def coherent_records(rng, n_rows, per_row, E_lo, E_hi):
    """Seeded line records with the ranges of the reference's coherent fixtures:
    phases to 6e7 rad, formation widths 0.5-60 per eV, escape optical depths to 12."""
    n = n_rows * per_row
    tau_s = rng.uniform(0.0, 6.0, n)
    tau_e = tau_s + rng.uniform(-tau_s, 6.0, n)
    a, b = np.exp(-0.5 * tau_s), np.exp(-0.5 * tau_e)
    rec = dict(E_vac=rng.uniform(E_lo, E_hi, n), a_vac=rng.uniform(0.5, 60.0, n),
               phase_slope=rng.uniform(-3000.0, 3000.0, n), g_phase=rng.uniform(-6e7, 6e7, n),
               cs_re=rng.normal(0, 1e-4, n), cs_im=rng.normal(0, 1e-5, n), cp_re=rng.normal(0, 1e-4, n),
               cp_im=rng.normal(0, 1e-5, n), L_esc=rng.uniform(0.0, 2e5, n), half_dL=rng.uniform(-1e5, 1e5, n),
               apb=a + b, bma=b - a, q=0.25 * (tau_e - tau_s))
    return rec, np.full(n_rows, per_row, dtype=np.int64), rng.uniform(0.1, 1.0, n_rows)


def run_coherent(args, torch):
    """The coherent (field-sum) CXR reduction: 8 rows (reflection x mosaic
    node) x 125,000 line records x 2048 energies (1-61 keV) per step, i.e.
    2.048e9 line-energy pairs. ``value``: records resident on the device,
    raw C-ABI calls; ``e2e``: the public host API from host records each
    step, spectrum read back; ``cpu_baseline``: the numpy FP64 oracle on one
    row of 4,000 lines over the same energies."""
    import ctypes as C

    from oracle import coherent as oc
    from pyrite_b200 import _lib as L
    from pyrite_b200.coherent import RECORD_FIELDS, coherent_reduce

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(3)
    n_rows, per_row = 8, 125_000
    rec, cnt, w = coherent_records(rng, n_rows, per_row, 2000.0, 60000.0)
    E = np.linspace(1000.0, 61000.0, 2048)
    dom = 2.3e-4 * (1e4 / (E + 500.0)) ** 2 * E / 1973.27
    n_line = int(cnt.sum())
    pairs = n_line * E.size
    lib = L.load()
    drec = {k: torch.as_tensor(rec[k], device=dev) for k in RECORD_FIELDS}
    row_off = torch.as_tensor(np.concatenate([[0], np.cumsum(cnt)]), dtype=torch.int64, device=dev)
    wt, Et, Dt = (torch.as_tensor(x, device=dev) for x in (w, E, dom))
    spec = torch.zeros(E.size, dtype=torch.float64, device=dev)
    nb = C.c_uint64()
    L.check(lib.pb_coherent_work_size(n_rows, n_line, E.size, C.byref(nb)), "pb_coherent_work_size")
    work = torch.empty(nb.value, dtype=torch.uint8, device=dev)
    a = L.PbCoherentArgs()
    a.n_row, a.n_E, a.n_line = n_rows, E.size, n_line
    a.row_off, a.row_weight, a.E, a.delta_omega = (t.data_ptr() for t in (row_off, wt, Et, Dt))
    for k in RECORD_FIELDS:
        setattr(a, k, drec[k].data_ptr())
    a.scale, a.spec, a.work, a.work_bytes = 1.0, spec.data_ptr(), work.data_ptr(), nb.value
    stream = torch.cuda.current_stream()

    def call():
        L.check(lib.pb_coherent_reduce(C.byref(a), stream.cuda_stream), "pb_coherent_reduce")

    for _ in range(max(args.warmup, 3)):
        call()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as sampler:
        ev0.record(stream)
        for _ in range(args.steps):
            call()
        ev1.record(stream)
        torch.cuda.synchronize()
    clocks = sampler.summary()
    ms = ev0.elapsed_time(ev1) / args.steps
    value = pairs / (ms * 1e-3)
    # e2e: the host API from host (pinned) records, spectrum read back every step
    host = {k: torch.as_tensor(rec[k]).pin_memory() for k in RECORD_FIELDS}
    coherent_reduce(host, cnt, w, E, dom, device=dev).cpu()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        out = coherent_reduce(host, cnt, w, E, dom, device=dev).cpu().numpy()
    e2e_s = (time.perf_counter() - t0) / args.steps
    h2d = 8 * (len(RECORD_FIELDS) * n_line + 2 * E.size + n_rows + n_rows + 1)
    # parity on every 64th energy against the FP64 oracle
    sub = np.arange(0, E.size, 64)
    ref = oc.coherent_spectrum(rec, cnt, w, E[sub], dom[sub])
    parity = float(np.max(np.abs(out[sub] - ref)) / np.max(ref))
    # CPU baseline: the numpy oracle on one row of 4,000 lines, all energies
    n_cpu = 4000
    sample = {k: v[:n_cpu] for k, v in rec.items()}
    t0 = time.perf_counter()
    oc.coherent_spectrum(sample, [n_cpu], [1.0], E, dom)
    cpu_rate = n_cpu * E.size / (time.perf_counter() - t0)
    peak_pairs = 148 * (clocks.get("sm_mhz") or 1965) * 1e6 * 128 / COH_INSTR_PER_PAIR
    line = {
        "metric": "coherent CXR reduction line-energy pairs/s on 1 B200", "value": value, "unit": "pairs/s",
        "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 phases, f32 trig",
        "data": "synthetic",
        "config": {"workload": "8 rows x 125,000 line records x 2048 energies (1-61 keV), records resident "
                               "(104 MB) above L2 between steps", "pairs_per_step": pairs},
        "gpu_launches": 3 * args.steps,
        "roofline": {"bound": "issue", "achieved": value, "peak": peak_pairs, "unit": "pairs/s",
                     "frac": value / peak_pairs, "traffic": None,
                     "note": "issue ceiling 148 SM x clock x 128 thread-instr per cycle / %.1f instr per pair "
                             "(ncu); no HBM or tensor roofline applies" % COH_INSTR_PER_PAIR},
        "e2e": {"value": pairs / e2e_s, "unit": "pairs/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": 8 * E.size},
        "cpu_baseline": {"value": cpu_rate, "unit": "pairs/s", "cores": 1, "kind": "port",
                         "sample": "numpy FP64 oracle, 1 row x 4,000 lines x 2048 energies"},
        "parity_vs_oracle_max_rel_to_peak": parity,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--histories", type=int, default=1 << 16)
    ap.add_argument("--cpu-per-process", type=int, default=4,
                    help="histories per host process in the CPU baseline (about 4 s each)")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true")
    ap.add_argument("--compare-batches", type=int, default=4,
                    help="batches of the comparison pass run through every arm on the same histories "
                         "(spectrum errors against FP64, and the FP64 rate from batches 2..C)")
    ap.add_argument("--exact-stride", type=int, default=150,
                    help="exact control-variate sub-sample: every n-th history")
    ap.add_argument("--train-segments", type=int, default=16384)
    ap.add_argument("--train-dirs", type=int, default=512)
    ap.add_argument("--train-epochs", type=int, default=6)
    ap.add_argument("--surrogate-form", default="tiles", choices=["pairwise", "tiles"],
                    help="pairwise: the direction is an input and every (segment, tile) pair runs the network; "
                         "tiles: one head per detector tile on shared segment features (one pass per segment)")
    ap.add_argument("--cv-exact-widths", type=float, default=2.0,
                    help="exact bin-mean window of the control variate's sub-sample scorer, in first-zero widths "
                         "(the exact arms keep the reference's 64)")
    ap.add_argument("--tile-segments", type=int, default=262144, help="training segments of the tiles form")
    ap.add_argument("--tile-epochs", type=int, default=40, help="training epochs of the tiles form")
    ap.add_argument("--train-domain", default="case", choices=["case", "uniform"],
                    help="surrogate training segments: the case's transport, or spread over the whole input "
                         "domain (5-100 MeV, +-5 mrad, every depth; adds a 1e5-segment held-out audit)")
    ap.add_argument("--workload", default="c2", choices=["c2", "sweep", "stack", "coherent"],
                    help="c2: the headline step (default); sweep: the 256-configuration design sweep, "
                         "one graph replay against sequential plain launches; stack: the 10 MeV HOPG / Si / W "
                         "stack with four detectors; coherent: the coherent CXR field-sum reduction "
                         "(each its own JSON line)")
    ap.add_argument("--sweep-scale", type=float, default=1.0, help="scale of every sweep case's histories")
    ap.add_argument("--sweep-streams", type=int, default=8, help="concurrent case streams of the tuned sweep")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        rate, cores, sample = run_cpu_reference(args)
        line = {
            "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(workload_config(args, 16, 238, 2048),
                           precision="FP64 (the CPU oracle port of the reference's algorithm)",
                           transport="exact SR core, the same Twiss entrance states",
                           l2="n/a (host cores)"),
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return

    import torch

    if args.workload == "sweep":
        if rank == 0:
            run_sweep(args, torch)
        return
    if args.workload == "stack":
        if rank == 0:
            run_stack(args, torch)
        return
    if args.workload == "coherent":
        if rank == 0:
            run_coherent(args, torch)
        return

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as tdist

        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    else:
        torch.cuda.set_device(0)
    from pyrite_b200 import configs
    from pyrite_b200.pipeline import ScoringCase

    spec = configs.c2_si_50mev(seed=BENCH_SEED)
    H = args.histories
    C = max(2, args.compare_batches)
    # History indices of the comparison pass: the same C batches in every arm,
    # disjoint from the timed ones.
    cmp_base = (1 << 40) + rank * C * H
    cases, results, clocks, compare = {}, {}, {}, {}

    def arm(name, case, n_steps):
        with ClockSampler(local) as clk:
            total_ms, t_tr, t_cxr, t_brem = time_pipeline(case, args, rank, world, torch, dist, n_steps, args.warmup)
        clocks[name] = clk.summary()
        cases[name] = case
        results[name] = dict(total_ms=total_ms, n_steps=n_steps, t_tr=t_tr, t_cxr=t_cxr, t_brem=t_brem,
                             status=case.device_status(), res=case.results())

    def compare_pass(name, case, timed=False):
        """The comparison batches through a reset case; per-batch FP64 spectra
        (for the batch-means sigma) and, with ``timed``, CUDA-event times of
        batches 2..C (the first is the warm-up)."""
        case.reset()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(C + 1)]
        per_batch, prev, fine_by_batch = [], None, []
        for i in range(C):
            ev[i].record()
            case.run_batch(cmp_base + i * H, H)
            if getattr(case, "surrogates", None):
                # the cumulative surrogate+CV fine spectrum after every batch
                # (the arm is not timed): its error trajectory against FP64
                fine_by_batch.append(case.surrogate_spectrum_fine())
            if timed:
                cur = {k: v.detach().clone() for k, v in (("cxr", case.spec_cxr), ("brem", case.spec_brem))}
                if prev is not None:
                    per_batch.append({k: (cur[k] - prev[k]).cpu().numpy() / H for k in cur})
                else:
                    per_batch.append({k: cur[k].cpu().numpy() / H for k in cur})
                prev = cur
        ev[C].record()
        torch.cuda.synchronize()
        out = {"res": case.results(), "status": case.device_status()}
        if getattr(case, "surrogates", None):
            out["report"] = case.surrogate_report()  # the probe ran on these batches
            out["sur_coarse"] = case.surrogate_spectrum()
            out["sur_fine"] = case.surrogate_spectrum_fine()
            out["sur_fine_by_batch"] = fine_by_batch
            out["sur_alone"] = case._head(case.sur_hsum, case.sur_lsum).cpu().numpy() / max(case.histories, 1)
        if timed:
            # the per-batch snapshots sit between the events; each batch is
            # seconds long, the snapshot copies 0.5 MB
            out["ms_per_step"] = float(np.mean([ev[i].elapsed_time(ev[i + 1]) for i in range(1, C)]))
            out["per_batch"] = per_batch
        case.reset()
        compare[name] = out

    # 1. exact mixed precision (FP32 flight and lines, FP64 bookkeeping)
    mixed_case = ScoringCase(spec, precision="mixed", rng="philox", lut=True, batch_histories=H)
    cxr_counters = torch.zeros(2, dtype=torch.int64, device="cuda")
    mixed_case.cargs.counters = cxr_counters.data_ptr()  # kept lines, deposit items (comparison pass only)
    compare_pass("mixed", mixed_case)
    mixed_case.cargs.counters = None
    cxr_work = {"lines_kept": int(cxr_counters[0].item()), "deposit_items": int(cxr_counters[1].item()),
                "segments": int(mixed_case.seg_count.item()) * C}  # approximate: last batch's count x C
    arm("mixed", mixed_case, args.steps)
    # 2. surrogate + exact control variate on the same histories
    sur = None
    if not args.no_surrogate:
        from pyrite_b200 import surrogate as S

        torch.cuda.synchronize()
        t0 = time.perf_counter()
        # Data-parallel on N > 1 GPUs: each rank builds 1/N of the segments of
        # the training set (its own seed) and the gradients are averaged.
        pg = dist.group.WORLD if dist is not None else None
        if args.surrogate_form == "tiles":
            n_seg_rank = max(8192, args.tile_segments // world)
            data = S.make_tile_training_set(spec, n_seg=n_seg_rank, seed=1000 + rank, device="cuda",
                                            process_group=pg)
            model = S.Surrogate("cuda", seed=0, n_tiles=int(data["n_tiles"]))
            epochs = args.tile_epochs
        else:
            n_seg_rank = max(1024, args.train_segments // world)
            data = S.make_training_set(spec, n_seg=n_seg_rank, n_dir=args.train_dirs,
                                       dir_chunk=max(1, 2 ** 20 // n_seg_rank), seed=1000 + rank, device="cuda",
                                       process_group=pg, domain=args.train_domain)
            model = S.Surrogate("cuda", seed=0)
            epochs = args.train_epochs
        losses = model.train(data, epochs=epochs, lr=2e-3, lr_final=2e-5, process_group=pg)
        n_pairs = int(data["X"].shape[0]) * world
        n_dropped = int(data.get("nonfinite_pairs_dropped", 0))
        del data
        torch.cuda.synchronize()
        train_s = time.perf_counter() - t0
        cs = ScoringCase(spec, precision="mixed", rng="philox", lut=True, batch_histories=H)
        cs.use_surrogate([model], exact_stride=args.exact_stride, sample_exact_widths=args.cv_exact_widths)
        sub_counters = torch.zeros(2, dtype=torch.int64, device="cuda")
        cs.cargs_s.counters = sub_counters.data_ptr()  # the sub-sample scorer's lines and items (comparison pass)
        compare_pass("surrogate", cs)
        cs.cargs_s.counters = None
        sub_work = {"lines_kept": int(sub_counters[0].item()), "deposit_items": int(sub_counters[1].item()),
                    "segments": int(cs.smp["count"].item()) * C}  # approximate: last batch's count x C
        gate_report = compare["surrogate"]["report"]
        arm("surrogate", cs, args.steps)
        form = ("MLP 6 -> 4x256 SiLU -> 512 bins per (segment, tile) pair" if model.n_tiles == 1 else
                "MLP 4 segment features -> 4x256 SiLU -> %d tile heads x 512 bins (one pass per segment)"
                % model.n_tiles)
        sur = {"model": form + ", bf16 weights and activations, FP32 accumulate (tcgen05)",
               "form": args.surrogate_form,
               "train_s": train_s, "train_pairs": n_pairs, "epochs": epochs,
               "final_mse": losses[-1], "epoch_mse": [float(x) for x in losses],
               "diverged_epochs_redone": int(model.retries), "nonfinite_pairs_dropped": n_dropped,
               "train_domain": args.train_domain, "exact_stride": args.exact_stride,
               "cv_exact_widths": args.cv_exact_widths,
               "coarse_bins": int(model.n_bins),
               "error_estimate": {"what": "the product path's own per-tile estimate after its probe batches "
                                          "(3 standard errors of the control-variate correction, worst bin, "
                                          "relative to the tile peak), the tiles moved to the exact scorer, and "
                                          "the run's audit (surrogate alone vs the exact sum on the sub-sample)",
                                  **gate_report}}
        if args.train_domain == "uniform":
            # held-out segments over the whole input domain, surrogate alone
            au = S.audit_uniform(model, spec, n_seg=100_000, device="cuda")
            sur["audit_uniform_1e5"] = {"max_over_tiles": au["err_tile_max"], "detector_total": au["err_total"],
                                        "segments": au["segments"], "status": au["status"]}
    # 3. plain all-FP64 exact path: the comparison batches (its rate from batches 2..C)
    if not args.skip_fp64:
        compare_pass("fp64", ScoringCase(spec, precision="fp64", rng="philox", lut=True, batch_histories=H),
                     timed=True)
    for name, r in results.items():
        if not (r["res"]["cxr"].sum() > 0 or name == "surrogate") or not r["res"].get("brem", np.ones(1)).sum() > 0:
            raise SystemExit(f"bench: the {name} spectra are empty; refusing to report a rate")

    # ---- spectrum errors on the comparison batches (same histories in every arm) ----
    n_dir_c = int(mixed_case.n_dir)
    n_out = int(sur["coarse_bins"]) if sur is not None else 512

    def coarse(x):
        return np.asarray(x).reshape(n_dir_c, n_out, -1).mean(-1)

    errors = {"histories": C * H, "batches": C, "history_indices": f"[{cmp_base}, {cmp_base + C * H})"}
    ref_name = "fp64" if "fp64" in compare else "mixed"
    ref_cxr = compare[ref_name]["res"]["cxr"]
    ref_brem = compare[ref_name]["res"]["brem"]
    sigma = None
    if ref_name == "fp64":
        pb = compare["fp64"]["per_batch"]
        sigma = {k: np.std(np.stack([b[k] for b in pb]), axis=0, ddof=1) / np.sqrt(len(pb)) for k in ("cxr", "brem")}
    errors["reference"] = ("plain FP64 exact path" if ref_name == "fp64"
                           else "exact mixed path (FP64 arm skipped)")
    if ref_name == "fp64":
        errors["mixed_exact"] = {
            "fine_2048": spectrum_error_stats(compare["mixed"]["res"]["cxr"], ref_cxr),
            "coarse_512": spectrum_error_stats(coarse(compare["mixed"]["res"]["cxr"]), coarse(ref_cxr)),
            "fine_2048_in_fp64_sigma": sigma_stats(compare["mixed"]["res"]["cxr"], ref_cxr, sigma["cxr"])}
        errors["brem_mixed"] = {
            "fine_2048": spectrum_error_stats(compare["mixed"]["res"]["brem"], ref_brem),
            "fine_2048_in_fp64_sigma": sigma_stats(compare["mixed"]["res"]["brem"], ref_brem, sigma["brem"])}
    if sur is not None:
        errors["surrogate_cv"] = {
            "coarse_512": spectrum_error_stats(compare["surrogate"]["sur_coarse"], coarse(ref_cxr)),
            "fine_2048": spectrum_error_stats(compare["surrogate"]["sur_fine"], ref_cxr)}
        if sigma is not None:
            errors["surrogate_cv"]["fine_2048_in_fp64_sigma"] = sigma_stats(compare["surrogate"]["sur_fine"], ref_cxr,
                                                                            sigma["cxr"])
        if ref_name == "fp64":
            # The fine-bin error is the exact sub-sample's sampling noise: it
            # falls as 1 / sqrt(histories). Its trajectory over the comparison
            # batches (cumulative estimates against the cumulative FP64
            # spectra), the fitted exponent, and the value it extrapolates to
            # at the configuration's 1e8 histories.
            pb = compare["fp64"]["per_batch"]
            traj = []
            for k in range(1, C + 1):
                ref_k = np.mean(np.stack([b["cxr"] for b in pb[:k]]), axis=0)
                traj.append(spectrum_error_stats(compare["surrogate"]["sur_fine_by_batch"][k - 1], ref_k))
            ks = np.arange(1, C + 1, dtype=float)
            rms = np.array([t["rms_over_tiles"] for t in traj])
            slope = float(np.polyfit(np.log(ks), np.log(np.maximum(rms, 1e-300)), 1)[0]) if C >= 2 else float("nan")
            scale = np.sqrt(C * H / 1.0e8)
            errors["surrogate_cv"]["fine_2048_by_batches"] = {
                "histories": [int(k * H) for k in ks],
                "max_over_tiles": [t["max_over_tiles"] for t in traj],
                "rms_over_tiles": [t["rms_over_tiles"] for t in traj],
                "rms_exponent_vs_histories": slope,
                "projected_at_1e8_histories": {
                    "max_over_tiles": traj[-1]["max_over_tiles"] * scale,
                    "rms_over_tiles": traj[-1]["rms_over_tiles"] * scale,
                    "rule": "measured at %d histories x sqrt(%d / 1e8)" % (C * H, C * H)}}
        # the surrogate alone (no control variate), coarse: what the network
        # gains over the exact sub-sample alone is the gap between the two
        errors["surrogate_alone_coarse_512"] = spectrum_error_stats(compare["surrogate"]["sur_alone"],
                                                                    coarse(ref_cxr))
        # The gate: the headline variant's PXR+CBS on the surrogate's grid
        # and its bremsstrahlung on the case's grid as measured, and its
        # PXR+CBS on the case's 2048 bins at the configuration's 1e8
        # histories (the measured fine-bin error scaled by its 1/sqrt(N)
        # law, whose exponent the trajectory above reports), worst tile,
        # against the reference arm on the same histories.
        fine_proj = (errors["surrogate_cv"].get("fine_2048_by_batches", {})
                     .get("projected_at_1e8_histories", {}).get("max_over_tiles", 0.0))
        parts = [errors["surrogate_cv"]["coarse_512"]["max_over_tiles"],
                 errors.get("brem_mixed", {}).get("fine_2048", {}).get("max_over_tiles", 0.0), fine_proj]
        t = torch.tensor(parts, device="cuda", dtype=torch.float64)
        if dist is not None:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        parts = [float(x) for x in t.cpu()]
        e_gate = max(parts)
        sur["gate"] = {"bound": 0.01, "error": e_gate,
                       "parts": {"pxr_cbs_512_measured": parts[0], "brem_2048_measured": parts[1],
                                 "pxr_cbs_2048_projected_1e8": parts[2]},
                       "measured_on": "worst tile relative to the tile peak, against the %s on the same "
                                      "histories: surrogate+CV PXR/CBS on 512 bins and mixed brem on 2048 "
                                      "bins as measured; surrogate+CV PXR/CBS on 2048 bins projected to 1e8 "
                                      "histories" % errors["reference"]}
        sur["passed"] = bool(e_gate <= 0.01)

    def rate(name):
        r = results[name]
        return world * H / (r["total_ms"] / r["n_steps"] / 1e3), r["total_ms"] / r["n_steps"]

    head = "surrogate" if sur is not None and sur["passed"] else "mixed"
    value, ms_per_step = rate(head)
    r_head = results[head]
    mixed = results["mixed"]
    ce = cases["mixed"]
    n_seg = mixed["res"]["segments_last_batch"]
    n_g, n_dir, n_E = int(ce.rows.G.shape[0]), ce.n_dir, ce.n_E
    n_g_cxr = n_g
    pairs = n_seg * n_g * n_dir
    peak_fp32 = 148 * 128 * 2 * 1.965e9 / 1e12
    cxr_tflops = pairs * ALG_FLOPS_PAIR / (mixed["t_cxr"] / 1e3) / 1e12
    # Second census with the bin-mean deposit: (line, bin) items per pair from
    # the comparison pass's counters, ~80 FP32 flops each (midpoint series,
    # closed far form or antiderivative difference).
    items_per_pair = cxr_work["deposit_items"] / max(1.0, cxr_work["segments"] * n_g_cxr * mixed_case.n_dir)
    cxr_tflops_dep = pairs * (ALG_FLOPS_PAIR + items_per_pair * ALG_FLOPS_ITEM) / (mixed["t_cxr"] / 1e3) / 1e12
    brem_pairs_s = n_seg * n_E / (r_head["t_brem"] / 1e3)
    thin = brem_thin_fraction(ce, spec, n_seg, torch)
    flops_brem = thin * ALG_FLOPS_BREM_THIN + (1.0 - thin) * ALG_FLOPS_BREM_THICK
    sfu_brem = thin * 1.0 + (1.0 - thin) * 2.0 + BREM_FIT_SFU_PER_PAIR
    sm_mhz = (clocks[head].get("sm_mhz") or 1965.0)
    sfu_ceiling = 148 * sm_mhz * 1e6 * SFU_OPS_PER_SM_CLOCK / sfu_brem
    rooflines = {
        "cxr_kernel": {"bound": "fp32", "kernel": "cxr_kernel<float> (exact PXR+CBS lines + bin-mean deposit)",
                       "achieved": cxr_tflops, "peak": peak_fp32, "unit": "TFLOP/s", "frac": cxr_tflops / peak_fp32,
                       "peak_source": "nominal FP32 CUDA-core peak (148 SM x 128 lanes x 2 x 1.965 GHz)",
                       "census": "%g FP32 flops per (segment, reflection, tile) pair" % ALG_FLOPS_PAIR,
                       "with_deposit": {"achieved": cxr_tflops_dep, "frac": cxr_tflops_dep / peak_fp32,
                                        "items_per_pair": items_per_pair, "lines_kept": cxr_work["lines_kept"],
                                        "deposit_items": cxr_work["deposit_items"],
                                        "census": "%g per pair + %g per (line, bin) item" % (ALG_FLOPS_PAIR,
                                                                                           ALG_FLOPS_ITEM)},
                       "traffic": DRAM_BYTES_PER_HISTORY["cxr_kernel"] * H},
    }
    node_state = cases[head].brem_node_state()
    if node_state and node_state[0]["ok"]:
        # the depth-node form scored the step: an HBM census of what it reads
        gbs = NODE_BYTES_PER_SEGMENT * n_seg / (r_head["t_brem"] / 1e3) / 1e9
        rooflines["brem_kernel"] = {
            "bound": "hbm", "kernel": "brem_node_* (depth-node form: energy window and depth grid, moment pass "
                                      "on the FP64 tensor cores, one contraction block per photon energy)",
            "achieved": gbs, "peak": MEASURED_HBM_GBS, "unit": "GB/s", "frac": gbs / MEASURED_HBM_GBS,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
            "census": "%g B per segment (energy, length, z, v_z, electron id); the five launches and the "
                      "left-out segments' per-pair launches all inside the timed brem span" % NODE_BYTES_PER_SEGMENT,
            "node": node_state[0], "segments": n_seg,
            "traffic": None}
    else:
        rooflines["brem_kernel"] = {
            "bound": "fp32", "kernel": "brem_moment_packed_kernel (Bethe-Heitler + Elwert, 16 tiles by direction "
                                       "moments, FP32x2, cubic cross section, thin-segment escape series)",
            "achieved": brem_pairs_s * flops_brem / 1e12, "peak": peak_fp32, "unit": "TFLOP/s",
            "frac": brem_pairs_s * flops_brem / 1e12 / peak_fp32,
            "peak_source": "nominal FP32 CUDA-core peak (148 SM x 128 lanes x 2 x 1.965 GHz)",
            "census": "%.2f FP32 flops per (segment, energy) pair (%g thin-segment, %g otherwise; %.3f of the "
                      "pairs thin)" % (flops_brem, ALG_FLOPS_BREM_THIN, ALG_FLOPS_BREM_THICK, thin),
            "thin_fraction": thin,
            "pairs_per_s": brem_pairs_s,
            "sfu": {"achieved": brem_pairs_s, "peak": sfu_ceiling, "unit": "(segment, energy) pairs/s",
                    "frac": brem_pairs_s / sfu_ceiling,
                    "peak_source": "148 SM x measured SM clock x 16 MUFU lanes / %.2f SFU operations per pair"
                                   % sfu_brem},
            "traffic": DRAM_BYTES_PER_HISTORY["brem_kernel"] * H}
    if sur is not None:
        t_sample, t_inf = cases["surrogate"].t_split
        tiles_form = sur["form"] == "tiles"
        # network rows per step: every (segment, tile) pair, or every segment once (tiles form)
        inf_pairs = n_seg * (1 if tiles_form else n_dir) * (1.0 + 1.0 / max(args.exact_stride, 1))
        inf_tflops = inf_pairs * ALG_FLOPS_INFER / (t_inf / 1e3) / 1e12
        rooflines["mlp_infer_kernel"] = {
            "bound": "tensor",
            "kernel": "mlp_infer_kernel (tcgen05 BF16, 4 hidden layers per %s)"
                      % ("segment; tile heads at readout" if tiles_form else "segment x tile"),
            "achieved": inf_tflops, "peak": MEASURED_BF16_SUSTAINED, "unit": "TFLOP/s",
            "frac": inf_tflops / MEASURED_BF16_SUSTAINED,
            "peak_source": "MEASURED_PEAKS.json bf16_tflops_sustained (of measured)",
            "traffic": None if tiles_form else DRAM_BYTES_PER_HISTORY["mlp_infer_kernel"] * H}
        # The exact control variate as it runs in the step: every exact_stride-th
        # segment through cxr_kernel<float> with the narrow exact window, plus
        # the segment sampler and the far-field convolution, all inside t_sample.
        n_sub = int(cases["surrogate"].smp["count"].item())
        sub_pairs = n_sub * n_g * n_dir
        sub_tflops = sub_pairs * ALG_FLOPS_PAIR / (t_sample / 1e3) / 1e12
        sub_items = sub_work["deposit_items"] / max(1.0, sub_work["segments"] * n_g * n_dir)
        sub_tflops_dep = sub_pairs * (ALG_FLOPS_PAIR + sub_items * ALG_FLOPS_ITEM) / (t_sample / 1e3) / 1e12
        rooflines["cxr_subsample"] = {
            "bound": "fp32",
            "kernel": "cxr_kernel<float> on the exact sub-sample (every %d-th segment, %g first-zero widths of "
                      "exact bin means) with the segment sampler and the far-field convolution"
                      % (args.exact_stride, args.cv_exact_widths),
            "achieved": sub_tflops, "peak": peak_fp32, "unit": "TFLOP/s", "frac": sub_tflops / peak_fp32,
            "peak_source": "nominal FP32 CUDA-core peak (148 SM x 128 lanes x 2 x 1.965 GHz)",
            "census": "%g FP32 flops per (segment, reflection, tile) pair" % ALG_FLOPS_PAIR,
            "pairs_per_step": sub_pairs,
            "with_deposit": {"achieved": sub_tflops_dep, "frac": sub_tflops_dep / peak_fp32,
                             "items_per_pair": sub_items, "lines_kept": sub_work["lines_kept"],
                             "deposit_items": sub_work["deposit_items"],
                             "census": "%g per pair + %g per (line, bin) item" % (ALG_FLOPS_PAIR, ALG_FLOPS_ITEM)},
            "traffic": (DRAM_BYTES_PER_SUBSAMPLE_SEGMENT * n_sub if DRAM_BYTES_PER_SUBSAMPLE_SEGMENT else None)}
        sur["kernel_ms"] = {"transport": results["surrogate"]["t_tr"], "exact_subsample": t_sample,
                            "surrogate_infer": t_inf, "brem": results["surrogate"]["t_brem"]}
        sur["value"], sur["ms_per_step"] = rate("surrogate")
        # Training is outside the timed step: its cost spread over a C2-size
        # run of 1e8 histories.
        sur["amortised_rate_1e8_histories_with_training"] = 1e8 / (1e8 / sur["value"] + train_s)
    if head == "mixed":
        cands = [("brem_kernel", r_head["t_brem"]), ("cxr_kernel", r_head["t_cxr"])]
    else:
        t_sample, t_inf = cases["surrogate"].t_split
        cands = [("brem_kernel", r_head["t_brem"]), ("mlp_infer_kernel", t_inf), ("cxr_subsample", t_sample)]
    dominant = max(cands, key=lambda kv: kv[1])[0]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16+f32+f64" if head == "surrogate" else "f32+f64", "data": "synthetic",
        "variant": "surrogate+mixed" if head == "surrogate" else "mixed (surrogate off or failed its gate)",
        "config": workload_config(args, n_dir, n_g, n_E),
        "segments_per_s": world * n_seg / (ms_per_step / 1e3),
        "kernel_ms": {"transport": r_head["t_tr"], "cxr": r_head["t_cxr"], "brem": r_head["t_brem"]},
        "device_status": r_head["status"],
        "roofline": dict(rooflines[dominant], dominant_in_step=True),
        "rooflines": rooflines,
        "gpu_launches": cases[head].kernel_launches_per_batch() * args.steps,
        "clocks": clocks[head],
        "surrogate": sur,
        "spectrum_error_vs_fp64_same_histories": errors,
        "mixed_exact": {"value": rate("mixed")[0], "ms_per_step": rate("mixed")[1], "pairs_per_s": world * pairs /
                        (rate("mixed")[1] / 1e3), "kernel_ms": {"transport": mixed["t_tr"], "cxr": mixed["t_cxr"],
                                                                 "brem": mixed["t_brem"]},
                        "spectrum_check": {"cxr_integral": float(mixed["res"]["cxr"].sum()),
                                           "brem_integral": float(mixed["res"]["brem"].sum()),
                                           "fates": [int(v) for v in mixed["res"]["fates"]]}},
    }
    if "fp64" in compare:
        fp64_ms = compare["fp64"]["ms_per_step"]
        if dist is not None:
            t = torch.tensor([fp64_ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            fp64_ms = float(t.item())
        fp64_value = world * H / (fp64_ms / 1e3)
        line["fp64"] = {"value": fp64_value, "ms_per_step": fp64_ms, "steps": C - 1, "warmup": 1,
                        "timed_on": "the comparison batches 2..C (batch 1 is the warm-up)",
                        "device_status": compare["fp64"]["status"]}
        line["speedup_vs_fp64"] = value / fp64_value
    # e2e through the public API with host buffers.
    line["e2e"] = e2e_measure(spec, args, torch, rank, world, dist,
                              surrogates=cases["surrogate"].surrogates if head == "surrogate" else None)
    if world > 1:
        # Final tally exchange: one all-reduce per FP64 spectrum / int64 tally.
        from pyrite_b200.shard import reduce_results

        reduce_results(cases[head].device_results())
        torch.cuda.synchronize()
    if rank == 0 and world == 1 and not args.skip_cpu:
        rate_c, cores, sample = run_cpu_reference(args)
        line["cpu_baseline"] = {"value": rate_c, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
                                "same_config": True}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def e2e_measure(spec, args, torch, rank, world, dist, surrogates=None):
    """Same batches through ``pyrite_b200.simulate_case_host`` with host buffers.

    Whole-job rate: every rank runs its own histories; the slowest rank's
    time sets the rate of all of them.
    """
    from pyrite_b200.pipeline import simulate_case_host

    steps = max(1, args.steps)
    res = simulate_case_host(spec, args.histories, steps=steps, warmup=args.warmup, precision="mixed",
                             e_start=10_000_000 + rank * 10_000_000, surrogates=surrogates,
                             exact_stride=args.exact_stride,
                             sample_exact_widths=args.cv_exact_widths if surrogates else None)
    ms = float(res["ms_per_step"])
    if dist is not None:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return {"value": world * args.histories / (ms / 1e3), "unit": UNIT,
            "h2d_bytes_per_step": res["h2d_bytes_per_step"], "d2h_bytes_per_step": res["d2h_bytes_per_step"],
            "steps": steps, "warmup": args.warmup}


if __name__ == "__main__":
    main()
