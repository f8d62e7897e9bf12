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
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
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

    e_start, n, directions = payload
    spec = configs.c2_si_50mev()
    st = spec.stack
    lt = oracle.LayerTables(st.z_top, st.z_bot, st.n_el, st.Z, st.J, st.N, st.E_cross)
    # Entry: Twiss beam sampled like the device (reference SplitMix64 stream
    # needs the reference's ndtri; the CPU arm uses the mean beam direction).
    bd = np.asarray(spec.beam.beam_dir, float)
    pos = np.zeros((n, 3))
    dirs = np.tile(bd, (n, 1))
    E = np.full(n, spec.beam.E0_keV)
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
    sample = (f"{done} histories of the same scene ({per} per process x {cores} processes), "
              f"transport + PXR/CBS bin means + Bethe-Heitler on all {n_dir} tiles")
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
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(n_steps)]
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
    if dist is not None:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    return total_ms, t_tr, t_cxr, t_brem


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
            "config": {"workload": "50 MeV e- on 500 um Si (220), 16 tiles, 2048 bins (CPU oracle port)"},
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return

    import torch

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

    spec = configs.c2_si_50mev(seed=12345)
    cases = {}
    results = {}
    for precision in (["mixed"] if args.skip_fp64 else ["mixed", "fp64"]):
        case = ScoringCase(spec, precision=precision, rng="philox", lut=True, batch_histories=args.histories)
        cases[precision] = case
        if precision == "mixed":
            with ClockSampler(local) as clk:
                total_ms, t_tr, t_cxr, t_brem = time_pipeline(case, args, rank, world, torch, dist,
                                                              args.steps, args.warmup)
            clocks = clk.summary()
        else:
            total_ms, t_tr, t_cxr, t_brem = time_pipeline(case, args, rank, world, torch, dist,
                                                          max(1, args.steps // 2), args.warmup)
        n_steps = args.steps if precision == "mixed" else max(1, args.steps // 2)
        results[precision] = dict(total_ms=total_ms, n_steps=n_steps, t_tr=t_tr, t_cxr=t_cxr, t_brem=t_brem,
                                  status=case.device_status(), res=case.results())
    mixed = results["mixed"]
    for name, r in results.items():
        if not (r["res"]["cxr"].sum() > 0 and r["res"].get("brem", np.ones(1)).sum() > 0):
            raise SystemExit(f"bench: the {name} spectra are empty; refusing to report a rate")
    ms_per_step = mixed["total_ms"] / mixed["n_steps"]
    value = world * args.histories / (ms_per_step / 1e3)
    case = cases["mixed"]
    n_seg = mixed["res"]["segments_last_batch"]
    n_g, n_dir, n_E = int(case.rows.G.shape[0]), case.n_dir, case.n_E
    pairs = n_seg * n_g * n_dir
    achieved_tflops = pairs * ALG_FLOPS_PAIR / (mixed["t_cxr"] / 1e3) / 1e12
    peak_fp32 = 148 * 128 * 2 * 1.965e9 / 1e12
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": workload_config(args, n_dir, n_g, n_E),
        "segments_per_s": world * n_seg / (ms_per_step / 1e3),
        "pairs_per_s": world * pairs / (ms_per_step / 1e3),
        "kernel_ms": {"transport": mixed["t_tr"], "cxr": mixed["t_cxr"], "brem": mixed["t_brem"]},
        "device_status": mixed["status"],
        "spectrum_check": {
            "cxr_integral": float(mixed["res"]["cxr"].sum()),
            "brem_integral": float(mixed["res"]["brem"].sum()) if "brem" in mixed["res"] else None,
            "fates": [int(v) for v in mixed["res"]["fates"]],
        },
        "roofline": {
            "bound": "fp32", "kernel": "cxr_kernel<float> (PXR+CBS lines + bin-mean deposit)",
            "achieved": achieved_tflops, "peak": peak_fp32, "unit": "TFLOP/s",
            "frac": achieved_tflops / peak_fp32,
            "peak_source": "nominal FP32 CUDA-core peak (148 SM x 128 lanes x 2 x 1.965 GHz); "
                           "MEASURED_PEAKS.json has HBM and bf16 tensor figures only",
            "traffic": None,
        },
        "gpu_launches": case.kernel_launches_per_batch() * args.steps,
        "clocks": clocks,
    }
    if "fp64" in results:
        f = results["fp64"]
        fp64_ms = f["total_ms"] / f["n_steps"]
        line["fp64"] = {"value": world * args.histories / (fp64_ms / 1e3), "ms_per_step": fp64_ms,
                        "kernel_ms": {"transport": f["t_tr"], "cxr": f["t_cxr"], "brem": f["t_brem"]}}
        line["speedup_vs_fp64"] = line["value"] / line["fp64"]["value"]
        a, b = mixed["res"]["cxr"], f["res"]["cxr"]
        peak = np.max(np.abs(b))
        line["spectrum_error_vs_fp64"] = {
            "note": "different history batches; statistical comparison of the tile-summed CXR spectra",
            "max_rel_to_peak": float(np.max(np.abs(a.sum(0) - b.sum(0))) / (n_dir * peak)) if peak > 0 else None,
        }
    # e2e through the public API with host buffers.
    line["e2e"] = e2e_measure(spec, args, torch, rank, world, dist)
    if world > 1:
        # Final tally exchange: one all-reduce per FP64 spectrum / int64 tally.
        from pyrite_b200.shard import reduce_results

        reduce_results(cases["mixed"].device_results())
        torch.cuda.synchronize()
    if rank == 0 and world == 1 and not args.skip_cpu:
        rate, cores, sample = run_cpu_reference(args)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def e2e_measure(spec, args, torch, rank, world, dist):
    """Same batches through ``pyrite_b200.simulate_case_host`` with host buffers.

    Whole-job rate: every rank runs its own histories; the slowest rank's
    time sets the rate of all of them.
    """
    from pyrite_b200.pipeline import simulate_case_host

    steps = max(1, args.steps // 2)
    res = simulate_case_host(spec, args.histories, steps=steps, warmup=args.warmup, precision="mixed",
                             e_start=10_000_000 + rank * 10_000_000)
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
