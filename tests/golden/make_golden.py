"""Generate the golden vectors the oracle is pinned against, by running the reference.

Run from the repository root, in a container that holds the reference tree::

    python tests/golden/make_golden.py [--only NAME ...]

It imports PyRITE v0.36.2 through ``oracle.ref_harness`` (stand-ins for the
absent third-party packages; ``PYRITE_MC_BACKEND=cpu``) and calls the
reference's own CPU functions on seeded inputs. Every fixture stores the
inputs it was made from next to the reference's outputs, so the tests never
need the reference at run time. Data the reference would read from absent
tables (EPDL attenuation, Chantler refraction, the CXR tabulation mesh) is
injected through the reference's own module seams with the smooth analytic
tables of ``synthetic_tables`` below; the arithmetic that consumes them is
the reference's.
"""

from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from oracle.ref_harness import import_reference  # noqa: E402

# The reference tree this recipe reads: $PYRITE_REFERENCE_ROOT, else the
# read-only mount of the build container.
REFERENCE_ROOT = Path(os.environ.get("PYRITE_REFERENCE_ROOT", "/root/reference"))
import_reference(REFERENCE_ROOT)

from pyrite.montecarlo import geometry as ref_geometry  # noqa: E402
from pyrite.montecarlo.transport import TransportLUTConfig, _simulate_trajectories  # noqa: E402
from pyrite.montecarlo.transport import kinematics as ref_kin  # noqa: E402
from pyrite.montecarlo.transport import scattering as ref_scat  # noqa: E402
from pyrite.montecarlo.transport import stopping as ref_stop  # noqa: E402


def _save(name, **arrays):
    path = OUT / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    print(f"wrote {path.relative_to(ROOT)} ({path.stat().st_size / 1024:.1f} KiB)")


# ---------------------------------------------------------------------------
# RNG: SplitMix64 counter stream (pyrite/montecarlo/transport/kinematics.py:205-246)
# and the Philox4x32-10 published vector quoted by the reference's tests.
# ---------------------------------------------------------------------------
def gen_rng():
    xs = np.array([0, 1, 2, 3, 2**32 - 1, 2**63 + 7, 2**64 - 1], dtype=np.uint64)
    sm = np.array([int(ref_kin._splitmix64(np.uint64(x))) for x in xs], dtype=np.uint64)
    keys = ref_kin.stream_keys(7, 64)
    keys_block = ref_kin.stream_keys(7, 16, start=100)
    pairs = []
    for elec in (0, 1, 4095, 123456789):
        key = int(ref_kin._stream_key_scalar(3, elec))
        for counter in (0, 1, 2, 997, 10**6):
            u = ref_kin._stream_uniform_scalar(np.uint64(key), np.uint64(counter))
            pairs.append((elec, counter, key, u))
    pairs = np.array(pairs, dtype=object)
    cu = ref_kin.counter_uniforms(np.uint64(2**40 + 5), 8, 3, start=11)
    # Random123 Philox4x32-10, counter = key = 0 (tests/montecarlo/quantum/
    # test_channeling_axial_cuda.py:129).
    philox_words = np.array([0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8], dtype=np.uint32)
    _save(
        "rng",
        splitmix_in=xs,
        splitmix_out=sm,
        stream_keys_seed7=keys,
        stream_keys_seed7_start100=keys_block,
        uniform_elec=pairs[:, 0].astype(np.int64),
        uniform_counter=pairs[:, 1].astype(np.int64),
        uniform_key=np.array([int(k) for k in pairs[:, 2]], dtype=np.uint64),
        uniform_value=pairs[:, 3].astype(np.float64),
        counter_uniforms_root=np.uint64(2**40 + 5),
        counter_uniforms_out=cu,
        philox_zero_words=philox_words,
    )


# ---------------------------------------------------------------------------
# Transport physics leaves (scattering.py:208,114,234; stopping.py:384)
# ---------------------------------------------------------------------------
def _layer_coefficients(composition):
    from pyrite.materials._transport_data import TRANSPORT_ELEMENTS

    rows = []
    for el, n in composition:
        p = TRANSPORT_ELEMENTS[el]
        Z, A, J = float(p["Z"]), float(p["A"]), float(p["J_keV"])
        rows.append(
            dict(
                el=el,
                Z=Z,
                A=A,
                J=J,
                n=n,
                k=0.731 + 0.0688 * np.log10(Z),
                coeff=(n / 0.602214076) * Z,
                E_cross=ref_stop._element_crossover_keV(el, Z, A, J),
                sr_rate_numer=5.21e-21 * Z * Z * 4.0 * np.pi * (n * 1e24),
                sr_joy_numer=3.4e-3 * Z**0.67,
            )
        )
    return rows


def gen_physics_leaves():
    comps = {
        "C": [("C", 0.1133)],
        "Si": [("Si", 0.04994)],
        "W": [("W", 0.0632)],
        "SiO2": [("Si", 0.0227), ("O", 0.0454)],
    }
    E = np.geomspace(5.0, 1.2e5, 97)
    out = {"E_keV": E}
    for name, comp in comps.items():
        rows = _layer_coefficients(comp)
        J = np.array([r["J"] for r in rows])
        k = np.array([r["k"] for r in rows])
        coeff = np.array([r["coeff"] for r in rows])
        Ec = np.array([r["E_cross"] for r in rows])
        srn = np.array([r["sr_rate_numer"] for r in rows])
        sjn = np.array([r["sr_joy_numer"] for r in rows])
        out[f"{name}_Z"] = np.array([r["Z"] for r in rows])
        out[f"{name}_A"] = np.array([r["A"] for r in rows])
        out[f"{name}_J"] = J
        out[f"{name}_n"] = np.array([r["n"] for r in rows])
        out[f"{name}_E_cross"] = Ec
        out[f"{name}_dEds"] = np.array(
            [ref_stop._dEds_spliced_compound_scalar(J, k, coeff, Ec, 0.0, e) for e in E]
        )
        rates = np.array(
            [[ref_scat._scatter_rates_sr_scalar(e, srn[i], sjn[i]) for i in range(len(rows))] for e in E]
        )
        out[f"{name}_sr_rates"] = rates
        out[f"{name}_alpha"] = np.array([[sjn[i] / e for i in range(len(rows))] for e in E])
    R = np.linspace(0.0, 0.999, 11)
    alphas = np.array([1e-7, 1e-4, 0.3])
    out["cos_R"] = R
    out["cos_alpha"] = alphas
    out["cos_theta"] = np.array(
        [[ref_scat._sample_cos_theta_from_alpha(a, r) for r in R] for a in alphas]
    )
    _save("physics_leaves", **out)


# ---------------------------------------------------------------------------
# Transport, per-electron core (pyrite/montecarlo/transport/cores.py:96-1230)
# ---------------------------------------------------------------------------
ROW_KEYS = (
    "r_mid",
    "v_hat",
    "L_ang",
    "E_keV",
    "E_end_keV",
    "E_repr_keV",
    "t_ang",
    "t_end_ang",
    "elec_id",
    "layer",
    "flight_id",
    "event_kind",
)
COUNT_KEYS = (
    "n_backscattered",
    "n_transmitted",
    "n_side_exited",
    "n_cutoff_stopped",
    "n_step_limited",
    "n_missed",
)

TRANSPORT_CASES = {
    # HOPG-density carbon, 20 MeV, 100 um, 45 deg tilt, 1 mm FWHM spot.
    "c20mev": dict(
        E0_keV=20000.0, Ne=48, layers=[(0.0, 1.0e6, [("C", 0.1133)])], seed=0,
        tilt_deg=45.0, theta_obs_deg=90.0, beam_fwhm_mm=1.1774,
    ),
    # Si 50 MeV, 500 um, 10 deg tilt.
    "si50mev": dict(
        E0_keV=50000.0, Ne=24, layers=[(0.0, 5.0e6, [("Si", 0.04994)])], seed=3,
        tilt_deg=10.0, theta_obs_deg=20.0, beam_fwhm_mm=2.3548,
    ),
    # Three-layer stack C / Si / W at 10 MeV.
    "stack10mev": dict(
        E0_keV=10000.0, Ne=12,
        layers=[
            (0.0, 2.0e5, [("C", 0.1133)]),
            (2.0e5, 2.2e6, [("Si", 0.04994)]),
            (2.2e6, 2.4e6, [("W", 0.0632)]),
        ],
        seed=5, tilt_deg=0.0, theta_obs_deg=20.0, beam_fwhm_mm=None,
    ),
    # Low-energy Si: backscatter and cutoff exits (the reference test BASE_CASE).
    "si30kev": dict(
        E0_keV=30.0, Ne=16, layers=[(0.0, 5.0e4, [("Si", 0.04996)])], seed=11,
        tilt_deg=0.0, theta_obs_deg=119.0, beam_fwhm_mm=None,
    ),
    # Two-element compound: element choice by partial rate.
    "sio2_300kev": dict(
        E0_keV=300.0, Ne=16, layers=[(0.0, 2.0e5, [("Si", 0.0227), ("O", 0.0454)])], seed=2,
        tilt_deg=30.0, theta_obs_deg=90.0, beam_fwhm_mm=0.5,
    ),
}


def run_reference_transport(case, lut=False):
    layers = case["layers"]
    tp = np.deg2rad(case["tilt_deg"])
    beam_dir, n_hat = ref_geometry.tilted_geometry(np.deg2rad(case["theta_obs_deg"]), tp, 0.0)
    kwargs = dict(
        E0_keV=case["E0_keV"],
        Ne=case["Ne"],
        thickness_ang=layers[-1][1],
        seed=case["seed"],
        elastic_model="sr",
        transport_core="per-electron",
        radiative_model="uncoupled",
        beam_dir=beam_dir,
        tilt_polar_rad=tp,
        beam_fwhm_mm=case["beam_fwhm_mm"],
        transport_lut_config=TransportLUTConfig(enabled=bool(lut)),
    )
    if len(layers) == 1:
        kwargs["composition"] = layers[0][2]
    else:
        kwargs["layers"] = layers
    out = _simulate_trajectories(**kwargs)
    return out, beam_dir, n_hat


def _pack_layers(layers):
    z_top = np.array([l[0] for l in layers])
    z_bot = np.array([l[1] for l in layers])
    n_el = np.array([len(l[2]) for l in layers], dtype=np.int32)
    syms = [[el for el, _ in l[2]] for l in layers]
    dens = [[n for _, n in l[2]] for l in layers]
    width = int(n_el.max())
    from pyrite.materials._transport_data import TRANSPORT_ELEMENTS

    Z = np.zeros((len(layers), width))
    A = np.zeros((len(layers), width))
    J = np.zeros((len(layers), width))
    N = np.zeros((len(layers), width))
    for i, (ss, dd) in enumerate(zip(syms, dens)):
        for j, (s, d) in enumerate(zip(ss, dd)):
            p = TRANSPORT_ELEMENTS[s]
            Z[i, j], A[i, j], J[i, j], N[i, j] = p["Z"], p["A"], p["J_keV"], d
    return z_top, z_bot, n_el, Z, A, J, N


def gen_transport():
    for name, case in TRANSPORT_CASES.items():
        out, beam_dir, n_hat = run_reference_transport(case)
        z_top, z_bot, n_el, Z, A, J, N = _pack_layers(case["layers"])
        E_cross = np.zeros_like(Z)
        from pyrite.materials._transport_data import TRANSPORT_ELEMENTS

        for i, layer in enumerate(case["layers"]):
            for j, (s, _d) in enumerate(layer[2]):
                p = TRANSPORT_ELEMENTS[s]
                E_cross[i, j] = ref_stop._element_crossover_keV(s, float(p["Z"]), float(p["A"]), float(p["J_keV"]))
        arrays = {k: np.asarray(out[k]) for k in ROW_KEYS}
        counts = np.array([int(out[k]) for k in COUNT_KEYS], dtype=np.int64)
        _save(
            f"transport_{name}",
            E0_keV=case["E0_keV"],
            E_cut_keV=5.0,
            seed=case["seed"],
            Ne=case["Ne"],
            beam_dir=beam_dir,
            n_hat=n_hat,
            z_top=z_top,
            z_bot=z_bot,
            n_el=n_el,
            Z=Z,
            A=A,
            J=J,
            N=N,
            E_cross=E_cross,
            initial_r=out["initial_r_ang"],
            initial_v=out["initial_v_hat"],
            initial_E=out["initial_E_keV"],
            count_names=np.array(COUNT_KEYS),
            counts=counts,
            **arrays,
        )


# ---------------------------------------------------------------------------
# Synthetic data tables injected into the reference's CXR/brem data seams.
# Smooth, positive, analytic; stand-ins for the absent Chantler/EPDL data.
# ---------------------------------------------------------------------------
def synthetic_E_tab(E_grid):
    pad = 0.2 * (float(E_grid[-1]) - float(E_grid[0]))
    lo, hi = max(float(E_grid[0]) - pad, 1.0), float(E_grid[-1]) + pad
    return np.geomspace(lo, hi, 700)


def synthetic_delta(E):
    E = np.asarray(E, dtype=float)
    return 4.5e-6 * (1.0e4 / (E + 500.0)) ** 2


def synthetic_log_mu(composition, E):
    E = np.asarray(E, dtype=float)
    rows = []
    for i, (el, n) in enumerate(composition):
        scale = (1.0 + 0.7 * i) * n / 0.05
        rows.append(np.log(scale * (2.0e-4 * (1.0e4 / E) ** 2.8 + 3.0e-7)))
    return np.stack(rows, axis=0)


def synthetic_mu_total(composition, E):
    return np.exp(synthetic_log_mu(composition, E)).sum(axis=0)


def synthetic_couplings(g_mags, E_tab):
    E = np.asarray(E_tab, dtype=float)[None, :]
    g = np.asarray(g_mags, dtype=float)[:, None]
    lam2 = (1.0e4 / E) ** 2
    chi_re = -2.5e-6 * lam2 * np.exp(-0.012 * g * g) * (1.0 + 0.05 * np.cos(3.0 * g))
    chi_im = 0.03 * chi_re * (1.0e4 / (E + 2.0e3)) + 1.0e-9 * np.sin(g)
    u_re = 3.0e-6 * np.exp(-0.006 * g * g) / (1.0 + 0.08 * g * g) + 0.0 * E
    u_im = 2.0e-8 * np.cos(g) + 0.0 * E
    return chi_re, chi_im, u_re, u_im


CXR_CASES = {
    # HOPG-density carbon rows at 20 MeV, 45 deg tilt, 90 deg detector,
    # fibre (00l) rows, Gauss-Hermite mosaic; grid 1-40 keV in 50 eV steps.
    "hopg20": dict(
        transport="c20mev", crystal="hopg", absorber="C", surface_hkl=(0, 0, 1),
        hkl=[(0, 0, l) for l in range(-8, 9) if l != 0],
        mosaic_fwhm_deg=0.4 * 2.3548200450309493, mosaic_nodes=3,
        E_grid=np.arange(1000.0, 40000.0 + 1e-6, 50.0),
    ),
    # Si rows at 50 MeV, (220) cut, 10 deg tilt, 20 deg detector, perfect
    # crystal; grid 1-60 keV in 2048 nodes.
    "si50": dict(
        transport="si50mev", crystal="silicon", absorber="Si", surface_hkl=(2, 2, 0),
        hkl="diamond<=4", mosaic_fwhm_deg=None, mosaic_nodes=1,
        E_grid=np.linspace(1000.0, 60000.0, 2048),
    ),
}


def _diamond_hkls(hmax):
    out = []
    r = range(-hmax, hmax + 1)
    for h in r:
        for k in r:
            for l in r:
                if (h, k, l) == (0, 0, 0):
                    continue
                odd = h % 2 and k % 2 and l % 2
                even = (h % 2 == 0) and (k % 2 == 0) and (l % 2 == 0) and (h + k + l) % 4 == 0
                if odd or even:
                    out.append((h, k, l))
    return out


def gen_cxr():
    from pyrite.materials.crystal import CRYSTALS, reciprocal_g_vector
    from pyrite.montecarlo.spectrum.cxr import _batched, _setup
    from pyrite.montecarlo.spectrum.cxr._spectrum import mc_cxr_spectrum

    for name, case in CXR_CASES.items():
        tr = np.load(OUT / f"transport_{case['transport']}.npz")
        seg = {
            "r_mid": tr["r_mid"], "v_hat": tr["v_hat"], "L_ang": tr["L_ang"],
            "E_keV": tr["E_keV"], "E_repr_keV": tr["E_repr_keV"], "elec_id": tr["elec_id"],
            "Ne": int(tr["Ne"]), "thickness_ang": float(tr["z_bot"][-1]),
        }
        info = CRYSTALS[case["crystal"]]
        hkl = _diamond_hkls(4) if case["hkl"] == "diamond<=4" else case["hkl"]
        g_mags = np.array([reciprocal_g_vector(h, info["lattice"])[1] for h in hkl])
        E_grid = case["E_grid"]
        E_tab = synthetic_E_tab(E_grid)
        n_atoms = len(info["basis"]) / info["V_cell"]
        comp = [(case["absorber"], n_atoms)]
        tables = synthetic_couplings(g_mags, E_tab)
        captured = {}
        orig_brt = _batched._batched_reflection_tables

        def capture(st, _orig=orig_brt):
            out = _orig(st)
            captured["rows"] = out
            return out

        patches = [
            (_setup, "_line_tabulation_grid", lambda *a, **k: E_tab),
            (_setup, "_elemental_log_mu_table", lambda c, E: synthetic_log_mu(c, E)),
            (_setup, "refractive_index", lambda cr, E, uh=True: (1.0 - synthetic_delta(E)) + 0j),
            (_batched, "_reflection_tables", lambda *a, **k: tuple(np.array(t) for t in tables)),
            (_batched, "_batched_reflection_tables", capture),
        ]
        saved = [(m, n, getattr(m, n)) for m, n, _ in patches]
        for m, n, f in patches:
            setattr(m, n, f)
        try:
            common = dict(
                crystal=case["crystal"], hkl_list=[tuple(h) for h in hkl],
                B_ang2=float(info.get("B_ang2", 0.0) or 0.0), absorber_element=case["absorber"],
                n_hat=tr["n_hat"], surface_hkl=case["surface_hkl"],
                mosaic_fwhm_rad=None if case["mosaic_fwhm_deg"] is None else np.deg2rad(case["mosaic_fwhm_deg"]),
                mosaic_nodes=case["mosaic_nodes"], node_support_cutoff=None,
            )
            spec_node = np.asarray(mc_cxr_spectrum(seg, E_grid, line_quadrature="node", **common))
            spec_bin = np.asarray(mc_cxr_spectrum(seg, E_grid, line_quadrature="bin-mean", **common))
        finally:
            for m, n, f in saved:
                setattr(m, n, f)
        G, ES, EP, WM, _cr, _ci, _ur, _ui, ROW_TABLE = captured["rows"][:9]
        _save(
            f"cxr_{name}",
            transport=case["transport"], crystal=case["crystal"], hkl=np.array(hkl, dtype=np.int64),
            g_mags=g_mags, lattice_a=float(info["lattice"]["a"]),
            n_hat=tr["n_hat"], thickness=seg["thickness_ang"], Ne=seg["Ne"],
            surface_hkl=np.array(case["surface_hkl"]),
            mosaic_fwhm_rad=np.nan if case["mosaic_fwhm_deg"] is None else np.deg2rad(case["mosaic_fwhm_deg"]),
            mosaic_nodes=case["mosaic_nodes"],
            E_grid=E_grid, E_tab=E_tab, delta=synthetic_delta(E_tab),
            log_mu=synthetic_log_mu(comp, E_tab), absorber_n=n_atoms,
            chi_re=tables[0], chi_im=tables[1], u_re=tables[2], u_im=tables[3],
            G=np.asarray(G), ES=np.asarray(ES), EP=np.asarray(EP), WM=np.asarray(WM).reshape(-1),
            row_table=np.asarray(ROW_TABLE), spec_node=spec_node, spec_binmean=spec_bin,
        )


def gen_brem():
    from pyrite.montecarlo.spectrum import brem as ref_brem

    for name, tname, comp_el in (("c20", "c20mev", "C"), ("sio2", "sio2_300kev", None)):
        tr = np.load(OUT / f"transport_{tname}.npz")
        seg = {
            "r_mid": tr["r_mid"], "v_hat": tr["v_hat"], "L_ang": tr["L_ang"],
            "E_keV": tr["E_keV"], "E_repr_keV": tr["E_repr_keV"], "elec_id": tr["elec_id"],
            "Ne": int(tr["Ne"]), "thickness_ang": float(tr["z_bot"][-1]),
        }
        n_el = int(tr["n_el"][0])
        comp = [(["C", "Si", "O", "W"][[6, 14, 8, 74].index(int(z))], float(n)) for z, n in zip(tr["Z"][0][:n_el], tr["N"][0][:n_el])]
        E_grid = np.linspace(1000.0, 40000.0, 391) if comp_el else np.linspace(1000.0, 250000.0, 300)
        saved = ref_brem._mu_total_inv_ang
        ref_brem._mu_total_inv_ang = lambda c, E: synthetic_mu_total(c, np.asarray(E, dtype=float))
        try:
            spec = np.asarray(ref_brem.mc_brem_spectrum(
                seg, E_grid, composition=comp, n_hat=tr["n_hat"],
                cross_section_model="bethe-heitler",
            ))
        finally:
            ref_brem._mu_total_inv_ang = saved
        from pyrite.materials._transport_data import TRANSPORT_ELEMENTS

        _save(
            f"brem_{name}", transport=tname, E_grid=E_grid,
            Z=np.array([float(TRANSPORT_ELEMENTS[e]["Z"]) for e, _ in comp]),
            n_ang3=np.array([n for _, n in comp]),
            mu_grid=synthetic_mu_total(comp, E_grid), n_hat=tr["n_hat"],
            thickness=seg["thickness_ang"], Ne=seg["Ne"], spec=spec,
        )


def gen_cxr_leaves():
    from pyrite.montecarlo.spectrum.cxr._bin_quadrature import sincsq_bin_masses, sincsq_tail
    from pyrite.montecarlo.spectrum.cxr._recoil import _quantum_line_factors
    from pyrite.montecarlo.spectrum.segment_escape import mean_transmission

    rng = np.random.default_rng(344)
    n = 64
    args = dict(
        h=np.full(n, 1973.269804 / 510998.95),
        gamma=rng.uniform(10.0, 200.0, n),
        vdg=rng.uniform(0.2, 4.0, n),
        k_dot_v=rng.uniform(0.5, 30.0, n),
        k_dot_g=rng.uniform(-3.0, 3.0, n),
        g2=rng.uniform(1.0, 40.0, n),
        k2=rng.uniform(1.0, 900.0, n),
        v_dot_e=rng.uniform(-0.5, 0.5, n),
        g_dot_e=rng.uniform(-3.0, 3.0, n),
        k_dot_e=rng.uniform(-1e-3, 1e-3, n),
    )
    pxr, cbs = _quantum_line_factors(*args.values())
    x = np.concatenate([np.linspace(-30.0, 30.0, 241), [1e-9, -1e-9, 0.0, 3.7e3, -8.1e4, 2.5e6]])
    tails = sincsq_tail(x)
    a_w = rng.uniform(0.002, 3.0, 40)
    e_r = rng.uniform(900.0, 41000.0, 40)
    edges = np.linspace(975.0, 40025.0, 782)
    masses = sincsq_bin_masses(a_w, e_r, edges)
    t0 = np.concatenate([rng.uniform(0, 5, 50), [0.3, 0.3, 2.0]])
    t1 = np.concatenate([rng.uniform(0, 5, 50), [0.3 + 5e-5, 0.3, 2.0 + 2e-4]])
    mt = mean_transmission(t0, t1)
    _save(
        "cxr_leaves", **{f"qlf_{k}": v for k, v in args.items()}, qlf_pxr=pxr, qlf_cbs=cbs,
        tail_x=x, tail=tails, bm_a=a_w, bm_E=e_r, bm_edges=edges, bm_mass=masses,
        mt_t0=t0, mt_t1=t1, mt=mt,
    )


def gen_transport_lut():
    """Same cases through the reference's default LUT core (lut.py, cores.py lut=True)."""
    from pyrite.montecarlo.transport import host_pass

    for name in ("c20mev", "stack10mev", "si30kev", "sio2_300kev"):
        case = TRANSPORT_CASES[name]
        captured = {}
        orig = host_pass.build_transport_energy_lut

        def wrapped(*a, _orig=orig, **k):
            out = _orig(*a, **k)
            captured["lut"] = out
            return out

        host_pass.build_transport_energy_lut = wrapped
        try:
            out, beam_dir, n_hat = run_reference_transport(case, lut=True)
        finally:
            host_pass.build_transport_energy_lut = orig
        lut = captured["lut"]
        arrays = {k: np.asarray(out[k]) for k in ROW_KEYS}
        counts = np.array([int(out[k]) for k in COUNT_KEYS], dtype=np.int64)
        _save(
            f"transport_lut_{name}",
            log_E_min=np.float64(lut.log_E_min), inv_dlogE=np.float64(lut.inv_dlogE),
            n_energy=int(lut.n_energy), lut_n_el=np.asarray(lut.n_el),
            lut_total_rate=lut.total_rate, lut_dEds=lut.dEds, lut_inv_beta=lut.inv_beta,
            lut_cdf=lut.cdf, lut_alpha=lut.alpha, E_min_keV=np.float64(lut.E_min_keV),
            E_max_keV=np.float64(lut.E_max_keV), initial_r=out["initial_r_ang"],
            initial_v=out["initial_v_hat"], initial_E=out["initial_E_keV"],
            counts=counts, **arrays,
        )


# ---------------------------------------------------------------------------
# Characteristic lines (pyrite/montecarlo/spectrum/characteristic.py:1033):
# the EEDL/EADL tables are absent, so a synthetic element table (smooth shell
# ionisation cross sections on per-shell grids, line energies and widths) and
# a synthetic cascade response are injected through the module's own seams;
# the reference's arithmetic turns them into Lorentzian profiles, escape
# paths, line yields and the spectrum.
# ---------------------------------------------------------------------------
CHAR_ELEMENTS = {
    # binding energies [eV] of the ionised shells; lines (energy, FWHM) [eV]
    "Si": dict(Z=14, shells=[1839.0, 149.7, 99.8, 99.2],
               lines=[(1739.98, 0.52), (1739.38, 0.52), (1835.94, 0.60), (91.5, 0.3)]),
    "W": dict(Z=74, shells=[69525.0, 12100.0, 11544.0, 10207.0, 2820.0, 2575.0],
              lines=[(59318.2, 43.0), (57981.7, 45.0), (8397.6, 6.2), (8335.2, 6.4), (9672.4, 7.1),
                     (9961.5, 7.3), (11285.9, 8.4), (2775.0, 3.0), (67244.3, 52.0)]),
    "C": dict(Z=6, shells=[288.0], lines=[(277.0, 0.2)]),
}


def synthetic_char_table(element):
    from types import SimpleNamespace

    spec = CHAR_ELEMENTS[element]
    rng = np.random.default_rng(spec["Z"])
    grids, sigmas = [], []
    for i, Eb in enumerate(spec["shells"]):
        n_pts = 60 + 7 * i
        E = np.geomspace(Eb, 1.0e9, n_pts)
        u = E / Eb
        sig = 1.0e-20 * (spec["Z"] / 14.0) ** -1.5 * (1.0 + 0.3 * i) * np.log(u) / (u + 0.5) * (1.0 + 0.02 * np.sin(3.0 * np.log(u)))
        sig[0] = 0.0
        grids.append(E)
        sigmas.append(sig)
    lines = np.array([e for e, _ in spec["lines"]])
    fwhm = np.array([w for _, w in spec["lines"]])
    response = rng.uniform(0.0, 0.3, size=(len(spec["shells"]), lines.size))
    response[rng.uniform(size=response.shape) < 0.25] = 0.0
    return SimpleNamespace(
        element=element, atomic_number=spec["Z"], recommended_cutoff_eV=50.0,
        projectile_energy_eV_by_shell=tuple(grids), ionization_cross_sections_cm2_by_shell=tuple(sigmas),
        ionization_shell_labels=tuple(f"S{i}" for i in range(len(spec["shells"]))),
        line_energy_eV=lines, cxr_fwhm_eV=fwhm, line_labels=np.array([f"L{i}" for i in range(lines.size)]),
        _response=response,
    )


def synthetic_char_mu(composition, E):
    E = np.asarray(E, dtype=float)
    return 1.0e-4 * synthetic_mu_total(composition, E)


def gen_char():
    from pyrite.montecarlo.spectrum import characteristic as CH

    cases = (
        # name, transport, element, emitting composition, layers, grid
        ("si50", "si50mev", "Si", [("Si", 0.04994)], None, np.linspace(1000.0, 60000.0, 2048)),
        ("stack_w", "stack10mev", "W", [("W", 0.0632)], True, np.linspace(1000.0, 80000.0, 1024)),
        ("c20", "c20mev", "C", [("C", 0.1133)], None, np.linspace(1000.0, 40000.0, 780)),
    )
    saved = (CH.load_characteristic_cross_sections, CH._cascade_line_yields, CH._mu_total_inv_ang)
    tables = {}
    try:
        CH.load_characteristic_cross_sections = lambda el, **kw: tables.setdefault(el, synthetic_char_table(el))
        CH._cascade_line_yields = lambda table, cutoff: (None, table._response)
        CH._mu_total_inv_ang = lambda comp, E: synthetic_char_mu(comp, E)
        for name, tname, el, comp, layered, E_grid in cases:
            tr = np.load(OUT / f"transport_{tname}.npz")
            seg = {
                "r_mid": tr["r_mid"], "v_hat": tr["v_hat"], "L_ang": tr["L_ang"], "E_keV": tr["E_keV"],
                "E_repr_keV": tr["E_repr_keV"], "elec_id": tr["elec_id"], "layer": tr["layer"],
                "Ne": int(tr["Ne"]), "thickness_ang": float(tr["z_bot"][-1]),
            }
            layers = None
            if layered:
                z_top, z_bot = tr["z_top"], tr["z_bot"]
                layers = []
                for i in range(z_top.size):
                    n = int(tr["n_el"][i])
                    syms = [["C", "Si", "O", "W"][[6, 14, 8, 74].index(int(z))] for z in tr["Z"][i][:n]]
                    layers.append((float(z_top[i]), float(z_bot[i]), list(zip(syms, [float(x) for x in tr["N"][i][:n]]))))
                keep = tr["layer"] == z_top.size - 1  # segments of the emitting (last) layer
                seg = {k: (v[keep] if isinstance(v, np.ndarray) and v.shape[:1] == tr["layer"].shape else v)
                       for k, v in seg.items()}
            spec = np.asarray(CH.mc_characteristic_spectrum(seg, E_grid, composition=comp, n_hat=tr["n_hat"],
                                                            layers=layers))
            table = tables[el]
            edges, widths = CH._energy_bin_edges_and_widths(E_grid)
            prep = CH._prepare_lines(table, comp, layers, edges, widths, 50.0)
            absorbers = [comp] if layers is None else [c for _a, _b, c in layers]
            offs = np.cumsum([0] + [g.size for g in table.projectile_energy_eV_by_shell])
            _save(
                f"char_{name}", transport=tname, element=el, n_atoms=float(comp[0][1]), E_grid=E_grid,
                n_hat=tr["n_hat"], thickness=seg["thickness_ang"], Ne=seg["Ne"],
                layer_z_top=np.array([l[0] for l in layers]) if layers else np.zeros(0),
                layer_z_bot=np.array([l[1] for l in layers]) if layers else np.zeros(0),
                seg_mask=(tr["layer"] == tr["z_top"].size - 1) if layered else np.ones(tr["layer"].size, bool),
                shell_E=np.concatenate(table.projectile_energy_eV_by_shell),
                shell_sigma=np.concatenate(table.ionization_cross_sections_cm2_by_shell),
                shell_offset=offs.astype(np.int64), line_E=table.line_energy_eV, line_fwhm=table.cxr_fwhm_eV,
                response_all=table._response, kept_response=np.asarray(prep.response),
                mu_by_line=np.asarray(prep.mu_by_line), profiles=np.asarray(prep.profiles),
                absorber_mu_check=np.stack([synthetic_char_mu(c, table.line_energy_eV) for c in absorbers]),
                spec=spec,
            )
    finally:
        CH.load_characteristic_cross_sections, CH._cascade_line_yields, CH._mu_total_inv_ang = saved


def synthetic_exact_mu(composition, knots=None):
    """Piecewise-linear mu(E) tables of one composition on a fixed knot set
    (the shape of cxr/_escape_mu.py:ExactMuTable), from synthetic_mu_total."""
    kn = np.geomspace(500.0, 2.0e5, 400) if knots is None else np.asarray(knots, dtype=float)
    val = synthetic_mu_total(composition, kn)
    slope = np.empty_like(val)
    slope[:-1] = np.diff(val) / np.diff(kn)
    slope[-1] = slope[-2]
    return kn, val, slope


def _stack_layers(tr):
    layers = []
    for i in range(tr["z_top"].size):
        n = int(tr["n_el"][i])
        syms = [["C", "Si", "O", "W"][[6, 14, 8, 74].index(int(z))] for z in tr["Z"][i][:n]]
        layers.append((float(tr["z_top"][i]), float(tr["z_bot"][i]), list(zip(syms, [float(x) for x in tr["N"][i][:n]]))))
    return layers


def _layer_segments(tr, L):
    keep = tr["layer"] == L
    seg = {
        "r_mid": tr["r_mid"][keep], "v_hat": tr["v_hat"][keep], "L_ang": tr["L_ang"][keep],
        "E_keV": tr["E_keV"][keep], "E_repr_keV": tr["E_repr_keV"][keep], "elec_id": tr["elec_id"][keep],
        "layer": tr["layer"][keep], "Ne": int(tr["Ne"]), "thickness_ang": float(tr["z_bot"][-1]),
    }
    return seg, keep


def gen_layered():
    """Layered-absorber escape on the 10 MeV C / Si / W stack: per-layer
    Bethe-Heitler (each layer its own composition, escape through the whole
    stack; runner/emission.py:155-172) and PXR+CBS of the two crystalline
    layers (runner/case_driver.py:742-770) with exact per-layer mu tables."""
    from pyrite.materials._transport_data import TRANSPORT_ELEMENTS
    from pyrite.materials.crystal import CRYSTALS, reciprocal_g_vector
    from pyrite.montecarlo.spectrum import brem as ref_brem
    from pyrite.montecarlo.spectrum.cxr import _batched, _setup
    from pyrite.montecarlo.spectrum.cxr._escape_mu import ExactMuTable
    from pyrite.montecarlo.spectrum.cxr._spectrum import mc_cxr_spectrum

    tr = np.load(OUT / "transport_stack10mev.npz")
    layers = _stack_layers(tr)
    out = {"z_top": tr["z_top"], "z_bot": tr["z_bot"], "n_hat": tr["n_hat"], "Ne": int(tr["Ne"]),
           "thickness": float(tr["z_bot"][-1])}
    # bremsstrahlung, every layer
    E_brem = np.linspace(1000.0, 80000.0, 300)
    saved = ref_brem._mu_total_inv_ang
    ref_brem._mu_total_inv_ang = lambda c, E: synthetic_mu_total(c, np.asarray(E, dtype=float))
    try:
        for L, (_zt, _zb, comp) in enumerate(layers):
            seg, _keep = _layer_segments(tr, L)
            out[f"brem_spec_{L}"] = np.asarray(ref_brem.mc_brem_spectrum(
                seg, E_brem, composition=comp, n_hat=tr["n_hat"], layers=layers,
                cross_section_model="bethe-heitler"))
            out[f"brem_Z_{L}"] = np.array([float(TRANSPORT_ELEMENTS[e]["Z"]) for e, _ in comp])
            out[f"brem_n_{L}"] = np.array([n for _, n in comp])
    finally:
        ref_brem._mu_total_inv_ang = saved
    out["brem_E_grid"] = E_brem
    out["brem_mu_layer"] = np.stack([synthetic_mu_total(c, E_brem) for _a, _b, c in layers])
    # PXR + CBS of the HOPG-like carbon layer and the Si layer
    E_grid = np.linspace(1000.0, 60000.0, 1024)
    E_tab = synthetic_E_tab(E_grid)
    mu_tabs = [synthetic_exact_mu(c) for _a, _b, c in layers]
    for k, (kn, val, sl) in enumerate(mu_tabs):
        out[f"mu_knot_{k}"], out[f"mu_value_{k}"], out[f"mu_slope_{k}"] = kn, val, sl
    radiators = {0: ("hopg", (0, 0, 1), [(0, 0, l) for l in range(-8, 9) if l != 0]),
                 1: ("silicon", (2, 2, 0), _diamond_hkls(4))}
    for L, (crystal, surface, hkl) in radiators.items():
        info = CRYSTALS[crystal]
        g_mags = np.array([reciprocal_g_vector(h, info["lattice"])[1] for h in hkl])
        tables = synthetic_couplings(g_mags, E_tab)
        comp = layers[L][2]
        seg, keep = _layer_segments(tr, L)
        captured = {}
        orig_brt = _batched._batched_reflection_tables

        def capture(st, _orig=orig_brt):
            res = _orig(st)
            captured["rows"] = res
            return res

        def exact_tables(req, abs_comp):
            return tuple(ExactMuTable(knots=kn, value=val, slope=sl) for kn, val, sl in mu_tabs)

        patches = [
            (_setup, "_line_tabulation_grid", lambda *a, **k: E_tab),
            (_setup, "_elemental_log_mu_table", lambda c, E: synthetic_log_mu(c, E)),
            (_setup, "refractive_index", lambda cr, E, uh=True: (1.0 - synthetic_delta(E)) + 0j),
            (_batched, "_reflection_tables", lambda *a, **k: tuple(np.array(t) for t in tables)),
            (_batched, "_batched_reflection_tables", capture),
            (_batched, "escape_mu_tables", exact_tables),
        ]
        saved_p = [(m, n, getattr(m, n)) for m, n, _ in patches]
        for m, n, f in patches:
            setattr(m, n, f)
        try:
            common = dict(
                crystal=crystal, hkl_list=[tuple(h) for h in hkl],
                B_ang2=float(info.get("B_ang2", 0.0) or 0.0), composition=comp,
                n_hat=tr["n_hat"], surface_hkl=surface, layers=layers,
                mosaic_fwhm_rad=None, mosaic_nodes=1, node_support_cutoff=None,
            )
            spec_node = np.asarray(mc_cxr_spectrum(seg, E_grid, line_quadrature="node", **common))
            spec_bin = np.asarray(mc_cxr_spectrum(seg, E_grid, line_quadrature="bin-mean", **common))
        finally:
            for m, n, f in saved_p:
                setattr(m, n, f)
        G, ES, EP, WM, _cr, _ci, _ur, _ui, ROW_TABLE = captured["rows"][:9]
        out.update({
            f"cxr_hkl_{L}": np.array(hkl, dtype=np.int64), f"cxr_g_mags_{L}": g_mags,
            f"cxr_chi_re_{L}": tables[0], f"cxr_chi_im_{L}": tables[1], f"cxr_u_re_{L}": tables[2],
            f"cxr_u_im_{L}": tables[3], f"cxr_G_{L}": np.asarray(G), f"cxr_ES_{L}": np.asarray(ES),
            f"cxr_EP_{L}": np.asarray(EP), f"cxr_WM_{L}": np.asarray(WM).reshape(-1),
            f"cxr_row_table_{L}": np.asarray(ROW_TABLE), f"cxr_log_mu_{L}": synthetic_log_mu(comp, E_tab),
            f"cxr_spec_node_{L}": spec_node, f"cxr_spec_binmean_{L}": spec_bin,
        })
    out.update(cxr_E_grid=E_grid, cxr_E_tab=E_tab, cxr_delta=synthetic_delta(E_tab))
    _save("layered_stack10", **out)


COHERENT_FIELDS = ("E_vac", "a_vac", "phase_slope", "g_phase", "cs_re", "cs_im", "cp_re", "cp_im",
                   "L_esc", "elec_id", "half_dL", "apb", "bma", "q")
# The reference's coherent route on the first electrons of two CXR cases
# (fixture size), with segment start ages, so the emission-time phase is live.
COHERENT_CASES = {"hopg20": 8, "si50": 6}


def gen_coherent():
    """Coherent (field-sum) CXR on the batched route (cxr/_batched.py:1029-1240).

    Captures the per-row line records the block loop hands to
    ``_batched_coherent_finalize`` (cxr/_batched_finalize.py:22; record
    layout cxr/_batched.py:646-660), concatenated per row in the finalize's
    order, and the reference's coherent spectrum from those records. Inter-
    electron decoherence is off (no initial beam offsets), so the reduction is
    the flat per-row field sum of _batched_finalize.py:209-243.
    """
    from pyrite.materials.crystal import CRYSTALS, reciprocal_g_vector
    from pyrite.montecarlo.spectrum.cxr import _batched, _setup
    from pyrite.montecarlo.spectrum.cxr._spectrum import mc_cxr_spectrum

    for name, n_elec in COHERENT_CASES.items():
        case = CXR_CASES[name]
        tr = np.load(OUT / f"transport_{case['transport']}.npz")
        sel = tr["elec_id"] < n_elec
        seg = {k: tr[k][sel] for k in ("r_mid", "v_hat", "L_ang", "E_keV", "E_repr_keV", "elec_id", "t_ang")}
        seg.update(Ne=n_elec, thickness_ang=float(tr["z_bot"][-1]))
        info = CRYSTALS[case["crystal"]]
        hkl = _diamond_hkls(4) if case["hkl"] == "diamond<=4" else case["hkl"]
        g_mags = np.array([reciprocal_g_vector(h, info["lattice"])[1] for h in hkl])
        E_grid = case["E_grid"]
        E_tab = synthetic_E_tab(E_grid)
        tables = synthetic_couplings(g_mags, E_tab)
        captured = {}
        orig_fin = _batched._batched_coherent_finalize

        def capture(st, bt, coh_blocks, coh_counts, *a, _orig=orig_fin, **k):
            captured.update(st=st, bt=bt, blocks=[[np.array(f) for f in b] for b in coh_blocks],
                            counts=[np.array(c) for c in coh_counts])
            return _orig(st, bt, coh_blocks, coh_counts, *a, **k)

        patches = [
            (_setup, "_line_tabulation_grid", lambda *a, **k: E_tab),
            (_setup, "_elemental_log_mu_table", lambda c, E: synthetic_log_mu(c, E)),
            (_setup, "refractive_index", lambda cr, E, uh=True: (1.0 - synthetic_delta(E)) + 0j),
            (_batched, "_reflection_tables", lambda *a, **k: tuple(np.array(t) for t in tables)),
            (_batched, "_batched_coherent_finalize", capture),
        ]
        saved = [(m, n, getattr(m, n)) for m, n, _ in patches]
        for m, n, f in patches:
            setattr(m, n, f)
        try:
            spec = np.asarray(mc_cxr_spectrum(
                seg, E_grid, crystal=case["crystal"], hkl_list=[tuple(h) for h in hkl],
                B_ang2=float(info.get("B_ang2", 0.0) or 0.0), absorber_element=case["absorber"],
                n_hat=tr["n_hat"], surface_hkl=case["surface_hkl"],
                mosaic_fwhm_rad=None if case["mosaic_fwhm_deg"] is None else np.deg2rad(case["mosaic_fwhm_deg"]),
                mosaic_nodes=case["mosaic_nodes"], node_support_cutoff=None, coherent=True))
        finally:
            for m, n, f in saved:
                setattr(m, n, f)
        st, bt = captured["st"], captured["bt"]
        if st.decoherence_active:
            raise RuntimeError("coherent fixture expects the flat reduction (no beam offsets)")
        counts = np.stack(captured["counts"])                      # (n_block, N_g)
        starts = np.concatenate([np.zeros((counts.shape[0], 1), counts.dtype), np.cumsum(counts, axis=1)], axis=1)
        rows = {f: [] for f in COHERENT_FIELDS}
        for i_row in range(int(bt.N_g)):
            for b, flat in enumerate(captured["blocks"]):
                for f, arr in zip(COHERENT_FIELDS, flat, strict=True):
                    rows[f].append(arr[int(starts[b, i_row]):int(starts[b, i_row + 1])])
        _save(
            f"coherent_{name}",
            transport=case["transport"], n_elec=n_elec, Ne=n_elec, E_grid=np.asarray(st.E_grid),
            delta_omega=np.asarray(st.delta_omega_grid), row_weight=np.asarray(bt.wm_rows, dtype=float).reshape(-1),
            row_count=counts.sum(axis=0).astype(np.int64), spec=spec,
            **{f: np.concatenate(rows[f]) for f in COHERENT_FIELDS},
        )


def gen_coherent_decoherence():
    """Coherent route with sampled beam offsets on the infinite slab: the
    inter-electron decoherence blend of cxr/_batched_finalize.py:163-243.

    The first 8 electrons of the HOPG 20 MeV case get their transport entry
    points as face offsets (``initial_r_ang``) and seeded arrival offsets
    (``initial_t0_ang``, 0.3 Angstrom RMS of c t), so the route builds
    offset-free records (cxr/_setup.py:637-642), a per-row factor
    F = |<exp(i(omega A_e - g.xy0_e))>|^2 (cxr/_per_hkl.py:121-160), the
    per-electron sum of squared fields (cxr/_per_hkl.py:457-500) and the blend
    (1 - F) grouped + F flat (spectrum/coherent_population.py:83-96). Saves the
    records with their electron ids, the population offsets, each row's
    reciprocal vector, F and grouped term, and the spectrum.
    """
    from pyrite.materials.crystal import CRYSTALS, reciprocal_g_vector
    from pyrite.montecarlo.spectrum.cxr import _batched, _batched_finalize, _setup
    from pyrite.montecarlo.spectrum.cxr._spectrum import mc_cxr_spectrum

    name, n_elec = "hopg20", 8
    case = CXR_CASES[name]
    tr = np.load(OUT / f"transport_{case['transport']}.npz")
    sel = tr["elec_id"] < n_elec
    seg = {k: tr[k][sel] for k in ("r_mid", "v_hat", "L_ang", "E_keV", "E_repr_keV", "elec_id", "t_ang")}
    rng = np.random.default_rng(17)
    r0 = np.array(tr["initial_r"][:n_elec], dtype=float)
    t0 = rng.normal(0.0, 0.3, n_elec)
    seg.update(Ne=n_elec, thickness_ang=float(tr["z_bot"][-1]), initial_r_ang=r0, initial_t0_ang=t0)
    info = CRYSTALS[case["crystal"]]
    hkl = case["hkl"]
    g_mags = np.array([reciprocal_g_vector(h, info["lattice"])[1] for h in hkl])
    E_grid = case["E_grid"]
    E_tab = synthetic_E_tab(E_grid)
    tables = synthetic_couplings(g_mags, E_tab)
    cap = {"F": {}, "grouped": []}
    orig_fin = _batched._batched_coherent_finalize
    orig_F = _batched_finalize._row_decoherence_factor
    orig_grp = _batched_finalize._coherent_electron_grouped_row

    def capture(st, bt, coh_blocks, coh_counts, *a, _orig=orig_fin, **k):
        cap.update(st=st, bt=bt, blocks=[[np.array(f) for f in b] for b in coh_blocks],
                   counts=[np.array(c) for c in coh_counts])
        return _orig(st, bt, coh_blocks, coh_counts, *a, **k)

    def capture_F(st, g_vec, _orig=orig_F):
        out = _orig(st, g_vec)
        cap["F"][tuple(np.asarray(g_vec, dtype=float))] = np.array(out)
        return out

    def capture_grp(*a, _orig=orig_grp, **k):
        out = _orig(*a, **k)
        cap["grouped"].append(np.array(out))
        return out

    patches = [
        (_setup, "_line_tabulation_grid", lambda *a, **k: E_tab),
        (_setup, "_elemental_log_mu_table", lambda c, E: synthetic_log_mu(c, E)),
        (_setup, "refractive_index", lambda cr, E, uh=True: (1.0 - synthetic_delta(E)) + 0j),
        (_batched, "_reflection_tables", lambda *a, **k: tuple(np.array(t) for t in tables)),
        (_batched, "_batched_coherent_finalize", capture),
        (_batched_finalize, "_row_decoherence_factor", capture_F),
        (_batched_finalize, "_coherent_electron_grouped_row", capture_grp),
    ]
    saved = [(m, n, getattr(m, n)) for m, n, _ in patches]
    for m, n, f in patches:
        setattr(m, n, f)
    try:
        spec = np.asarray(mc_cxr_spectrum(
            seg, E_grid, crystal=case["crystal"], hkl_list=[tuple(h) for h in hkl],
            B_ang2=float(info.get("B_ang2", 0.0) or 0.0), absorber_element=case["absorber"],
            n_hat=tr["n_hat"], surface_hkl=case["surface_hkl"],
            mosaic_fwhm_rad=np.deg2rad(case["mosaic_fwhm_deg"]), mosaic_nodes=case["mosaic_nodes"],
            node_support_cutoff=None, coherent=True))
    finally:
        for m, n, f in saved:
            setattr(m, n, f)
    st, bt = cap["st"], cap["bt"]
    if not st.decoherence_active or st.analytic_offsets:
        raise RuntimeError("decoherence fixture expects the sampled (empirical) blend")
    counts = np.stack(cap["counts"])
    starts = np.concatenate([np.zeros((counts.shape[0], 1), counts.dtype), np.cumsum(counts, axis=1)], axis=1)
    rows = {f: [] for f in COHERENT_FIELDS}
    for i_row in range(int(bt.N_g)):
        for b, flat in enumerate(cap["blocks"]):
            for f, arr in zip(COHERENT_FIELDS, flat, strict=True):
                rows[f].append(arr[int(starts[b, i_row]):int(starts[b, i_row + 1])])
    row_count = counts.sum(axis=0).astype(np.int64)
    G = np.asarray(bt.G, dtype=float)
    active = np.flatnonzero(row_count > 0)
    F_rows = np.stack([cap["F"][tuple(G[r])] for r in active])
    if len(cap["grouped"]) != active.size:
        raise RuntimeError("expected one grouped term per row with lines")
    _save(
        "coherent_decoherence_hopg20",
        transport=case["transport"], n_elec=n_elec, Ne=n_elec, E_grid=np.asarray(st.E_grid),
        delta_omega=np.asarray(st.delta_omega_grid), omega=np.asarray(st.omega_grid),
        row_weight=np.asarray(bt.wm_rows, dtype=float).reshape(-1), row_count=row_count, G=G,
        n_hat=np.asarray(tr["n_hat"], dtype=float), initial_r_ang=r0, initial_t0_ang=t0,
        A_pop=np.asarray(st.decoherence_A_pop), xy0_pop=np.asarray(st.xy0_pop),
        active_rows=active, F_rows=F_rows, grouped_rows=np.stack(cap["grouped"]), spec=spec,
        **{f: np.concatenate(rows[f]) for f in COHERENT_FIELDS},
    )


# ---------------------------------------------------------------------------
# Urban energy-loss straggling (pyrite/montecarlo/transport/straggling.py):
# the sampler's leaves on seeded keys, and whole histories of the per-electron
# exact core with straggling=True.
# ---------------------------------------------------------------------------
STRAGGLING_CASES = ("c20mev", "si30kev", "sio2_300kev")


def gen_straggling():
    from pyrite.materials._transport_data import TRANSPORT_ELEMENTS
    from pyrite.montecarlo.transport import straggling as ref_str

    rng = np.random.default_rng(17)
    rows = []
    for el in ("C", "O", "Si", "W"):
        p = TRANSPORT_ELEMENTS[el]
        Z, A, J = float(p["Z"]), float(p["A"]), float(p["J_keV"])
        n = 0.05
        k = 0.731 + 0.0688 * np.log10(Z)
        coeff = (n / 0.602214076) * Z
        E_cross = ref_stop._element_crossover_keV(el, Z, A, J)
        for E in (0.5, 3.0, 30.0, 300.0, 5000.0, 50000.0):
            C = -float(ref_str._dEds_spliced_element_scalar(J, k, coeff, E_cross, 0.0, E))
            for s in (1.0, 1e2, 1e4, 1e6):
                key = int(rng.integers(0, 2**63))
                dE, ctr = ref_str._urban_sample_element_keV(Z, J, C, E, s, np.uint64(key), np.uint64(0))
                m, v = ref_str._urban_moments_element_scalar(Z, J, C, E, s)
                rows.append((Z, J, k, coeff, E_cross, E, s, key, C, float(dE), int(ctr), float(m), float(v)))
    a = np.array([r[:7] for r in rows])
    _save("straggling_leaves", Z=a[:, 0], J=a[:, 1], k=a[:, 2], coeff=a[:, 3], E_cross=a[:, 4], E=a[:, 5],
          s=a[:, 6], key=np.array([r[7] for r in rows], dtype=np.uint64), C=np.array([r[8] for r in rows]),
          dE=np.array([r[9] for r in rows]), counter=np.array([r[10] for r in rows], dtype=np.uint64),
          mean=np.array([r[11] for r in rows]), var=np.array([r[12] for r in rows]))
    for name in STRAGGLING_CASES:
        case = TRANSPORT_CASES[name]
        layers = case["layers"]
        tp = np.deg2rad(case["tilt_deg"])
        beam_dir, n_hat = ref_geometry.tilted_geometry(np.deg2rad(case["theta_obs_deg"]), tp, 0.0)
        kwargs = dict(E0_keV=case["E0_keV"], Ne=case["Ne"], thickness_ang=layers[-1][1], seed=case["seed"],
                      elastic_model="sr", transport_core="per-electron", radiative_model="uncoupled",
                      beam_dir=beam_dir, tilt_polar_rad=tp, beam_fwhm_mm=case["beam_fwhm_mm"],
                      transport_lut_config=TransportLUTConfig(enabled=False), straggling=True)
        if len(layers) == 1:
            kwargs["composition"] = layers[0][2]
        else:
            kwargs["layers"] = layers
        out = _simulate_trajectories(**kwargs)
        arrays = {k: np.asarray(out[k]) for k in ROW_KEYS}
        counts = np.array([int(out[k]) for k in COUNT_KEYS], dtype=np.int64)
        _save(f"straggling_{name}", E0_keV=case["E0_keV"], E_cut_keV=5.0, seed=case["seed"], Ne=case["Ne"],
              initial_r=out["initial_r_ang"], initial_v=out["initial_v_hat"], initial_E=out["initial_E_keV"],
              count_names=np.array(COUNT_KEYS), counts=counts, **arrays)


# ---------------------------------------------------------------------------
# ELSEPA tabulated elastic scattering (transport/scattering.py:330-640,
# cores.py:425-440 and 1120-1180) with synthetic tables passed through the
# reference's public ``elastic_tables`` argument: smooth total cross sections
# and angular densities on a shared mu grid, shaped like screened Rutherford
# with a mild modulation so neither the rates nor the inversion are the
# analytic model's.
# ---------------------------------------------------------------------------
ELSEPA_CASES = ("si30kev", "sio2_300kev", "c20mev")


def synthetic_elsepa_table(symbol):
    """One element's table in the reference's ``elastic_tables`` layout."""
    from pyrite.materials._transport_data import TRANSPORT_ELEMENTS

    Z = float(TRANSPORT_ELEMENTS[symbol]["Z"])
    energy_eV = np.geomspace(1.0e3, 1.0e8, 48)
    E = energy_eV / 1e3
    a = 3.4e-3 * Z ** 0.67 / E
    r = (E + 511.0) / (E + 1024.0)
    sigma = 5.21e-21 * Z * Z * 4.0 * np.pi / (E * E) / (a * (1.0 + a)) * r * r
    sigma = sigma * (1.0 + 0.15 * np.sin(np.log(energy_eV)))
    mu = np.concatenate([[0.0], np.geomspace(1.0e-9, 1.0, 199)])
    dcs = (1.0 + 0.4 * mu[None, :]) / (mu[None, :] + a[:, None]) ** 2
    dcs = dcs * (1.0 + 0.05 * np.cos(7.0 * mu[None, :] + np.log(E)[:, None]))
    return dict(energy_eV=energy_eV, total_elastic_cm2=sigma, mu=mu, dcs_cm2_sr=dcs)


def gen_elsepa():
    rng = np.random.default_rng(29)
    for name in ELSEPA_CASES:
        case = TRANSPORT_CASES[name]
        layers = case["layers"]
        tables = [[synthetic_elsepa_table(el) for el, _n in layer[2]] for layer in layers]
        L_ncm3 = [np.array([n * 1e24 for _el, n in layer[2]]) for layer in layers]
        has, start, length, logE, log_rate, cdf, pdf, mu, guide = ref_scat.pack_elsepa_tables(tables, L_ncm3)
        tp = np.deg2rad(case["tilt_deg"])
        beam_dir, n_hat = ref_geometry.tilted_geometry(np.deg2rad(case["theta_obs_deg"]), tp, 0.0)
        kwargs = dict(E0_keV=case["E0_keV"], Ne=case["Ne"], thickness_ang=layers[-1][1], seed=case["seed"],
                      elastic_model="elsepa", elastic_tables=tables, transport_core="per-electron",
                      radiative_model="uncoupled", beam_dir=beam_dir, tilt_polar_rad=tp,
                      beam_fwhm_mm=case["beam_fwhm_mm"], transport_lut_config=TransportLUTConfig(enabled=False))
        if len(layers) == 1:
            kwargs["composition"] = layers[0][2]
        else:
            kwargs["layers"] = layers
        out = _simulate_trajectories(**kwargs)
        arrays = {k: np.asarray(out[k]) for k in ROW_KEYS}
        counts = np.array([int(out[k]) for k in COUNT_KEYS], dtype=np.int64)
        # leaves: rates and polar cosines at seeded (E, xi) of every element
        n_leaf = 64
        leaf_E = np.exp(rng.uniform(np.log(1.0), np.log(1.0e5), n_leaf))
        leaf_E[:4] = (1.0, 1.0e5, 30.0, 0.5)  # both table ends, a mid value, below the table
        leaf_xi = rng.uniform(0.0, 1.0, n_leaf)
        leaf_xi[4:8] = (0.0, 1.0, 0.5, 1.0 - 2.0 ** -40)
        leaf_rate = np.zeros((len(layers), has.shape[1], n_leaf))
        leaf_cos = np.zeros_like(leaf_rate)
        for L in range(len(layers)):
            for k in range(len(layers[L][2])):
                for j in range(n_leaf):
                    E = float(leaf_E[j])  # below the table the bracket clamps to its first node
                    leaf_rate[L, k, j] = ref_scat._elsepa_rate_scalar(E, logE, log_rate, start[L, k], length[L, k])
                    leaf_cos[L, k, j] = ref_scat._sample_cos_theta_elsepa(E, leaf_xi[j], logE, cdf, pdf, mu, guide,
                                                                          start[L, k], length[L, k])
        raw = {}
        for L, layer in enumerate(tables):
            for k, t in enumerate(layer):
                for f in ("energy_eV", "total_elastic_cm2", "dcs_cm2_sr"):
                    raw[f"raw_{L}_{k}_{f}"] = t[f]
        _save(f"elsepa_{name}", E0_keV=case["E0_keV"], E_cut_keV=5.0, seed=case["seed"], Ne=case["Ne"],
              initial_r=out["initial_r_ang"], initial_v=out["initial_v_hat"], initial_E=out["initial_E_keV"],
              count_names=np.array(COUNT_KEYS), counts=counts,
              el_has=has, el_start=start, el_length=length, el_logE=logE, el_log_rate=log_rate, el_cdf=cdf,
              el_pdf=pdf, el_mu=mu, el_guide=guide, leaf_E=leaf_E, leaf_xi=leaf_xi, leaf_rate=leaf_rate,
              leaf_cos=leaf_cos, **raw, **arrays)


# ---------------------------------------------------------------------------
# SBETHE table stopping (transport/stopping.py:11-103, cores.py:581-600 and
# 720-780) with synthetic per-layer tables passed through the reference's
# public ``stopping_tables`` argument: the layer's spliced analytic stopping
# with a smooth modulation, on a geometric grid from 1 keV to 1 GeV.
# ---------------------------------------------------------------------------
SBETHE_CASES = (("si30kev", False), ("sio2_300kev", False), ("c20mev", False), ("sio2_300kev", True))


def synthetic_sbethe_table(composition):
    from pyrite.materials._transport_data import TRANSPORT_ELEMENTS
    from pyrite.montecarlo.transport import straggling as ref_str

    E_eV = np.geomspace(1.0e3, 1.0e9, 120)
    S = np.zeros_like(E_eV)
    for el, n in composition:
        p = TRANSPORT_ELEMENTS[el]
        Z, A, J = float(p["Z"]), float(p["A"]), float(p["J_keV"])
        k = 0.731 + 0.0688 * np.log10(Z)
        coeff = (n / 0.602214076) * Z
        E_cross = ref_stop._element_crossover_keV(el, Z, A, J)
        S += np.array([-float(ref_str._dEds_spliced_element_scalar(J, k, coeff, E_cross, 0.0, e / 1e3))
                       for e in E_eV])
    S_eV = S * 1e3 * (1.0 + 0.08 * np.sin(2.0 * np.log(E_eV)))
    return dict(stopping_energy_eV=E_eV, stopping_eV_per_angstrom=S_eV)


def gen_sbethe():
    for name, stg in SBETHE_CASES:
        case = TRANSPORT_CASES[name]
        layers = case["layers"]
        tables = [synthetic_sbethe_table(layer[2]) for layer in layers]
        prepared = ref_stop.prepare_sbethe_stopping_tables(tables, len(layers))
        _on, count, logE, logS = ref_stop.pack_sbethe_stopping_tables(prepared, len(layers))
        tp = np.deg2rad(case["tilt_deg"])
        beam_dir, n_hat = ref_geometry.tilted_geometry(np.deg2rad(case["theta_obs_deg"]), tp, 0.0)
        kwargs = dict(E0_keV=case["E0_keV"], Ne=case["Ne"], thickness_ang=layers[-1][1], seed=case["seed"],
                      elastic_model="sr", stopping_tables=tables, transport_core="per-electron",
                      radiative_model="uncoupled", beam_dir=beam_dir, tilt_polar_rad=tp,
                      beam_fwhm_mm=case["beam_fwhm_mm"], transport_lut_config=TransportLUTConfig(enabled=False),
                      straggling=stg)
        if len(layers) == 1:
            kwargs["composition"] = layers[0][2]
        else:
            kwargs["layers"] = layers
        out = _simulate_trajectories(**kwargs)
        arrays = {k: np.asarray(out[k]) for k in ROW_KEYS}
        counts = np.array([int(out[k]) for k in COUNT_KEYS], dtype=np.int64)
        leaf_E = np.geomspace(0.5, 2.0e6, 97)
        leaf_S = np.array([[ref_stop._dEds_sbethe_packed_scalar(logE, logS, L, count[L], e) for e in leaf_E]
                           for L in range(len(layers))])
        raw = {}
        for L, t in enumerate(tables):
            for f in ("stopping_energy_eV", "stopping_eV_per_angstrom"):
                raw[f"raw_{L}_{f}"] = t[f]
        _save(f"sbethe_{name}{'_straggled' if stg else ''}", E0_keV=case["E0_keV"], E_cut_keV=5.0,
              seed=case["seed"], Ne=case["Ne"], straggling=stg,
              initial_r=out["initial_r_ang"], initial_v=out["initial_v_hat"], initial_E=out["initial_E_keV"],
              count_names=np.array(COUNT_KEYS), counts=counts, sb_count=count, sb_logE=logE, sb_logS=logS,
              leaf_E=leaf_E, leaf_S=leaf_S, **raw, **arrays)


# ---------------------------------------------------------------------------
# Summary tables (pyrite/montecarlo/trajectory_summary.py:147-260) of the
# golden transport cases: the reference's own reductions of its own rows.
# ---------------------------------------------------------------------------
SUMMARY_BINS = dict(exit_E=64, exit_theta=36, depth=8)


def gen_summary():
    from pyrite.montecarlo import trajectory_summary as ts

    for name, case in TRANSPORT_CASES.items():
        out, _beam_dir, _n_hat = run_reference_transport(case)
        block = {k: np.asarray(out[k]) for k in ("r_mid", "L_ang", "v_hat", "E_start_keV", "E_end_keV",
                                                  "event_kind", "flight_id", "substep_id", "layer")}
        block["electron_id"] = np.asarray(out["elec_id"])
        rows = ts._history_rows(block)
        names = ("backscattered", "transmitted", "side_exited", "cutoff_stopped")
        fates = np.array([sum(1 for r in rows if r[1] == n) for n in names], dtype=np.int64)
        esc = [r for r in rows if r[1] in names[:3]]
        E_edges = np.linspace(0.0, case["E0_keV"], SUMMARY_BINS["exit_E"] + 1)
        th_edges = np.linspace(0.0, np.pi, SUMMARY_BINS["exit_theta"] + 1)
        exit_E = ts._histogram(np.array([r[4] for r in esc]), E_edges)
        exit_theta = ts._histogram(np.array([r[5] for r in esc]), th_edges)
        layers = case["layers"]
        edges = np.unique(np.concatenate([np.linspace(a, b, SUMMARY_BINS["depth"] + 1) for a, b, _ in layers]))
        prof = ts.depth_loss_profile(block, edges)
        per_layer = prof.groupby("layer")["continuous_loss_keV"].sum()
        deposit = np.array([float(per_layer.get(k, 0.0)) for k in range(len(layers))])
        _save(f"summary_{name}", E_edges=E_edges, theta_edges=th_edges, fates=fates, fate_names=np.array(names),
              exit_E=exit_E, exit_theta=exit_theta, depth_edges=edges,
              depth_layer=prof["layer"].to_numpy(), depth_low=prof["depth_low_ang"].to_numpy(),
              depth_loss=prof["continuous_loss_keV"].to_numpy(), deposit_per_layer=deposit,
              escaped_exit_E=np.array([r[4] for r in esc]), escaped_exit_theta=np.array([r[5] for r in esc]))


# ---------------------------------------------------------------------------
# Full run (statistical pin): the 20 MeV HOPG scene with its Twiss beam through
# the reference's per-electron core, then PXR/CBS bin means, Bethe-Heitler and
# the exit / fate / depth-loss summaries, in electron groups so the tests can
# form the reference's own statistical error (batch means).
# ---------------------------------------------------------------------------
FULLRUN = dict(E0_keV=20000.0, Ne=20000, groups=10, seed=11, thickness=1.0e6, n_C=0.1133, tilt_deg=45.0,
               theta_obs_deg=90.0, sigma_mm=0.5, sigma_prime_rad=0.5e-3,
               E_grid=np.arange(1000.0, 40000.0 + 1e-6, 50.0), exit_E_bins=64, exit_theta_bins=36,
               depth_bins=10)


def gen_fullrun():
    from pyrite.materials.crystal import CRYSTALS, reciprocal_g_vector
    from pyrite.montecarlo import trajectory_summary as ts
    from pyrite.montecarlo.spectrum import brem as ref_brem
    from pyrite.montecarlo.spectrum.cxr import _batched, _setup
    from pyrite.montecarlo.spectrum.cxr._spectrum import mc_cxr_spectrum
    from dataclasses import asdict

    from pyrite.montecarlo.transverse import TransverseDistribution, resolve_transverse_distribution

    c = FULLRUN
    E0 = c["E0_keV"]
    bg = float(np.sqrt((1.0 + E0 / 510.99895) ** 2 - 1.0))
    eps_n = c["sigma_mm"] * c["sigma_prime_rad"] * bg * 1e3  # mm mrad
    beta_m = c["sigma_mm"] / c["sigma_prime_rad"] * 1e-3
    tp = np.deg2rad(c["tilt_deg"])
    beam_dir, n_hat = ref_geometry.tilted_geometry(np.deg2rad(c["theta_obs_deg"]), tp, 0.0)
    out = _simulate_trajectories(
        E0_keV=E0, Ne=c["Ne"], thickness_ang=c["thickness"], composition=[("C", c["n_C"])], seed=c["seed"],
        elastic_model="sr", transport_core="per-electron", radiative_model="uncoupled", beam_dir=beam_dir,
        tilt_polar_rad=tp,
        transverse_distribution=asdict(resolve_transverse_distribution(TransverseDistribution(eps_n, beta_m),
                                                                       energy_keV=E0)),
        transport_lut_config=TransportLUTConfig(enabled=True))
    hkl = [(0, 0, l) for l in range(-8, 9) if l != 0]
    info = CRYSTALS["hopg"]
    g_mags = np.array([reciprocal_g_vector(h, info["lattice"])[1] for h in hkl])
    E_grid = c["E_grid"]
    E_tab = synthetic_E_tab(E_grid)
    comp = [("C", c["n_C"])]
    tables = synthetic_couplings(g_mags, E_tab)
    mosaic = np.deg2rad(0.4 * 2.3548200450309493)
    patches = [
        (_setup, "_line_tabulation_grid", lambda *a, **k: E_tab),
        (_setup, "_elemental_log_mu_table", lambda cc, E: synthetic_log_mu(cc, E)),
        (_setup, "refractive_index", lambda cr, E, uh=True: (1.0 - synthetic_delta(E)) + 0j),
        (_batched, "_reflection_tables", lambda *a, **k: tuple(np.array(t) for t in tables)),
    ]
    saved = [(m, n, getattr(m, n)) for m, n, _ in patches]
    for m, n, f in patches:
        setattr(m, n, f)
    saved_mu = ref_brem._mu_total_inv_ang
    ref_brem._mu_total_inv_ang = lambda cc, E: synthetic_mu_total(cc, np.asarray(E, dtype=float))
    K, Ne = c["groups"], c["Ne"]
    per = Ne // K
    eid = np.asarray(out["elec_id"])
    E_edges = np.linspace(0.0, E0, c["exit_E_bins"] + 1)
    th_edges = np.linspace(0.0, np.pi, c["exit_theta_bins"] + 1)
    depth_edges = np.linspace(0.0, c["thickness"], c["depth_bins"] + 1)
    cxr, brem, exE, exT, fates, dep = [], [], [], [], [], []
    try:
        for g in range(K):
            m = (eid >= g * per) & (eid < (g + 1) * per)
            seg = {k: np.asarray(out[k])[m] for k in ("r_mid", "v_hat", "L_ang", "E_keV", "E_repr_keV")}
            seg["elec_id"] = eid[m] - g * per
            seg["Ne"], seg["thickness_ang"] = per, c["thickness"]
            cxr.append(np.asarray(mc_cxr_spectrum(
                seg, E_grid, crystal="hopg", hkl_list=hkl, B_ang2=float(info.get("B_ang2", 0.0) or 0.0),
                absorber_element="C", n_hat=n_hat, surface_hkl=(0, 0, 1), mosaic_fwhm_rad=mosaic, mosaic_nodes=3,
                node_support_cutoff=None, line_quadrature="bin-mean")))
            brem.append(np.asarray(ref_brem.mc_brem_spectrum(seg, E_grid, composition=comp, n_hat=n_hat,
                                                             cross_section_model="bethe-heitler")))
            block = {k: np.asarray(out[k])[m] for k in ("r_mid", "L_ang", "v_hat", "E_start_keV", "E_end_keV",
                                                        "event_kind", "flight_id", "substep_id", "layer")}
            block["electron_id"] = eid[m]
            rows = ts._history_rows(block)
            names = ("backscattered", "transmitted", "side_exited", "cutoff_stopped")
            fates.append([sum(1 for r in rows if r[1] == n) for n in names])
            esc = [r for r in rows if r[1] in names[:3]]
            exE.append(ts._histogram(np.array([r[4] for r in esc]), E_edges))
            exT.append(ts._histogram(np.array([r[5] for r in esc]), th_edges))
            prof = ts.depth_loss_profile(block, depth_edges)
            dep.append(prof["continuous_loss_keV"].to_numpy() / per)
    finally:
        for m_, n_, f_ in saved:
            setattr(m_, n_, f_)
        ref_brem._mu_total_inv_ang = saved_mu
    _save("fullrun_hopg20", E0_keV=E0, Ne=Ne, groups=K, seed=c["seed"], thickness=c["thickness"], n_C=c["n_C"],
          tilt_deg=c["tilt_deg"], beam_dir=beam_dir, n_hat=n_hat, eps_n_mm_mrad=eps_n, beta_m=beta_m,
          hkl=np.array(hkl), mosaic_fwhm_rad=mosaic, E_grid=E_grid, E_tab=E_tab, delta=synthetic_delta(E_tab),
          log_mu=synthetic_log_mu(comp, E_tab), chi_re=tables[0], chi_im=tables[1], u_re=tables[2],
          u_im=tables[3], mu_grid=synthetic_mu_total(comp, E_grid), E_edges=E_edges, theta_edges=th_edges,
          depth_edges=depth_edges, cxr=np.array(cxr), brem=np.array(brem), exit_E=np.array(exE),
          exit_theta=np.array(exT), fates=np.array(fates), depth_loss=np.array(dep),
          fate_names=np.array(["backscattered", "transmitted", "side_exited", "cutoff_stopped"]))


GENERATORS = {
    "elsepa": gen_elsepa,
    "sbethe": gen_sbethe,
    "rng": gen_rng,
    "physics_leaves": gen_physics_leaves,
    "transport": gen_transport,
    "transport_lut": gen_transport_lut,
    "cxr": gen_cxr,
    "brem": gen_brem,
    "cxr_leaves": gen_cxr_leaves,
    "char": gen_char,
    "layered": gen_layered,
    "coherent": gen_coherent,
    "coherent_decoherence": gen_coherent_decoherence,
    "fullrun": gen_fullrun,
    "summary": gen_summary,
    "straggling": gen_straggling,
}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*", default=None)
    args = ap.parse_args(argv)
    for name, fn in GENERATORS.items():
        if args.only and name not in args.only:
            continue
        fn()


if __name__ == "__main__":
    main()
