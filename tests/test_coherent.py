"""Coherent (field-sum) CXR reduction: oracle pinned to the reference, the
kernel's precision plan emulated on the CPU, the C ABI's checks, and (GPU)
``pb_coherent_reduce`` against the reference's spectra and the oracle.

Golden vectors: ``tests/golden/coherent_{hopg20,si50}.npz``, made by
``make_golden.py --only coherent`` from the reference's own coherent route
(``cxr/_batched.py:1029-1240`` -> ``_batched_finalize.py:209-243``).

Tolerance of the device path against FP64: the spectrum within 2e-5 of its
peak everywhere and within 1e-4 relative wherever it exceeds 1e-3 of the
peak. Phases reach 1e8 rad; they are formed and reduced in FP64, the
trigonometry and the per-chunk field sums are FP32.
"""

import ctypes as C
import math

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import coherent as oc
from pyrite_b200 import _lib as L

CASES = ("hopg20", "si50")
PEAK_TOL = 2e-5
REL_TOL = 1e-4


def _golden(name):
    return oc.load_golden(GOLDEN / f"coherent_{name}.npz")


def _assert_close(got, ref, peak_tol=PEAK_TOL, rel_tol=REL_TOL):
    peak = float(np.max(np.abs(ref)))
    assert peak > 0
    err = np.abs(got - ref)
    assert err.max() <= peak_tol * peak, (err.max() / peak)
    big = np.abs(ref) > 1e-3 * peak
    assert np.all(err[big] <= rel_tol * np.abs(ref[big])), np.max(err[big] / np.abs(ref[big]))


# ---------------------------------------------------------------------------
# oracle against the reference
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_coherent_spectrum(name):
    rec, cnt, w, E, dom, Ne, spec = _golden(name)
    got = oc.coherent_spectrum(rec, cnt, w, E, dom, Ne)
    assert np.max(np.abs(got - spec)) <= 1e-12 * np.max(spec)


COHERENT_ELECTRONS = {"hopg20": 8, "si50": 6}


def _oracle_records(name):
    """The oracle's coherent records from the fixture's segments and tables."""
    import oracle

    c = np.load(GOLDEN / f"cxr_{name}.npz")
    tr = np.load(GOLDEN / f"transport_{c['transport']}.npz")
    n_elec = COHERENT_ELECTRONS[name]
    sel = tr["elec_id"] < n_elec
    seg = dict(v_hat=tr["v_hat"][sel], E_keV=tr["E_repr_keV"][sel], L_ang=tr["L_ang"][sel],
               r_mid=tr["r_mid"][sel], elec_id=tr["elec_id"][sel], t_ang=tr["t_ang"][sel])
    t = {k: c[k] for k in ("G", "ES", "EP", "WM", "row_table", "E_tab", "chi_re", "chi_im", "u_re", "u_im",
                           "log_mu", "delta")}
    pad = 0.2 * (c["E_grid"][-1] - c["E_grid"][0])
    t["lo_keep"], t["hi_keep"] = c["E_grid"][0] - pad, c["E_grid"][-1] + pad
    pairs, good = oracle.cxr_coherent_records(t, c["n_hat"], c["thickness"], seg, n_elec)
    return oc.rows_from_pairs(pairs, good, c["G"].shape[0])


@pytest.mark.parametrize("name", CASES)
def test_oracle_coherent_records_match_reference(name):
    """Segments + line tables -> the reference's per-row line records: the same
    pairs kept, in the same order, every field to 1e-10."""
    rec, cnt = _oracle_records(name)
    z = np.load(GOLDEN / f"coherent_{name}.npz")
    assert np.array_equal(cnt, z["row_count"])
    for f in oc.FIELDS:
        np.testing.assert_allclose(rec[f], z[f], rtol=1e-10, atol=0, err_msg=f)


@pytest.mark.parametrize("name", CASES)
def test_oracle_coherent_route_end_to_end(name):
    """Segments -> records -> spectrum, all in the oracle, against the
    reference's coherent spectrum. Phases of 1e8 rad carry 1e-8 rad of FP64
    rounding from the record differences, hence 1e-8 of the peak."""
    rec, cnt = _oracle_records(name)
    _, _, w, E, dom, Ne, spec = _golden(name)
    got = oc.coherent_spectrum(rec, cnt, w, E, dom, Ne)
    assert np.max(np.abs(got - spec)) <= 1e-8 * np.max(spec)


def test_oracle_decoherence_blend_matches_reference():
    """Sampled beam offsets on the infinite slab: the row factor F, each
    row's per-electron sum of squared fields and the blended spectrum."""
    z = np.load(GOLDEN / "coherent_decoherence_hopg20.npz")
    rec = {k: z[k] for k in oc.FIELDS}
    cnt, w, G, E, dom = z["row_count"], z["row_weight"], z["G"], z["E_grid"], z["delta_omega"]
    off = np.concatenate([[0], np.cumsum(cnt)])
    assert 0.0 < z["F_rows"].min() < 1e-3 and z["F_rows"].max() > 0.5  # a real blend
    for i, r in enumerate(z["active_rows"]):
        F = oc.decoherence_factor(z["A_pop"], z["xy0_pop"], G[r], z["omega"])
        np.testing.assert_allclose(F, z["F_rows"][i], rtol=1e-12, atol=1e-15)
        if i % 8 == 0:
            g = oc.grouped_row(rec, off[r], off[r + 1], z["elec_id"], E, dom)
            assert np.max(np.abs(g - z["grouped_rows"][i])) <= 1e-12 * np.max(z["grouped_rows"][i])
    spec = oc.coherent_spectrum_decoherent(rec, z["elec_id"], cnt, w, G, z["A_pop"], z["xy0_pop"], E, dom,
                                           z["omega"], int(z["Ne"]))
    assert np.max(np.abs(spec - z["spec"])) <= 1e-12 * np.max(z["spec"])


def test_oracle_offset_free_records_match_reference():
    """With each electron's face offset removed from the midpoints
    (cxr/_setup.py:637-642) the record prologue gives the reference's
    offset-free records."""
    import oracle

    z = np.load(GOLDEN / "coherent_decoherence_hopg20.npz")
    c = np.load(GOLDEN / "cxr_hopg20.npz")
    tr = np.load(GOLDEN / f"transport_{c['transport']}.npz")
    n = int(z["n_elec"])
    sel = tr["elec_id"] < n
    eid = tr["elec_id"][sel]
    r_geom = tr["r_mid"][sel].copy()
    r_geom[:, :2] -= z["xy0_pop"][np.clip(eid, 0, n - 1)]
    seg = dict(v_hat=tr["v_hat"][sel], E_keV=tr["E_repr_keV"][sel], L_ang=tr["L_ang"][sel], r_mid=r_geom,
               elec_id=eid, t_ang=tr["t_ang"][sel])
    t = {k: c[k] for k in ("G", "ES", "EP", "WM", "row_table", "E_tab", "chi_re", "chi_im", "u_re", "u_im",
                           "log_mu", "delta")}
    pad = 0.2 * (c["E_grid"][-1] - c["E_grid"][0])
    t["lo_keep"], t["hi_keep"] = c["E_grid"][0] - pad, c["E_grid"][-1] + pad
    pairs, good = oracle.cxr_coherent_records(t, c["n_hat"], c["thickness"], seg, n)
    rec, cnt = oc.rows_from_pairs(pairs, good, c["G"].shape[0])
    assert np.array_equal(cnt, z["row_count"])
    for f in oc.FIELDS:
        np.testing.assert_allclose(rec[f], z[f], rtol=1e-10, atol=0, err_msg=f)


@pytest.mark.parametrize("pieces", [2, 4])
def test_oracle_coherent_sum_is_invariant_under_segment_splitting(pieces):
    """A straight segment and its collinear pieces (own midpoints, lengths and
    start ages advanced by the flight time) radiate the same coherent field
    (cxr/_formation.py:26-36; the reference's segment-escape split
    invariance, tests/montecarlo/spectrum/test_segment_escape.py:75-86, in its
    coherent form). Pieces buried under optical depths that underflow drop out
    with no effect on the spectrum."""
    import oracle

    c = np.load(GOLDEN / "cxr_hopg20.npz")
    z = np.load(GOLDEN / "coherent_hopg20.npz")
    tr = np.load(GOLDEN / f"transport_{c['transport']}.npz")
    sel = tr["elec_id"] < 1
    seg = dict(v_hat=tr["v_hat"][sel], E_keV=tr["E_repr_keV"][sel], L_ang=tr["L_ang"][sel],
               r_mid=tr["r_mid"][sel], elec_id=tr["elec_id"][sel], t_ang=tr["t_ang"][sel])
    t = {k: c[k] for k in ("G", "ES", "EP", "WM", "row_table", "E_tab", "chi_re", "chi_im", "u_re", "u_im",
                           "log_mu", "delta")}
    pad = 0.2 * (c["E_grid"][-1] - c["E_grid"][0])
    t["lo_keep"], t["hi_keep"] = c["E_grid"][0] - pad, c["E_grid"][-1] + pad

    def spectrum(sg):
        pairs, good = oracle.cxr_coherent_records(t, c["n_hat"], c["thickness"], sg, 1)
        rec, cnt = oc.rows_from_pairs(pairs, good, c["G"].shape[0])
        return oc.coherent_spectrum(rec, cnt, z["row_weight"], z["E_grid"], z["delta_omega"], 1)

    n = seg["L_ang"].size
    frac = (np.arange(pieces) + 0.5) / pieces - 0.5
    L = np.repeat(seg["L_ang"], pieces) / pieces
    E = np.repeat(seg["E_keV"], pieces)
    gam = 1.0 + E / 510.99895
    beta = np.sqrt(1.0 - 1.0 / (gam * gam))
    v = np.repeat(seg["v_hat"], pieces, axis=0)
    split = dict(v_hat=v, E_keV=E, L_ang=L, elec_id=np.repeat(seg["elec_id"], pieces),
                 r_mid=np.repeat(seg["r_mid"], pieces, axis=0) + (np.tile(frac, n) * np.repeat(seg["L_ang"], pieces))[:, None] * v,
                 t_ang=np.repeat(seg["t_ang"], pieces) + np.tile(np.arange(pieces), n) * L / beta)
    whole = spectrum(seg)
    assert np.max(np.abs(spectrum(split) - whole)) <= 1e-8 * np.max(whole)


def test_golden_records_exercise_the_hard_cases():
    """Phases near 1e8 rad, formation arguments far from resonance, heavy
    absorption (apb underflowing FP32) and several rows with weights."""
    rec, cnt, w, E, dom, Ne, _ = _golden("si50")
    phi_max = np.max(np.abs(rec["phase_slope"])) * E.max() + np.max(np.abs(rec["g_phase"]))
    assert phi_max > 1e7
    assert np.min(rec["apb"]) < 1e-38
    rec_h, cnt_h, w_h, *_ = _golden("hopg20")
    assert len(np.unique(w_h)) > 1 and np.count_nonzero(cnt_h) > 50


def test_formation_factor_limits():
    v = np.linspace(-40.0, 40.0, 4001)
    # no absorption: the real sinc
    F = oc.formation_factor(v, np.full_like(v, 2.0), np.zeros_like(v), np.zeros_like(v))
    np.testing.assert_allclose(F.real, np.sinc(v / np.pi), atol=1e-12)
    assert np.max(np.abs(F.imag)) == 0.0
    # series branch and closed form agree at the switch
    for q in (1e-4, 3e-4):
        vv = np.array([math.sqrt(max(1e-6 - q * q, 0.0)) * (1 - 1e-9), math.sqrt(1e-6 - q * q) * (1 + 1e-9)])
        a, b = math.exp(-0.1), math.exp(-0.1 - 2 * q)
        Fs = oc.formation_factor(vv, np.full(2, a + b), np.full(2, b - a), np.full(2, q))
        assert abs(Fs[0] - Fs[1]) < 1e-9


def test_formation_parseval():
    """int |F|^2 dv = pi <exp(-tau)> over the piece (_formation.py:37-40)."""
    tau_s, tau_e = 0.3, 2.1
    q = 0.25 * (tau_e - tau_s)
    a, b = math.exp(-0.5 * tau_s), math.exp(-0.5 * tau_e)
    v = np.linspace(-4000.0, 4000.0, 4_000_001)
    F = oc.formation_factor(v, np.full_like(v, a + b), np.full_like(v, b - a), np.full_like(v, q))
    integral = np.trapezoid(np.abs(F) ** 2, v)
    mean_T = (math.exp(-tau_s) - math.exp(-tau_e)) / (tau_e - tau_s)
    assert abs(integral - math.pi * mean_T) < 2e-3 * math.pi * mean_T


def test_rows_add_incoherently_lines_coherently():
    rec, cnt, w, E, dom, Ne, spec = _golden("hopg20")
    off = np.concatenate([[0], np.cumsum(cnt)])
    total = np.zeros_like(spec)
    for r in np.flatnonzero(cnt)[:12]:
        sub = {k: v[off[r]:off[r + 1]] for k, v in rec.items()}
        total += oc.coherent_spectrum(sub, [cnt[r]], [w[r]], E, dom, Ne)
    rows = np.flatnonzero(cnt)[:12]
    sel = np.concatenate([np.arange(off[r], off[r + 1]) for r in rows])
    both = oc.coherent_spectrum({k: v[sel] for k, v in rec.items()}, cnt[rows], w[rows], E, dom, Ne)
    np.testing.assert_allclose(both, total, rtol=1e-12, atol=1e-14 * total.max())
    # one row holding two rows' lines interferes: not the incoherent sum
    r0, r1 = rows[-2], rows[-1]
    pair = np.concatenate([np.arange(off[r0], off[r0 + 1]), np.arange(off[r1], off[r1 + 1])])
    one = oc.coherent_spectrum({k: v[pair] for k, v in rec.items()}, [pair.size], [1.0], E, dom, Ne)
    two = oc.coherent_spectrum({k: v[pair] for k, v in rec.items()}, [cnt[r0], cnt[r1]], [1.0, 1.0], E, dom, Ne)
    assert np.max(np.abs(one - two)) > 1e-3 * np.max(two)


# ---------------------------------------------------------------------------
# the kernel's arithmetic, emulated in float32 numpy
# ---------------------------------------------------------------------------
def _chunk_lines(n_line, n_E):
    """pb_coherent.cu chunk_lines: items for ~8 CTAs per SM over 512-energy tiles."""
    tiles = -(-n_E // 512)
    items = max(1, (148 * 8) // tiles)
    k = max(-(-n_line // items), 256)
    return -(-k // 128) * 128


def _taylor_sincos(v):
    """pb_coherent.cu sincos_taylor in float32: Taylor series to v^11 / v^12."""
    f32 = np.float32
    v = np.where(np.abs(v) <= 1, v, f32(0))  # the kernel takes this branch only for |v| <= 1
    z = v * v
    ps = z * f32(-1 / 39916800) + f32(1 / 362880)
    for c in (-1 / 5040, 1 / 120, -1 / 6):
        ps = z * ps + f32(c)
    pc = z * f32(1 / 479001600) + f32(-1 / 3628800)
    for c in (1 / 40320, -1 / 720, 1 / 24, -0.5):
        pc = z * pc + f32(c)
    return (v * z * ps + v).astype(f32), (z * pc + f32(1)).astype(f32)


TURN_BASE = 805306368.0  # 1.5 * 2^29
FAST_LIMIT = 2.0 ** 27
INV2PI = 0.15915494309189535


def _fma(a, b, c):
    """Fused multiply-add in float64, emulated through the x87 extended type."""
    ld = np.longdouble
    return (np.asarray(a, dtype=ld) * np.asarray(b, dtype=ld) + np.asarray(c, dtype=ld)).astype(np.float64)


def turn_fraction_offset(x):
    """pb_coherent.cu sincos_turns_offset: f - 1/2 from the low 23 mantissa bits of x in [2^29, 2^30)."""
    bits = np.asarray(x, dtype=np.float64).view(np.uint64) & np.uint64(0x7FFFFF)
    return (np.float32(1.0) + (bits.astype(np.float64) / 2.0 ** 23).astype(np.float32)) - np.float32(1.5)


def kernel_emulation(rec, cnt, w, E, dom, Ne, tile=1024):
    """The field kernel's arithmetic with numpy: per line and energy tile the
    offset-binade FP64 path (or the plain FP64 reduction when a line's terms
    could leave the binade), FP32 formation factor, rotation and per-item
    sums, FP64 across items (SFU errors not modelled)."""
    f32 = np.float32
    E = np.asarray(E, dtype=np.float64)
    spec = np.zeros(E.size)
    K = _chunk_lines(int(np.sum(cnt)), E.size)
    off = np.concatenate([[0], np.cumsum(cnt)])
    two_pi = f32(2 * np.pi)
    Emax = np.zeros(E.size)
    Dmax = np.zeros(E.size)
    for t0 in range(0, E.size, tile):
        Emax[t0:t0 + tile] = np.max(np.abs(E[t0:t0 + tile]))
        Dmax[t0:t0 + tile] = np.max(np.abs(dom[t0:t0 + tile]))
    for r in range(len(cnt)):
        F = np.zeros((4, E.size))
        for j0 in range(off[r], off[r + 1], K):
            acc = np.zeros((4, E.size), dtype=f32)
            for j in range(j0, min(j0 + K, off[r + 1])):
                ps_t, L_t = rec["phase_slope"][j] * INV2PI, rec["L_esc"][j] * INV2PI
                a_t, h_t = rec["a_vac"][j] * INV2PI, rec["half_dL"][j] * INV2PI
                gt, Ev = rec["g_phase"][j] * INV2PI, rec["E_vac"][j]
                fast = ((abs(ps_t) * Emax + abs(gt) + abs(L_t) * Dmax < FAST_LIMIT)
                        & (abs(a_t) * (Emax + abs(Ev)) + abs(h_t) * Dmax < FAST_LIMIT))
                # fast: offset sums, fraction from the mantissa; sin/cos negated back
                vx = _fma(a_t, E, _fma(-h_t, dom, TURN_BASE - a_t * Ev))
                px = _fma(ps_t, E, _fma(-L_t, dom, TURN_BASE - gt))
                vf_fast = ((vx - TURN_BASE).astype(f32) * two_pi).astype(f32)
                gv, gp = turn_fraction_offset(vx), turn_fraction_offset(px)
                sv_f = -np.sin((gv * two_pi).astype(f32)).astype(f32)
                cv_f = -np.cos((gv * two_pi).astype(f32)).astype(f32)
                sp_f = -np.sin((gp * two_pi).astype(f32)).astype(f32)
                cp_f = -np.cos((gp * two_pi).astype(f32)).astype(f32)
                # plain: turns reduced in FP64
                vt = _fma(a_t, E - Ev, -h_t * dom)
                vf_slow = (vt.astype(f32) * two_pi).astype(f32)
                xv = ((vt - np.rint(vt)).astype(f32) * two_pi).astype(f32)
                pt = _fma(ps_t, E, -_fma(L_t, dom, gt))
                xp = ((pt - np.rint(pt)).astype(f32) * two_pi).astype(f32)
                vf = np.where(fast, vf_fast, vf_slow)
                st, ct = _taylor_sincos(vf)
                near = np.abs(vf) <= 1
                sv = np.where(near, st, np.where(fast, sv_f, np.sin(xv).astype(f32)))
                cv = np.where(near, ct, np.where(fast, cv_f, np.cos(xv).astype(f32)))
                sp = np.where(fast, sp_f, np.sin(xp).astype(f32))
                cp = np.where(fast, cp_f, np.cos(xp).astype(f32))
                q, apb, bma = f32(rec["q"][j]), f32(rec["apb"][j]), f32(rec["bma"][j])
                w2 = (q.astype(np.float64) * q + (vf * vf).astype(np.float64)).astype(f32)
                with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
                    inv = (f32(0.5) / w2).astype(f32)
                fr = ((vf * apb).astype(np.float64) * sv - (q * bma * cv).astype(np.float64)).astype(f32) * inv
                fi = -((vf * bma).astype(np.float64) * cv + (q * apb * sv).astype(np.float64)).astype(f32) * inv
                series = w2 < f32(1e-6)
                half = f32(0.5) * apb
                fr = np.where(series, half * (f32(1) - q * q * f32(1 / 3) - vf * vf * f32(1 / 6)), fr)
                fi = np.where(series, -half * q * vf * f32(1 / 3), fi)
                pr, pi = fr * cp - fi * sp, fr * sp + fi * cp
                csr, csi, cpr, cpi = (f32(rec[k][j]) for k in ("cs_re", "cs_im", "cp_re", "cp_im"))
                acc[0] += csr * pr - csi * pi
                acc[1] += csr * pi + csi * pr
                acc[2] += cpr * pr - cpi * pi
                acc[3] += cpr * pi + cpi * pr
            F += acc.astype(np.float64)
        spec += w[r] * np.sum(F * F, axis=0)
    return spec / Ne


def _whole_turns_added(rec, every=2, turns=1e9):
    """Every other line's g_phase moved by a whole number of turns: the same
    physics, but beyond the offset binade, so those lines take the plain path."""
    out = dict(rec)
    gp = rec["g_phase"].copy()
    gp[::every] += 2.0 * np.pi * turns
    out["g_phase"] = gp
    return out


def test_float_plan_mixes_both_phase_paths():
    rec, cnt, w, E, dom, Ne, spec = _golden("hopg20")
    moved = _whole_turns_added(rec)
    gt = moved["g_phase"] * INV2PI
    assert np.count_nonzero(np.abs(gt) > FAST_LIMIT) * 3 > rec["g_phase"].size
    _assert_close(kernel_emulation(moved, cnt, w, E, dom, Ne), spec, PEAK_TOL / 4, REL_TOL / 4)


def test_turn_fraction_from_the_offset_binade():
    """x = 1.5 * 2^29 + t in [2^29, 2^30): the low 23 mantissa bits are t's
    fractional turn to 2^-23; the extracted f - 1/2 matches it."""
    rng = np.random.default_rng(2)
    t = np.concatenate([rng.uniform(-2.0 ** 27, 2.0 ** 27, 100000), rng.uniform(-3, 3, 1000), [0.0, 0.25, -0.5]])
    x = TURN_BASE + t
    assert np.all((x >= 2.0 ** 29) & (x < 2.0 ** 30))
    g = turn_fraction_offset(x).astype(np.float64)
    frac = (x - TURN_BASE) - np.floor(x - TURN_BASE)  # exact: x - base is exact (Sterbenz)
    d = (g + 0.5) - frac
    d -= np.rint(d)
    assert np.max(np.abs(d)) == 0.0
    assert np.max(np.abs(((x - TURN_BASE) - t))) <= 2.0 ** -24 + 1e-30


def test_taylor_sincos_accuracy():
    v = np.linspace(-1.0, 1.0, 20001).astype(np.float32)
    s, c = _taylor_sincos(v)
    assert np.max(np.abs(s - np.sin(v.astype(np.float64)))) < 2e-7
    assert np.max(np.abs(c - np.cos(v.astype(np.float64)))) < 2e-7
    small = np.abs(v) > 1e-30
    assert np.max(np.abs(s[small] / np.sin(v[small].astype(np.float64)) - 1)) < 3e-7


@pytest.mark.parametrize("name", CASES)
def test_float_plan_meets_tolerance_on_reference_records(name):
    rec, cnt, w, E, dom, Ne, spec = _golden(name)
    _assert_close(kernel_emulation(rec, cnt, w, E, dom, Ne), spec, PEAK_TOL / 4, REL_TOL / 4)


def test_phase_in_float32_would_not_do():
    """The reason the phase stays FP64: formed in FP32, the si50 spectrum is off."""
    rec, cnt, w, E, dom, Ne, spec = _golden("si50")
    f32 = np.float32
    off = np.concatenate([[0], np.cumsum(cnt)])
    r = int(np.argmax(cnt))
    sl = slice(off[r], off[r + 1])
    phi64 = rec["phase_slope"][sl, None] * E[None, :] - rec["g_phase"][sl, None]
    phi32 = (rec["phase_slope"][sl, None].astype(f32) * E[None, :].astype(f32) - rec["g_phase"][sl, None].astype(f32))
    assert np.max(np.abs(np.angle(np.exp(1j * (phi32.astype(np.float64) - phi64))))) > 1.0


# ---------------------------------------------------------------------------
# C ABI (no device work)
# ---------------------------------------------------------------------------
def test_abi_work_size_and_argument_errors():
    lib = L.load()
    nb = C.c_uint64()
    assert lib.pb_coherent_work_size(144, 6003, 781, C.byref(nb)) == 0
    # item offsets (145 int64, 256-aligned) + (144 + 6003 // 256) items x 4 x 781 floats
    assert nb.value == 1280 + (144 + 6003 // 256) * 4 * 781 * 4
    assert lib.pb_coherent_work_size(0, 10, 10, C.byref(nb)) == 1
    assert lib.pb_coherent_work_size(1, 10, 0, C.byref(nb)) == 1
    assert lib.pb_coherent_work_size(1, -1, 10, C.byref(nb)) == 1
    a = L.PbCoherentArgs()
    a.n_row, a.n_E, a.n_line = 2, 16, 0
    assert lib.pb_coherent_reduce(C.byref(a), None) == 1
    assert b"must be set" in lib.pb_last_error()
    fake = 1 << 20
    a.row_off = a.row_weight = a.E = a.delta_omega = a.spec = fake
    a.work = fake + 8
    assert lib.pb_coherent_reduce(C.byref(a), None) == 1
    assert b"aligned" in lib.pb_last_error()
    a.work = fake
    a.work_bytes = 16
    assert lib.pb_coherent_reduce(C.byref(a), None) == 4
    a.work_bytes = 1 << 30
    a.sinc_cutoff = -1.0
    assert lib.pb_coherent_reduce(C.byref(a), None) == 1
    a.sinc_cutoff = 0.0
    assert lib.pb_coherent_reduce(C.byref(a), None) == 0  # no lines: nothing to launch
    a.n_line = 5
    assert lib.pb_coherent_reduce(C.byref(a), None) == 1
    assert b"line record" in lib.pb_last_error()


# ---------------------------------------------------------------------------
# GPU: the kernel
# ---------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_coherent_matches_reference(name):
    from pyrite_b200.coherent import coherent_spectrum

    rec, cnt, w, E, dom, Ne, spec = _golden(name)
    got = coherent_spectrum(rec, cnt, w, E, dom, Ne)
    _assert_close(got, spec)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_coherent_records_and_route_match_reference(name):
    """The device record prologue (``pb_coherent_records``) from the fixture's
    segments (with start ages) and line tables: the reference's per-row line
    records -- the same pairs kept in the same order, every field within
    1e-10 (a polarisation coefficient within 1e-10 of its record's complex
    pair) -- and the whole device route, segments -> records -> reduction,
    the reference's coherent spectrum within the reduction's tolerance (2e-5
    of the peak, 1e-4 relative above 1e-3 of it).

    One exception is allowed and checked: a pair whose escape optical depth
    puts its formation coefficient apb = exp(-tau_s/2) + exp(-tau_e/2) at the
    last subnormal (the reference keeps apb = 5e-324 when glibc's exp rounds
    up to it, CUDA's exp may round to 0 and drop the pair). Such a record
    adds nothing to any field; records with apb below 1e-300 are compared
    as absent."""
    from pyrite_b200 import LineTables
    from pyrite_b200.coherent import coherent_records, coherent_route_spectrum
    from pyrite_b200.tables import ReflectionRows

    c = np.load(GOLDEN / f"cxr_{name}.npz")
    tr = np.load(GOLDEN / f"transport_{c['transport']}.npz")
    n_elec = COHERENT_ELECTRONS[name]
    sel = tr["elec_id"] < n_elec
    seg = dict(v_hat=tr["v_hat"][sel], E_keV=tr["E_repr_keV"][sel], L_ang=tr["L_ang"][sel],
               r_mid=tr["r_mid"][sel], elec_id=tr["elec_id"][sel], t_ang=tr["t_ang"][sel], Ne=n_elec,
               thickness_ang=float(c["thickness"]))
    tables = LineTables(c["E_tab"], c["chi_re"], c["chi_im"], c["u_re"], c["u_im"], c["log_mu"], c["delta"])
    rows = ReflectionRows(c["G"], c["ES"][None], c["EP"][None], c["WM"], c["row_table"])
    rec, cnt = coherent_records(seg, c["E_grid"], tables=tables, rows=rows, n_hat=c["n_hat"])
    z = np.load(GOLDEN / f"coherent_{name}.npz")
    got_rec = {f: rec[f].cpu().numpy() for f in oc.FIELDS}
    live_got, live_ref = got_rec["apb"] > 1e-300, z["apb"] > 1e-300
    row_got = np.repeat(np.arange(cnt.size), cnt)
    row_ref = np.repeat(np.arange(z["row_count"].size), z["row_count"])
    assert np.array_equal(np.bincount(row_got[live_got], minlength=cnt.size),
                          np.bincount(row_ref[live_ref], minlength=cnt.size))
    assert abs(int(cnt.sum()) - int(z["row_count"].sum())) <= int((~live_ref).sum()) + int((~live_got).sum())
    # the four polarisation coefficients of a record are one complex pair:
    # a component that nearly cancels is held to 1e-10 of the pair's size
    coef = ("cs_re", "cs_im", "cp_re", "cp_im")
    size = np.sqrt(sum(z[f][live_ref] ** 2 for f in coef))
    for f in oc.FIELDS:
        atol = 1e-10 * size if f in coef else 1e-300
        g, r = got_rec[f][live_got], z[f][live_ref]
        bad = np.abs(g - r) > 1e-10 * np.abs(r) + atol
        assert not np.any(bad), (f, int(bad.sum()), float(np.max(np.abs(g - r)[bad])))
    got = coherent_route_spectrum(seg, z["E_grid"], z["delta_omega"], tables=tables, rows=rows, n_hat=c["n_hat"])
    _assert_close(got, z["spec"])


def _random_rows(rng, n_rows, n_per_row, E_lo, E_hi):
    n = n_rows * n_per_row
    E_vac = rng.uniform(E_lo, E_hi, n)
    a_vac = rng.uniform(0.5, 60.0, n)
    tau_s = rng.uniform(0.0, 6.0, n)
    tau_e = tau_s + rng.uniform(-tau_s, 6.0, n)
    q = 0.25 * (tau_e - tau_s)
    a, b = np.exp(-0.5 * tau_s), np.exp(-0.5 * tau_e)
    rec = dict(
        E_vac=E_vac, a_vac=a_vac, phase_slope=rng.uniform(-3000.0, 3000.0, n),
        g_phase=rng.uniform(-6e7, 6e7, n), cs_re=rng.normal(0, 1e-4, n), cs_im=rng.normal(0, 1e-5, n),
        cp_re=rng.normal(0, 1e-4, n), cp_im=rng.normal(0, 1e-5, n), L_esc=rng.uniform(0.0, 2e5, n),
        half_dL=rng.uniform(-1e5, 1e5, n), apb=a + b, bma=b - a, q=q,
    )
    return rec, np.full(n_rows, n_per_row), rng.uniform(0.1, 1.0, n_rows)


@pytest.mark.gpu
def test_gpu_coherent_both_phase_paths_agree():
    """Whole turns added to half the lines' g_phase (plain FP64 path) leave
    the reference spectrum unchanged."""
    from pyrite_b200.coherent import coherent_spectrum

    rec, cnt, w, E, dom, Ne, spec = _golden("hopg20")
    _assert_close(coherent_spectrum(_whole_turns_added(rec), cnt, w, E, dom, Ne), spec)


@pytest.mark.gpu
def test_gpu_coherent_random_rows_against_oracle():
    """3 rows x 20k lines over 4096 energies (2.5e8 line-energy pairs), the
    oracle on every 16th energy; deterministic across calls."""
    import torch

    from pyrite_b200.coherent import coherent_reduce

    rng = np.random.default_rng(11)
    rec, cnt, w = _random_rows(rng, 3, 20000, 2000.0, 40000.0)
    E = np.linspace(1000.0, 41000.0, 4096)
    dom = 2.3e-4 * (1e4 / (E + 500.0)) ** 2 * E / 1973.27
    got = coherent_reduce(rec, cnt, w, E, dom).cpu().numpy()
    again = coherent_reduce(rec, cnt, w, E, dom).cpu().numpy()
    assert np.array_equal(got, again)
    sub = np.arange(0, E.size, 16)
    ref = oc.coherent_spectrum(rec, cnt, w, E[sub], dom[sub])
    _assert_close(got[sub], ref)
    torch.cuda.synchronize()


@pytest.mark.gpu
def test_gpu_coherent_sinc_window_and_one_row_signature():
    """The reference's one-row call: vacuum sinc lines (no medium, no
    formation group) and the |v| window."""
    import torch

    from pyrite_b200.coherent import run_coherent_reduction_kernel

    rng = np.random.default_rng(5)
    n = 3000
    E = np.linspace(5000.0, 15000.0, 1500)
    rec = dict(E_vac=rng.uniform(6000, 14000, n), a_vac=rng.uniform(0.05, 2.0, n),
               phase_slope=rng.uniform(-50, 50, n), g_phase=rng.uniform(-1e5, 1e5, n),
               cs_re=rng.normal(0, 1, n), cs_im=rng.normal(0, 1, n), cp_re=rng.normal(0, 1, n),
               cp_im=rng.normal(0, 1, n))
    out = torch.zeros(E.size, dtype=torch.float64, device="cuda")
    run_coherent_reduction_kernel(rec["E_vac"], rec["a_vac"], rec["phase_slope"], rec["g_phase"], rec["cs_re"],
                                  rec["cs_im"], rec["cp_re"], rec["cp_im"], E, out=out, mosaic_weight=0.5)
    full = dict(rec, L_esc=np.zeros(n), half_dL=np.zeros(n), apb=np.full(n, 2.0), bma=np.zeros(n), q=np.zeros(n))
    ref = 0.5 * oc.coherent_spectrum(full, [n], [1.0], E, np.zeros(E.size))
    _assert_close(out.cpu().numpy(), ref)
    # window: lines beyond |v| > 30 add nothing
    out.zero_()
    run_coherent_reduction_kernel(rec["E_vac"], rec["a_vac"], rec["phase_slope"], rec["g_phase"], rec["cs_re"],
                                  rec["cs_im"], rec["cp_re"], rec["cp_im"], E, out=out, sinc_cutoff=30.0)
    f_s = np.zeros(E.size, complex)
    f_p = np.zeros(E.size, complex)
    for j in range(n):
        v = rec["a_vac"][j] * (E - rec["E_vac"][j])
        keep = np.abs(v) <= 30.0
        sp = np.where(keep, np.sinc(v / np.pi), 0.0) * np.exp(1j * (rec["phase_slope"][j] * E - rec["g_phase"][j]))
        f_s += (rec["cs_re"][j] + 1j * rec["cs_im"][j]) * sp
        f_p += (rec["cp_re"][j] + 1j * rec["cp_im"][j]) * sp
    _assert_close(out.cpu().numpy(), np.abs(f_s) ** 2 + np.abs(f_p) ** 2)


@pytest.mark.gpu
def test_gpu_coherent_bad_row_offsets_are_clamped_and_flagged():
    """A row_off that is not a partition (a row ending before it starts, one
    past n_line) stays inside the record arrays and sets PB_DEV_BAD_INPUT."""
    import torch

    lib = L.load()
    dev = torch.device("cuda")
    n_line, n_E = 10, 64
    f = {k: torch.ones(n_line, dtype=torch.float64, device=dev) for k in oc.FIELDS}
    E = torch.linspace(1000.0, 2000.0, n_E, dtype=torch.float64, device=dev)
    dom = torch.zeros(n_E, dtype=torch.float64, device=dev)
    for offs in ([0, 5, 3, 10], [0, 20, 10, 10]):
        row_off = torch.tensor(offs, dtype=torch.int64, device=dev)
        w = torch.ones(3, dtype=torch.float64, device=dev)
        spec = torch.zeros(n_E, dtype=torch.float64, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        nb = C.c_uint64()
        assert lib.pb_coherent_work_size(3, n_line, n_E, C.byref(nb)) == 0
        work = torch.empty(nb.value, dtype=torch.uint8, device=dev)
        a = L.PbCoherentArgs()
        a.n_row, a.n_E, a.n_line = 3, n_E, n_line
        a.row_off, a.row_weight, a.E, a.delta_omega = row_off.data_ptr(), w.data_ptr(), E.data_ptr(), dom.data_ptr()
        for k in oc.FIELDS:
            setattr(a, k, f[k].data_ptr())
        a.scale = 1.0
        a.spec, a.work, a.work_bytes, a.status = spec.data_ptr(), work.data_ptr(), nb.value, status.data_ptr()
        L.check(lib.pb_coherent_reduce(C.byref(a), torch.cuda.current_stream().cuda_stream), "pb_coherent_reduce")
        torch.cuda.synchronize()
        assert int(status.item()) & L.PB_DEV_BAD_INPUT
        assert torch.isfinite(spec).all()


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the behaviour without a GPU")
def test_no_cpu_fallback_without_a_device():
    """Without a CUDA device the coherent API refuses instead of computing
    on the host."""
    from pyrite_b200 import PyriteB200Error
    from pyrite_b200.coherent import coherent_reduce, coherent_spectrum

    rec, cnt, w, E, dom, Ne, _ = _golden("hopg20")
    with pytest.raises(PyriteB200Error, match="CUDA"):
        coherent_reduce(rec, cnt, w, E, dom)
    with pytest.raises(PyriteB200Error, match="CUDA"):
        coherent_spectrum(rec, cnt, w, E, dom, Ne)


@pytest.mark.gpu
def test_gpu_decoherence_blend_matches_reference():
    """The sampled-bunch blend on the device: the row factors F against the
    reference's (FP64, 1e-12), and the blended spectrum -- flat and
    per-electron fields from one pass, mixed by F -- against the reference's
    within the reduction's tolerance."""
    from pyrite_b200.coherent import coherent_spectrum_decoherent, decoherence_factor

    z = np.load(GOLDEN / "coherent_decoherence_hopg20.npz")
    rec = {k: z[k] for k in oc.FIELDS}
    F = decoherence_factor(z["G"], z["A_pop"], z["xy0_pop"], z["omega"]).cpu().numpy()[z["active_rows"]]
    # The phase omega A - g.xy0 reaches ~1e8 rad, so the last bit of its FP64
    # value (and of the reference's g.xy0, a BLAS dot product) moves it by
    # ~2e-8 rad; F = |chi|^2 moves by at most 2 |chi| that much.
    B = np.abs(z["xy0_pop"]) @ np.abs(z["G"][z["active_rows"], :2]).T
    phase = np.abs(z["omega"])[None, :] * np.abs(z["A_pop"]).max() + B.max(axis=0)[:, None]
    bound = 2.0 * np.sqrt(z["F_rows"]) * 4.0 * np.spacing(phase) + 1e-15
    err = np.abs(F - z["F_rows"])
    assert np.all(err <= bound), float(np.max(err / bound))
    assert np.max(err) < 1e-9
    spec = coherent_spectrum_decoherent(rec, z["elec_id"], z["row_count"], z["row_weight"], z["G"], z["A_pop"],
                                        z["xy0_pop"], z["E_grid"], z["delta_omega"], z["omega"], int(z["Ne"]))
    _assert_close(spec, z["spec"])


@pytest.mark.gpu
def test_gpu_blend_limits_and_long_electrons():
    """Random rows whose electrons hold 1 to 40 lines, one of them 700 (longer
    than a work item, so item bounds move to electron ends): F = 1 gives the
    plain reduction, F = 0 the oracle's per-electron sum on every 16th
    energy; repeated calls are bit-identical."""
    import torch

    from pyrite_b200.coherent import coherent_reduce

    rng = np.random.default_rng(17)
    n_rows, n_per_row = 3, 6000
    rec, cnt, w = _random_rows(rng, n_rows, n_per_row, 2000.0, 40000.0)
    eid = []
    for r in range(n_rows):
        ids, e = [], 1000 * r
        while len(ids) < n_per_row:
            k = 700 if (r == 1 and e == 1003) else int(rng.integers(1, 41))
            ids += [e] * k
            e += 1
        eid.append(np.asarray(ids[:n_per_row], dtype=np.int64))
    eid = np.concatenate(eid)
    E = np.linspace(1000.0, 41000.0, 2048)
    dom = 2.3e-4 * (1e4 / (E + 500.0)) ** 2 * E / 1973.27
    ones, zeros = np.ones((n_rows, E.size)), np.zeros((n_rows, E.size))
    plain = coherent_reduce(rec, cnt, w, E, dom).cpu().numpy()
    flat = coherent_reduce(rec, cnt, w, E, dom, elec_id=eid, F_row=ones).cpu().numpy()
    _assert_close(flat, plain)
    grouped = coherent_reduce(rec, cnt, w, E, dom, elec_id=eid, F_row=zeros).cpu().numpy()
    again = coherent_reduce(rec, cnt, w, E, dom, elec_id=eid, F_row=zeros).cpu().numpy()
    assert np.array_equal(grouped, again)
    sub = np.arange(0, E.size, 16)
    off = np.concatenate([[0], np.cumsum(cnt)])
    rec64 = {k: np.asarray(rec[k], dtype=np.float64) for k in oc.FIELDS}
    ref = sum(w[r] * oc.grouped_row(rec64, off[r], off[r + 1], eid, E[sub], dom[sub]) for r in range(n_rows))
    _assert_close(grouped[sub], ref)
    torch.cuda.synchronize()


@pytest.mark.gpu
def test_gpu_blend_flags_unordered_electrons():
    """Electron ids that decrease inside a row set PB_DEV_BAD_INPUT."""
    import torch

    from pyrite_b200 import _lib as L
    from pyrite_b200.coherent import coherent_reduce

    rng = np.random.default_rng(23)
    rec, cnt, w = _random_rows(rng, 1, 600, 2000.0, 40000.0)
    eid = np.repeat(np.arange(60, dtype=np.int64), 10)[::-1].copy()
    E = np.linspace(1000.0, 41000.0, 256)
    dom = np.zeros_like(E)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    coherent_reduce(rec, cnt, w, E, dom, elec_id=eid, F_row=np.zeros((1, E.size)), status=status)
    assert int(status.item()) & L.PB_DEV_BAD_INPUT


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_streamed_route_equals_the_whole_route(name):
    """The streamed field-plane route (records of three segment blocks folded
    into persistent FP64 fields, squared once) gives the reference's coherent
    spectrum, as the one-shot route does."""
    from pyrite_b200 import LineTables
    from pyrite_b200.coherent import coherent_route_spectrum, coherent_route_spectrum_streamed
    from pyrite_b200.tables import ReflectionRows

    c = np.load(GOLDEN / f"cxr_{name}.npz")
    tr = np.load(GOLDEN / f"transport_{c['transport']}.npz")
    n_elec = COHERENT_ELECTRONS[name]
    sel = tr["elec_id"] < n_elec
    seg = dict(v_hat=tr["v_hat"][sel], E_keV=tr["E_repr_keV"][sel], L_ang=tr["L_ang"][sel],
               r_mid=tr["r_mid"][sel], elec_id=tr["elec_id"][sel], t_ang=tr["t_ang"][sel], Ne=n_elec,
               thickness_ang=float(c["thickness"]))
    tables = LineTables(c["E_tab"], c["chi_re"], c["chi_im"], c["u_re"], c["u_im"], c["log_mu"], c["delta"])
    rows = ReflectionRows(c["G"], c["ES"][None], c["EP"][None], c["WM"], c["row_table"])
    z = np.load(GOLDEN / f"coherent_{name}.npz")
    whole = coherent_route_spectrum(seg, z["E_grid"], z["delta_omega"], tables=tables, rows=rows, n_hat=c["n_hat"])
    block = max(1, int(sel.sum()) // 3)
    got = coherent_route_spectrum_streamed(seg, z["E_grid"], z["delta_omega"], tables=tables, rows=rows,
                                           n_hat=c["n_hat"], block_segments=block)
    _assert_close(got, z["spec"])
    assert float(np.max(np.abs(got - whole))) <= 1e-5 * float(np.max(whole))


@pytest.mark.gpu
def test_gpu_streamed_decoherence_blend_matches_reference():
    """The streamed route with the sampled-bunch blend: records carry their
    electrons, per-electron fields are accumulated beside the flat ones, and
    the finalize mixes them by the rows' factors -- the reference's blended
    spectrum from the fixture's offset-free segments."""
    from pyrite_b200 import LineTables
    from pyrite_b200.coherent import coherent_route_spectrum_streamed
    from pyrite_b200.tables import ReflectionRows

    z = np.load(GOLDEN / "coherent_decoherence_hopg20.npz")
    c = np.load(GOLDEN / "cxr_hopg20.npz")
    tr = np.load(GOLDEN / f"transport_{c['transport']}.npz")
    n = int(z["n_elec"])
    sel = tr["elec_id"] < n
    eid = tr["elec_id"][sel]
    r_geom = tr["r_mid"][sel].copy()
    r_geom[:, :2] -= z["xy0_pop"][np.clip(eid, 0, n - 1)]
    seg = dict(v_hat=tr["v_hat"][sel], E_keV=tr["E_repr_keV"][sel], L_ang=tr["L_ang"][sel], r_mid=r_geom,
               elec_id=eid, t_ang=tr["t_ang"][sel], Ne=int(z["Ne"]), thickness_ang=float(c["thickness"]))
    tables = LineTables(c["E_tab"], c["chi_re"], c["chi_im"], c["u_re"], c["u_im"], c["log_mu"], c["delta"])
    rows = ReflectionRows(c["G"], c["ES"][None], c["EP"][None], c["WM"], c["row_table"])
    got = coherent_route_spectrum_streamed(seg, z["E_grid"], z["delta_omega"], tables=tables, rows=rows,
                                           n_hat=c["n_hat"], block_segments=max(1, int(sel.sum()) // 3),
                                           decoherence=dict(A_pop=z["A_pop"], xy0_pop=z["xy0_pop"], omega=z["omega"]))
    _assert_close(got, z["spec"])
