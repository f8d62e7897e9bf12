"""The float path's rewrites of the reference's expressions, emulated in
float32 NumPy against the double-precision forms (CPU; the kernels' own
results are checked against the reference on the GPU).

- Bethe-Heitler + Elwert (brem.py:396-479): the float kernel takes
  1/p_f = m c^2 / sqrt(q), 1/beta_f = (1 + T_f / m c^2) m c^2 / sqrt(q) and
  ln((p_i + p_f)/(p_i - p_f)) = ln((p_i + p_f)^2 / (p_i^2 - p_f^2)) with
  p_i^2 - p_f^2 = k (T + T_f + 2 m c^2) / (m c^2)^2, free of cancellation;
- the segment-mean escape (segment_escape.py:276-289) as the difference
  2^(-A f) - 2^(-(A+B) f) over B (D > 0.01) or its series (D <= 0.01), with
  D = B f ln 2 (directions that leave through both faces);
- the direction-moment form of the escape for directions that share an exit
  face (pb_brem.cu brem_moment_chunk): Taylor coefficients of
  f Tbar(f) about the band centre f_c, summed over segments, evaluated per
  direction.
"""

import math

import numpy as np

import oracle

MC2 = 510.99895
ALPHA = 1.0 / 137.035999
RE_CM = 2.8179403262e-13


def bh_double(T, k, Z):
    """brem.py:431-479 in float64, the reference's expression order."""
    T_f = T - k
    p_i = np.sqrt(T * (T + 2 * MC2)) / MC2
    p_f = np.sqrt(T_f * (T_f + 2 * MC2)) / MC2
    b_i = p_i / (1 + T / MC2)
    b_f = p_f / (1 + T_f / MC2)
    born = np.log((p_i + p_f) / np.maximum(p_i - p_f, 1e-30))
    elw = b_i / b_f * (1 - np.exp(-2 * np.pi * Z * ALPHA / b_i)) / (1 - np.exp(-2 * np.pi * Z * ALPHA / b_f))
    return 16 / 3 * ALPHA * RE_CM ** 2 * Z * Z / (k * 1e3) / (p_i * p_i) * born * elw


def bh_float_form(T, k, Z):
    f = np.float32
    T, k, Z = f(T), f(k), f(Z)
    mc2, inv = f(MC2), f(1.0 / MC2)
    T_f = T - k
    q = T_f * (T_f + f(2) * mc2)
    rs = f(1) / np.sqrt(q)
    p_f = q * rs * inv
    p_i = np.sqrt(T * (T + f(2) * mc2)) * inv
    b_i = p_i / (f(1) + T * inv)
    g_i = b_i / (p_i * p_i)
    sp = p_i + p_f
    dpp = f(k / (MC2 * MC2)) * (f(2) * T + f(2 * MC2 - float(k)))
    lg = np.log2(sp * sp / dpp)
    inv_b_f = (T_f * inv + f(1)) * (rs * mc2)
    za = f(2 * np.pi * ALPHA)
    den_i = f(1) - np.exp(-za * Z / b_i)
    den_f = f(1) - np.exp2(-f(2 * np.pi * ALPHA * 1.4426950408889634) * Z * inv_b_f)
    c0k = f(16 / 3 * ALPHA * RE_CM ** 2 * np.log(2) / (float(k) * 1e3))
    return float(c0k * g_i * lg * inv_b_f * Z * Z * den_i / den_f)


def test_cross_section_rewrite():
    """Within 2e-5 up to k = 0.99 T; at the tip (k -> T of a 50-100 MeV
    electron) T_f = T - k itself loses digits in float (its spacing near
    1e5 keV is 0.008 keV), so the bound there is 2e-4."""
    worst, worst_tip = 0.0, 0.0
    for T in (20.0, 300.0, 5000.0, 50000.0, 100000.0):
        for frac in (1e-4, 0.01, 0.3, 0.9, 0.99, 0.999):
            k = T * frac
            for Z in (6.0, 14.0, 74.0):
                ref = bh_double(T, k, Z)
                err = abs(bh_float_form(T, k, Z) - ref) / ref
                if frac <= 0.99:
                    worst = max(worst, err)
                else:
                    worst_tip = max(worst_tip, err)
    assert worst < 2e-5, worst
    assert worst_tip < 2e-4, worst_tip


def escape_float(A, B, f):
    """The per-direction form (pb_brem.cu, directions on both faces)."""
    f32 = np.float32
    A, B, f = f32(A), f32(B), f32(f)
    fl = f * f32(np.log(2))
    D = B * fl
    e_lo = np.exp2(-A * f)
    if D > f32(0.01):
        t = (f32(1) / B) * (f32(1) - np.exp2(-B * f))
    else:
        t = fl * (f32(1) + D * (f32(-0.5) + D * (f32(1 / 6) + D * f32(-1 / 24))))
    return float(t * e_lo / fl)


def test_escape_forms():
    """The per-direction form, divided by f ln 2 as the kernel does per chunk,
    against the reference's mean transmission of the base-e depths A f ln 2
    and (A + B) f ln 2 (A, B are the base-2 depths the kernel carries)."""
    worst = 0.0
    for A in (0.0, 0.3, 4.0, 30.0):
        for B in (0.0, 1e-6, 1e-3, 0.02, 0.5, 8.0):
            for f in (1.0, 1.06, 3.0):
                ln2 = np.log(2.0)
                ref = oracle.mean_transmission(A * f * ln2, (A + B) * f * ln2)
                got = escape_float(A, B, f)
                scale = max(ref, 1e-30)
                worst = max(worst, abs(got - ref) / scale)
    assert worst < 1e-4, worst


def moment_escape_float(nsig, e_lo, e2, mu, f_dirs, order):
    """float32 emulation of brem_moment_chunk + brem_moment_eval: the sums
    sum_seg nsig Tbar(f_d) over segments (nsig, e_lo exit-side depth, e2 depth
    extent) at one photon energy (mu) for every direction factor f_d, in the
    kernel's operation order."""
    f32 = np.float32
    f_dirs = np.asarray(f_dirs, dtype=np.float64)
    f_lo, f_hi = f_dirs.min(), f_dirs.max()
    f_c, dl = 0.5 * (f_lo + f_hi), 0.5 * (f_hi - f_lo)
    mu_l2fc, mu_fc = f32(mu * 1.4426950408889634 * f_c), f32(mu * f_c)
    inv_mu, mu_dl, fcf, dlf = f32(1) / f32(mu), f32(mu * dl), f32(f_c), f32(dl)
    Q = [f32(0)] * (order + 1)
    for ns, es, d2 in zip(nsig, e_lo, e2):
        ns, es, d2 = f32(ns), f32(es), f32(d2)
        inv_e2 = f32(1) / d2 if d2 > 0 else f32(np.inf)
        ef = es + d2
        Ea, Ec = np.exp2(-mu_l2fc * es), np.exp2(-mu_l2fc * ef)
        x = mu_fc * d2
        phi = x * (x * (x * (x * (x * f32(-1 / 720) + f32(1 / 120)) + f32(-1 / 24)) + f32(1 / 6)) + f32(-0.5)) + f32(1)
        P = (Ea - Ec) * (inv_mu * inv_e2) if x > f32(0.1) else Ea * fcf * phi
        Q[0] = ns * P + Q[0]
        ah, ch = -mu_dl * es, -mu_dl * ef
        R = dlf * Ec
        for n in range(1, order + 1):
            P = ah * P + R
            if n < order:
                R = R * ch
            Q[n] = ns * P + Q[n]
    inv_fact = [f32(1.0 / math.factorial(n)) for n in range(order + 1)]
    out = []
    for f in f_dirs:
        h = f32((f - f_c) / dl) if dl > 0 else f32(0)
        r = Q[order] * inv_fact[order]
        for n in range(order - 1, -1, -1):
            r = r * h + Q[n] * inv_fact[n]
        out.append(float(r) * float(f32(1.0 / f)))
    return np.array(out)


def test_moment_escape_form_against_fp64():
    """The moment form against the FP64 per-direction mean transmission
    (segment_escape.py:276-289) summed over a segment population spanning
    every regime: exit-side depths 0-500 um, depth extents from 0 (parallel
    to the face) to 40 um, photon energies from strongly (mu L >> 1) to
    weakly absorbed. Directions: the 16 tiles of the 50 MeV Si detector
    (rho = 0.13 %, order 3) and a 10 % spread (order 7). Bound: 1e-6
    relative (float rounding, measured 3.2e-7; the series truncation is below
    3e-9; order 3 on the 10 % spread would give 6e-6)."""
    from pyrite_b200 import configs

    rng = np.random.default_rng(5)
    n = 256
    e_lo = np.concatenate([[0.0, 0.0], rng.uniform(0.0, 5.0e6, n - 2)])
    e2 = np.concatenate([[0.0, 1.0e-3], rng.uniform(0.0, 4.0e5, n - 2)])
    e2[5:12] = 0.0
    nsig = rng.uniform(0.5, 2.0, n)
    tiles = 1.0 / np.abs(configs.c2_si_50mev().n_hats[:, 2])
    wide = np.linspace(1.0, 1.2, 9)
    worst = 0.0
    for f_dirs, order in ((tiles, 3), (wide, 7)):
        for mu in (1e-9, 1e-7, 3e-6, 1e-5, 1e-4, 1e-3):
            got = moment_escape_float(nsig, e_lo, e2, mu, f_dirs, order)
            for g, f in zip(got, f_dirs):
                ref = sum(w * oracle.mean_transmission(mu * a * f, mu * (a + b) * f)
                          for w, a, b in zip(nsig, e_lo, e2))
                worst = max(worst, abs(g - ref) / ref)
    assert worst < 1e-6, worst


def test_float32_doppler_factor_at_tens_of_mev():
    """The mixed CXR scorer's FP32 Doppler factor (pb_cxr.cu seg_precompute:
    gamma = 1 + E/mc^2, 1 - beta v.n = 1/(gamma^2 (1 + beta)) + beta |v - n|^2/2)
    within the reference's float32 bounds (4 ulp gamma, 16 ulp denominator;
    tests/montecarlo/spectrum/test_line_kinematics_precision.py:56-66) at
    30 and 100 MeV, forward (1 mrad, 1/gamma scale) and backward; beta
    carries up to 3 ulp of the rsqrt-based square root."""
    f32 = np.float32
    eps = float(np.finfo(f32).eps)
    angles = np.array([1e-3, 5e-3, 0.3, 2.0])
    for E in (3.0e4, 1.0e5):
        gamma_ref = 1.0 + E / MC2
        omb_ref = 1.0 / (gamma_ref * gamma_ref * (1.0 + np.sqrt(1.0 - 1.0 / gamma_ref ** 2)))
        denom_ref = omb_ref + (1.0 - omb_ref) * 2.0 * np.sin(angles / 2.0) ** 2
        Ef = f32(E)
        g0 = f32(1) + Ef / f32(510.99895)
        beta0 = np.sqrt(f32(1) - f32(1) / (g0 * g0)).astype(f32)
        gamma = f32(1) + Ef / f32(MC2)
        assert abs(float(gamma) / gamma_ref - 1.0) < 4 * eps
        vh = np.array([0.0, 0.0, 1.0], dtype=f32)
        for k in range(-3, 4):
            beta = f32(beta0 + f32(k) * np.spacing(beta0))
            omb = f32(1) / (gamma * gamma * (f32(1) + beta))
            for a, ref in zip(angles, denom_ref):
                n = np.array([np.sin(a), 0.0, np.cos(a)], dtype=f32)
                d = vh - n
                omc = f32(0.5) * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
                denom = omb + beta * omc
                assert abs(float(denom) / ref - 1.0) < 16 * eps, (E, a, k)
