"""The depth-node form of the mixed bremsstrahlung scorer, restated in numpy
and checked against the oracle's per-(segment, energy) spectrum on CPU.

The restatement follows pb_brem_node.cu step by step: the electron-energy
window and its degree-5 Chebyshev fit of J_el(T, k), the depth grid (five
cells of 1/lambda_max, then cells a fifth of their start depth), the exact
segment means of the cell polynomials through the divided differences
D_{j+1}(t_a, t_b), the Lagrange basis of the eight Chebyshev nodes, and the
contraction per energy and direction. Segments outside the window are scored
by the oracle, as the device hands them to the per-pair kernels. In FP64 the
form reproduces the per-pair sums to rounding; the device's float moment sums
add ~1e-7 (tests/test_gpu_brem_node.py).
"""

import numpy as np
import pytest

import oracle

MC2 = 510.99895
ALPHA = 1.0 / 137.035999
RE2 = 7.9407877e-26
ZA = 2 * np.pi * ALPHA
C0 = 16.0 / 3.0 * ALPHA * RE2


def _J(T, k, Z):
    Tf = T - k
    p_i = np.sqrt(T * (T + 2 * MC2)) / MC2
    b_i = p_i / (1 + T / MC2)
    p_f = np.sqrt(Tf * (Tf + 2 * MC2)) / MC2
    b_f = p_f / (1 + Tf / MC2)
    dpp = k * (T + Tf + 2 * MC2) / MC2 ** 2
    return b_i / p_i ** 2 * np.log((p_i + p_f) ** 2 / dpp) / b_f / (1 - np.exp(-ZA * Z / b_f))


def _fit5(f):
    um = np.cos((2 * np.arange(6) + 1) * np.pi / 12)
    fv = f(um)
    Tm = np.array([np.cos(p * np.arccos(um)) for p in range(6)])
    c = (2.0 / 6) * fv @ Tm.T
    c[..., 0] *= 0.5
    return np.stack([c[..., 0] - c[..., 2] + c[..., 4], c[..., 1] - 3 * c[..., 3] + 5 * c[..., 5],
                     2 * c[..., 2] - 8 * c[..., 4], 4 * c[..., 3] - 20 * c[..., 5], 8 * c[..., 4], 16 * c[..., 5]], -1)


def _lagrange8():
    x = np.cos((2 * np.arange(8) + 1) * np.pi / 16)
    Tc = np.zeros((8, 8))
    Tc[0, 0] = Tc[1, 1] = 1
    for m in range(1, 7):
        Tc[m + 1] = 2 * np.roll(Tc[m], 1) - Tc[m - 1]
    w = np.full(8, 2.0 / 8)
    w[0] = 1.0 / 8
    Tx = np.array([np.cos(m * np.arccos(x)) for m in range(8)])
    return x, np.einsum("m,mi,mj->ij", w, Tx, Tc)


def _grid(thickness, lam_max):
    h = min(1.0 / lam_max, thickness) if lam_max > 0 else thickness
    zb, c = [0.0], 0
    while zb[-1] < thickness:
        c += 1
        zb.append(c * h if c <= 5 else 5 * h * 1.2 ** (c - 5))
    zb[-1] = thickness
    return np.array(zb)


def node_spectrum(seg, Z, n_ang3, thickness, n_hats, E_grid, mu):
    T = seg["E_keV"]
    L = seg["L_ang"]
    z, vz = seg["r_mid"][:, 2], seg["v_hat"][:, 2]
    k = E_grid / 1e3
    T_hi = T.max()
    T_lo = max(T.min(), T_hi / 1.1, 2.5 * k.max())
    win = T >= T_lo
    Tc, Th = 0.5 * (T_lo + T_hi), 0.5 * (T_hi - T_lo)
    A = np.stack([_fit5(lambda u, Ze=Ze: _J(Tc + Th * u[None, :], k[:, None], Ze)) for Ze in Z], 1)
    f = 1.0 / np.maximum(np.abs(n_hats[:, 2]), 1e-12)
    face = np.where(n_hats[:, 2] < 0, 0, 1)
    zb = _grid(thickness, mu.max() * f.max())
    nc = zb.size - 1
    x, Lm = _lagrange8()
    S = np.zeros((len(Z), 2, nc, 6, 8))
    d0 = np.clip(z - 0.5 * L * vz, 0, thickness)
    d1 = np.clip(z + 0.5 * L * vz, 0, thickness)
    lo, hi = np.minimum(d0, d1), np.maximum(d0, d1)
    b_i = np.sqrt(T * (T + 2 * MC2)) / (T + MC2)
    for s in np.nonzero(win)[0]:
        up = ((T[s] - Tc) / Th if Th > 0 else 0.0) ** np.arange(6)
        w = np.array([n * 1e24 * L[s] * 1e-8 * Ze ** 2 * (1 - np.exp(-ZA * Ze / b_i[s])) for Ze, n in zip(Z, n_ang3)])
        for fc in (0, 1):
            a, b = (lo[s], hi[s]) if fc == 0 else (thickness - hi[s], thickness - lo[s])
            ca = min(max(np.searchsorted(zb, a, side="right") - 1, 0), nc - 1)
            cb = min(max(np.searchsorted(zb, b, side="right") - 1, 0), nc - 1)
            for c in range(ca, cb + 1):
                mid, hw = 0.5 * (zb[c] + zb[c + 1]), 0.5 * (zb[c + 1] - zb[c])
                if b - a <= 1e-9 * 2 * hw:
                    M = ((a - mid) / hw) ** np.arange(8)
                else:
                    oa, ob = max(a, zb[c]), min(b, zb[c + 1])
                    if ob <= oa:
                        continue
                    ta, tb = (oa - mid) / hw, (ob - mid) / hw
                    D, tan, M = 1.0, ta, np.zeros(8)
                    M[0] = 1.0
                    for j in range(1, 8):
                        D = tb * D + tan
                        tan *= ta
                        M[j] = D / (j + 1)
                    M *= (ob - oa) / (b - a)
                S[:, fc, c] += w[:, None, None] * up[None, :, None] * M[None, None, :]
    nodes = 0.5 * (zb[:-1] + zb[1:])[:, None] + 0.5 * (zb[1:] - zb[:-1])[:, None] * x[None, :]
    spec = np.zeros((n_hats.shape[0], k.size))
    for e in range(k.size):
        W = np.einsum("ij,fcj->fci", Lm, np.einsum("lp,lfcpj->fcj", A[e], S))
        for d in range(n_hats.shape[0]):
            spec[d, e] = C0 / E_grid[e] * np.sum(np.exp(-mu[e] * f[d] * nodes) * W[face[d]])
    return spec, win


@pytest.fixture(scope="module")
def scene():
    from pyrite_b200 import configs
    from pyrite_b200.api import _fill_beam

    spec = configs.c2_si_50mev(seed=12345)
    st = spec.stack
    lt = oracle.LayerTables(st.z_top, st.z_bot, st.n_el, st.Z, st.J, st.N, st.E_cross)
    pos, dirs, E = oracle.beam_entries(_fill_beam(None, spec.beam, spec.seed), 0, 12, rng=oracle.RNG_PHILOX)
    out = oracle.transport(lt, pos, dirs, E, seed=spec.seed, E_cut=spec.E_cut_keV, rng=oracle.RNG_PHILOX,
                           e_start=0, cap=256)
    seg = dict(E_keV=0.5 * (np.asarray(out["E_start"]) + np.asarray(out["E_end"])), L_ang=np.asarray(out["L"]),
               r_mid=np.asarray(out["r_mid"]).reshape(-1, 3), v_hat=np.asarray(out["v_hat"]).reshape(-1, 3))
    return spec, seg


@pytest.mark.parametrize("spread", [False, True])
def test_node_form_matches_the_oracle(scene, spread):
    """The bench scene's segments (a narrow window: every segment in it), and
    the same segments with their energies spread so that half fall below the
    window and take the per-pair oracle: both within 1e-10 of the peak."""
    spec, seg = scene
    seg = dict(seg)
    if spread:
        seg["E_keV"] = seg["E_keV"] * np.random.default_rng(3).uniform(0.8, 1.0, seg["E_keV"].size)
    st = spec.stack
    Z, n3 = [14.0], [spec.brem_composition[0][1]]
    Eg, mu = np.asarray(spec.E_grid)[::32], np.asarray(spec.brem_mu)[::32]
    nh = np.asarray(spec.n_hats)[[0, 5, 15]].copy()
    nh[1, 2] *= -1.0  # a direction through the other face
    sp, win = node_spectrum(seg, Z, n3, st.thickness, nh, Eg, mu)
    assert win.any() and (win.all() != spread)
    rest = {kk: v[~win] for kk, v in seg.items()}
    for d in range(nh.shape[0]):
        ref = oracle.brem_spectrum(seg, Z, n3, st.thickness, nh[d], Eg, mu, 1) * 4 * np.pi
        tot = sp[d] + (oracle.brem_spectrum(rest, Z, n3, st.thickness, nh[d], Eg, mu, 1) * 4 * np.pi
                       if (~win).any() else 0.0)
        assert np.max(np.abs(tot - ref)) <= 1e-10 * np.max(np.abs(ref))
