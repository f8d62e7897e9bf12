/*
 * CPU ORACLE -- test infrastructure, never the product.
 *
 * C restatement of the reference's incoherent PXR + CBS line chain for a
 * fixed segment list on a single slab (the batched route,
 * src/pyrite/montecarlo/spectrum/cxr/_batched.py:461-931), its two line
 * reductions (node sampling, cxr/_cpu_reduce.py:26-50; exact bin means,
 * cxr/_bin_quadrature.py:280-520) and the Bethe-Heitler + Elwert
 * bremsstrahlung track-length estimator (spectrum/brem.py:396-505,1196-1239).
 * Evaluation order follows the reference expression by expression, so FP64
 * results agree with it to rounding (pinned by tests/golden/cxr_*.npz and
 * brem_*.npz).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "oracle.h"

#define HBARC_EV_ANG 1973.269804
#define M_E_EV 510998.95
#define ALPHA_FS (1.0 / 137.035999)
#define RESONANCE_ROOT_RTOL 1e-3

/* cxr/_kernels.py:328-349: bracket index against an ascending grid. */
static void interp_index(double x, const double *grid, int n, int *idx, double *frac, int *below,
                         int *above) {
    int i;
    if (isnan(x)) {
        i = n; /* NaN sorts last in searchsorted */
    } else {
        int lo = 0, hi = n; /* searchsorted side="left" */
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (grid[mid] < x) lo = mid + 1; else hi = mid;
        }
        i = lo;
    }
    if (i < 1) i = 1;
    if (i > n - 1) i = n - 1;
    *idx = i;
    *frac = (x - grid[i - 1]) / (grid[i] - grid[i - 1]);
    *below = x <= grid[0];
    *above = x >= grid[n - 1];
}

/* cxr/_kernels.py:495-506 */
static double gather1(const double *f, int n, int idx, double frac, int below, int above) {
    double f0 = f[idx - 1];
    double y = f0 + frac * (f[idx] - f0);
    if (below) y = f[0];
    if (above) y = f[n - 1];
    return y;
}

/* cxr/_kernels.py:352-366 */
static double log_interp_fraction(double x, const double *grid, int idx) {
    double x0 = grid[idx - 1], x1 = grid[idx];
    double bx = fmin(fmax(x, x0), x1);
    if (isnan(x)) bx = x;
    return log1p((bx - x0) / x0) / log1p((x1 - x0) / x0);
}

/* segment_escape.py:276-289 */
double or_mean_transmission(double t0, double t1) {
    double lo = fmin(t0, t1);
    if (isnan(t0) || isnan(t1)) lo = NAN;
    double d = fabs(t1 - t0);
    double safe = d > 1.0e-4 ? d : 1.0;
    double ratio = d > 1.0e-4 ? -expm1(-safe) / safe : 1.0 - 0.5 * d + d * d / 6.0;
    return exp(-lo) * ratio;
}

/* cxr/_recoil.py:35-76 */
void or_quantum_line_factors(double h, double gamma, double vdg, double k_dot_v, double k_dot_g,
                             double g2, double k2, double v_dot_e, double g_dot_e, double k_dot_e,
                             double *pxr_num, double *f_cbs) {
    double gg = gamma * gamma;
    double n_1 = h * g2 - 2.0 * gamma * vdg;
    double n_2 = n_1 + 2.0 * h * k_dot_g;
    double n_f = h * (g2 + 2.0 * k_dot_g + k2) - 2.0 * gamma * (vdg + k_dot_v);
    double e_1 = sqrt(gg + h * n_1);
    double e_2 = sqrt(gg + h * (h * k2 - 2.0 * gamma * k_dot_v));
    double e_f = sqrt(gg + h * n_f);
    double s_if = gamma + e_f;
    double ge_ke = g_dot_e + k_dot_e;
    *pxr_num = (-n_f * ge_ke - k2 * (2.0 * gamma * v_dot_e - h * ge_ke)) / s_if;
    double s_1 = e_1 + gamma;
    double s_3 = e_1 + e_f;
    double s_4 = gamma + e_2;
    double x = 2.0 * gamma * v_dot_e - h * k_dot_e;
    double sigma = s_if + e_1 + e_2;
    *f_cbs = 2.0 * g_dot_e * s_1 / (s_3 * n_1) +
             x * (n_1 * (n_f / s_if) * sigma - 2.0 * s_1 * s_4 * k_dot_g) / (s_3 * s_4 * n_1 * n_2);
}

/* segment_escape.py:50-75: slab escape path [Angstrom] from depth z along n. */
static double slab_path(double z, double thickness, double nz) {
    double inv_nz = 1.0 / fmax(fabs(nz), 1.0e-12);
    double depth = fmin(fmax(z, 0.0), thickness);
    return nz < 0 ? depth * inv_nz : (thickness - depth) * inv_nz;
}

/* attenuation.py:270-277: z-extent of layer [z_top, z_bot] crossed leaving depth z. */
static double layer_dz(double z, double n_z, double z_top, double z_bot) {
    if (n_z < 0) return fmax(fmin(z, z_bot) - z_top, 0.0);
    return fmax(z_bot - fmax(z, z_top), 0.0);
}

/* segment_escape.py:134-140 */
static double cut_at_zero(double start, double end) {
    double den = start - end;
    double fr = start / (den == 0.0 ? 1.0 : den);
    return (fr > 0.0 && fr < 1.0) ? fr : 1.0;
}

#define OR_MAX_LAYERS 8

/* segment_escape.py:193-272 (layers, no footprint): cut at the tops of
 * layers 1..K-1, keep pieces wider than 1e-12, per-layer paths at the 1/4 and
 * 3/4 points (segment_escape.py:59-70) extrapolated to the piece ends and
 * clipped at zero. */
int or_layer_pieces(double z0, double z1, const or_layer_escape *ly, double n_z, double *frac,
                    double *path0, double *path1) {
    const int K = ly->n_layer;
    double cuts[OR_MAX_LAYERS + 1];
    int nc = 0;
    cuts[nc++] = 0.0;
    cuts[nc++] = 1.0;
    for (int k = 1; k < K; ++k) cuts[nc++] = cut_at_zero(z0 - ly->z_top[k], z1 - ly->z_top[k]);
    for (int i = 1; i < nc; ++i) {  /* np.sort */
        double v = cuts[i];
        int j = i - 1;
        while (j >= 0 && cuts[j] > v) { cuts[j + 1] = cuts[j]; --j; }
        cuts[j + 1] = v;
    }
    const double inv_nz = 1.0 / fmax(fabs(n_z), 1.0e-12);
    int P = 0;
    for (int i = 0; i + 1 < nc; ++i) {
        double w = cuts[i + 1] - cuts[i];
        if (!(w > 1.0e-12)) continue;
        double left = cuts[i];
        double delta = z1 - z0;
        double zq = z0 + (left + 0.25 * w) * delta;
        double z3 = z0 + (left + 0.75 * w) * delta;
        frac[P] = w;
        for (int k = 0; k < K; ++k) {
            double q = layer_dz(zq, n_z, ly->z_top[k], ly->z_bot[k]) * inv_nz;
            double tq = layer_dz(z3, n_z, ly->z_top[k], ly->z_bot[k]) * inv_nz;
            path0[P * K + k] = fmax(1.5 * q - 0.5 * tq, 0.0);
            path1[P * K + k] = fmax(1.5 * tq - 0.5 * q, 0.0);
        }
        ++P;
    }
    return P;
}

/* cxr/_escape_mu.py:49-57 */
static double exact_mu(const or_layer_escape *ly, int k, double E) {
    const int o = ly->mu_off[k], n = ly->mu_off[k + 1] - o;
    const double *kn = ly->mu_knot + o;
    int lo = 0, hi = n;
    while (lo < hi) {  /* searchsorted(..., side="right") */
        int mid = (lo + hi) / 2;
        if (kn[mid] <= E) lo = mid + 1; else hi = mid;
    }
    int j = lo - 1;
    if (j < 0) j = 0;
    if (j > n - 1) j = n - 1;
    double mu = ly->mu_value[o + j] + (E - kn[j]) * ly->mu_slope[o + j];
    if (E < kn[0]) mu = 0.0;
    return mu;
}

/* Per-segment quantities every row shares (cxr/_setup.py:945-1005). */
typedef struct {
    double vhz, beta, vx, vy, vz, gamma, denom_row, inv_E;
    double gx, gy, gz, grad2, v_dot_grad;
    int cxr_electron;
} seg_state;

static void seg_setup(const double *n_hat, double thickness, double E, const double *vh, double z_mid,
                      int cxr_electron, seg_state *q) {
    const double mec2_kev = M_E_EV / 1e3;
    q->vhz = vh[2];
    q->beta = or_beta_from_keV(E);
    q->vx = q->beta * vh[0];
    q->vy = q->beta * vh[1];
    q->vz = q->beta * vh[2];
    /* cxr/_kernels.py:678-699 (_vacuum_doppler) */
    q->gamma = 1.0 + E / mec2_kev;
    const double one_minus_beta = 1.0 / (q->gamma * q->gamma * (1.0 + q->beta));
    const double dvx = vh[0] - n_hat[0], dvy = vh[1] - n_hat[1], dvz = vh[2] - n_hat[2];
    const double omc = 0.5 * (dvx * dvx + dvy * dvy + dvz * dvz);
    q->denom_row = one_minus_beta + q->beta * omc;
    /* segment_escape.py:95-131: grad L = -z_hat / (z_hat . n), zero outside */
    const double nz = n_hat[2];
    q->gx = -0.0 / nz;
    q->gy = -0.0 / nz;
    q->gz = -1.0 / nz;
    if (z_mid < 0.0 || z_mid > thickness) { q->gx = 0.0; q->gy = 0.0; q->gz = 0.0; }
    q->grad2 = q->gx * q->gx + q->gy * q->gy + q->gz * q->gz;
    q->v_dot_grad = q->vx * q->gx + q->vy * q->gy + q->vz * q->gz;
    q->cxr_electron = cxr_electron;
    q->inv_E = HBARC_EV_ANG / (q->gamma * M_E_EV); /* cxr/_recoil.py:19-24 */
}

/* One (segment, row) pair up to the complex amplitudes of both
 * polarisations: cxr/_batched.py:461-559 and 600-625. */
typedef struct {
    double G[3], g2, n_dot_g, r_num, r_den, v_dot_g;
    double omega, E_res, slope, mu;
    double A_re[2], A_im[2];
    int keep;
} pair_state;

static void pair_chain(const or_cxr_tables *t, const double *n_hat, const seg_state *q, int g, pair_state *p) {
    const double h = HBARC_EV_ANG / M_E_EV; /* cxr/_recoil.py:27-32 */
    const double Gx = t->G[3 * g], Gy = t->G[3 * g + 1], Gz = t->G[3 * g + 2];
    const double vx = q->vx, vy = q->vy, vz = q->vz, gx = q->gx, gy = q->gy, gz = q->gz;
    p->G[0] = Gx;
    p->G[1] = Gy;
    p->G[2] = Gz;
    const double g2 = Gx * Gx + Gy * Gy + Gz * Gz;
    const double n_dot_g = Gx * n_hat[0] + Gy * n_hat[1] + Gz * n_hat[2];
    /* cxr/_block_prologue.py:18-38 + cxr/_recoil.py:79-97 */
    const double r_num = 0.5 * g2 * q->inv_E;
    const double r_den = n_dot_g * q->inv_E;
    const double v_dot_g_exact = (vx * Gx + vy * Gy + vz * Gz) - r_num;
    const double denom_vac = q->denom_row + r_den;
    /* cxr/_kernels.py:702-765: three fixed-point Snell passes */
    double denom = denom_vac, previous = denom, delta = NAN;
    for (int pass = 0; pass < 3; ++pass) {
        double Er = HBARC_EV_ANG * (v_dot_g_exact / denom);
        int ix, bl, ab;
        double fr;
        interp_index(Er, t->E_tab, t->n_tab, &ix, &fr, &bl, &ab);
        delta = gather1(t->delta, t->n_tab, ix, fr, bl, ab);
        previous = denom;
        denom = denom_vac - delta * q->v_dot_grad;
    }
    int settled = fabs(denom - previous) <= RESONANCE_ROOT_RTOL * fabs(denom);
    settled = settled && (2.0 * fabs(delta) * q->grad2 < 1.0);
    if (!settled) denom = NAN;
    /* cxr/_block_prologue.py:41-50 */
    const double n_dot_g_blk = n_dot_g + delta * (gx * Gx + gy * Gy + gz * Gz);
    /* cxr/_kernels.py:624-655 (_cxr_kin_core) */
    const double v_dot_g = vx * Gx + vy * Gy + vz * Gz;
    const double omega = (v_dot_g - r_num) / denom;
    const double k_dot_v = omega * ((1.0 - denom) + r_den);
    const double k_dot_g = omega * n_dot_g_blk;
    const double detuning = g2 + 2.0 * k_dot_g;
    /* cxr/_batched.py:435-458 (_line_bracket) */
    const double k_mag = omega * sqrt(q->grad2 == 0.0 ? 1.0 : 1.0 - 2.0 * delta + delta * delta * q->grad2);
    const double E_res = HBARC_EV_ANG * omega;
    int keep = q->cxr_electron && (E_res > t->lo_keep) && (E_res > 10.0) && (E_res < t->hi_keep);
    int ix, bl, ab;
    double fr;
    interp_index(E_res, t->E_tab, t->n_tab, &ix, &fr, &bl, &ab);
    const double lfr = log_interp_fraction(E_res, t->E_tab, ix);
    /* cxr/_block_prologue.py:53-62 + cxr/_recoil.py:100-118 */
    p->slope = denom * (1.0 / (1.0 - omega * q->inv_E));
    keep = keep && (denom > 0) && (omega * q->inv_E <= 1.0 - 1.0 / q->gamma);
    /* cxr/_kernels.py:482-506,369-388: couplings and attenuation */
    const int row = t->row_table[g];
    const double chi_re = gather1(t->chi_re + (int64_t)row * t->n_tab, t->n_tab, ix, fr, bl, ab);
    const double chi_im = gather1(t->chi_im + (int64_t)row * t->n_tab, t->n_tab, ix, fr, bl, ab);
    const double u_re = gather1(t->u_re + (int64_t)row * t->n_tab, t->n_tab, ix, fr, bl, ab);
    const double u_im = gather1(t->u_im + (int64_t)row * t->n_tab, t->n_tab, ix, fr, bl, ab);
    double mu = 0.0;
    for (int el = 0; el < t->n_mu; ++el) {
        const double *lm = t->log_mu + (int64_t)el * t->n_tab;
        double f0 = lm[ix - 1];
        double v = exp(f0 + lfr * (lm[ix] - f0));
        if (bl) v = exp(lm[0]);
        if (ab) v = exp(lm[t->n_tab - 1]);
        mu += v;
    }
    /* cxr/_batched.py:789-826 + cxr/_line_amplitude.py:14-37: PXR + CBS per polarization */
    for (int pol = 0; pol < 2; ++pol) {
        const double *Ev = pol == 0 ? t->ES + 3 * g : t->EP + 3 * g;
        const double ex = Ev[0], ey = Ev[1], ez = Ev[2];
        const double g_dot_e = Gx * ex + Gy * ey + Gz * ez;
        const double v_dot_e = vx * ex + vy * ey + vz * ez;
        const double k_dot_e = omega * delta * (gx * ex + gy * ey + gz * ez);
        double pxr_num, f_cbs;
        or_quantum_line_factors(h, q->gamma, v_dot_g, k_dot_v, k_dot_g, g2, k_mag * k_mag, v_dot_e, g_dot_e,
                                k_dot_e, &pxr_num, &f_cbs);
        const double f_pxr = pxr_num / detuning;
        p->A_re[pol] = chi_re * f_pxr + u_re * f_cbs;
        p->A_im[pol] = chi_im * f_pxr + u_im * f_cbs;
    }
    p->g2 = g2;
    p->n_dot_g = n_dot_g;
    p->r_num = r_num;
    p->r_den = r_den;
    p->v_dot_g = v_dot_g;
    p->omega = omega;
    p->E_res = E_res;
    p->mu = mu;
    p->keep = keep;
}

void or_cxr_lines(const or_cxr_tables *t, const or_cxr_geom *geo, int64_t n_seg,
                  const double *v_hat, const double *E_keV, const double *L_ang,
                  const double *r_mid, const int64_t *elec_id, int64_t Ne, double *E_res_out,
                  double *a_width_out, double *weight_out, uint8_t *good_out, int n_threads) {
    const double nz = geo->n_hat[2];
    const double T = geo->thickness;
    const double pref_c1 = 4.0 * (M_PI * M_PI) * HBARC_EV_ANG; /* cxr/_kernels.py:325 */
#pragma omp parallel for schedule(dynamic, 64) num_threads(n_threads > 0 ? n_threads : 1)
    for (int64_t s = 0; s < n_seg; ++s) {
        seg_state q;
        const double z_mid = r_mid[3 * s + 2];
        seg_setup(geo->n_hat, T, E_keV[s], v_hat + 3 * s, z_mid, elec_id[s] < Ne, &q);
        const double t_L = L_ang[s] / q.beta;
        /* segment_escape.py:239-270 (one linear piece on a single slab) */
        const double half = 0.5 * L_ang[s];
        const double path0 = slab_path(z_mid - half * q.vhz, T, nz);
        const double path1 = slab_path(z_mid + half * q.vhz, T, nz);
        /* layered absorber: linear escape pieces (cxr/_setup.py:1089) */
        const or_layer_escape *ly = geo->layers;
        double pf[OR_MAX_LAYERS], pp0[OR_MAX_LAYERS * OR_MAX_LAYERS], pp1[OR_MAX_LAYERS * OR_MAX_LAYERS];
        int n_piece = 0;
        if (ly) n_piece = or_layer_pieces(z_mid - half * q.vhz, z_mid + half * q.vhz, ly, nz, pf, pp0, pp1);
        for (int g = 0; g < t->n_g; ++g) {
            const int64_t o = s * t->n_g + g;
            pair_state p;
            pair_chain(t, geo->n_hat, &q, g, &p);
            const double A2 = (p.A_re[0] * p.A_re[0] + p.A_im[0] * p.A_im[0]) +
                              (p.A_re[1] * p.A_re[1] + p.A_im[1] * p.A_im[1]);
            /* cxr/_batched.py:702-730 + cxr/_kernels.py:658-668 */
            double T_abs;
            if (!ly) {
                T_abs = or_mean_transmission(path0 * p.mu, path1 * p.mu);
            } else {
                /* piece_mean_transmission (segment_escape.py:335-355) with the
                 * exact per-layer mu at E_res (cxr/_batched.py:714-720) */
                double mu_k[OR_MAX_LAYERS];
                for (int k = 0; k < ly->n_layer; ++k) mu_k[k] = exact_mu(ly, k, p.E_res);
                T_abs = 0.0;
                for (int i = 0; i < n_piece; ++i) {
                    double t0 = 0.0, t1 = 0.0;
                    for (int k = 0; k < ly->n_layer; ++k) {
                        t0 += pp0[i * ly->n_layer + k] * mu_k[k];
                        t1 += pp1[i * ly->n_layer + k] * mu_k[k];
                    }
                    T_abs += pf[i] * or_mean_transmission(t0, t1);
                }
            }
            const double pref = ALPHA_FS * p.omega / pref_c1 * (t_L * t_L) * T_abs;
            const double a_width = p.slope * t_L / (2.0 * HBARC_EV_ANG) * 1.0;
            const double weight = pref * A2 * t->WM[g];
            const int good = p.keep && isfinite(weight) && (weight > 0);
            E_res_out[o] = p.E_res;
            a_width_out[o] = a_width;
            weight_out[o] = weight;
            good_out[o] = (uint8_t)good;
        }
    }
}

/* cxr/_formation.py:58-81 (formation_coefficients) */
static void formation_coefficients(double tau_start, double tau_end, double *apb, double *bma, double *q) {
    const double qq = 0.25 * (tau_end - tau_start);
    if (fabs(qq) < 0.5) { /* FORMATION_SMALL_Q */
        const double c0 = exp(-0.25 * (tau_start + tau_end));
        *apb = 2.0 * c0 * cosh(qq);
        *bma = -2.0 * c0 * sinh(qq);
    } else {
        const double a = exp(-0.5 * tau_start), b = exp(-0.5 * tau_end);
        *apb = a + b;
        *bma = b - a;
    }
    *q = qq;
}

void or_cxr_coherent_records(const or_cxr_tables *t, const or_cxr_geom *geo, int64_t n_seg,
                             const double *v_hat, const double *E_keV, const double *L_ang,
                             const double *r_mid, const double *t_ang, const int64_t *elec_id,
                             int64_t Ne, double *const rec[OR_COH_FIELDS], uint8_t *good_out) {
    const double nx = geo->n_hat[0], ny = geo->n_hat[1], nz = geo->n_hat[2];
    const double T = geo->thickness;
    const double pref_c1 = 4.0 * (M_PI * M_PI) * HBARC_EV_ANG; /* cxr/_kernels.py:325 */
    for (int64_t s = 0; s < n_seg; ++s) {
        seg_state q;
        const double z_mid = r_mid[3 * s + 2];
        seg_setup(geo->n_hat, T, E_keV[s], v_hat + 3 * s, z_mid, elec_id[s] < Ne, &q);
        /* coherent rows keep their own length and unit piece fraction (cxr/_setup.py:1001-1005) */
        const double t_L = L_ang[s] / q.beta;
        /* escape distance at the piece ends, ordered along travel (cxr/_formation.py:168-200) */
        const double half = 0.5 * L_ang[s];
        const double L_start = slab_path(z_mid - half * q.vhz, T, nz);
        const double L_end = slab_path(z_mid + half * q.vhz, T, nz);
        /* cxr/_setup.py:1023-1026: midpoint age and retardation d = t_mid - n.r */
        const double t_mid = (t_ang ? t_ang[s] : 0.0) + 0.5 * t_L;
        const double rx = r_mid[3 * s], ry = r_mid[3 * s + 1], rz = r_mid[3 * s + 2];
        const double d_geom = t_mid - (rx * nx + ry * ny + rz * nz);
        for (int g = 0; g < t->n_g; ++g) {
            const int64_t o = s * t->n_g + g;
            pair_state p;
            pair_chain(t, geo->n_hat, &q, g, &p);
            /* formation factor constants of the piece (cxr/_batched.py:627-633) */
            double apb, bma, qq;
            formation_coefficients(L_start * p.mu, L_end * p.mu, &apb, &bma, &qq);
            /* exact vacuum centre / width and recoil phase over the age (cxr/_recoil.py:118-147),
             * with the vacuum denominator and n.g of the batched tables */
            const double numerator = p.v_dot_g - p.r_num;
            const double den = q.denom_row + p.r_den;
            const double E_c = HBARC_EV_ANG * numerator / den;
            const double x = numerator / den * q.inv_E;
            const double kappa = 1.0 / (1.0 - x);
            const double a_vac = kappa * den * t_L / (2.0 * HBARC_EV_ANG);
            const double d_shift = kappa * (x * q.denom_row + p.r_den) * t_mid;
            const double g_shift = kappa * (x * p.v_dot_g - p.r_num) * t_mid;
            const double amp = sqrt(ALPHA_FS * p.omega / pref_c1);
            int good = p.keep && isfinite(amp) && (amp > 0) && (t_L > 0) && isfinite(apb) && (apb > 0) &&
                       isfinite(bma);
            const double cs_re = amp * t_L * p.A_re[0], cs_im = amp * t_L * p.A_im[0];
            const double cp_re = amp * t_L * p.A_re[1], cp_im = amp * t_L * p.A_im[1];
            good = good && isfinite(cs_re) && isfinite(cs_im) && isfinite(cp_re) && isfinite(cp_im);
            /* record fields (cxr/_batched.py:646-660) */
            rec[0][o] = E_c;
            rec[1][o] = a_vac;
            rec[2][o] = (d_geom + d_shift) / HBARC_EV_ANG;
            rec[3][o] = rx * p.G[0] + ry * p.G[1] + rz * p.G[2] + g_shift;
            rec[4][o] = cs_re;
            rec[5][o] = cs_im;
            rec[6][o] = cp_re;
            rec[7][o] = cp_im;
            rec[8][o] = 0.5 * (L_start + L_end);
            rec[9][o] = 0.5 * (L_end - L_start);
            rec[10][o] = apb;
            rec[11][o] = bma;
            rec[12][o] = qq;
            good_out[o] = (uint8_t)good;
        }
    }
}

/* ---- line reductions ---------------------------------------------------- */

void or_reduce_node(int64_t n_lines, const double *E_res, const double *a_width,
                    const double *weight, int64_t n_e, const double *E_grid, double *spec,
                    int n_threads) {
#pragma omp parallel for schedule(static) num_threads(n_threads > 0 ? n_threads : 1)
    for (int64_t e = 0; e < n_e; ++e) {
        const double E = E_grid[e];
        double acc = 0.0;
        for (int64_t j = 0; j < n_lines; ++j) {
            double x = a_width[j] * (E - E_res[j]) / M_PI;
            if (x == 0.0) x = 1.0e-20;
            double y = M_PI * x;
            double s = sin(y) / y;
            acc += weight[j] * (s * s);
        }
        spec[e] += acc;
    }
}

/* Si(t) - pi/2 for t >= 0: power series below t = 4, else the continued
 * fraction of E1(i t) evaluated by the modified Lentz method (Numerical
 * Recipes, "cisi"), with E1(i t) = -Ci(t) + i (Si(t) - pi/2). */
double or_si_minus_half_pi(double t) {
    if (t <= 4.0) {
        double t2 = t * t, term = t, sum = t;
        for (int k = 1; k < 40; ++k) {
            term *= -t2 / ((2.0 * k) * (2.0 * k + 1.0));
            double add = term / (2.0 * k + 1.0);
            sum += add;
            if (fabs(add) < 1e-18 * fabs(sum)) break;
        }
        return sum - 0.5 * M_PI;
    }
    /* b = 1 + i t; h = 1/b; c = big; d = 1/b */
    double br = 1.0, bi = t;
    double den = br * br + bi * bi;
    double dr = br / den, di = -bi / den;
    double hr = dr, hi = di;
    double cr = 1e300, ci = 0.0;
    for (int i = 2; i < 400; ++i) {
        double a = -(double)(i - 1) * (double)(i - 1);
        br += 2.0;
        /* d = 1 / (a d + b) */
        double xr = a * dr + br, xi = a * di + bi;
        den = xr * xr + xi * xi;
        dr = xr / den;
        di = -xi / den;
        /* c = b + a / c */
        den = cr * cr + ci * ci;
        double qr = a * cr / den, qi = -a * ci / den;
        cr = br + qr;
        ci = bi + qi;
        double delr = cr * dr - ci * di, deli = cr * di + ci * dr;
        double nhr = hr * delr - hi * deli, nhi = hr * deli + hi * delr;
        hr = nhr;
        hi = nhi;
        if (fabs(delr - 1.0) + fabs(deli) < 1e-16) break;
    }
    /* E1(i t) = (cos t - i sin t) h */
    double c = cos(t), s = sin(t);
    double e_im = c * hi - s * hr;
    return e_im;
}

/* R(x) = F(x) - sign(x)/2 with F(x) = Si(2 pi x)/pi - x sinc^2(x), the
 * integral of sinc^2 from 0 (cxr/_bin_quadrature.py:351-375). */
double or_sincsq_tail(double x) {
    double u = fabs(x);
    double t = 2.0 * M_PI * u;
    double s = u == 0.0 ? 1.0 : sin(M_PI * u) / (M_PI * u);
    double r = or_si_minus_half_pi(t) / M_PI - u * s * s;
    return x >= 0.0 ? r : -r;
}

void or_reduce_binmean(int64_t n_lines, const double *E_res, const double *a_width,
                       const double *weight, int64_t n_bins, const double *edges, double *spec,
                       int n_threads) {
    double *partial = (double *)calloc((size_t)n_bins, sizeof(double));
#pragma omp parallel num_threads(n_threads > 0 ? n_threads : 1)
    {
        double *local = (double *)calloc((size_t)n_bins, sizeof(double));
#pragma omp for schedule(dynamic, 64)
        for (int64_t j = 0; j < n_lines; ++j) {
            const double a = a_width[j], Er = E_res[j], w = weight[j];
            double x_lo = a * (edges[0] - Er) / M_PI;
            double r_lo = or_sincsq_tail(x_lo);
            for (int64_t b = 0; b < n_bins; ++b) {
                double x_hi = a * (edges[b + 1] - Er) / M_PI;
                double r_hi = or_sincsq_tail(x_hi);
                double mass = r_hi - r_lo + ((x_lo < 0.0 && x_hi >= 0.0) ? 1.0 : 0.0);
                double mean = mass * (M_PI / a) / (edges[b + 1] - edges[b]);
                local[b] += w * mean;
                x_lo = x_hi;
                r_lo = r_hi;
            }
        }
#pragma omp critical
        for (int64_t b = 0; b < n_bins; ++b) partial[b] += local[b];
        free(local);
    }
    for (int64_t b = 0; b < n_bins; ++b) spec[b] += partial[b];
    free(partial);
}

/* ---- Bethe-Heitler + Elwert (spectrum/brem.py:431-479) ------------------ */
#define R_E_CM2 7.9407877e-26
#define BREM_MC2_KEV 510.99895

static double brem_dsigma_dk(double T_i, double k_keV, double Z) {
    double mc2 = BREM_MC2_KEV;
    double T_f = T_i - k_keV;
    int ok = (T_f > 1e-6) && (k_keV > 0.0);
    if (!ok) return 0.0;
    double p_i = sqrt(T_i * (T_i + 2.0 * mc2)) / mc2;
    double p_f = sqrt(T_f * (T_f + 2.0 * mc2)) / mc2;
    double beta_i = p_i / (1.0 + T_i / mc2);
    double beta_f = p_f / (1.0 + T_f / mc2);
    double born_log = log((p_i + p_f) / fmax(p_i - p_f, 1e-30));
    double elwert = beta_i / beta_f * (1.0 - exp(-2.0 * M_PI * Z * ALPHA_FS / beta_i)) /
                    (1.0 - exp(-2.0 * M_PI * Z * ALPHA_FS / beta_f));
    return 16.0 / 3.0 * ALPHA_FS * R_E_CM2 * (Z * Z) / fmax(k_keV * 1e3, 1e-30) / (p_i * p_i) *
           born_log * elwert;
}

void or_brem_spectrum(int64_t n_seg, const double *E_keV, const double *L_ang,
                      const double *r_mid, const double *v_hat, int n_el, const double *Z,
                      const double *n_ang3, double thickness, const double n_hat[3], int64_t n_e,
                      const double *E_grid, const double *mu_grid, double *spec, int n_threads) {
#pragma omp parallel for schedule(static) num_threads(n_threads > 0 ? n_threads : 1)
    for (int64_t e = 0; e < n_e; ++e) {
        const double k = E_grid[e] / 1e3;
        double acc = 0.0;
        for (int64_t s = 0; s < n_seg; ++s) {
            const double half = 0.5 * L_ang[s];
            const double z = r_mid[3 * s + 2];
            const double p0 = slab_path(z - half * v_hat[3 * s + 2], thickness, n_hat[2]);
            const double p1 = slab_path(z + half * v_hat[3 * s + 2], thickness, n_hat[2]);
            const double T_abs = or_mean_transmission(p0 * mu_grid[e], p1 * mu_grid[e]);
            const double path_cm = L_ang[s] * 1e-8;
            for (int el = 0; el < n_el; ++el) {
                double d = brem_dsigma_dk(E_keV[s], k, Z[el]);
                acc += (n_ang3[el] * 1e24 * 1.0 * path_cm) * (d * T_abs);
            }
        }
        spec[e] += acc;
    }
}

void or_brem_spectrum_layered(int64_t n_seg, const double *E_keV, const double *L_ang,
                              const double *r_mid, const double *v_hat, int n_el, const double *Z,
                              const double *n_ang3, const or_layer_escape *ly, const double n_hat[3],
                              int64_t n_e, const double *E_grid, const double *mu_layer, double *spec,
                              int n_threads) {
    const int K = ly->n_layer;
#pragma omp parallel for schedule(static) num_threads(n_threads > 0 ? n_threads : 1)
    for (int64_t e = 0; e < n_e; ++e) {
        const double k = E_grid[e] / 1e3;
        double acc = 0.0;
        for (int64_t s = 0; s < n_seg; ++s) {
            const double half = 0.5 * L_ang[s];
            const double z = r_mid[3 * s + 2];
            double pf[OR_MAX_LAYERS], p0[OR_MAX_LAYERS * OR_MAX_LAYERS], p1[OR_MAX_LAYERS * OR_MAX_LAYERS];
            const int P = or_layer_pieces(z - half * v_hat[3 * s + 2], z + half * v_hat[3 * s + 2], ly, n_hat[2],
                                          pf, p0, p1);
            for (int p = 0; p < P; ++p) {
                /* _layer_depth (brem.py:814-820): fixed layer order */
                double t0 = p0[p * K] * mu_layer[e], t1 = p1[p * K] * mu_layer[e];
                for (int kk = 1; kk < K; ++kk) {
                    t0 = t0 + p0[p * K + kk] * mu_layer[(int64_t)kk * n_e + e];
                    t1 = t1 + p1[p * K + kk] * mu_layer[(int64_t)kk * n_e + e];
                }
                const double T_abs = or_mean_transmission(t0, t1);
                const double path_cm = (L_ang[s] * pf[p]) * 1e-8;
                for (int el = 0; el < n_el; ++el) {
                    double d = brem_dsigma_dk(E_keV[s], k, Z[el]);
                    acc += (n_ang3[el] * 1e24 * 1.0 * path_cm) * (d * T_abs);
                }
            }
        }
        spec[e] += acc;
    }
}
