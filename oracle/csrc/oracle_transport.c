/*
 * CPU ORACLE -- test infrastructure, never the product.
 *
 * Plain-C restatement of the reference's per-electron transport core with the
 * data-free physics set (screened-Rutherford elastic, spliced Joy-Luo /
 * Berger-Seltzer stopping, midpoint energy rule, no straggling, no
 * substeps), used by the tests as the checker for the CUDA transport kernel
 * and by bench.py as the timed CPU baseline. Each block cites the reference
 * lines it follows (paths relative to the reference project root).
 *
 * Parity: pinned bit for bit against rows produced by the reference itself
 * (tests/golden/transport_*.npz, made by tests/golden/make_golden.py).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "oracle.h"

/* ---- counter RNGs ------------------------------------------------------ */

/* SplitMix64 finalizer: src/pyrite/montecarlo/transport/kinematics.py:205-211 */
uint64_t or_splitmix64(uint64_t x) {
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

/* kinematics.py:219-222: key_e = sm64(seed + phi (e + 1)) */
uint64_t or_stream_key(uint64_t seed, uint64_t elec) {
    return or_splitmix64(seed + 0x9E3779B97F4A7C15ULL * (elec + 1ULL));
}

/* kinematics.py:225-229: u = (sm64(key + phi (c + 1)) >> 11) 2^-53 */
double or_stream_uniform(uint64_t key, uint64_t counter) {
    uint64_t z = or_splitmix64(key + 0x9E3779B97F4A7C15ULL * (counter + 1ULL));
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

/* Random123 Philox4x32-10 (Salmon et al., SC11), round mapping as in
 * src/pyrite/montecarlo/channeling/_axial_cuda_rng.py:17-43. */
void or_philox4x32_10(uint32_t ctr[4], uint32_t key[2]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = 0xD2511F53ULL * (uint64_t)c0;
        uint64_t p1 = 0xCD9E8D57ULL * (uint64_t)c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c0 = n0;
        c1 = (uint32_t)p1;
        c2 = n2;
        c3 = (uint32_t)p0;
        k0 += 0x9E3779B9U;
        k1 += 0xBB67AE85U;
    }
    ctr[0] = c0; ctr[1] = c1; ctr[2] = c2; ctr[3] = c3;
}

/* Draw ``draw`` of the Philox stream with 64-bit key ``key``: block draw/2 is
 * the counter, even draws use words (0,1), odd draws (2,3), 53-bit mantissa. */
double or_philox_uniform(uint64_t key, uint64_t draw) {
    uint64_t block = draw >> 1;
    uint32_t ctr[4] = {(uint32_t)block, (uint32_t)(block >> 32), 0u, 0u};
    uint32_t k[2] = {(uint32_t)key, (uint32_t)(key >> 32)};
    or_philox4x32_10(ctr, k);
    uint32_t a = (draw & 1ULL) ? ctr[2] : ctr[0];
    uint32_t b = (draw & 1ULL) ? ctr[3] : ctr[1];
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) / 9007199254740992.0;
}

static double draw_uniform(int rng_kind, uint64_t key, uint64_t counter) {
    return rng_kind == OR_RNG_PHILOX ? or_philox_uniform(key, counter)
                                     : or_stream_uniform(key, counter);
}

/* ---- physics leaves ------------------------------------------------------ */

#define MC2_KEV 510.99895
#define LN2 0.6931471805599453
#define BS_PREFACTOR 1.535e-6

/* kinematics.py:162-166 */
double or_beta_from_keV(double E) {
    double g = 1.0 + E / 510.99895;
    double gis = 1.0 / (g * g);
    return sqrt(1.0 - gis);
}

/* stopping.py:384-410, _dEds_spliced_packed_scalar (delta = 0) */
double or_dEds_spliced(const or_layers *ly, int L, double E) {
    double tau = E / MC2_KEV;
    double gamma = 1.0 + tau;
    double beta_sq = 1.0 - 1.0 / (gamma * gamma);
    double f_minus = 1.0 - beta_sq + (tau * tau / 8.0 - (2.0 * tau + 1.0) * LN2) / (gamma * gamma);
    double jl = 0.0, bs = 0.0;
    int n_el = ly->n_el[L];
    for (int i = 0; i < n_el; ++i) {
        int ix = L * ly->max_el + i;
        double J = ly->J[ix], coeff = ly->coeff[ix];
        if (E < ly->E_cross[ix]) {
            jl += coeff * log(1.166 * (E + ly->k[ix] * J) / J);
        } else {
            double I_rel = J / MC2_KEV;
            bs += coeff * (log(tau * tau * (tau + 2.0) / (2.0 * I_rel * I_rel)) + f_minus - 0.0);
        }
    }
    return -7.85e-4 / E * jl - BS_PREFACTOR / beta_sq * bs;
}

/* ---- Urban energy-loss straggling (straggling.py) ------------------------
 * The loss over a flight of length s is the compound Poisson sum of two
 * excitation levels and a 1/E^2 ionisation continuum whose mean is C s,
 * C = |dE/dx| of the element (straggling.py:57-120, the Urban model of the
 * Geant4 Physics Reference Manual). Each flight draws from its own SplitMix64
 * stream: urban key = sm64(electron key ^ salt) (straggling.py:37-43), flight
 * key = sm64(urban key + phi ((flight << 32) + substep)) (straggling.py:46-59),
 * draws (flight key, counter) from counter 0. */
#define URBAN_SALT 0xD6E8FEB86659FD93ULL
#define URBAN_E0_KEV 1.0e-2
#define URBAN_E2_PER_Z2 1.0e-2
#define URBAN_RATE 0.55
#define URBAN_CHUNK_MAX 64.0

/* stopping.py via straggling.py:278-298, _dEds_spliced_element_scalar (delta = 0) */
double or_dEds_element(double J, double k, double coeff, double E_cross, double E) {
    double tau = E / MC2_KEV;
    double gamma = 1.0 + tau;
    double beta_sq = 1.0 - 1.0 / (gamma * gamma);
    if (E < E_cross) return -7.85e-4 / E * coeff * log(1.166 * (E + k * J) / J);
    double f_minus = 1.0 - beta_sq + (tau * tau / 8.0 - (2.0 * tau + 1.0) * LN2) / (gamma * gamma);
    double I_rel = J / MC2_KEV;
    return -BS_PREFACTOR / beta_sq * coeff * (log(tau * tau * (tau + 2.0) / (2.0 * I_rel * I_rel)) + f_minus - 0.0);
}

/* straggling.py:127-157, _urban_levels_scalar */
static void urban_levels(double Z, double J, double T_up, double two_mc2_bg2, double beta_sq, double *f1,
                         double *E1, double *f2, double *E2) {
    double e2 = URBAN_E2_PER_Z2 * Z * Z;
    double g2 = Z > 2.0 ? 2.0 / Z : 1.0;
    *E2 = e2;
    if (Z > 2.0 && e2 < T_up && log(two_mc2_bg2 / e2) - beta_sq > 0.0) {
        double g1 = 1.0 - g2;
        double e1 = exp((log(J) - g2 * log(e2)) / g1);
        if (log(two_mc2_bg2 / e1) - beta_sq > 0.0) {
            *f1 = g1; *E1 = e1; *f2 = g2;
            return;
        }
    }
    *f1 = 1.0; *E1 = J; *f2 = 0.0;
}

/* straggling.py:160-201, _urban_channels_scalar; returns valid */
static int urban_channels(double Z, double J, double C, double E, double *s1, double *E1, double *s2,
                          double *E2, double *s3) {
    double tau = E / MC2_KEV;
    double gamma = 1.0 + tau;
    double beta_sq = 1.0 - 1.0 / (gamma * gamma);
    double two_mc2_bg2 = 2.0 * MC2_KEV * tau * (tau + 2.0);
    double T_up = 0.5 * E;
    *s1 = *s2 = *s3 = 0.0;
    *E1 = J;
    *E2 = 0.0;
    if (T_up <= URBAN_E0_KEV || C <= 0.0) return 0;
    double L_I = log(two_mc2_bg2 / J) - beta_sq;
    if (L_I <= 0.0) return 0;
    double f1, f2;
    urban_levels(Z, J, T_up, two_mc2_bg2, beta_sq, &f1, E1, &f2, E2);
    double soft = C * (1.0 - URBAN_RATE) / L_I;
    *s1 = soft * (f1 / *E1) * (log(two_mc2_bg2 / *E1) - beta_sq);
    if (f2 > 0.0) *s2 = soft * (f2 / *E2) * (log(two_mc2_bg2 / *E2) - beta_sq);
    *s3 = C * URBAN_RATE * (T_up - URBAN_E0_KEV) / (URBAN_E0_KEV * T_up * log(T_up / URBAN_E0_KEV));
    return 1;
}

/* straggling.py:204-222, _urban_moments_element_scalar */
void or_urban_moments_element(double Z, double J, double C, double E, double s, double *mean, double *var) {
    double s1, E1, s2, E2, s3;
    if (!urban_channels(Z, J, C, E, &s1, &E1, &s2, &E2, &s3)) {
        *mean = C * s;
        *var = 0.0;
        return;
    }
    double T_up = 0.5 * E;
    double mean3 = URBAN_E0_KEV * T_up * log(T_up / URBAN_E0_KEV) / (T_up - URBAN_E0_KEV);
    *mean = s * (s1 * E1 + s2 * E2 + s3 * mean3);
    *var = s * (s1 * E1 * E1 + s2 * E2 * E2 + s3 * URBAN_E0_KEV * T_up);
}

/* straggling.py:225-262, _urban_poisson_scalar: inverse CDF per chunk of
 * mean <= 64, one uniform per chunk */
static int64_t urban_poisson(double lam, uint64_t key, uint64_t *counter) {
    if (lam <= 0.0) return 0;
    int64_t n_chunks = (int64_t)ceil(lam / URBAN_CHUNK_MAX);
    double chunk = lam / (double)n_chunks;
    int64_t total = 0;
    for (int64_t c = 0; c < n_chunks; ++c) {
        double u = or_stream_uniform(key, *counter);
        *counter += 1;
        double p = exp(-chunk);
        double cdf = p;
        int64_t k = 0;
        while (u >= cdf) {
            k += 1;
            p = p * chunk / (double)k;
            double next = cdf + p;
            if (next <= cdf) break;
            cdf = next;
        }
        total += k;
    }
    return total;
}

/* straggling.py:277-275, _urban_sample_element_keV (inverse CDF of the
 * continuum, straggling.py:265-274) */
double or_urban_sample_element(double Z, double J, double C, double E, double s, uint64_t key,
                               uint64_t *counter) {
    double s1, E1, s2, E2, s3;
    if (!urban_channels(Z, J, C, E, &s1, &E1, &s2, &E2, &s3) || s <= 0.0) return C * s;
    int64_t n1 = urban_poisson(s1 * s, key, counter);
    int64_t n2 = urban_poisson(s2 * s, key, counter);
    int64_t n3 = urban_poisson(s3 * s, key, counter);
    double dE = (double)n1 * E1 + (double)n2 * E2;
    double T_up = 0.5 * E;
    for (int64_t i = 0; i < n3; ++i) {
        double u = or_stream_uniform(key, *counter);
        *counter += 1;
        dE += URBAN_E0_KEV / (1.0 - u * (T_up - URBAN_E0_KEV) / T_up);
    }
    return dE;
}

/* scattering.py:208-218, _scatter_rates_sr_scalar [1/cm] */
double or_sr_rate(double E, double sr_rate_numer, double sr_joy_numer) {
    double a = sr_joy_numer / E;
    double p511 = E + 511.0;
    double p1024 = E + 1024.0;
    double r = p511 / p1024;
    return sr_rate_numer / (E * E) / (a * (1.0 + a)) * (r * r);
}

/* scattering.py:234-236 */
double or_cos_theta_sr(double alpha, double R) { return 1.0 - 2.0 * alpha * R / (1.0 + alpha - R); }

/* ---- ELSEPA tabulated elastic scattering (scattering.py:516-640) -------- */

/* _elsepa_bracket: grid interval and fraction of logE, clamped to the ends */
static void elsepa_bracket(const or_elsepa *t, double logE, int64_t start, int64_t length, int64_t *row,
                           double *f) {
    int64_t first = start, last = start + length - 1;
    if (logE <= t->logE[first]) { *row = first; *f = 0.0; return; }
    if (logE >= t->logE[last]) { *row = last - 1; *f = 1.0; return; }
    int64_t lo = first, hi = last;
    while (hi - lo > 1) {
        int64_t mid = (lo + hi) / 2;
        if (t->logE[mid] <= logE) lo = mid; else hi = mid;
    }
    *row = lo;
    *f = (logE - t->logE[lo]) / (t->logE[hi] - t->logE[lo]);
}

/* _elsepa_rate_scalar: macroscopic elastic rate [1/cm], log-log in energy */
double or_elsepa_rate(const or_elsepa *t, int64_t start, int64_t length, double E_keV) {
    int64_t row;
    double f;
    elsepa_bracket(t, log(E_keV * 1e3), start, length, &row, &f);
    return exp(t->log_rate[row] + f * (t->log_rate[row + 1] - t->log_rate[row]));
}

/* _elsepa_panel: last panel k with cdf[row, k] <= xi, bisection inside the
 * guide window of xi's cell */
static int64_t elsepa_panel(const or_elsepa *t, int64_t row, double xi) {
    int cells = t->cells;
    double scaled = xi * cells;
    int cell;
    if (scaled >= cells) cell = cells - 1;
    else if (scaled > 0.0) cell = (int)scaled;
    else cell = 0;
    const int32_t *g = t->guide + row * (int64_t)(cells + 1);
    int64_t lo = g[cell], hi = (int64_t)g[cell + 1] + 1;
    const double *cdf = t->cdf + row * (int64_t)t->n_mu;
    while (hi - lo > 1) {
        int64_t mid = (lo + hi) / 2;
        if (cdf[mid] <= xi) lo = mid; else hi = mid;
    }
    return lo;
}

/* _elsepa_invert_row: the quadratic CDF of the linear panel density solved
 * in its cancellation-free form, t clamped to [0, 1] */
static double elsepa_invert_row(const or_elsepa *t, int64_t row, double xi) {
    int64_t lo = elsepa_panel(t, row, xi);
    const double *cdf = t->cdf + row * (int64_t)t->n_mu;
    const double *pdf = t->pdf + row * (int64_t)t->n_mu;
    double dmu = t->mu[lo + 1] - t->mu[lo];
    double p0 = pdf[lo], p1 = pdf[lo + 1];
    double r = xi - cdf[lo];
    double b = dmu * p0;
    double disc = b * b + 2.0 * dmu * (p1 - p0) * r;
    if (disc < 0.0) disc = 0.0;
    double denom = b + sqrt(disc);
    double tt = denom > 0.0 ? 2.0 * r / denom : 0.0;
    if (tt < 0.0) tt = 0.0;
    else if (tt > 1.0) tt = 1.0;
    return t->mu[lo] + tt * dmu;
}

/* _sample_cos_theta_elsepa: one xi inverted on both bracketing energy rows,
 * quantiles interpolated linearly in ln E */
double or_elsepa_cos_theta(const or_elsepa *t, int64_t start, int64_t length, double E_keV, double xi) {
    int64_t row;
    double f;
    elsepa_bracket(t, log(E_keV * 1e3), start, length, &row, &f);
    double mu0 = elsepa_invert_row(t, row, xi);
    double mu1 = elsepa_invert_row(t, row + 1, xi);
    return 1.0 - 2.0 * ((1.0 - f) * mu0 + f * mu1);
}

/* stopping.py:86-103, _dEds_sbethe_scalar: log-log interpolation of layer
 * L's table, hi the first node at or above ln E, clamped at both ends */
double or_sbethe_dEds(const or_layers *ly, int L, double E) {
    const double *lE = ly->sb_logE + (int64_t)L * ly->sb_width;
    const double *lS = ly->sb_logS + (int64_t)L * ly->sb_width;
    int n = ly->sb_count[L];
    double x = log(E);
    if (x <= lE[0]) return -exp(lS[0]);
    if (x >= lE[n - 1]) return -exp(lS[n - 1]);
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        int mid = (lo + hi) / 2;
        if (lE[mid] < x) lo = mid; else hi = mid;
    }
    double f = (x - lE[lo]) / (lE[hi] - lE[lo]);
    return -exp(lS[lo] + f * (lS[hi] - lS[lo]));
}

/* cores.py:581-590: the continuous stopping of layer L, SBETHE or spliced */
static double stopping(const or_layers *ly, int L, double E) {
    return ly->sb_count ? or_sbethe_dEds(ly, L, E) : or_dEds_spliced(ly, L, E);
}

/* the elastic rate of element slot ix at E: ELSEPA or screened Rutherford */
static double elastic_rate(const or_layers *ly, int ix, double E) {
    if (ly->elsepa) return or_elsepa_rate(ly->elsepa, ly->elsepa->start[ix], ly->elsepa->length[ix], E);
    return or_sr_rate(E, ly->sr_rate_numer[ix], ly->sr_joy_numer[ix]);
}

/* core_geometry.py:16-35, _rotate_direction_scalar */
void or_rotate(double *dx, double *dy, double *dz, double cos_t, double phi) {
    double st2 = 1.0 - cos_t * cos_t;
    double sin_t = sqrt(st2 > 0.0 ? st2 : 0.0);
    double cp = cos(phi), sp = sin(phi);
    double refx, refy;
    if (fabs(*dx) < 0.9) { refx = 1.0; refy = 0.0; } else { refx = 0.0; refy = 1.0; }
    double ux = -(*dz) * refy, uy = (*dz) * refx, uz = (*dx) * refy - (*dy) * refx;
    double um = sqrt(ux * ux + uy * uy + uz * uz);
    ux /= um; uy /= um; uz /= um;
    double wx = (*dy) * uz - (*dz) * uy, wy = (*dz) * ux - (*dx) * uz, wz = (*dx) * uy - (*dy) * ux;
    double a = sin_t * cp, b = sin_t * sp;
    double ox = cos_t * (*dx) + a * ux + b * wx;
    double oy = cos_t * (*dy) + a * uy + b * wy;
    double oz = cos_t * (*dz) + a * uz + b * wz;
    double m = sqrt(ox * ox + oy * oy + oz * oz);
    *dx = ox / m; *dy = oy / m; *dz = oz / m;
}

/* core_geometry.py:78-86, searchsorted(side="right") over the internal bounds */
static int layer_of(const or_layers *ly, double z) {
    int n = ly->n_layers - 1, lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) / 2;
        if (ly->z_top[mid + 1] <= z) lo = mid + 1; else hi = mid;
    }
    return lo;
}

/* ---- the per-electron event loop ----------------------------------------
 * cores.py:379-1230 with per_electron=True, lut=False, grooved=False,
 * inelastic=False, radiative=False, mixed=False, cone_split=False,
 * elastic_model_code=0 (SR) or 2 (ELSEPA, ly->elsepa), energy_model_code=1 (midpoint), straggling
 * off or Urban (ly->straggling), max_dE_frac=0, infinite lateral footprint. With spliced stopping the lazy
 * cutoff bound is never armed (_jit_cutoff_bound.py:47-56), so the midpoint
 * cutoff solve always runs.
 */
void or_transport_one(const or_layers *ly, int rng_kind, uint64_t key, int64_t elec, double E_cut,
                      int64_t max_steps, int64_t cap, double *pos, double *dir, double *E_io,
                      double *clock_io, or_rows *rows, int64_t row_base, int64_t *seg_count,
                      int8_t *exit_code) {
    double px = pos[0], py = pos[1], pz = pos[2];
    double dx = dir[0], dy = dir[1], dz = dir[2];
    double E = *E_io, clk = *clock_io;
    double tau_left = -1.0;
    uint64_t draws = 0;
    int64_t nseg = 0, flight = 0, steps = 0;
    int8_t code = OR_EXIT_STEP_LIMITED;
    const double EPS = 1e-6;
    double z_total = ly->z_bot[ly->n_layers - 1];
    while (steps < max_steps) {
        int L = ly->n_layers == 1 ? 0 : layer_of(ly, pz);
        int n_el = ly->n_el[L];
        double z_top = ly->z_top[L], z_bot = ly->z_bot[L];
        const double E_j = E;
        double total_rate = 0.0;
        for (int i = 0; i < n_el; ++i) {
            int ix = L * ly->max_el + i;
            total_rate += elastic_rate(ly, ix, E_j);
        }
        double lam = 1e8 / total_rate;
        if (tau_left < 0.0) {
            tau_left = -log(draw_uniform(rng_kind, key, draws));
            draws += 1;
        }
        double step = tau_left * lam;
        int cross_up = 0, cross_dn = 0;
        if (dz < 0.0) {
            double sb = (pz - z_top) / (-dz);
            if (step > sb) { step = sb; cross_up = 1; }
        } else if (dz > 0.0) {
            double sb = (z_bot - pz) / dz;
            if (step > sb) { step = sb; cross_dn = 1; }
        }
        int exit_top = cross_up && z_top <= 0.0;
        int exit_bot = cross_dn && z_bot >= z_total;
        double dEds = stopping(ly, L, E_j);
        int geometry_event = cross_up || cross_dn;
        int cutoff = 0;
        double E_end;
        if (ly->straggling) {
            /* cores.py:654-700: the Urban loss of the flight, element by
             * element (straggling.py:301-333), a loss beyond E - E_cut
             * shortening the step in proportion and ending at the cutoff. */
            uint64_t urban_key = or_splitmix64(key ^ URBAN_SALT);
            uint64_t fkey = or_splitmix64(urban_key + 0x9E3779B97F4A7C15ULL * ((uint64_t)flight << 32));
            uint64_t ctr = 0;
            double loss = 0.0;
            /* cores.py:595-604: with SBETHE each element's C is scaled by the
             * table's stopping over the spliced one at the row's energy */
            const double scale = ly->sb_count ? dEds / or_dEds_spliced(ly, L, E_j) : 1.0;
            for (int i = 0; i < n_el; ++i) {
                int ix = L * ly->max_el + i;
                double C = -or_dEds_element(ly->J[ix], ly->k[ix], ly->coeff[ix], ly->E_cross[ix], E_j);
                C *= scale;
                loss += or_urban_sample_element(ly->Z[ix], ly->J[ix], C, E_j, step, fkey, &ctr);
            }
            double delta_cut = E_j - E_cut;
            if (loss > delta_cut || (loss == delta_cut && !geometry_event)) {
                step = loss > 0.0 ? step * (delta_cut / loss) : 0.0;
                cutoff = 1;
                cross_up = cross_dn = exit_top = exit_bot = 0;
                E_end = E_cut;
            } else {
                E_end = E_j - loss;
            }
        } else {
            /* cores.py:734-776: midpoint cutoff distance */
            double cutoff_rate = stopping(ly, L, 0.5 * (E_j + E_cut));
            double cutoff_distance = (E_cut - E_j) / cutoff_rate;
            if (cutoff_distance < step || (cutoff_distance == step && !geometry_event)) {
                step = cutoff_distance;
                cutoff = 1;
                cross_up = cross_dn = exit_top = exit_bot = 0;
            }
            /* cores.py:783-809: midpoint (RK2) end energy and clock */
            if (cutoff) {
                E_end = E_cut;
            } else {
                double E_pred = E_j + dEds * step;
                double E_mid = 0.5 * (E_j + E_pred);
                E_end = E_j + step * stopping(ly, L, E_mid);
            }
        }
        double t_end = clk + step / or_beta_from_keV(0.5 * (E_j + E_end));
        int8_t event;
        if (cutoff) event = OR_EVENT_CUTOFF;
        else if (exit_top) event = OR_EVENT_EXIT_TOP;
        else if (exit_bot) event = OR_EVENT_EXIT_BOTTOM;
        else if (cross_up || cross_dn) event = OR_EVENT_LAYER_BOUNDARY;
        else event = OR_EVENT_ELASTIC;
        /* cores.py:911-935: row written to slot i*cap + s while it fits */
        if (rows && nseg < cap) {
            int64_t s = row_base + nseg;
            rows->v_hat[3 * s + 0] = dx; rows->v_hat[3 * s + 1] = dy; rows->v_hat[3 * s + 2] = dz;
            rows->r_mid[3 * s + 0] = px + 0.5 * step * dx;
            rows->r_mid[3 * s + 1] = py + 0.5 * step * dy;
            rows->r_mid[3 * s + 2] = pz + 0.5 * step * dz;
            rows->L[s] = step;
            rows->E_start[s] = E_j;
            rows->E_end[s] = E_end;
            rows->t_start[s] = clk;
            rows->t_end[s] = t_end;
            rows->elec_id[s] = elec;
            rows->layer[s] = (int16_t)L;
            rows->flight[s] = flight;
            rows->event[s] = event;
        }
        nseg += 1;
        px = px + step * dx; py = py + step * dy; pz = pz + step * dz;
        E = E_end;
        clk = t_end;
        tau_left -= step / lam;
        if (tau_left < 0.0) tau_left = 0.0;
        /* cores.py:1060-1066: every row closes the flight and resets tau */
        flight += 1;
        tau_left = -1.0;
        if (exit_top || exit_bot || cutoff) {
            code = exit_top ? OR_EXIT_BACKSCATTERED : exit_bot ? OR_EXIT_TRANSMITTED : OR_EXIT_CUTOFF;
            break;
        }
        if (cross_up || cross_dn) {
            pz += (dz > 0.0 ? 1.0 : -1.0) * EPS;
            steps += 1;
            continue;
        }
        /* cores.py:1082-1141: element by partial rate at the row-start energy,
         * SR screening at the post-step energy, then two angle draws. */
        int i_el = 0;
        if (n_el > 1) {
            double u = draw_uniform(rng_kind, key, draws) * total_rate;
            draws += 1;
            double cum = 0.0;
            i_el = n_el - 1;
            for (int k = 0; k < n_el; ++k) {
                int ix = L * ly->max_el + k;
                cum += elastic_rate(ly, ix, E_j);
                if (cum > u) { i_el = k; break; }
            }
        }
        const int ix_el = L * ly->max_el + i_el;
        double cos_u = draw_uniform(rng_kind, key, draws);
        draws += 1;
        double phi_u = draw_uniform(rng_kind, key, draws);
        draws += 1;
        /* cores.py:1158-1188: ELSEPA tables at the post-step energy, else SR */
        double cos_t = ly->elsepa ? or_elsepa_cos_theta(ly->elsepa, ly->elsepa->start[ix_el],
                                                        ly->elsepa->length[ix_el], E, cos_u)
                                  : or_cos_theta_sr(ly->sr_joy_numer[ix_el] / E, cos_u);
        or_rotate(&dx, &dy, &dz, cos_t, 2.0 * M_PI * phi_u);
        steps += 1;
    }
    pos[0] = px; pos[1] = py; pos[2] = pz;
    dir[0] = dx; dir[1] = dy; dir[2] = dz;
    *E_io = E;
    *clock_io = clk;
    *seg_count = nseg;
    *exit_code = code;
}

void or_transport(const or_layers *ly, int rng_kind, uint64_t seed, int64_t e_start, int64_t n,
                  double E_cut, int64_t max_steps, int64_t cap, double *pos, double *dir, double *E,
                  double *clock, or_rows *rows, int64_t *seg_count, int8_t *exit_code, int n_threads) {
#pragma omp parallel for schedule(dynamic, 16) num_threads(n_threads > 0 ? n_threads : 1)
    for (int64_t i = 0; i < n; ++i) {
        uint64_t key = or_stream_key(seed, (uint64_t)(e_start + i));
        or_transport_one(ly, rng_kind, key, e_start + i, E_cut, max_steps, cap, pos + 3 * i,
                         dir + 3 * i, E + i, clock + i, rows, i * cap, seg_count + i, exit_code + i);
    }
}

/* ---- the LUT core (the reference's default exact-physics path) -----------
 * cores.py:379-1230 with lut=True: one uniform-log-energy table per layer for
 * the total elastic rate, the stopping power and the element CDF / screening,
 * one shared 1/beta table (lut.py:64-283), read by the closed-form index of
 * lut.py:118-137 and linear interpolation.
 */
static void lut_index(const or_lut *t, double E, int *i, double *f) {
    double x = (log(E) - t->log_E_min) * t->inv_dlogE;
    int last = t->n_energy - 1;
    if (x >= last) { *i = last - 1; *f = 1.0; return; }
    if (x > 0.0) { int ii = (int)x; *i = ii; *f = x - ii; return; }
    *i = 0; *f = 0.0;
}

static double lerp(const double *row, int i, double f) { return row[i] + f * (row[i + 1] - row[i]); }

void or_transport_lut_one(const or_lut *t, int rng_kind, uint64_t key, int64_t elec, double E_cut,
                          int64_t max_steps, int64_t cap, double *pos, double *dir, double *E_io,
                          double *clock_io, or_rows *rows, int64_t row_base, int64_t *seg_count,
                          int8_t *exit_code) {
    double px = pos[0], py = pos[1], pz = pos[2];
    double dx = dir[0], dy = dir[1], dz = dir[2];
    double E = *E_io, clk = *clock_io;
    double tau_left = -1.0;
    uint64_t draws = 0;
    int64_t nseg = 0, flight = 0, steps = 0;
    int8_t code = OR_EXIT_STEP_LIMITED;
    const double EPS = 1e-6;
    const int ne = t->n_energy;
    double z_total = t->z_bot[t->n_layers - 1];
    while (steps < max_steps) {
        int L = 0;
        if (t->n_layers > 1) {
            int n = t->n_layers - 1, lo = 0, hi = n;
            while (lo < hi) {
                int mid = (lo + hi) / 2;
                if (t->z_top[mid + 1] <= pz) lo = mid + 1; else hi = mid;
            }
            L = lo;
        }
        int n_el = t->n_el[L];
        double z_top = t->z_top[L], z_bot = t->z_bot[L];
        const double E_j = E;
        const double *rate_row = t->total_rate + (int64_t)L * ne;
        const double *dEds_row = t->dEds + (int64_t)L * ne;
        int li;
        double lf;
        lut_index(t, E_j, &li, &lf);
        double total_rate = lerp(rate_row, li, lf);
        double lam = 1e8 / total_rate;
        if (tau_left < 0.0) {
            tau_left = -log(draw_uniform(rng_kind, key, draws));
            draws += 1;
        }
        double step = tau_left * lam;
        int cross_up = 0, cross_dn = 0;
        if (dz < 0.0) {
            double sb = (pz - z_top) / (-dz);
            if (step > sb) { step = sb; cross_up = 1; }
        } else if (dz > 0.0) {
            double sb = (z_bot - pz) / dz;
            if (step > sb) { step = sb; cross_dn = 1; }
        }
        int exit_top = cross_up && z_top <= 0.0;
        int exit_bot = cross_dn && z_bot >= z_total;
        double dEds = lerp(dEds_row, li, lf);
        int geometry_event = cross_up || cross_dn;
        int cutoff = 0;
        int ci;
        double cf;
        lut_index(t, 0.5 * (E_j + E_cut), &ci, &cf);
        double cutoff_distance = (E_cut - E_j) / lerp(dEds_row, ci, cf);
        if (cutoff_distance < step || (cutoff_distance == step && !geometry_event)) {
            step = cutoff_distance;
            cutoff = 1;
            cross_up = cross_dn = exit_top = exit_bot = 0;
        }
        double E_end;
        if (cutoff) {
            E_end = E_cut;
        } else {
            double E_pred = E_j + dEds * step;
            int mi;
            double mf;
            lut_index(t, 0.5 * (E_j + E_pred), &mi, &mf);
            E_end = E_j + step * lerp(dEds_row, mi, mf);
        }
        int ki;
        double kf;
        lut_index(t, 0.5 * (E_j + E_end), &ki, &kf);
        double t_end = clk + step * lerp(t->inv_beta, ki, kf);
        int8_t event;
        if (cutoff) event = OR_EVENT_CUTOFF;
        else if (exit_top) event = OR_EVENT_EXIT_TOP;
        else if (exit_bot) event = OR_EVENT_EXIT_BOTTOM;
        else if (cross_up || cross_dn) event = OR_EVENT_LAYER_BOUNDARY;
        else event = OR_EVENT_ELASTIC;
        if (rows && nseg < cap) {
            int64_t s = row_base + nseg;
            rows->v_hat[3 * s + 0] = dx; rows->v_hat[3 * s + 1] = dy; rows->v_hat[3 * s + 2] = dz;
            rows->r_mid[3 * s + 0] = px + 0.5 * step * dx;
            rows->r_mid[3 * s + 1] = py + 0.5 * step * dy;
            rows->r_mid[3 * s + 2] = pz + 0.5 * step * dz;
            rows->L[s] = step;
            rows->E_start[s] = E_j;
            rows->E_end[s] = E_end;
            rows->t_start[s] = clk;
            rows->t_end[s] = t_end;
            rows->elec_id[s] = elec;
            rows->layer[s] = (int16_t)L;
            rows->flight[s] = flight;
            rows->event[s] = event;
        }
        nseg += 1;
        px = px + step * dx; py = py + step * dy; pz = pz + step * dz;
        E = E_end;
        clk = t_end;
        flight += 1;
        tau_left = -1.0;
        if (exit_top || exit_bot || cutoff) {
            code = exit_top ? OR_EXIT_BACKSCATTERED : exit_bot ? OR_EXIT_TRANSMITTED : OR_EXIT_CUTOFF;
            break;
        }
        if (cross_up || cross_dn) {
            pz += (dz > 0.0 ? 1.0 : -1.0) * EPS;
            steps += 1;
            continue;
        }
        int i_el = 0;
        if (n_el > 1) {
            double u = draw_uniform(rng_kind, key, draws);
            draws += 1;
            i_el = n_el - 1;
            for (int k = 0; k < n_el; ++k) {
                const double *cdf = t->cdf + ((int64_t)L * t->max_el + k) * ne;
                if (lerp(cdf, li, lf) > u) { i_el = k; break; }
            }
        }
        int ai;
        double af;
        lut_index(t, E, &ai, &af);
        double alpha = lerp(t->alpha + ((int64_t)L * t->max_el + i_el) * ne, ai, af);
        double cos_u = draw_uniform(rng_kind, key, draws);
        draws += 1;
        double phi_u = draw_uniform(rng_kind, key, draws);
        draws += 1;
        or_rotate(&dx, &dy, &dz, or_cos_theta_sr(alpha, cos_u), 2.0 * M_PI * phi_u);
        steps += 1;
    }
    pos[0] = px; pos[1] = py; pos[2] = pz;
    dir[0] = dx; dir[1] = dy; dir[2] = dz;
    *E_io = E;
    *clock_io = clk;
    *seg_count = nseg;
    *exit_code = code;
}

void or_transport_lut(const or_lut *t, int rng_kind, uint64_t seed, int64_t e_start, int64_t n,
                      double E_cut, int64_t max_steps, int64_t cap, double *pos, double *dir,
                      double *E, double *clock, or_rows *rows, int64_t *seg_count,
                      int8_t *exit_code) {
    for (int64_t i = 0; i < n; ++i) {
        uint64_t key = or_stream_key(seed, (uint64_t)(e_start + i));
        or_transport_lut_one(t, rng_kind, key, e_start + i, E_cut, max_steps, cap, pos + 3 * i,
                             dir + 3 * i, E + i, clock + i, rows, i * cap, seg_count + i,
                             exit_code + i);
    }
}
