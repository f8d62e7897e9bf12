// Persistent electron-transport kernel (sm_100a).
//
// One history per thread, structure-of-arrays state in registers, refilled
// from a global work counter: after every event the warp ballots its idle
// lanes and one lane claims that many new histories with a single atomic, so
// lanes never sit on a finished history while the rest of the warp works.
//
// Physics is the reference's per-electron core with the data-free set
// (src/pyrite/montecarlo/transport/cores.py:379-1230): screened-Rutherford
// elastic scattering, spliced Joy-Luo / Berger-Seltzer stopping, the
// midpoint (RK2) energy rule, layered slabs. Two forms of the energy
// dependence are compiled: the exact analytic expressions (FP64 parity with
// the reference's exact core) and the reference's default uniform-log-energy
// LUT (transport/lut.py), staged once per block into shared memory by a
// non-multicast bulk copy. The RNG is either the reference's SplitMix64
// counter stream (bit-compatible draws) or Philox4x32-10 keyed by
// (seed, history) with the draw index as counter.
//
// Precision: PB_FP64 runs everything in double. PB_MIXED runs rates,
// geometry and flight steps in float and keeps the per-history energy and
// clock bookkeeping in double.
#include <cstdint>
#include <cstdio>

#include "pb_common.cuh"
#include "pb_internal.h"

namespace pb {

constexpr int kMaxLayers = 8;
constexpr int kMaxEl = 8;
constexpr double kEps = 1e-6;

enum : int8_t {
    EV_ELASTIC = 0,
    EV_LAYER_BOUNDARY = 2,
    EV_EXIT_TOP = 4,
    EV_EXIT_BOTTOM = 5,
    EV_CUTOFF = 7
};
enum : int8_t {
    EXIT_CUTOFF = 0,
    EXIT_BACK = 1,
    EXIT_TRANS = 2,
    EXIT_SIDE = 3,
    EXIT_STEP = 4,
    EXIT_NOT_ENTERED = 5
};

// Layer geometry and exact-physics coefficients, copied to shared memory.
struct LayerSmem {
    double z_top[kMaxLayers];
    double z_bot[kMaxLayers];
    int n_el[kMaxLayers];
    double J[kMaxLayers * kMaxEl];
    double k[kMaxLayers * kMaxEl];
    double coeff[kMaxLayers * kMaxEl];
    double E_cross[kMaxLayers * kMaxEl];
    double srn[kMaxLayers * kMaxEl];
    double sjn[kMaxLayers * kMaxEl];
    double Z[kMaxLayers * kMaxEl];  // atomic numbers (straggling only)
};

// Math in the precision of the flight arithmetic.
__device__ __forceinline__ double m_log(double x) { return log(x); }
__device__ __forceinline__ float m_log(float x) { return logf(x); }
__device__ __forceinline__ double m_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float m_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double m_sin(double x) { return sin(x); }
__device__ __forceinline__ float m_sin(float x) { return sinf(x); }
__device__ __forceinline__ double m_cos(double x) { return cos(x); }
__device__ __forceinline__ float m_cos(float x) { return cosf(x); }

// stopping.py:384-410 (_dEds_spliced_packed_scalar), density effect 0.
template <class Real>
__device__ __forceinline__ Real dEds_spliced(const LayerSmem &ly, int max_el, int L, Real E) {
    const Real tau = E / (Real)kMc2Kev;
    const Real gamma = (Real)1 + tau;
    const Real beta_sq = (Real)1 - (Real)1 / (gamma * gamma);
    const Real f_minus = (Real)1 - beta_sq +
                         (tau * tau / (Real)8 - ((Real)2 * tau + (Real)1) * (Real)kLn2) / (gamma * gamma);
    Real jl = 0, bs = 0;
    const int n = ly.n_el[L];
    for (int i = 0; i < n; ++i) {
        const int ix = L * max_el + i;
        const Real J = (Real)ly.J[ix], coeff = (Real)ly.coeff[ix];
        if (E < (Real)ly.E_cross[ix]) {
            jl += coeff * m_log((Real)1.166 * (E + (Real)ly.k[ix] * J) / J);
        } else {
            const Real I_rel = J / (Real)kMc2Kev;
            bs += coeff * (m_log(tau * tau * (tau + (Real)2) / ((Real)2 * I_rel * I_rel)) + f_minus - (Real)0);
        }
    }
    return -(Real)7.85e-4 / E * jl - (Real)kBsPrefactor / beta_sq * bs;
}

// ---------------------------------------------------------------------------
// Urban energy-loss straggling (transport/straggling.py), FP64 in both
// precisions. A flight's loss is the compound Poisson sum of two excitation
// levels and a 1/E^2 ionisation continuum, per element of the layer, whose
// mean is the element's |dE/dx| times the path (the model's closure
// identity). Each flight draws from its own counter stream keyed by the
// history's key and the flight index (straggling.py:37-59), so the flight's
// draw count never moves the elastic draws.
// ---------------------------------------------------------------------------
constexpr uint64_t kUrbanSalt = 0xD6E8FEB86659FD93ULL;
constexpr double kUrbanE0 = 1.0e-2;         // ionisation threshold [keV]
constexpr double kUrbanE2PerZ2 = 1.0e-2;    // K-shell level 10 Z^2 eV [keV]
constexpr double kUrbanRate = 0.55;         // continuum share of the mean
constexpr double kUrbanChunkMax = 64.0;     // Poisson means split into chunks <= this

// straggling.py:278-298: one element's spliced stopping power (delta = 0).
__device__ __forceinline__ double dEds_element(double J, double k, double coeff, double E_cross, double E) {
    const double tau = E / kMc2Kev;
    const double gamma = 1.0 + tau;
    const double beta_sq = 1.0 - 1.0 / (gamma * gamma);
    if (E < E_cross) return -7.85e-4 / E * coeff * log(1.166 * (E + k * J) / J);
    const double f_minus = 1.0 - beta_sq + (tau * tau / 8.0 - (2.0 * tau + 1.0) * kLn2) / (gamma * gamma);
    const double I_rel = J / kMc2Kev;
    return -kBsPrefactor / beta_sq * coeff * (log(tau * tau * (tau + 2.0) / (2.0 * I_rel * I_rel)) + f_minus - 0.0);
}

// straggling.py:225-262: Poisson count of mean lam, one uniform per chunk.
template <int kRng>
__device__ __forceinline__ int64_t urban_poisson(double lam, uint64_t key, uint64_t &ctr) {
    if (lam <= 0.0) return 0;
    const int64_t n_chunks = (int64_t)ceil(lam / kUrbanChunkMax);
    const double chunk = lam / (double)n_chunks;
    int64_t total = 0;
    for (int64_t c = 0; c < n_chunks; ++c) {
        const double u = uniform<kRng>(key, ctr);
        ctr += 1;
        double pk = exp(-chunk);
        double cdf = pk;
        int64_t k = 0;
        while (u >= cdf) {  // ends: cdf grows to 1 or stops growing
            k += 1;
            pk = pk * chunk / (double)k;
            const double next = cdf + pk;
            if (next <= cdf) break;
            cdf = next;
        }
        total += k;
    }
    return total;
}

// straggling.py:127-201,277-298: one element's sampled loss over s [keV].
template <int kRng>
__device__ __forceinline__ double urban_sample_element(double Z, double J, double C, double E, double s,
                                                      uint64_t key, uint64_t &ctr) {
    const double tau = E / kMc2Kev;
    const double gamma = 1.0 + tau;
    const double beta_sq = 1.0 - 1.0 / (gamma * gamma);
    const double two_mc2_bg2 = 2.0 * kMc2Kev * tau * (tau + 2.0);
    const double T_up = 0.5 * E;
    if (T_up <= kUrbanE0 || C <= 0.0 || s <= 0.0) return C * s;
    const double L_I = log(two_mc2_bg2 / J) - beta_sq;
    if (L_I <= 0.0) return C * s;
    // Levels (straggling.py:127-157): K shell 10 Z^2 eV with f_2 = 2/Z and the
    // loosely bound level from the log sum rule, else one level at I.
    double f1 = 1.0, E1 = J, f2 = 0.0;
    const double E2 = kUrbanE2PerZ2 * Z * Z;
    const double g2 = Z > 2.0 ? 2.0 / Z : 1.0;
    if (Z > 2.0 && E2 < T_up && log(two_mc2_bg2 / E2) - beta_sq > 0.0) {
        const double g1 = 1.0 - g2;
        const double e1 = exp((log(J) - g2 * log(E2)) / g1);
        if (log(two_mc2_bg2 / e1) - beta_sq > 0.0) {
            f1 = g1;
            E1 = e1;
            f2 = g2;
        }
    }
    const double soft = C * (1.0 - kUrbanRate) / L_I;
    const double s1 = soft * (f1 / E1) * (log(two_mc2_bg2 / E1) - beta_sq);
    const double s2 = f2 > 0.0 ? soft * (f2 / E2) * (log(two_mc2_bg2 / E2) - beta_sq) : 0.0;
    const double s3 = C * kUrbanRate * (T_up - kUrbanE0) / (kUrbanE0 * T_up * log(T_up / kUrbanE0));
    const int64_t n1 = urban_poisson<kRng>(s1 * s, key, ctr);
    const int64_t n2 = urban_poisson<kRng>(s2 * s, key, ctr);
    const int64_t n3 = urban_poisson<kRng>(s3 * s, key, ctr);
    double dE = (double)n1 * E1 + (double)n2 * E2;
    for (int64_t i = 0; i < n3; ++i) {  // inverse CDF of the continuum (straggling.py:265-274)
        const double u = uniform<kRng>(key, ctr);
        ctr += 1;
        dE += kUrbanE0 / (1.0 - u * (T_up - kUrbanE0) / T_up);
    }
    return dE;
}

// The Urban loss of one flight of length s at energy E over the n elements
// of layer L (straggling.py:301-333), from the flight's own stream (key: the
// history's key, flight: its row index). The kernel instances with
// straggling off carry none of it.
template <int kRng>
__device__ __forceinline__ double straggled_loss(const LayerSmem &ly, int max_el, int L, int n_el, double E,
                                              double s, uint64_t key, int64_t flight, double scale = 1.0) {
    const uint64_t fkey = splitmix64(splitmix64(key ^ kUrbanSalt) + kPhi * ((uint64_t)flight << 32));
    uint64_t ctr = 0;
    double loss = 0.0;
    for (int k = 0; k < n_el; ++k) {
        const int ix = L * max_el + k;
        double C = -dEds_element(ly.J[ix], ly.k[ix], ly.coeff[ix], ly.E_cross[ix], E);
        C *= scale;
        loss += urban_sample_element<kRng>(ly.Z[ix], ly.J[ix], C, E, s, fkey, ctr);
    }
    return loss;
}

// scattering.py:208-218
template <class Real>
__device__ __forceinline__ Real sr_rate(Real E, Real srn, Real sjn) {
    const Real a = sjn / E;
    const Real r = (E + (Real)511) / (E + (Real)1024);
    return srn / (E * E) / (a * ((Real)1 + a)) * (r * r);
}

// ---- ELSEPA tabulated elastic scattering (scattering.py:516-640) ----------
// The tables stay in global memory: a case's rows (tens of energies x a few
// hundred mu nodes per element) are L2-resident, and one event reads two
// short guide windows and four table entries, so staging them would cost
// more shared memory than the reads it saves. FP64 throughout: the exact
// core replays the reference's draws.

// _elsepa_bracket: energy row and fraction of lnE within one slot, clamped.
__device__ __forceinline__ int64_t elsepa_bracket(const pb_elsepa &t, double lnE, int64_t start, int64_t len,
                                                  double &f) {
    const int64_t first = start, last = start + len - 1;
    if (lnE <= t.logE[first]) { f = 0.0; return first; }
    if (lnE >= t.logE[last]) { f = 1.0; return last - 1; }
    int64_t lo = first, hi = last;
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (t.logE[mid] <= lnE) lo = mid;
        else hi = mid;
    }
    f = (lnE - t.logE[lo]) / (t.logE[hi] - t.logE[lo]);
    return lo;
}

// _elsepa_rate_scalar: n sigma [1/cm] of one element, log-log in energy.
__device__ __forceinline__ double elsepa_rate(const pb_elsepa &t, int ix, double E_keV) {
    double f;
    const int64_t r = elsepa_bracket(t, log(E_keV * 1e3), t.start[ix], t.length[ix], f);
    return exp(t.log_rate[r] + f * (t.log_rate[r + 1] - t.log_rate[r]));
}

// _elsepa_panel + _elsepa_invert_row: the panel k whose CDF bracket holds
// xi, found by bisection inside the guide window of xi's cell, then the
// linear-density panel's quadratic CDF solved in its cancellation-free form.
__device__ __forceinline__ double elsepa_invert(const pb_elsepa &t, int64_t row, double xi) {
    const int cells = t.cells;
    const double scaled = xi * (double)cells;
    const int cell = scaled >= (double)cells ? cells - 1 : scaled > 0.0 ? (int)scaled : 0;
    const int32_t *g = t.guide + row * (int64_t)(cells + 1);
    const double *cdf = t.cdf + row * (int64_t)t.n_mu;
    int64_t lo = g[cell], hi = (int64_t)g[cell + 1] + 1;
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (cdf[mid] <= xi) lo = mid;
        else hi = mid;
    }
    const double *pdf = t.pdf + row * (int64_t)t.n_mu;
    const double dmu = t.mu[lo + 1] - t.mu[lo];
    const double p0 = pdf[lo], p1 = pdf[lo + 1];
    const double r = xi - cdf[lo];
    const double b = dmu * p0;
    double disc = b * b + 2.0 * dmu * (p1 - p0) * r;
    if (disc < 0.0) disc = 0.0;
    const double denom = b + sqrt(disc);
    double u = denom > 0.0 ? 2.0 * r / denom : 0.0;
    u = u < 0.0 ? 0.0 : (u > 1.0 ? 1.0 : u);
    return t.mu[lo] + u * dmu;
}

// _sample_cos_theta_elsepa: one uniform on both bracketing energy rows, the
// quantiles interpolated linearly in ln E.
__device__ __forceinline__ double elsepa_cos_theta(const pb_elsepa &t, int ix, double E_keV, double xi) {
    double f;
    const int64_t r = elsepa_bracket(t, log(E_keV * 1e3), t.start[ix], t.length[ix], f);
    const double mu0 = elsepa_invert(t, r, xi);
    const double mu1 = elsepa_invert(t, r + 1, xi);
    return 1.0 - 2.0 * ((1.0 - f) * mu0 + f * mu1);
}

// ---- SBETHE table stopping (stopping.py:86-103) -----------------------------
// Layer L's log-log table; hi is the first node at or above ln E (numpy's
// searchsorted on the left), both ends clamped. FP64, negative.
__device__ __forceinline__ double sbethe_dEds(const pb_stopping &t, int L, double E) {
    const double *lE = t.logE + (int64_t)L * t.width;
    const double *lS = t.logS + (int64_t)L * t.width;
    const int n = t.count[L];
    const double x = log(E);
    if (x <= lE[0]) return -exp(lS[0]);
    if (x >= lE[n - 1]) return -exp(lS[n - 1]);
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (lE[mid] < x) lo = mid;
        else hi = mid;
    }
    const double f = (x - lE[lo]) / (lE[hi] - lE[lo]);
    return -exp(lS[lo] + f * (lS[hi] - lS[lo]));
}

// kinematics.py:162-166
template <class Real>
__device__ __forceinline__ Real beta_from_keV(Real E) {
    const Real g = (Real)1 + E / (Real)kMc2Kev;
    const Real gis = (Real)1 / (g * g);
    return m_sqrt((Real)1 - gis);
}

// core_geometry.py:16-35
template <class Real>
__device__ __forceinline__ void rotate(Real &dx, Real &dy, Real &dz, Real cos_t, Real phi) {
    const Real st2 = (Real)1 - cos_t * cos_t;
    const Real sin_t = m_sqrt(st2 > (Real)0 ? st2 : (Real)0);
    const Real cp = m_cos(phi), sp = m_sin(phi);
    Real refx, refy;
    if (fabs(dx) < (Real)0.9) { refx = 1; refy = 0; } else { refx = 0; refy = 1; }
    Real ux = -dz * refy, uy = dz * refx, uz = dx * refy - dy * refx;
    const Real um = m_sqrt(ux * ux + uy * uy + uz * uz);
    ux /= um; uy /= um; uz /= um;
    const Real wx = dy * uz - dz * uy, wy = dz * ux - dx * uz, wz = dx * uy - dy * ux;
    const Real a = sin_t * cp, b = sin_t * sp;
    const Real ox = cos_t * dx + a * ux + b * wx;
    const Real oy = cos_t * dy + a * uy + b * wy;
    const Real oz = cos_t * dz + a * uz + b * wz;
    const Real m = m_sqrt(ox * ox + oy * oy + oz * oz);
    dx = ox / m; dy = oy / m; dz = oz / m;
}

// LUT view (shared or global memory) in the flight precision.
template <class Real>
struct LutView {
    const Real *rate;
    const Real *dEds;
    const Real *inv_beta;
    const Real *cdf;
    const Real *alpha;
    int ne;
    double log_E_min;
    double inv_dlogE;
};

// lut.py:118-137: one log, one multiply, clamped index and fraction.
template <class Real>
__device__ __forceinline__ void lut_index(const LutView<Real> &t, double E, int &i, Real &f) {
    Real x;
    if constexpr (sizeof(Real) == 8) x = (log(E) - t.log_E_min) * t.inv_dlogE;
    else x = (logf((float)E) - (float)t.log_E_min) * (float)t.inv_dlogE;
    const int last = t.ne - 1;
    if (x >= (Real)last) { i = last - 1; f = 1; return; }
    if (x > (Real)0) { const int ii = (int)x; i = ii; f = x - (Real)ii; return; }
    i = 0;
    f = 0;
}

template <class Real>
__device__ __forceinline__ Real lerp(const Real *row, int i, Real f) {
    return row[i] + f * (row[i + 1] - row[i]);
}

// Normal quantile of an open uniform (the reference uses scipy ndtri,
// kinematics.py:302-311; normcdfinv is CUDA's inverse normal CDF).
__device__ __forceinline__ double normal_from(double u) { return normcdfinv(u); }

// Entrance state of history ``e`` (global index) at local index ``i``.
template <int kRng>
__device__ void sample_entry(const pb_transport_args &p, int64_t i, int64_t e, double pos[3],
                             double dir[3], double &E) {
    const pb_beam &b = p.beam;
    if (b.mode == PB_BEAM_EXPLICIT) {
        pos[0] = b.pos0[3 * i]; pos[1] = b.pos0[3 * i + 1]; pos[2] = b.pos0[3 * i + 2];
        dir[0] = b.dir0[3 * i]; dir[1] = b.dir0[3 * i + 1]; dir[2] = b.dir0[3 * i + 2];
        E = b.E0[i];
        return;
    }
    // Counter-addressed normals of the entry namespace (kinematics.py:270-311).
    const uint64_t key = stream_key(b.root, (uint64_t)e);
    double z[4];
    const int nz = b.mode == PB_BEAM_TWISS ? 4 : 2;
    for (int c = 0; c < nz; ++c) {
        double u;
        if constexpr (kRng == PB_RNG_PHILOX) {
            // 52-bit open uniform built from one Philox draw.
            const double w = philox_uniform(key, (uint64_t)c);
            u = (floor(w * 4503599627370496.0) + 0.5) * (1.0 / 4503599627370496.0);
        } else {
            u = splitmix_open_uniform(key, (uint64_t)c);
        }
        z[c] = normal_from(u);
    }
    double u_off, v_off, xp = 0.0, yp = 0.0;
    if (b.mode == PB_BEAM_TWISS) {
        // transverse.py:177-186 with eps [mm rad], beta [mm/rad]
        const double ex = b.twiss_x[0], bx = b.twiss_x[1], ax = b.twiss_x[2];
        const double ey = b.twiss_y[0], by = b.twiss_y[1], ay = b.twiss_y[2];
        const double x_mm = sqrt(ex * bx) * z[0];
        xp = sqrt(ex / bx) * (z[1] - ax * z[0]);
        const double y_mm = sqrt(ey * by) * z[2];
        yp = sqrt(ey / by) * (z[3] - ay * z[2]);
        u_off = x_mm * 1.0e7;
        v_off = y_mm * 1.0e7;
    } else {
        u_off = z[0] * b.sigma_x_ang;
        v_off = z[1] * b.sigma_y_ang;
    }
    // geometry.py:374-390 (_project_entry_rows)
    if (b.tilted) {
        const double s_star = -(u_off * b.e_x[2] + v_off * b.e_y[2]) / b.beam_dir[2];
        pos[0] = (u_off * b.e_x[0] + v_off * b.e_y[0]) + s_star * b.beam_dir[0];
        pos[1] = (u_off * b.e_x[1] + v_off * b.e_y[1]) + s_star * b.beam_dir[1];
    } else {
        pos[0] = u_off;
        pos[1] = v_off;
    }
    pos[2] = 0.0;
    if (b.mode == PB_BEAM_TWISS) {
        // beam_entry.py:347-359: (x', y', 1) in the beam frame, normalised
        double d[3];
        for (int c = 0; c < 3; ++c)
            d[c] = (xp * b.basis[3 * c + 0] + yp * b.basis[3 * c + 1]) + b.beam_dir[c];
        const double nrm = sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]);
        dir[0] = d[0] / nrm; dir[1] = d[1] / nrm; dir[2] = d[2] / nrm;
    } else {
        dir[0] = b.beam_dir[0]; dir[1] = b.beam_dir[1]; dir[2] = b.beam_dir[2];
    }
    E = b.E0_keV;
}

struct TallySmem {
    unsigned long long fates[6];
    unsigned long long exit_E[258];
    unsigned long long exit_theta[258];
    double deposit[kMaxLayers];
};

__device__ __forceinline__ int hist_slot(double v, double lo, double hi, int n) {
    if (!(v >= lo)) return 0;  // underflow (NaN counts as underflow)
    if (v > hi) return n + 1;
    int b = (int)((v - lo) / (hi - lo) * n);
    if (b >= n) b = n - 1;
    return b + 1;
}

// kTab: the exact core with the table-driven physics switched on at run time
// (ELSEPA elastic rates and angles, SBETHE stopping); kLut is false with it.
// The analytic exact core and the LUT core compile without those branches.
template <class Real, bool kLut, int kRng, bool kStrag, bool kTab>
__global__ void __launch_bounds__(256) transport_kernel(const pb_transport_args p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ LayerSmem ly;
    __shared__ TallySmem tal;
    __shared__ __align__(8) uint64_t mbar;
    __shared__ int lut_in_smem;

    const int tid = threadIdx.x;
    const int n_layers = p.layers.n_layers;
    const int max_el = p.layers.max_el;
    for (int j = tid; j < n_layers; j += blockDim.x) {
        ly.z_top[j] = p.layers.z_top[j];
        ly.z_bot[j] = p.layers.z_bot[j];
        ly.n_el[j] = p.layers.n_el[j];
    }
    for (int j = tid; j < n_layers * max_el; j += blockDim.x) {
        ly.J[j] = p.layers.J[j];
        ly.k[j] = p.layers.k[j];
        ly.coeff[j] = p.layers.coeff[j];
        ly.E_cross[j] = p.layers.E_cross[j];
        ly.srn[j] = p.layers.sr_rate_numer[j];
        ly.sjn[j] = p.layers.sr_joy_numer[j];
        ly.Z[j] = p.straggling ? p.Z[j] : 0.0;
    }
    for (int j = tid; j < 6; j += blockDim.x) tal.fates[j] = 0;
    const bool want_E = p.tallies.exit_E != nullptr && p.tallies.n_E <= 256;
    const bool want_th = p.tallies.exit_theta != nullptr && p.tallies.n_theta <= 256;
    for (int j = tid; j < 258; j += blockDim.x) { tal.exit_E[j] = 0; tal.exit_theta[j] = 0; }
    for (int j = tid; j < kMaxLayers; j += blockDim.x) tal.deposit[j] = 0.0;

    // Stage the LUT into shared memory with one bulk copy per 64 KiB chunk.
    LutView<Real> lut{};
    if constexpr (kLut) {
        const Real *base = reinterpret_cast<const Real *>(p.lut.base);
        const uint32_t bytes = (uint32_t)p.lut.total_bytes;
        const bool fits = p.lut.total_bytes <= (int64_t)kLutSmemBytes;
        if (tid == 0) {
            lut_in_smem = 0;
            if (fits) {
                mbar_init(&mbar, 1);
                mbar_expect_tx(&mbar, bytes);
                for (uint32_t off = 0; off < bytes; off += 65536u) {
                    const uint32_t chunk = bytes - off < 65536u ? bytes - off : 65536u;
                    bulk_g2s(smem_raw + off, reinterpret_cast<const unsigned char *>(base) + off,
                             chunk, &mbar);
                }
                if (mbar_wait(&mbar, 0)) {
                    lut_in_smem = 1;
                } else {
                    set_status(p.status, PB_DEV_WAIT_TIMEOUT);
                }
            }
        }
        __syncthreads();
        const Real *src = lut_in_smem ? reinterpret_cast<const Real *>(smem_raw) : base;
        lut.rate = src + p.lut.off_total_rate;
        lut.dEds = src + p.lut.off_dEds;
        lut.inv_beta = src + p.lut.off_inv_beta;
        lut.cdf = src + p.lut.off_cdf;
        lut.alpha = src + p.lut.off_alpha;
        lut.ne = p.lut.n_energy;
        lut.log_E_min = p.lut.log_E_min;
        lut.inv_dlogE = p.lut.inv_dlogE;
    }
    __syncthreads();

    const unsigned lane = tid & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;
    const double E_cut = p.E_cut_keV;
    const double z_total = ly.z_bot[n_layers - 1];
    const bool want_rows = p.rows.L != nullptr;
    const bool want_seg = p.seg.L != nullptr;
    double dep_acc[kMaxLayers];
#pragma unroll
    for (int j = 0; j < kMaxLayers; ++j) dep_acc[j] = 0.0;

    // Per-history state.
    int64_t i = -1;  // local history index; -1 idle, -2 drained
    uint64_t key = 0, draws = 0;
    // Positions stay FP64 in both precisions: deep in a thick stack (z ~ 1e7
    // Angstrom) a float position cannot resolve the boundary nudge or an
    // Angstrom-scale step, and a particle leaving a layer upward would sit on
    // the boundary for ever. Flight lengths and physics follow Real.
    double px = 0, py = 0, pz = 0;
    Real dx = 0, dy = 0, dz = 1;
    double E = 0.0, clk = 0.0;
    int64_t nseg = 0, steps = 0;
    Real tau_left = -1;

    while (true) {
        const bool idle = (i == -1);
        const unsigned idle_mask = __ballot_sync(0xffffffffu, idle);
        if (idle_mask) {
            const int leader = __ffs(idle_mask) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) base = atomicAdd(p.work_counter, (unsigned long long)__popc(idle_mask));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (idle) {
                const unsigned long long mine = base + __popc(idle_mask & lt_mask);
                if (mine < (unsigned long long)p.n) {
                    i = (int64_t)mine;
                    const int64_t e = p.e_start + i;
                    double pos[3], dir[3], E0;
                    sample_entry<kRng>(p, i, e, pos, dir, E0);
                    px = pos[0]; py = pos[1]; pz = pos[2];
                    dx = (Real)dir[0]; dy = (Real)dir[1]; dz = (Real)dir[2];
                    E = E0;
                    clk = 0.0;
                    key = stream_key(p.seed, (uint64_t)e);
                    draws = 0;
                    nseg = 0;
                    steps = 0;
                    tau_left = -1;
                } else {
                    i = -2;
                }
            }
        }
        if (__ballot_sync(0xffffffffu, i >= 0) == 0u) break;
        if (i < 0) continue;

        // ---- one event (cores.py:402-1230) ----
        int8_t code = -1;
        if (steps >= p.max_steps) {
            code = EXIT_STEP;
            set_status(p.status, PB_DEV_STEP_LIMIT);
        } else {
            int L = 0;
            if (n_layers > 1) {
                // searchsorted(internal_bounds, z, side="right")
                for (int j = 1; j < n_layers; ++j) L += (ly.z_top[j] <= pz) ? 1 : 0;
            }
            const double z_top = ly.z_top[L], z_bot = ly.z_bot[L];
            const int n_el = ly.n_el[L];
            const double E_j = E;
            const Real Er = (Real)E_j;
            int li = 0;
            Real lf = 0;
            Real total_rate = 0;
            if constexpr (kLut) {
                lut_index(lut, E_j, li, lf);
                total_rate = lerp(lut.rate + (int64_t)L * lut.ne, li, lf);
            } else {
                for (int k = 0; k < n_el; ++k) {
                    const int ix = L * max_el + k;
                    if (kTab && p.elastic_model == PB_ELASTIC_ELSEPA) total_rate += (Real)elsepa_rate(p.elsepa, ix, E_j);
                    else total_rate += sr_rate<Real>(Er, (Real)ly.srn[ix], (Real)ly.sjn[ix]);
                }
            }
            const Real lam = (Real)1e8 / total_rate;
            if (tau_left < (Real)0) {
                tau_left = (Real)(-log(uniform<kRng>(key, draws)));
                draws += 1;
            }
            Real step = tau_left * lam;
            bool cross_up = false, cross_dn = false;
            if (dz < (Real)0) {
                const Real sb = (Real)((pz - z_top) / (double)(-dz));
                if (step > sb) { step = sb; cross_up = true; }
            } else if (dz > (Real)0) {
                const Real sb = (Real)((z_bot - pz) / (double)dz);
                if (step > sb) { step = sb; cross_dn = true; }
            }
            bool exit_top = cross_up && z_top <= 0.0;
            bool exit_bot = cross_dn && z_bot >= z_total;
            const bool geometry_event = cross_up || cross_dn;
            bool cutoff = false;
            double E_end;
            Real dEds = 0;
            if constexpr (kStrag) {
                // cores.py:654-700: the flight's Urban loss, element by element
                // (straggling.py:301-333) from the flight's own stream; a loss
                // beyond E - E_cut shortens the step in proportion and ends
                // the history at the cutoff.
                // cores.py:595-604: SBETHE scales each element's Urban mean
                // by the table's stopping over the spliced one at E_j.
                double scale = 1.0;
                if constexpr (kTab)
                    if (p.stopping.count)
                        scale = sbethe_dEds(p.stopping, L, E_j) / (double)dEds_spliced<double>(ly, max_el, L, E_j);
                const double loss = straggled_loss<kRng>(ly, max_el, L, n_el, E_j, (double)step, key, nseg, scale);
                const double delta_cut = E_j - E_cut;
                if (loss > delta_cut || (loss == delta_cut && !geometry_event)) {
                    step = loss > 0.0 ? (Real)((double)step * (delta_cut / loss)) : (Real)0;
                    cutoff = true;
                    cross_up = cross_dn = exit_top = exit_bot = false;
                    E_end = E_cut;
                } else {
                    E_end = E_j - loss;
                }
            } else {
            Real cutoff_rate;
            if constexpr (kLut) {
                const Real *row = lut.dEds + (int64_t)L * lut.ne;
                dEds = lerp(row, li, lf);
                int ci;
                Real cf;
                lut_index(lut, 0.5 * (E_j + E_cut), ci, cf);
                cutoff_rate = lerp(row, ci, cf);
            } else if (kTab && p.stopping.count) {
                dEds = (Real)sbethe_dEds(p.stopping, L, E_j);
                cutoff_rate = (Real)sbethe_dEds(p.stopping, L, 0.5 * (E_j + E_cut));
            } else {
                dEds = dEds_spliced<Real>(ly, max_el, L, Er);
                cutoff_rate = dEds_spliced<Real>(ly, max_el, L, (Real)(0.5 * (E_j + E_cut)));
            }
            const Real cutoff_distance = (Real)(E_cut - E_j) / cutoff_rate;
            if (cutoff_distance < step || (cutoff_distance == step && !geometry_event)) {
                step = cutoff_distance;
                cutoff = true;
                cross_up = cross_dn = exit_top = exit_bot = false;
            }
            if (cutoff) {
                E_end = E_cut;
            } else {
                const double E_pred = E_j + (double)(dEds * step);
                const double E_mid = 0.5 * (E_j + E_pred);
                Real mid_rate;
                if constexpr (kLut) {
                    int mi;
                    Real mf;
                    lut_index(lut, E_mid, mi, mf);
                    mid_rate = lerp(lut.dEds + (int64_t)L * lut.ne, mi, mf);
                } else if (kTab && p.stopping.count) {
                    mid_rate = (Real)sbethe_dEds(p.stopping, L, E_mid);
                } else {
                    mid_rate = dEds_spliced<Real>(ly, max_el, L, (Real)E_mid);
                }
                E_end = E_j + (double)(step * mid_rate);
            }
            }
            Real inv_beta_mid;
            if constexpr (kLut) {
                int ki;
                Real kf;
                lut_index(lut, 0.5 * (E_j + E_end), ki, kf);
                inv_beta_mid = lerp(lut.inv_beta, ki, kf);
            }
            double t_end;
            if constexpr (kLut) t_end = clk + (double)(step * inv_beta_mid);
            else t_end = clk + (double)step / (double)beta_from_keV<Real>((Real)(0.5 * (E_j + E_end)));
            int8_t event;
            if (cutoff) event = EV_CUTOFF;
            else if (exit_top) event = EV_EXIT_TOP;
            else if (exit_bot) event = EV_EXIT_BOTTOM;
            else if (cross_up || cross_dn) event = EV_LAYER_BOUNDARY;
            else event = EV_ELASTIC;
            const Real half = (Real)0.5 * step;
            if (want_rows) {
                if (nseg < p.cap) {
                    const int64_t s = i * p.cap + nseg;
                    p.rows.v_hat[3 * s] = (double)dx;
                    p.rows.v_hat[3 * s + 1] = (double)dy;
                    p.rows.v_hat[3 * s + 2] = (double)dz;
                    p.rows.r_mid[3 * s] = px + (double)(half * dx);
                    p.rows.r_mid[3 * s + 1] = py + (double)(half * dy);
                    p.rows.r_mid[3 * s + 2] = pz + (double)(half * dz);
                    p.rows.L[s] = (double)step;
                    p.rows.E_start[s] = E_j;
                    p.rows.E_end[s] = E_end;
                    p.rows.t_start[s] = clk;
                    p.rows.t_end[s] = t_end;
                    p.rows.elec_id[s] = p.e_start + i;
                    p.rows.layer[s] = (int16_t)L;
                    p.rows.flight[s] = nseg;
                    p.rows.event[s] = event;
                } else {
                    set_status(p.status, PB_DEV_ROW_OVERFLOW);
                }
            }
            if (want_seg) {
                // Warp-aggregated append to the compact segment list.
                const unsigned active = __activemask();
                const int leader = __ffs(active) - 1;
                unsigned long long base = 0;
                if ((int)lane == leader) base = atomicAdd(p.seg.count, (unsigned long long)__popc(active));
                base = __shfl_sync(active, base, leader);
                const unsigned long long slot = base + __popc(active & lt_mask);
                if (slot < (unsigned long long)p.seg.capacity) {
                    p.seg.v_hat[3 * slot] = (double)dx;
                    p.seg.v_hat[3 * slot + 1] = (double)dy;
                    p.seg.v_hat[3 * slot + 2] = (double)dz;
                    p.seg.r_mid[3 * slot] = px + (double)(half * dx);
                    p.seg.r_mid[3 * slot + 1] = py + (double)(half * dy);
                    p.seg.r_mid[3 * slot + 2] = pz + (double)(half * dz);
                    p.seg.L[slot] = (double)step;
                    p.seg.E_repr[slot] = 0.5 * (E_j + E_end);
                    p.seg.elec_id[slot] = p.e_start + i;
                    p.seg.layer[slot] = L;
                } else {
                    set_status(p.status, PB_DEV_QUEUE_OVERFLOW);
                }
            }
#pragma unroll
            for (int j = 0; j < kMaxLayers; ++j)
                if (j == L) dep_acc[j] += E_j - E_end;
            nseg += 1;
            px = px + (double)(step * dx);
            py = py + (double)(step * dy);
            pz = pz + (double)(step * dz);
            E = E_end;
            clk = t_end;
            tau_left = (Real)-1;
            if (exit_top || exit_bot || cutoff) {
                code = exit_top ? EXIT_BACK : exit_bot ? EXIT_TRANS : EXIT_CUTOFF;
            } else if (cross_up || cross_dn) {
                pz += (dz > (Real)0 ? 1.0 : -1.0) * kEps;
                steps += 1;
            } else {
                int i_el = 0;
                if (n_el > 1) {
                    const double u = uniform<kRng>(key, draws);
                    draws += 1;
                    i_el = n_el - 1;
                    if constexpr (kLut) {
                        for (int k = 0; k < n_el; ++k) {
                            const Real *cdf = lut.cdf + ((int64_t)L * max_el + k) * lut.ne;
                            if ((double)lerp(cdf, li, lf) > u) { i_el = k; break; }
                        }
                    } else {
                        const Real target = (Real)u * total_rate;
                        Real cum = 0;
                        for (int k = 0; k < n_el; ++k) {
                            const int ix = L * max_el + k;
                            if (kTab && p.elastic_model == PB_ELASTIC_ELSEPA) cum += (Real)elsepa_rate(p.elsepa, ix, E_j);
                            else cum += sr_rate<Real>(Er, (Real)ly.srn[ix], (Real)ly.sjn[ix]);
                            if (cum > target) { i_el = k; break; }
                        }
                    }
                }
                Real alpha = 0;
                if constexpr (kLut) {
                    int ai;
                    Real af;
                    lut_index(lut, E, ai, af);
                    alpha = lerp(lut.alpha + ((int64_t)L * max_el + i_el) * lut.ne, ai, af);
                } else {
                    alpha = (Real)ly.sjn[L * max_el + i_el] / (Real)E;
                }
                const double cos_ud = uniform<kRng>(key, draws);
                const Real cos_u = (Real)cos_ud;
                draws += 1;
                const Real phi_u = (Real)uniform<kRng>(key, draws);
                draws += 1;
                Real cos_t;
                if (kTab && p.elastic_model == PB_ELASTIC_ELSEPA)
                    cos_t = (Real)elsepa_cos_theta(p.elsepa, L * max_el + i_el, E, cos_ud);
                else
                    cos_t = (Real)1 - (Real)2 * alpha * cos_u / ((Real)1 + alpha - cos_u);
                rotate<Real>(dx, dy, dz, cos_t, (Real)(2.0 * kPi) * phi_u);
                steps += 1;
            }
        }
        if (code >= 0) {
            if (p.seg_count) p.seg_count[i] = nseg;
            if (p.exit_code) p.exit_code[i] = code;
            if (p.final_pos) {
                p.final_pos[3 * i] = (double)px;
                p.final_pos[3 * i + 1] = (double)py;
                p.final_pos[3 * i + 2] = (double)pz;
            }
            if (p.final_dir) {
                p.final_dir[3 * i] = (double)dx;
                p.final_dir[3 * i + 1] = (double)dy;
                p.final_dir[3 * i + 2] = (double)dz;
            }
            if (p.final_E) p.final_E[i] = E;
            if (p.tallies.fates) atomicAdd(&tal.fates[code], 1ULL);
            const bool escaped = code == EXIT_BACK || code == EXIT_TRANS || code == EXIT_SIDE;
            if (escaped && want_E)
                atomicAdd(&tal.exit_E[hist_slot(E, p.tallies.E_lo, p.tallies.E_hi, p.tallies.n_E)], 1ULL);
            if (escaped && want_th) {
                const double th = acos(fmin(fmax((double)dz, -1.0), 1.0));
                atomicAdd(&tal.exit_theta[hist_slot(th, p.tallies.theta_lo, p.tallies.theta_hi,
                                                    p.tallies.n_theta)],
                          1ULL);
            }
            i = -1;
        }
    }

    // Flush block tallies.
    if (p.tallies.deposit) {
        for (int j = 0; j < n_layers && j < kMaxLayers; ++j) {
            double v = dep_acc[j];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0 && v != 0.0) atomicAdd(&tal.deposit[j], v);
        }
    }
    __syncthreads();
    if (p.tallies.fates)
        for (int j = tid; j < 6; j += blockDim.x)
            if (tal.fates[j]) atomicAdd(&p.tallies.fates[j], tal.fates[j]);
    if (want_E)
        for (int j = tid; j < p.tallies.n_E + 2; j += blockDim.x)
            if (tal.exit_E[j]) atomicAdd(&p.tallies.exit_E[j], tal.exit_E[j]);
    if (want_th)
        for (int j = tid; j < p.tallies.n_theta + 2; j += blockDim.x)
            if (tal.exit_theta[j]) atomicAdd(&p.tallies.exit_theta[j], tal.exit_theta[j]);
    if (p.tallies.deposit)
        for (int j = tid; j < n_layers && j < kMaxLayers; j += blockDim.x)
            if (tal.deposit[j] != 0.0) atomicAdd(&p.tallies.deposit[j], tal.deposit[j]);
}

template <class Real, bool kLut, int kRng, bool kStrag, bool kTab = false>
static cudaError_t launch_transport_t(const pb_transport_args &a, cudaStream_t s, int sms) {
    auto kern = transport_kernel<Real, kLut, kRng, kStrag, kTab>;
    size_t dyn = 0;
    if (kLut && a.lut.total_bytes <= (int64_t)kLutSmemBytes) dyn = (size_t)a.lut.total_bytes;
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kLutSmemBytes);
    if (err != cudaSuccess) return err;
    // Default: 256 threads, twice the histories in flight per block as 128 at
    // the same per-SM LUT staging (the LUT core is latency-bound: measured
    // 0.57 -> 0.44 ms for 65,536 histories of the 50 MeV Si scene).
    const int threads = a.block_threads > 0 ? a.block_threads : 256;
    int per_sm = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, dyn);
    if (err != cudaSuccess) return err;
    if (per_sm < 1) per_sm = 1;
    int64_t want = (a.n + threads - 1) / threads;
    int64_t grid = (int64_t)sms * per_sm;
    if (want < grid) grid = want < 1 ? 1 : want;
    kern<<<(unsigned)grid, threads, dyn, s>>>(a);
    return cudaGetLastError();
}

template <bool kStrag>
static cudaError_t launch_transport_s(const pb_transport_args &a, cudaStream_t s, int sms) {
    const bool mixed = a.precision == PB_MIXED;
    const bool lut = a.use_lut != 0;
    const bool philox = a.rng == PB_RNG_PHILOX;
    if (a.elastic_model == PB_ELASTIC_ELSEPA || a.stopping.count) {  // exact core only (checked by the caller)
        if (mixed) {
            if (philox) return launch_transport_t<float, false, PB_RNG_PHILOX, kStrag, true>(a, s, sms);
            return launch_transport_t<float, false, PB_RNG_SPLITMIX, kStrag, true>(a, s, sms);
        }
        if (philox) return launch_transport_t<double, false, PB_RNG_PHILOX, kStrag, true>(a, s, sms);
        return launch_transport_t<double, false, PB_RNG_SPLITMIX, kStrag, true>(a, s, sms);
    }
#define PB_DISPATCH(R, L, G) return launch_transport_t<R, L, G, kStrag>(a, s, sms)
    if (mixed) {
        if (lut) { if (philox) PB_DISPATCH(float, true, PB_RNG_PHILOX); PB_DISPATCH(float, true, PB_RNG_SPLITMIX); }
        if (philox) PB_DISPATCH(float, false, PB_RNG_PHILOX);
        PB_DISPATCH(float, false, PB_RNG_SPLITMIX);
    }
    if (lut) { if (philox) PB_DISPATCH(double, true, PB_RNG_PHILOX); PB_DISPATCH(double, true, PB_RNG_SPLITMIX); }
    if (philox) PB_DISPATCH(double, false, PB_RNG_PHILOX);
    PB_DISPATCH(double, false, PB_RNG_SPLITMIX);
#undef PB_DISPATCH
}

cudaError_t launch_transport(const pb_transport_args &a, cudaStream_t s, int sms) {
    return a.straggling ? launch_transport_s<true>(a, s, sms) : launch_transport_s<false>(a, s, sms);
}

}  // namespace pb
