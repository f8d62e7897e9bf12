// Incoherent PXR + CBS line scoring of a segment list (sm_100a).
//
// For every (segment, reflection row, detector direction) the kernels follow
// the reference's batched line chain (src/pyrite/montecarlo/spectrum/cxr/
// _batched.py:461-931): exact-recoil vacuum root, three fixed-point passes
// of the first-order Snell resonance (cxr/_kernels.py:702-765), the shared
// interpolation bracket for chi/U/mu (cxr/_kernels.py:482-620), the exact
// second-order PXR+CBS amplitude of both polarisations (cxr/_recoil.py:35),
// the segment-mean Beer-Lambert escape (segment_escape.py:276) and the
// line weight and width (cxr/_kernels.py:658, cxr/_batched.py:702-730).
//
// Reductions:
//  * bin-mean (production): each kept line is integrated exactly over the
//    bins within ``exact_widths`` sinc widths of its centre (FP64 sine
//    integral), and its far field -- the cycle-averaged envelope
//    1/(2 a^2 (E_lo - E_r)(E_hi - E_r)) -- is carried by three moments per
//    centre bin in shared memory and spread onto the grid by one finalize
//    pass (cxr/_bin_quadrature.py:280-560 for the exact and far forms).
//    Lines never leave the SM: warp work -> shared-memory spectrum -> one
//    global atomic per bin per block.
//  * node sampling: kept lines are appended to a line buffer and reduced
//    against the grid nodes by a separate kernel (cxr/_cpu_reduce.py:26-50).
//
// PB_FP64 evaluates the chain in double; PB_MIXED in float, with the line
// phase a (E - E_r) formed and range-reduced in double and every
// accumulation in double.
#include <algorithm>
#include <climits>
#include <type_traits>
#include <cstdint>
#include <cstdio>
#include <cuda.h>
#include <mutex>

#include "pb_common.cuh"
#include "pb_internal.h"
#include "pb_layers.cuh"

namespace pb {

constexpr int kSegTile = 16;
constexpr int kCxrThreads = 256;  // two resident blocks per SM (128 registers each)
// Reflection rows per pass: 120 on the float path (a pass's prefilter
// survivors then fill the block's threads about twice, with a smaller idle
// tail than at 64 rows, measured 10 % faster on the control variate's
// sub-sample), 64 on the FP64 path, whose staged tables need the room.
template <class Real>
constexpr int row_chunk() { return sizeof(Real) == 4 ? 120 : 64; }
template <class Real>
constexpr int pair_queue() { return kSegTile * row_chunk<Real>(); }  // every pair of a pass may keep a line
constexpr int kXQueue = 2048;   // queued exact-window bins per class and pass
constexpr int kMaxTab = 4096;   // E_tab / delta staged in shared memory up to this size
constexpr int kMaxMu = 4;

// Math of the line chain. FP64 uses IEEE operations throughout (parity with
// the reference's FP64 chain); the float path uses the SFU approximations
// (division by reciprocal, sqrt by reciprocal square root, base-2 exp/log),
// each within a few ulp, which the 1 % spectrum tolerance of the mixed path
// absorbs many times over.
__device__ __forceinline__ double r_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float r_sqrt(float x) { return x > 0.0f ? x * rsqrtf(x) : sqrtf(x); }
__device__ __forceinline__ double r_exp(double x) { return exp(x); }
__device__ __forceinline__ float r_exp(float x) { return __expf(x); }
__device__ __forceinline__ double r_expm1(double x) { return expm1(x); }
__device__ __forceinline__ float r_expm1(float x) { return expm1f(x); }
__device__ __forceinline__ double r_log1p(double x) { return log1p(x); }
__device__ __forceinline__ float r_log1p(float x) { return log1pf(x); }
__device__ __forceinline__ double rdiv(double a, double b) { return a / b; }
__device__ __forceinline__ float rdiv(float a, float b) { return __fdividef(a, b); }

// Per (segment, direction) quantities shared by every reflection row.
template <class Real>
struct SegPre {
    Real vx, vy, vz;        // beta v_hat
    Real gamma;
    Real denom_row;         // 1 - beta v_hat.n, cancellation free
    Real t_L;               // L / beta
    Real path0, path1;      // escape paths at the segment ends
    Real gx, gy, gz;        // grad L
    Real grad2;
    Real v_dot_grad;
    Real inv_E;             // hbar c / E
    int radiates;           // elec_id < Ne
};

template <class Real>
struct RowPre {
    Real G[3];
    Real ES[3];
    Real EP[3];
    Real g2, n_dot_g, g_dot_es, g_dot_ep, wm;
    int row;
};

template <class Real>
__device__ __forceinline__ Real slab_path(Real z, Real thickness, Real nz) {
    const Real inv_nz = (Real)1 / fmax(fabs(nz), (Real)1.0e-12);
    const Real depth = fmin(fmax(z, (Real)0), thickness);
    return nz < (Real)0 ? depth * inv_nz : (thickness - depth) * inv_nz;
}

template <class Real>
__device__ void seg_precompute(SegPre<Real> &sp, const pb_cxr_args &a, int64_t s, const double *nh) {
    const double E = a.E_keV[s];
    const Real Er = (Real)E;
    const Real vhx = (Real)a.v_hat[3 * s], vhy = (Real)a.v_hat[3 * s + 1], vhz = (Real)a.v_hat[3 * s + 2];
    const Real nx = (Real)nh[0], ny = (Real)nh[1], nz = (Real)nh[2];
    // cxr/_setup.py:945-1005; kinematics.py:151-154
    const Real g0 = (Real)1 + Er / (Real)510.99895;
    const Real beta = r_sqrt((Real)1 - (Real)1 / (g0 * g0));
    sp.vx = beta * vhx;
    sp.vy = beta * vhy;
    sp.vz = beta * vhz;
    // cxr/_kernels.py:678-699
    const Real gamma = (Real)1 + Er / (Real)(kMeEv / 1e3);
    const Real omb = (Real)1 / (gamma * gamma * ((Real)1 + beta));
    const Real dvx = vhx - nx, dvy = vhy - ny, dvz = vhz - nz;
    const Real omc = (Real)0.5 * (dvx * dvx + dvy * dvy + dvz * dvz);
    sp.gamma = gamma;
    sp.denom_row = omb + beta * omc;
    sp.t_L = (Real)a.L[s] / beta;
    // segment_escape.py:239-270, single slab
    const Real T = (Real)a.thickness;
    const Real half = (Real)0.5 * (Real)a.L[s];
    const Real z_mid = (Real)a.r_mid[3 * s + 2];
    sp.path0 = slab_path<Real>(z_mid - half * vhz, T, nz);
    sp.path1 = slab_path<Real>(z_mid + half * vhz, T, nz);
    // segment_escape.py:95-131
    Real gx = (Real)-0.0 / nz, gy = (Real)-0.0 / nz, gz = (Real)-1 / nz;
    if (z_mid < (Real)0 || z_mid > T) { gx = 0; gy = 0; gz = 0; }
    sp.gx = gx; sp.gy = gy; sp.gz = gz;
    sp.grad2 = gx * gx + gy * gy + gz * gz;
    sp.v_dot_grad = sp.vx * gx + sp.vy * gy + sp.vz * gz;
    sp.inv_E = (Real)kHbarcEvAng / (gamma * (Real)kMeEv);
    sp.radiates = a.elec_id[s] < a.Ne && (a.seg_layer == nullptr || a.seg_layer[s] == a.emit_layer);
}

// searchsorted(grid, x, side="left") clipped to [1, n-1] and the blend
// fraction (cxr/_kernels.py:328-349).
// Geometric tabulation grids (grid[i] = exp(log0 + i h)) are indexed in
// closed form and then corrected to the exact searchsorted answer, which
// replaces ~log2(n) dependent shared-memory loads by one logarithm.
struct TabIndex {
    bool geometric;
    double log0;
    double inv_h;
};

__device__ __forceinline__ double t_log(double x) { return log(x); }
__device__ __forceinline__ float t_log(float x) { return __logf(x); }

template <class Real>
__device__ __forceinline__ void bracket(const Real *grid, int n, Real x, int &idx, Real &frac,
                                        bool &below, bool &above, const TabIndex &ti) {
    int i;
    if (isnan(x)) {
        i = n;
    } else if (ti.geometric) {
        int c = 0;
        if (x > grid[0]) {
            const Real f = (t_log(x) - (Real)ti.log0) * (Real)ti.inv_h;
            c = f >= (Real)(n - 1) ? n : (int)ceil(f);
            if (c < 0) c = 0;
        }
        // searchsorted(side="left"): first index with grid[i] >= x
        while (c > 0 && !(grid[c - 1] < x)) --c;
        while (c < n && grid[c] < x) ++c;
        i = c;
    } else {
        int lo = 0, hi = n;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (grid[mid] < x) lo = mid + 1; else hi = mid;
        }
        i = lo;
    }
    i = i < 1 ? 1 : (i > n - 1 ? n - 1 : i);
    idx = i;
    frac = rdiv(x - grid[i - 1], grid[i] - grid[i - 1]);
    below = x <= grid[0];
    above = x >= grid[n - 1];
}

template <class Real, class T>
__device__ __forceinline__ Real gather(const T *f, int n, int idx, Real frac, bool below, bool above) {
    const Real f0 = (Real)f[idx - 1];
    Real y = f0 + frac * ((Real)f[idx] - f0);
    if (below) y = (Real)f[0];
    if (above) y = (Real)f[n - 1];
    return y;
}

// cxr/_recoil.py:35-76
template <class Real>
__device__ __forceinline__ void quantum_line_factors(Real h, Real gamma, Real vdg, Real k_dot_v,
                                                     Real k_dot_g, Real g2, Real k2, Real v_dot_e,
                                                     Real g_dot_e, Real k_dot_e, Real &pxr_num,
                                                     Real &f_cbs) {
    const Real gg = gamma * gamma;
    const Real n_1 = h * g2 - (Real)2 * gamma * vdg;
    const Real n_2 = n_1 + (Real)2 * h * k_dot_g;
    const Real n_f = h * (g2 + (Real)2 * k_dot_g + k2) - (Real)2 * gamma * (vdg + k_dot_v);
    const Real e_1 = r_sqrt(gg + h * n_1);
    const Real e_2 = r_sqrt(gg + h * (h * k2 - (Real)2 * gamma * k_dot_v));
    const Real e_f = r_sqrt(gg + h * n_f);
    const Real s_if = gamma + e_f;
    const Real ge_ke = g_dot_e + k_dot_e;
    pxr_num = rdiv(-n_f * ge_ke - k2 * ((Real)2 * gamma * v_dot_e - h * ge_ke), s_if);
    const Real s_1 = e_1 + gamma;
    const Real s_3 = e_1 + e_f;
    const Real s_4 = gamma + e_2;
    const Real x = (Real)2 * gamma * v_dot_e - h * k_dot_e;
    const Real sigma = s_if + e_1 + e_2;
    f_cbs = rdiv((Real)2 * g_dot_e * s_1, s_3 * n_1) +
            rdiv(x * (n_1 * rdiv(n_f, s_if) * sigma - (Real)2 * s_1 * s_4 * k_dot_g), s_3 * s_4 * n_1 * n_2);
}

// segment_escape.py:276-289. The float path switches to the series below
// d = 0.01, where 1 - exp(-d) in float would lose digits.
template <class Real>
__device__ __forceinline__ Real mean_transmission(Real t0, Real t1) {
    const Real lo = fmin(t0, t1);
    const Real d = fabs(t1 - t0);
    if constexpr (sizeof(Real) == 8) {
        const Real safe = d > (Real)1.0e-4 ? d : (Real)1;
        const Real ratio = d > (Real)1.0e-4 ? -r_expm1(-safe) / safe
                                             : (Real)1 - (Real)0.5 * d + d * d / (Real)6;
        return r_exp(-lo) * ratio;
    } else {
        const float ratio = d > 0.01f ? rdiv(1.0f - __expf(-d), d)
                                      : 1.0f - d * (0.5f - d * (1.0f / 6.0f - d * (1.0f / 24.0f)));
        return __expf(-lo) * ratio;
    }
}

// Layered escape of one (segment, direction): its pieces (pb_layers.cuh)
// with the exit-side depth inside the piece's layer at both ends, already
// divided by |n_z|.
template <class Real>
struct EscSeg {
    int np;
    int up;                 // exits through the entrance face (n_z < 0)
    Real inv_nz;
    int m[kMaxEscLayers];
    Real f[kMaxEscLayers], w0[kMaxEscLayers], w1[kMaxEscLayers];
};

template <class Real>
__device__ void esc_precompute(EscSeg<Real> &es, const pb_cxr_args &a, int64_t s, const double *nh,
                               const double *zt, const double *zb) {
    const double nz = nh[2];
    const double inv_nz = 1.0 / fmax(fabs(nz), 1.0e-12);
    const double half = 0.5 * a.L[s];
    const double z = a.r_mid[3 * s + 2], vz = a.v_hat[3 * s + 2];
    EscPiece pp[kMaxEscLayers];
    const int np = esc_pieces(z - half * vz, z + half * vz, a.n_layer, zt, zb, pp);
    es.np = np;
    es.up = nz < 0.0;
    es.inv_nz = (Real)inv_nz;
    for (int p = 0; p < np; ++p) {
        const double t = zb[pp[p].m] - zt[pp[p].m];
        es.m[p] = pp[p].m;
        es.f[p] = (Real)pp[p].f;
        es.w0[p] = (Real)((nz < 0.0 ? pp[p].u0 : t - pp[p].u0) * inv_nz);
        es.w1[p] = (Real)((nz < 0.0 ? pp[p].u1 : t - pp[p].u1) * inv_nz);
    }
}

// piece_mean_transmission (segment_escape.py:335-355) with every layer's
// exact mu at the line energy (cxr/_batched.py:702-720): the layers between
// a piece's layer and the exit face are crossed whole.
template <class Real>
__device__ Real esc_transmission(const EscSeg<Real> &es, const pb_cxr_args &a, const Real *lay_t, double E_eV) {
    Real mu[kMaxEscLayers], c[kMaxEscLayers];
    const int nl = a.n_layer;
#pragma unroll
    for (int k = 0; k < kMaxEscLayers; ++k) {
        mu[k] = 0;
        if (k < nl) {
            const int o = a.mu_off[k];
            mu[k] = (Real)esc_mu_at(a.mu_knot + o, a.mu_value + o, a.mu_slope + o, a.mu_off[k + 1] - o, E_eV);
        }
    }
    Real run = 0;
    if (es.up) {
#pragma unroll
        for (int k = 0; k < kMaxEscLayers; ++k) {
            c[k] = run;
            if (k < nl) run += mu[k] * lay_t[k];
        }
    } else {
#pragma unroll
        for (int k = kMaxEscLayers - 1; k >= 0; --k) {
            c[k] = run;
            if (k < nl) run += mu[k] * lay_t[k];
        }
    }
    Real T = 0;
    for (int p = 0; p < es.np; ++p) {
        const int m = es.m[p];
        const Real mm = esc_pick<Real>(mu, m), cm = esc_pick<Real>(c, m) * es.inv_nz;
        T += es.f[p] * mean_transmission<Real>(cm + mm * es.w0[p], cm + mm * es.w1[p]);
    }
    return T;
}

template <class Real>
struct Line {
    Real E_res, a_width, weight;
    bool good;
};

// Cheap test of whether a pair's resonance can reach the keep window under
// any refraction the table allows: omega <= 0 is never kept (denom > 0 is
// required); above the window, with D the largest |delta| the table holds at
// or above E_vac / 1.5, D |grad L| <= denom_vac / 2 keeps every root iterate
// (and so the root) at or above E_vac / 1.5, by induction over the passes.
template <class Real>
__device__ __forceinline__ bool pair_may_keep(const SegPre<Real> &sp, const RowPre<Real> &rw,
                                              const Real *E_tab, const Real *dtail, int n_tab,
                                              const pb_cxr_tables &t, const TabIndex &ti) {
    const Real r_num = (Real)0.5 * rw.g2 * sp.inv_E;
    const Real r_den = rw.n_dot_g * sp.inv_E;
    const Real num = (sp.vx * rw.G[0] + sp.vy * rw.G[1] + sp.vz * rw.G[2]) - r_num;
    const Real denom_vac = sp.denom_row + r_den;
    if (!sp.radiates || !(num > (Real)0) || !(denom_vac > (Real)0)) return false;
    if (dtail == nullptr) return true;
    const Real E_low = (Real)kHbarcEvAng * rdiv(num, denom_vac) * (Real)(1.0 / 1.5);
    if (E_low < (Real)t.hi_keep) return true;
    int ix;
    Real fr;
    bool bl, ab;
    bracket<Real>(E_tab, n_tab, E_low, ix, fr, bl, ab, ti);
    return !(dtail[ix - 1] * r_sqrt(sp.grad2) <= (Real)0.5 * denom_vac);
}

// The per-pair chain up to the complex PXR+CBS amplitude of both
// polarisations (cxr/_batched.py:461-559 and 789-826): the resonance (three
// Snell passes), the keep decision, the line's slope, the attenuation at the
// line energy and the amplitudes. Shared by the incoherent line (pair_line)
// and the coherent route's records (coh_records_kernel). ``E_tab`` /
// ``delta_tab`` / ``log_mu`` point at the shared-memory staging (or global
// memory for a large FP64 grid). The float path stops after the keep
// decision for dropped pairs.
template <class Real>
struct PairAmps {
    Real omega, E_res, slope, mu, v_dot_g, r_num, r_den;
    Real A_re[2], A_im[2];
    bool keep;
};

// The resonance of a pair: three Snell passes for the refraction at the line
// energy and the keep decision (delta and denom carry what the amplitude part
// needs; denom is NaN when the passes did not settle).
template <class Real>
struct Resonance {
    Real delta, denom;
    bool keep;
};

template <class Real>
__device__ __forceinline__ Resonance<Real> pair_resonance(const SegPre<Real> &sp, const RowPre<Real> &rw,
                                                          const Real *E_tab, const Real *delta_tab, int n_tab,
                                                          const pb_cxr_tables &t, const TabIndex &ti) {
    const Real Gx = rw.G[0], Gy = rw.G[1], Gz = rw.G[2];
    const Real g2 = rw.g2, n_dot_g = rw.n_dot_g;
    const Real hbarc = (Real)kHbarcEvAng;
    // cxr/_block_prologue.py:18-38, cxr/_recoil.py:79-97
    const Real r_num = (Real)0.5 * g2 * sp.inv_E;
    const Real r_den = n_dot_g * sp.inv_E;
    const Real v_dot_g = sp.vx * Gx + sp.vy * Gy + sp.vz * Gz;
    const Real v_dot_g_exact = v_dot_g - r_num;
    const Real denom_vac = sp.denom_row + r_den;
    // cxr/_kernels.py:702-765
    Real denom = denom_vac, previous = denom, delta = (Real)NAN;
    for (int pass = 0; pass < 3; ++pass) {
        const Real Er = hbarc * rdiv(v_dot_g_exact, denom);
        int ix;
        Real fr;
        bool bl, ab;
        bracket<Real>(E_tab, n_tab, Er, ix, fr, bl, ab, ti);
        delta = gather<Real>(delta_tab, n_tab, ix, fr, bl, ab);
        previous = denom;
        denom = denom_vac - delta * sp.v_dot_grad;
    }
    bool settled = fabs(denom - previous) <= (Real)1e-3 * fabs(denom);
    settled = settled && ((Real)2 * fabs(delta) * sp.grad2 < (Real)1);
    if (!settled) denom = (Real)NAN;
    const Real omega = rdiv(v_dot_g - r_num, denom);
    const Real E_res = hbarc * omega;
    bool keep = sp.radiates && (E_res > (Real)t.lo_keep) && (E_res > (Real)10) && (E_res < (Real)t.hi_keep);
    keep = keep && (denom > (Real)0) && (omega * sp.inv_E <= (Real)1 - rdiv((Real)1, sp.gamma));
    return Resonance<Real>{delta, denom, keep};
}

// The rest of the chain from the resonance: the line's slope, the attenuation
// at the line energy and the complex amplitudes. The float path stops after
// the resonance for dropped pairs; FP64 completes every pair so its per-pair
// output matches the reference's arrays.
template <class Real, bool kLayered>
__device__ __forceinline__ PairAmps<Real> pair_amps_from(const SegPre<Real> &sp, const RowPre<Real> &rw,
                                                         const Resonance<Real> &res, const Real *E_tab,
                                                         const Real *log_mu, int n_tab, int n_mu,
                                                         const pb_cxr_tables &t, const TabIndex &ti) {
    const Real Gx = rw.G[0], Gy = rw.G[1], Gz = rw.G[2];
    const Real g2 = rw.g2, n_dot_g = rw.n_dot_g;
    const Real hbarc = (Real)kHbarcEvAng;
    PairAmps<Real> o;
    const Real r_num = (Real)0.5 * g2 * sp.inv_E;
    const Real r_den = n_dot_g * sp.inv_E;
    const Real v_dot_g = sp.vx * Gx + sp.vy * Gy + sp.vz * Gz;
    o.r_num = r_num;
    o.r_den = r_den;
    o.v_dot_g = v_dot_g;
    const Real delta = res.delta, denom = res.denom;
    const Real n_dot_g_blk = n_dot_g + delta * (sp.gx * Gx + sp.gy * Gy + sp.gz * Gz);
    // cxr/_kernels.py:624-655
    const Real omega = rdiv(v_dot_g - r_num, denom);
    const Real k_dot_v = omega * (((Real)1 - denom) + r_den);
    const Real k_dot_g = omega * n_dot_g_blk;
    const Real detuning = g2 + (Real)2 * k_dot_g;
    // cxr/_batched.py:435-458
    const Real k_mag = omega * r_sqrt(sp.grad2 == (Real)0 ? (Real)1
                                                           : (Real)1 - (Real)2 * delta + delta * delta * sp.grad2);
    const Real E_res = hbarc * omega;
    o.omega = omega;
    o.E_res = E_res;
    o.mu = (Real)0;
    // cxr/_block_prologue.py:53-62, cxr/_recoil.py:100-118
    o.slope = denom * rdiv((Real)1, (Real)1 - omega * sp.inv_E);
    o.keep = res.keep;
    if constexpr (sizeof(Real) == 4) {
        if (!res.keep) return o;
    }
    int ix;
    Real fr;
    bool bl, ab;
    bracket<Real>(E_tab, n_tab, E_res, ix, fr, bl, ab, ti);
    Real lfr;
    {
        const Real x0 = E_tab[ix - 1], x1 = E_tab[ix];
        Real bx = fmin(fmax(E_res, x0), x1);
        if (isnan(E_res)) bx = E_res;
        if constexpr (sizeof(Real) == 8) {
            lfr = r_log1p((bx - x0) / x0) / r_log1p((x1 - x0) / x0);
        } else {
            // cxr/_kernels.py:352-366 on a geometric grid: log(bx/x0)/h.
            lfr = ti.geometric ? __logf(rdiv(bx, x0)) * (float)ti.inv_h
                               : rdiv(log1pf(rdiv(bx - x0, x0)), log1pf(rdiv(x1 - x0, x0)));
        }
    }
    // cxr/_kernels.py:482-506 couplings, 369-388 attenuation
    const int64_t base = (int64_t)rw.row * n_tab;
    const Real chi_re = gather<Real>(t.chi_re + base, n_tab, ix, fr, bl, ab);
    const Real chi_im = gather<Real>(t.chi_im + base, n_tab, ix, fr, bl, ab);
    const Real u_re = gather<Real>(t.u_re + base, n_tab, ix, fr, bl, ab);
    const Real u_im = gather<Real>(t.u_im + base, n_tab, ix, fr, bl, ab);
    Real mu = 0;
    for (int el = 0; el < (kLayered ? 0 : n_mu); ++el) {
        const Real *lm = log_mu + (int64_t)el * n_tab;
        const Real f0 = lm[ix - 1];
        Real v = r_exp(f0 + lfr * (lm[ix] - f0));
        if (bl) v = r_exp(lm[0]);
        if (ab) v = r_exp(lm[n_tab - 1]);
        mu += v;
    }
    o.mu = mu;
    // cxr/_batched.py:789-826, cxr/_line_amplitude.py:14-37
    const Real h = (Real)(kHbarcEvAng / kMeEv);
    const Real k2 = k_mag * k_mag;
#pragma unroll
    for (int pol = 0; pol < 2; ++pol) {
        const Real *Ev = pol == 0 ? rw.ES : rw.EP;
        const Real g_dot_e = pol == 0 ? rw.g_dot_es : rw.g_dot_ep;
        const Real v_dot_e = sp.vx * Ev[0] + sp.vy * Ev[1] + sp.vz * Ev[2];
        const Real k_dot_e = omega * delta * (sp.gx * Ev[0] + sp.gy * Ev[1] + sp.gz * Ev[2]);
        Real pxr_num, f_cbs;
        quantum_line_factors<Real>(h, sp.gamma, v_dot_g, k_dot_v, k_dot_g, g2, k2, v_dot_e, g_dot_e,
                                   k_dot_e, pxr_num, f_cbs);
        const Real f_pxr = rdiv(pxr_num, detuning);
        o.A_re[pol] = chi_re * f_pxr + u_re * f_cbs;
        o.A_im[pol] = chi_im * f_pxr + u_im * f_cbs;
    }
    return o;
}

template <class Real, bool kLayered>
__device__ __forceinline__ PairAmps<Real> pair_amps(const SegPre<Real> &sp, const RowPre<Real> &rw,
                                                    const Real *E_tab, const Real *delta_tab, const Real *log_mu,
                                                    int n_tab, int n_mu, const pb_cxr_tables &t,
                                                    const TabIndex &ti) {
    const Resonance<Real> res = pair_resonance<Real>(sp, rw, E_tab, delta_tab, n_tab, t, ti);
    return pair_amps_from<Real, kLayered>(sp, rw, res, E_tab, log_mu, n_tab, n_mu, t, ti);
}

// The incoherent line of a pair: resonance, width and weight
// (cxr/_batched.py:702-730, cxr/_kernels.py:658-668).
template <class Real, bool kLayered>
__device__ Line<Real> pair_line_from(const SegPre<Real> &sp, const RowPre<Real> &rw, const Resonance<Real> &res,
                                     const Real *E_tab, const Real *log_mu, int n_tab, int n_mu,
                                     const pb_cxr_tables &t, const TabIndex &ti, const EscSeg<Real> *es,
                                     const pb_cxr_args &a, const Real *lay_t) {
    const PairAmps<Real> p = pair_amps_from<Real, kLayered>(sp, rw, res, E_tab, log_mu, n_tab, n_mu, t, ti);
    Line<Real> out;
    out.good = false;
    out.E_res = p.E_res;
    out.a_width = (Real)NAN;
    out.weight = (Real)NAN;
    if constexpr (sizeof(Real) == 4) {
        if (!p.keep) return out;
    }
    const Real A2 = (p.A_re[0] * p.A_re[0] + p.A_im[0] * p.A_im[0]) + (p.A_re[1] * p.A_re[1] + p.A_im[1] * p.A_im[1]);
    Real T_abs;
    if constexpr (kLayered) T_abs = esc_transmission<Real>(*es, a, lay_t, (double)p.E_res);
    else T_abs = mean_transmission<Real>(sp.path0 * p.mu, sp.path1 * p.mu);
    const Real pref_c1 = (Real)(4.0 * (kPi * kPi) * kHbarcEvAng);
    const Real pref = rdiv((Real)kAlphaFs * p.omega, pref_c1) * (sp.t_L * sp.t_L) * T_abs;
    out.a_width = rdiv(p.slope * sp.t_L, (Real)2 * (Real)kHbarcEvAng) * (Real)1;
    out.weight = pref * A2 * rw.wm;
    out.good = p.keep && isfinite(out.weight) && (out.weight > (Real)0);
    return out;
}

template <class Real, bool kLayered>
__device__ __forceinline__ Line<Real> pair_line(const SegPre<Real> &sp, const RowPre<Real> &rw, const Real *E_tab,
                                                const Real *delta_tab, const Real *log_mu, int n_tab, int n_mu,
                                                const pb_cxr_tables &t, const TabIndex &ti, const EscSeg<Real> *es,
                                                const pb_cxr_args &a, const Real *lay_t) {
    const Resonance<Real> res = pair_resonance<Real>(sp, rw, E_tab, delta_tab, n_tab, t, ti);
    return pair_line_from<Real, kLayered>(sp, rw, res, E_tab, log_mu, n_tab, n_mu, t, ti, es, a, lay_t);
}

// ---- sine integral and the sinc^2 antiderivative --------------------------
// Si(t) - pi/2 for t >= 0: power series for t <= 13; the continued fraction of
// E1(i t) by the modified Lentz method (Numerical Recipes "cisi") for
// 13 < t < 40; the asymptotic auxiliary-function series beyond
// (Abramowitz & Stegun 5.2.34-5.2.35): Si - pi/2 = -f cos t - g sin t.
constexpr int kSiTerms = 31;  // k = 30 term at t = 13 is ~3e-18
struct SiSeries {
    double c[kSiTerms];  // (-1)^k / ((2k+1) (2k+1)!)
};
__host__ __device__ constexpr SiSeries make_si_series() {
    SiSeries s{};
    double fact = 1.0;
    for (int k = 0; k < kSiTerms; ++k) {
        if (k > 0) fact *= (2.0 * k) * (2.0 * k + 1.0);
        s.c[k] = ((k & 1) ? -1.0 : 1.0) / ((2.0 * k + 1.0) * fact);
    }
    return s;
}

__device__ double si_minus_half_pi(double t) {
    if (t <= 13.0) {
        // Power series in Horner form with compile-time coefficients; the
        // sum of |terms| at t = 13 is ~2e4, so ~5e-12 absolute accuracy.
        constexpr SiSeries kSi = make_si_series();
        const double t2 = t * t;
        double p = kSi.c[kSiTerms - 1];
#pragma unroll
        for (int k = kSiTerms - 2; k >= 0; --k) p = fma(p, t2, kSi.c[k]);
        return p * t - 0.5 * kPi;
    }
    double s, c;
    sincos(t, &s, &c);
    if (t >= 40.0) {
        const double inv_t = 1.0 / t;
        const double y = inv_t * inv_t;
        // f t = 1 - 2!/t^2 + 4!/t^4 - ..., g t^2 = 1 - 3!/t^2 + 5!/t^4 - ...
        double f = 1.0, g = 1.0, tf = 1.0, tg = 1.0;
        for (int k = 1; k < 12; ++k) {
            tf *= -(2.0 * k - 1.0) * (2.0 * k) * y;
            tg *= -(2.0 * k) * (2.0 * k + 1.0) * y;
            f += tf;
            g += tg;
            if (fabs(tf) < 1e-17 && fabs(tg) < 1e-17) break;
        }
        f *= inv_t;
        g *= y;
        return -f * c - g * s;
    }
    double br = 1.0, bi = t;
    double inv = 1.0 / (br * br + bi * bi);
    double dr = br * inv, di = -bi * inv;
    double hr = dr, hi = di;
    double cr = 1e300, ci = 0.0;
    for (int i = 2; i < 200; ++i) {
        const double a = -(double)(i - 1) * (double)(i - 1);
        br += 2.0;
        const double xr = a * dr + br, xi = a * di + bi;
        inv = 1.0 / (xr * xr + xi * xi);
        dr = xr * inv;
        di = -xi * inv;
        inv = a / (cr * cr + ci * ci);
        cr = br + cr * inv;
        ci = bi - ci * inv;
        const double delr = cr * dr - ci * di, deli = cr * di + ci * dr;
        const double nhr = hr * delr - hi * deli, nhi = hr * deli + hi * delr;
        hr = nhr;
        hi = nhi;
        if (fabs(delr - 1.0) + fabs(deli) < 1e-16) break;
    }
    return c * hi - s * hr;
}

// R(x) = F(x) - sign(x)/2, F the integral of sinc^2 from 0.
__device__ double sincsq_tail(double x) {
    const double u = fabs(x);
    const double t = 2.0 * kPi * u;
    double su;
    if (u == 0.0) {
        su = 1.0;
    } else {
        su = sin(kPi * u) / (kPi * u);
    }
    const double r = si_minus_half_pi(t) / kPi - u * su * su;
    return x >= 0.0 ? r : -r;
}

constexpr double kInvPi = 1.0 / kPi;
constexpr double kInv2Pi2 = 1.0 / (2.0 * kPi * kPi);

struct BinAxis {
    const double *edges;
    int n;
    double lo, w, inv_w;  // uniform axis: edges[b] = lo + b w
    bool uniform;
    int pad;              // virtual centre bins on each side (uniform axes)
};

__device__ __forceinline__ int bin_of(const BinAxis &ax, double E) {
    if (ax.uniform) return (int)floor((E - ax.lo) * ax.inv_w);
    if (E < ax.edges[0]) return -1;
    if (E >= ax.edges[ax.n]) return ax.n;
    int lo = 0, hi = ax.n;  // last edge index with edges[b] <= E
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (ax.edges[mid] <= E) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ double centre_of(const BinAxis &ax, int c) {
    if (ax.uniform) return ax.lo + ((double)c + 0.5) * ax.w;
    return 0.5 * (ax.edges[c] + ax.edges[c + 1]);
}

// Far-field envelope expansion about centre c: 1/((A-d)(B-d)) ~
// f0 + f1 d + f2 d^2 with A = E_lo - E_c, B = E_hi - E_c, d = E_r - E_c
// (any common unit: the form scales as 1/unit^2). Float on the mixed path.
template <bool kMixed>
__device__ __forceinline__ double far_envelope(double A, double B, double d) {
    if constexpr (kMixed) {
        const float Af = (float)A, Bf = (float)B, df = (float)d;
        const float AB = Af * Bf;
        const float r = __frcp_rn(AB);
        const float f1 = (Af + Bf) * r * r;
        const float f2 = (Af * Af + AB + Bf * Bf) * r * r * r;
        return (double)(r + df * (f1 + df * f2));
    } else {
        const double AB = A * B;
        const double r = 1.0 / AB;
        const double f1 = (A + B) * r * r;
        const double f2 = (A * A + AB + B * B) * r * r * r;
        return r + d * (f1 + d * f2);
    }
}

// Oscillatory part of the sinc^2 antiderivative beyond the asymptotic
// threshold (Abramowitz & Stegun 5.2.8, 5.2.34-35): with u = 2 pi |x|,
//   int sinc^2 = (1/(2 pi^2)) (1/x_a - 1/x_b) + (1/pi) [Q(u)]_a^b,
//   Q(u) = cos u (1/u - f(u)) - g(u) sin u,
// where 1/u - f(u) ~ (1/u) sum_{k>=1} (-1)^(k+1) (2k)!/u^2k and
// g(u) ~ (1/u^2) sum_{k>=0} (-1)^k (2k+1)!/u^2k. The envelope term carries
// the mass without the cancellation of a difference of antiderivatives.
__device__ __forceinline__ double q_osc_f64(double u) {
    const double inv_u = 1.0 / u;
    const double y = inv_u * inv_u;
    double p1 = 0.0, p2 = 0.0;
    // 13 terms: the first omitted one at u = 48 is below 1e-17 of the leading.
    double t1 = 2.0 * y, t2 = 1.0;
    for (int k = 1; k <= 13; ++k) {
        p1 += t1;
        p2 += t2;
        t1 *= -(2.0 * k + 1.0) * (2.0 * k + 2.0) * y;
        t2 *= -(2.0 * k) * (2.0 * k + 1.0) * y;
    }
    double sn, cs;
    sincos(u, &sn, &cs);
    return cs * p1 * inv_u - sn * p2 * y;
}

// Float form for the mixed path; the phase u is reduced in double first.
__device__ __forceinline__ double q_osc_f32(double u) {
    const float inv_u = __frcp_rn((float)u);
    const float yf = inv_u * inv_u;
    const float p1 = yf * (2.0f + yf * (-24.0f + yf * (720.0f + yf * (-40320.0f + yf * 3628800.0f))));
    const float p2 = 1.0f + yf * (-6.0f + yf * (120.0f + yf * (-5040.0f + yf * 362880.0f)));
    const double r = u - 2.0 * kPi * rint(u * (0.5 / kPi));
    float sn, cs;
    __sincosf((float)r, &sn, &cs);
    return (double)(cs * p1 * inv_u - sn * p2 * yf);
}

// One bin edge of a line, in both antiderivative forms it may be needed in.
struct EdgeCache {
    bool valid;
    double x;       // line-centred first-zero units
    bool has_r, has_q;
    double r;       // R(x), the sinc^2 antiderivative minus sign(x)/2
    double q;       // Q(2 pi |x|), the oscillatory part of the far form
};

template <bool kMixed>
__device__ __forceinline__ double edge_r(EdgeCache &e) {
    if (!e.has_r) { e.r = sincsq_tail(e.x); e.has_r = true; }
    return e.r;
}

template <bool kMixed>
__device__ __forceinline__ double edge_q(EdgeCache &e) {
    if (!e.has_q) {
        const double u = 2.0 * kPi * fabs(e.x);
        e.q = kMixed ? q_osc_f32(u) : q_osc_f64(u);
        e.has_q = true;
    }
    return e.q;
}

// Exact mass of sinc^2 over [lo.x, hi.x]: the far closed form when both
// edges are beyond the asymptotic threshold on one side, else the
// difference of antiderivatives.
template <bool kMixed>
__device__ __forceinline__ double bin_mass(EdgeCache &lo, EdgeCache &hi) {
    const double u_lim = kMixed ? 24.0 : 48.0;
    const double x_lo = lo.x, x_hi = hi.x;
    const double u_lo = 2.0 * kPi * fabs(x_lo), u_hi = 2.0 * kPi * fabs(x_hi);
    if ((x_lo > 0.0 || x_hi < 0.0) && fmin(u_lo, u_hi) >= u_lim) {
        const bool pos = x_lo > 0.0;
        const double a = pos ? x_lo : -x_hi;
        const double b = pos ? x_hi : -x_lo;
        double env;
        if constexpr (kMixed) {
            env = (double)__fdividef((float)((b - a) * kInv2Pi2), (float)a * (float)b);
        } else {
            env = (b - a) * kInv2Pi2 / (a * b);
        }
        const double osc = pos ? (edge_q<kMixed>(hi) - edge_q<kMixed>(lo))
                               : (edge_q<kMixed>(lo) - edge_q<kMixed>(hi));
        return env + osc / kPi;
    }
    return edge_r<kMixed>(hi) - edge_r<kMixed>(lo) + ((x_lo < 0.0 && x_hi >= 0.0) ? 1.0 : 0.0);
}

// Bin-mean deposit of a line: exact bin integrals within the line's window
// (``exact_widths`` first-zero widths, at least K_far bins); beyond it the far
// envelope w/(2 a^2) / ((E_lo - E_r)(E_hi - E_r)) is carried by three moments
// about the centre bin and spread by far_field_kernel onto every bin more
// than K_far bins away. A line whose window is wider than K_far removes the
// envelope again from its extra exact bins, so each bin takes exactly one of
// the two forms. Lines centred off a non-uniform axis, or too wide for a
// window, are integrated exactly over the whole axis.
struct LineWindow {
    int c;        // centre bin (may lie off the axis)
    int b0, nb;   // first exact bin and count
    bool mom;     // far field through the moments
};

__device__ __forceinline__ LineWindow line_window(double E_r, double a, const BinAxis &ax,
                                                  double exact_widths, int K_far, bool moments) {
    const int n = ax.n;
    LineWindow lw;
    lw.c = bin_of(ax, E_r);
    lw.mom = moments && K_far > 0 && lw.c >= -ax.pad && lw.c < n + ax.pad;
    int K;
    if (!lw.mom) {
        K = n + (lw.c < 0 ? -lw.c : (lw.c >= n ? lw.c - n + 1 : 0));
    } else {
        const double kk = ceil(exact_widths * kPi / (a * ax.w));
        K = kk > (double)(2 * n) ? 2 * n : (kk < (double)K_far ? K_far : (int)kk);
    }
    int b0 = lw.c - K, b1 = lw.c + K;
    if (b0 < 0) b0 = 0;
    if (b1 > n - 1) b1 = n - 1;
    lw.b0 = b0;
    lw.nb = b1 >= b0 ? b1 - b0 + 1 : 0;
    return lw;
}

// Mean of sinc^2 over [xc - dx/2, xc + dx/2] by its midpoint Taylor series
// f + f2 dx^2/24 + f4 dx^4/1920 + f6 dx^6/322560, f = (1 - cos 2 pi x)/(2 pi^2 x^2),
// with the derivatives by the Leibniz rule on (1 - cos 2 pi x) and x^-2
// (montecarlo/spectrum/cxr/_bin_quadrature.py:179-221, the reference's
// device bin mean, on by default there). Valid for dx <= 0.1 and |xc| >= 2, where the omitted term is below
// 2.5e-9 of the envelope 1/(2 pi^2 xc^2).
template <bool kMixed>
__device__ __forceinline__ double sincsq_midpoint_mean(double xc, double dx) {
    using R = typename std::conditional<kMixed, float, double>::type;
    // sin(pi xc), cos(pi xc) from the argument reduced to [-1, 1] in double.
    R sp, cp;
    if constexpr (kMixed) {
        // Reduce to [-1, 1] exactly in double before the float argument.
        const double red = xc - 2.0 * rint(0.5 * xc);
        __sincosf((float)(kPi * red), &sp, &cp);
    } else {
        sincospi(xc, &sp, &cp);
    }
    const R om = (R)(2.0 * kPi);
    const R a0 = (R)2 * sp * sp;
    const R s2 = (R)2 * sp * cp;
    const R c2 = (cp - sp) * (cp + sp);
    const R a1 = om * s2, a2 = om * om * c2;
    const R om3 = om * om * om;
    const R a3 = -om3 * s2, a4 = -om3 * om * c2;
    const R a5 = om3 * om * om * s2, a6 = om3 * om3 * c2;
    R q;
    if constexpr (kMixed) q = __frcp_rn((float)xc);
    else q = 1.0 / xc;
    const R h0 = q * q;
    const R h1 = (R)-2 * h0 * q;
    const R h2 = (R)-3 * h1 * q;
    const R h3 = (R)-4 * h2 * q;
    const R h4 = (R)-5 * h3 * q;
    const R h5 = (R)-6 * h4 * q;
    const R h6 = (R)-7 * h5 * q;
    const R f0 = a0 * h0;
    const R f2 = a2 * h0 + (R)2 * a1 * h1 + a0 * h2;
    const R f4 = a4 * h0 + (R)4 * a3 * h1 + (R)6 * a2 * h2 + (R)4 * a1 * h3 + a0 * h4;
    const R f6 = a6 * h0 + (R)6 * a5 * h1 + (R)15 * a4 * h2 + (R)20 * a3 * h3 + (R)15 * a2 * h4 +
                 (R)6 * a1 * h5 + a0 * h6;
    const R d2 = (R)(dx * dx);
    const R series = f0 + d2 * (f2 * (R)(1.0 / 24.0) + d2 * (f4 * (R)(1.0 / 1920.0) + d2 * (f6 * (R)(1.0 / 322560.0))));
    return (double)series * kInv2Pi2;
}

// Per-line constants of the deposit: s = a / pi converts energy to
// first-zero units and scale = w pi / a turns a bin's mass into its weighted
// mean; both are formed once per line, so a bin on a uniform axis costs no
// FP64 division beyond the far-envelope reciprocal.
struct LineDep {
    double E_r, s, scale;
};

// The far envelope this line's moments already spread onto bin b (more than
// K_far bins from the centre), which the exact window takes back out:
// w / (2 a^2) / ((E_lo - E_r)(E_hi - E_r)) = (w / (2 pi^2)) / (x_lo x_hi).
template <bool kMixed>
__device__ __forceinline__ double far_correction(const LineDep &L, int b, const LineWindow &lw, const BinAxis &ax,
                                                 int K_far, double e0, double e1) {
    if (!(lw.mom && (b - lw.c > K_far || lw.c - b > K_far))) return 0.0;
    const double E_c = centre_of(ax, lw.c);
    return (L.scale * L.s) * kInv2Pi2 *
           far_envelope<kMixed>(L.s * (e0 - E_c), L.s * (e1 - E_c), L.s * (L.E_r - E_c));
}

// Exact-window classes of a bin. The cheap ones are evaluated where they are
// found; the others are queued so that a warp evaluates one kind at a time.
enum BinClass { kBinDone = 0, kBinExact = 1, kBinExactCf = 2 };

// Evaluates bin b of a line when it is cheap: the midpoint series for a bin
// much narrower than the line, the far closed form when both edges lie past
// the asymptotic threshold on one side (ec carries the shared edge between
// consecutive such bins). Otherwise returns the class of exact work it needs:
// kBinExactCf when an edge falls in the continued-fraction range of Si.
template <bool kMixed>
__device__ __forceinline__ int bin_fast(const LineDep &L, int b, const LineWindow &lw, const BinAxis &ax,
                                        int K_far, EdgeCache &ec, double &v) {
    const double e0 = ax.edges[b], e1 = ax.edges[b + 1];
    const double x_lo = L.s * (e0 - L.E_r), x_hi = L.s * (e1 - L.E_r);
    const double dxw = L.s * (e1 - e0);
    const double xc = 0.5 * (x_lo + x_hi);
    if (dxw <= 0.1 && fabs(xc) >= 2.0) {
        ec.valid = false;
        v = (L.scale * L.s) * sincsq_midpoint_mean<kMixed>(xc, dxw);
    } else {
        constexpr double u_lim = kMixed ? 24.0 : 48.0;
        const double u_min = 2.0 * kPi * fmin(fabs(x_lo), fabs(x_hi));
        if (!((x_lo > 0.0 || x_hi < 0.0) && u_min >= u_lim)) {
            ec.valid = false;
            const double t_lo = 2.0 * kPi * fabs(x_lo), t_hi = 2.0 * kPi * fabs(x_hi);
            const bool cf = (t_lo > 13.0 && t_lo < 40.0) || (t_hi > 13.0 && t_hi < 40.0);
            return cf ? kBinExactCf : kBinExact;
        }
        EdgeCache lo_e;
        if (ec.valid && ec.x == x_lo) {
            lo_e = ec;
        } else {
            lo_e.valid = true;
            lo_e.x = x_lo;
            lo_e.has_r = lo_e.has_q = false;
        }
        EdgeCache hi_e;
        hi_e.valid = true;
        hi_e.x = x_hi;
        hi_e.has_r = hi_e.has_q = false;
        const double mass = bin_mass<kMixed>(lo_e, hi_e);
        ec = hi_e;
        const double inv_width = ax.uniform ? ax.inv_w : 1.0 / (e1 - e0);
        v = mass * L.scale * inv_width;
    }
    v -= far_correction<kMixed>(L, b, lw, ax, K_far, e0, e1);
    return kBinDone;
}

// Bin b of a line by the difference of sinc^2 antiderivatives at its edges.
template <bool kMixed>
__device__ __forceinline__ double bin_exact(const LineDep &L, int b, const LineWindow &lw, const BinAxis &ax,
                                            int K_far) {
    const double e0 = ax.edges[b], e1 = ax.edges[b + 1];
    EdgeCache lo_e, hi_e;
    lo_e.valid = hi_e.valid = true;
    lo_e.x = L.s * (e0 - L.E_r);
    hi_e.x = L.s * (e1 - L.E_r);
    lo_e.has_r = lo_e.has_q = hi_e.has_r = hi_e.has_q = false;
    const double mass = bin_mass<kMixed>(lo_e, hi_e);
    const double inv_width = ax.uniform ? ax.inv_w : 1.0 / (e1 - e0);
    return mass * L.scale * inv_width - far_correction<kMixed>(L, b, lw, ax, K_far, e0, e1);
}

// ---- mixed path: the cheap classes entirely in float ----------------------
// The line's E_r is float on this path already, so first-zero coordinates in
// float lose nothing further: |x| < ~2^8 in any window keeps ~1e-5 absolute.
struct EdgeCacheF {
    bool valid, has_r;
    float x, q, r;  // q = Q(2 pi |x|) of the far form, r = R(x)
    float iu;       // far form: 1 / (2 pi |x|) of the cached edge
    float ia;       // far correction: 1 / (s (edge - E_c)) of the cached edge (0: unset)
};

// Reciprocal on the SFU alone (rcp.approx, about 1 ulp): the mixed path's
// bin forms carry float rounding far below their tolerance.
__device__ __forceinline__ float rcp_fast(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Q(2 pi |x|) of q_osc_x_f32 with its reciprocal 1 / (2 pi |x|) returned in iu.
__device__ __forceinline__ float q_osc_iu_f32(float x, float &iu) {
    const float ax = fabsf(x);
    const float inv_u = rcp_fast(6.28318530717958648f * ax);
    iu = inv_u;
    const float yf = inv_u * inv_u;
    const float p1 = yf * (2.0f + yf * (-24.0f + yf * (720.0f + yf * (-40320.0f + yf * 3628800.0f))));
    const float p2 = 1.0f + yf * (-6.0f + yf * (120.0f + yf * (-5040.0f + yf * 362880.0f)));
    float sn, cs;
    __sincosf(6.28318530717958648f * (ax - rintf(ax)), &sn, &cs);
    return cs * p1 * inv_u - sn * p2 * yf;
}

// R(x) = F(x) - sign(x)/2 of sincsq_tail in float:
// Si(t) - pi/2 = -f(t) cos t - g(t) sin t with t = 2 pi |x| and the rational
// auxiliary functions of Abramowitz & Stegun 5.2.38-5.2.39 (|error| < 5e-7 for
// t >= 1); its Maclaurin series below t = 1.
__device__ __forceinline__ float sincsq_tail_f32(float x) {
    const float u = fabsf(x);
    const float red = u - rintf(u);
    float sp, cp;
    __sincosf(3.14159265358979324f * red, &sp, &cp);  // sin(pi u) up to sign
    const float t = 6.28318530717958648f * u;
    const float t2 = t * t;
    float si_m;  // Si(t) - pi/2
    if (t < 1.0f) {
        si_m = t * (1.0f + t2 * (-1.0f / 18.0f + t2 * (1.0f / 600.0f + t2 * (-1.0f / 35280.0f + t2 * (1.0f / 3265920.0f))))) -
               1.57079632679489662f;
    } else {
        const float f = __fdividef(t2 * (t2 * (t2 * (t2 + 38.027264f) + 265.187033f) + 335.677320f) + 38.102495f,
                                   (t2 * (t2 * (t2 * (t2 + 40.021433f) + 322.624911f) + 570.236280f) + 157.105423f) * t);
        const float g = __fdividef(t2 * (t2 * (t2 * (t2 + 42.242855f) + 302.757865f) + 352.018498f) + 21.821899f,
                                   (t2 * (t2 * (t2 * (t2 + 48.196927f) + 482.485984f) + 1114.978885f) + 449.690326f) * t2);
        const float sin_t = 2.0f * sp * cp, cos_t = (cp - sp) * (cp + sp);
        si_m = -f * cos_t - g * sin_t;
    }
    const float lobe = u > 0.0f ? __fdividef(sp * sp, 9.86960440108935862f * u) : 0.0f;
    const float r = si_m * (float)kInvPi - lobe;
    return x >= 0.0f ? r : -r;
}

// Q(2 pi |x|) of q_osc_f32 with the phase reduced in float.
__device__ __forceinline__ float q_osc_x_f32(float x) {
    const float u = 6.28318530717958648f * fabsf(x);
    const float inv_u = __frcp_rn(u);
    const float yf = inv_u * inv_u;
    const float p1 = yf * (2.0f + yf * (-24.0f + yf * (720.0f + yf * (-40320.0f + yf * 3628800.0f))));
    const float p2 = 1.0f + yf * (-6.0f + yf * (120.0f + yf * (-5040.0f + yf * 362880.0f)));
    // sin u, cos u with u = 2 pi |x|: reduce |x| to [-1/2, 1/2] turns.
    const float ax = fabsf(x);
    const float red = ax - rintf(ax);
    float sn, cs;
    __sincosf(6.28318530717958648f * red, &sn, &cs);
    return cs * p1 * inv_u - sn * p2 * yf;
}

// Mean of sinc^2 over a bin of width dx in first-zero units centred on xc
// (the midpoint series of sincsq_midpoint_mean), in float.
__device__ __forceinline__ float sincsq_midpoint_mean_f32(float xc, float dx) {
    const float red = xc - 2.0f * rintf(0.5f * xc);
    float sp, cp;
    __sincosf(3.14159265358979324f * red, &sp, &cp);
    const float om = 6.28318530717958648f;
    const float a0 = 2.0f * sp * sp;
    const float s2 = 2.0f * sp * cp;
    const float c2 = (cp - sp) * (cp + sp);
    const float a1 = om * s2, a2 = om * om * c2;
    const float om3 = om * om * om;
    const float a3 = -om3 * s2, a4 = -om3 * om * c2;
    const float a5 = om3 * om * om * s2, a6 = om3 * om3 * c2;
    const float q = __frcp_rn(xc);
    const float h0 = q * q;
    const float h1 = -2.0f * h0 * q;
    const float h2 = -3.0f * h1 * q;
    const float h3 = -4.0f * h2 * q;
    const float h4 = -5.0f * h3 * q;
    const float h5 = -6.0f * h4 * q;
    const float h6 = -7.0f * h5 * q;
    const float f0 = a0 * h0;
    const float f2 = a2 * h0 + 2.0f * a1 * h1 + a0 * h2;
    const float f4 = a4 * h0 + 4.0f * a3 * h1 + 6.0f * a2 * h2 + 4.0f * a1 * h3 + a0 * h4;
    const float f6 = a6 * h0 + 6.0f * a5 * h1 + 15.0f * a4 * h2 + 20.0f * a3 * h3 + 15.0f * a2 * h4 +
                     6.0f * a1 * h5 + a0 * h6;
    const float d2 = dx * dx;
    const float series = f0 + d2 * (f2 * (1.0f / 24.0f) + d2 * (f4 * (1.0f / 1920.0f) + d2 * (f6 * (1.0f / 322560.0f))));
    return series * (float)kInv2Pi2;
}

// Bin b of a line on the mixed path, every class in float (always returns
// kBinDone): edges_f is the float copy of the bin edges, c the line's centre
// bin when its far field goes through the moments (else INT_MIN), E_c that
// bin's centre.
__device__ __forceinline__ int bin_fast_f32(float E_r, float s, float scale, int b, int c, float E_c,
                                            const float *edges_f, bool uniform, float inv_w, int K_far,
                                            EdgeCacheF &ec, float &v) {
    const float e0 = edges_f[b], e1 = edges_f[b + 1];
    const float x_lo = s * (e0 - E_r), x_hi = s * (e1 - E_r);
    const float dxw = s * (e1 - e0);
    const float xc = 0.5f * (x_lo + x_hi);
    const float w = scale * s;
    const bool consec = ec.valid && ec.x == x_lo;  // the previous bin of this line, cached
    if (dxw <= 0.1f && fabsf(xc) >= 2.0f) {
        ec.valid = false;
        v = w * sincsq_midpoint_mean_f32(xc, dxw);
    } else {
        // Far closed form (u_lim = 24): both edges past 24 / (2 pi) on one side.
        constexpr float x_lim = (float)(24.0 / (2.0 * kPi));
        const bool cached = ec.valid && ec.x == x_lo;
        float mass;
        if (!((x_lo > 0.0f && x_lo >= x_lim) || (x_hi < 0.0f && -x_hi >= x_lim))) {
            // Difference of antiderivatives.
            const float r_lo = (cached && ec.has_r) ? ec.r : sincsq_tail_f32(x_lo);
            const float r_hi = sincsq_tail_f32(x_hi);
            ec.valid = true;
            ec.has_r = true;
            ec.x = x_hi;
            ec.r = r_hi;
            mass = r_hi - r_lo + ((x_lo < 0.0f && x_hi >= 0.0f) ? 1.0f : 0.0f);
        } else {
            // Far closed form: the envelope (1/lo - 1/hi) / (2 pi^2) from the
            // edges' reciprocals 1/(2 pi |x|), which the phase terms need
            // anyway, plus the oscillation (Q(hi) - Q(lo)) / pi.
            const bool reuse = cached && !ec.has_r;
            float iu_lo, iu_hi;
            const float q_lo = reuse ? ec.q : q_osc_iu_f32(x_lo, iu_lo);
            if (reuse) iu_lo = ec.iu;
            const float q_hi = q_osc_iu_f32(x_hi, iu_hi);
            ec.valid = true;
            ec.has_r = false;
            ec.x = x_hi;
            ec.q = q_hi;
            ec.iu = iu_hi;
            const bool pos = x_lo > 0.0f;
            const float env = (pos ? (iu_lo - iu_hi) : (iu_hi - iu_lo)) * (float)kInvPi;
            const float osc = pos ? (q_hi - q_lo) : (q_lo - q_hi);
            mass = env + osc * (float)kInvPi;
        }
        v = mass * scale * (uniform ? inv_w : __frcp_rn(e1 - e0));
    }
    if (c != INT_MIN && (b - c > K_far || c - b > K_far)) {
        // The envelope the moments spread here: with ra = 1/A, rb = 1/B,
        // A = s (e0 - E_c), B = s (e1 - E_c), r = ra rb:
        // r + d (r (ra + rb) + d r (ra^2 + ra rb + rb^2)), d = s (E_r - E_c).
        const float ra = (consec && ec.ia != 0.0f) ? ec.ia : rcp_fast(s * (e0 - E_c));
        const float rb = rcp_fast(s * (e1 - E_c));
        ec.ia = rb;
        const float d = s * (E_r - E_c);
        const float r = ra * rb;
        const float f1 = r * (ra + rb);
        const float f2 = r * fmaf(ra, ra + rb, rb * rb);
        v -= w * (float)kInv2Pi2 * (r + d * (f1 + d * f2));
    } else {
        ec.ia = 0.0f;
    }
    return kBinDone;
}

__device__ __forceinline__ void smem_add(float *p, float v) {
    asm volatile("red.shared.add.f32 [%0], %1;" ::"r"((uint32_t)__cvta_generic_to_shared(p)), "f"(v) : "memory");
}
__device__ __forceinline__ void smem_add(double *p, double v) {
    asm volatile("red.shared.add.f64 [%0], %1;" ::"r"((uint32_t)__cvta_generic_to_shared(p)), "d"(v) : "memory");
}

// A kept line's three far-field moments about its centre bin, added to the
// direction's moments in global memory (L2 reductions: a few per kept line,
// so the block keeps no on-chip copy of the moment array).
__device__ __forceinline__ void line_moments(double E_r, double a, double w, const LineWindow &lw,
                                             const BinAxis &ax, double *mom) {
    const int slot = lw.c + ax.pad;
    const double m = w / (2.0 * a * a);
    const double dd = E_r - centre_of(ax, lw.c);
    atomicAdd(&mom[3 * slot + 0], m);
    atomicAdd(&mom[3 * slot + 1], m * dd);
    atomicAdd(&mom[3 * slot + 2], m * dd * dd);
}

// Persistent blocks over the flattened (direction, segment tile) work, in
// contiguous ranges, so the grid is an exact multiple of the SM count; a
// block flushes its on-chip spectrum whenever its direction changes.
// Per pass (a segment tile x a chunk of reflection rows):
//   A0  a cheap prefilter drops pairs whose resonance cannot reach the keep
//       window and compacts the survivors into a shared queue (warp ballot);
//   A1  the full chain runs densely over the survivors and pushes kept lines
//       onto a second shared queue;
//   B   the queued lines' (line, bin) work is cut into 4-item chunks spread
//       over the block; edges shared by consecutive bins are evaluated once.
template <class Real, bool kLayered>
__global__ void __launch_bounds__(kCxrThreads, 2) cxr_kernel(const pb_cxr_args a, int K_far, int far_pad) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr bool kMixed = sizeof(Real) == 4;
    const int n_g = a.tables.n_g;
    const int n_tab = a.tables.n_tab;
    const int n_mu = a.tables.n_mu;
    const bool binmean = a.quadrature == PB_QUAD_BINMEAN;
    const int n_E = a.n_E;
    int64_t n_seg = a.n_seg;
    if (a.n_seg_device) n_seg = (int64_t)*a.n_seg_device;
    if (n_seg > a.n_seg && a.n_seg > 0) n_seg = a.n_seg;

    // Shared layout: [rows][segs][queues][tables][spec][moments][float spec]
    unsigned char *cur = smem_raw;
    RowPre<Real> *rows = reinterpret_cast<RowPre<Real> *>(cur);
    constexpr int kRowChunk = row_chunk<Real>();
    constexpr int kQueue = pair_queue<Real>();
    cur += sizeof(RowPre<Real>) * kRowChunk;
    SegPre<Real> *segs = reinterpret_cast<SegPre<Real> *>(cur);
    cur += sizeof(SegPre<Real>) * kSegTile;
    cur = (unsigned char *)(((uintptr_t)cur + 15) & ~(uintptr_t)15);
    Real *qE = reinterpret_cast<Real *>(cur);
    Real *qA = qE + kQueue;
    Real *qW = qA + kQueue;
    int *qStart = reinterpret_cast<int *>(qW + kQueue);   // kQueue + 1 prefix entries
    int *qB0 = qStart + kQueue + 1;
    int *qC = qB0 + kQueue;
    int *pq = qC + kQueue;                                  // surviving pair ids
    int *scratch = pq + kQueue;                             // warp sums + counters
    int *xq = scratch + 64;                                 // exact bins: [plain | continued fraction]
    // (the float path evaluates every bin class in place: no exact-bin queue)
    cur = reinterpret_cast<unsigned char *>(xq + ((binmean && !kMixed) ? 2 * kXQueue : 0));
    cur = (unsigned char *)(((uintptr_t)cur + 15) & ~(uintptr_t)15);
    const bool tab_smem = n_tab <= kMaxTab;
    Real *E_tab_s = reinterpret_cast<Real *>(cur);
    Real *delta_s = E_tab_s + (tab_smem ? n_tab : 0);
    Real *logmu_s = delta_s + (tab_smem ? n_tab : 0);
    Real *dtail_s = logmu_s + (tab_smem ? n_tab * n_mu : 0);
    const bool has_dtail = kMixed && tab_smem && a.tables.delta_tail_absmax != nullptr && a.pair_E == nullptr;
    cur = reinterpret_cast<unsigned char *>(dtail_s + (tab_smem ? n_tab : 0));
    cur = (unsigned char *)(((uintptr_t)cur + 15) & ~(uintptr_t)15);
    double *spec_s = reinterpret_cast<double *>(cur);
    const int n_mom = n_E + 2 * far_pad;
    float *spec_f = reinterpret_cast<float *>(spec_s + (binmean ? n_E : 0));
    float *edges_f = spec_f + (binmean ? n_E : 0);  // mixed path: float bin edges
    // Layered absorber: per-segment escape pieces, layer thicknesses and bounds.
    unsigned char *esc_raw = reinterpret_cast<unsigned char *>(edges_f + (binmean && kMixed ? n_E + 1 : 0));
    esc_raw = (unsigned char *)(((uintptr_t)esc_raw + 15) & ~(uintptr_t)15);
    EscSeg<Real> *esc = reinterpret_cast<EscSeg<Real> *>(esc_raw);
    double *lay_zt = reinterpret_cast<double *>(esc + (kLayered ? kSegTile : 0));
    double *lay_zb = lay_zt + (kLayered ? kMaxEscLayers : 0);
    Real *lay_t = reinterpret_cast<Real *>(lay_zb + (kLayered ? kMaxEscLayers : 0));
    int &q_count = scratch[40];
    int &p_count = scratch[42];
    int *xq_count = scratch + 44;  // two counters
    // A queued bin packs (line, bin) as line << 21 | bin.
    const bool use_xq = n_E < (1 << 21);

    const int tid = threadIdx.x;
    const unsigned lane = tid & 31u;
    if (tab_smem) {
        for (int j = tid; j < n_tab; j += blockDim.x) {
            E_tab_s[j] = (Real)a.tables.E_tab[j];
            delta_s[j] = (Real)a.tables.delta[j];
            if (has_dtail) dtail_s[j] = (Real)a.tables.delta_tail_absmax[j];
        }
        for (int j = tid; j < n_tab * n_mu; j += blockDim.x) logmu_s[j] = (Real)a.tables.log_mu[j];
    }
    const Real *dtail = has_dtail ? dtail_s : nullptr;
    if (binmean) {
        for (int j = tid; j < n_E; j += blockDim.x) { spec_s[j] = 0.0; spec_f[j] = 0.0f; }
        if (kMixed)
            for (int j = tid; j <= n_E; j += blockDim.x) edges_f[j] = (float)a.edges[j];
    }
    if (tid == 0) { q_count = 0; p_count = 0; xq_count[0] = 0; xq_count[1] = 0; }
    if constexpr (kLayered) {
        if (tid < a.n_layer) {
            lay_zt[tid] = a.z_top[tid];
            lay_zb[tid] = a.z_bot[tid];
            lay_t[tid] = (Real)(a.z_bot[tid] - a.z_top[tid]);
        }
        if (tid == 0) {
            // Contiguous layers in depth order, as the pieces assume.
            int bad = 0;
            for (int k = 0; k < a.n_layer; ++k) {
                if (!(a.z_bot[k] > a.z_top[k])) bad = 1;
                if (k + 1 < a.n_layer && fabs(a.z_bot[k] - a.z_top[k + 1]) > 1e-9 * fmax(1.0, fabs(a.z_bot[k])))
                    bad = 1;
            }
            scratch[46] = bad;
            if (bad && a.status) atomicOr(a.status, PB_DEV_BAD_INPUT);
        }
    }
    const Real *E_tab = tab_smem ? E_tab_s : reinterpret_cast<const Real *>(a.tables.E_tab);
    const Real *delta_tab = tab_smem ? delta_s : reinterpret_cast<const Real *>(a.tables.delta);
    const Real *log_mu = tab_smem ? logmu_s : reinterpret_cast<const Real *>(a.tables.log_mu);

    TabIndex ti{};
    ti.geometric = a.tables.tab_log_step > 0.0;
    ti.log0 = a.tables.tab_log0;
    ti.inv_h = ti.geometric ? 1.0 / a.tables.tab_log_step : 0.0;

    BinAxis ax{};
    if (binmean) {
        ax.edges = a.edges;
        ax.n = n_E;
        ax.uniform = K_far > 0;  // the launcher enables moments on uniform axes only
        ax.lo = a.edges[0];
        ax.w = (a.edges[n_E] - a.edges[0]) / n_E;
        ax.inv_w = 1.0 / ax.w;
        ax.pad = far_pad;
    }
    __syncthreads();
    if (kLayered && scratch[46]) return;

    const int64_t n_tiles = (n_seg + kSegTile - 1) / kSegTile;
    const int64_t n_work = n_tiles * a.n_dir;
    const int64_t w_begin = n_work * blockIdx.x / gridDim.x;
    const int64_t w_end = n_work * (blockIdx.x + 1) / gridDim.x;
    const bool pairs_out = a.pair_E != nullptr;
    const bool lines_out = a.line_E != nullptr;
    const double exact_widths = K_far > 0 ? a.exact_widths : 0.0;
    const int n_warps = blockDim.x >> 5;
    int d_cur = -1;

    auto flush = [&](int d) {
        // Publish (and clear) the block's spectrum of direction d.
        __syncthreads();
        if (binmean && d >= 0) {
            double *gspec = a.spec + (int64_t)d * n_E;
            for (int j = tid; j < n_E; j += blockDim.x) {
                if (spec_s[j] != 0.0) atomicAdd(&gspec[j], spec_s[j]);
                spec_s[j] = 0.0;
            }
        }
        __syncthreads();
    };

    for (int64_t wk = w_begin; wk < w_end; ++wk) {
        const int d = (int)(wk / n_tiles);
        const int64_t tile = wk - (int64_t)d * n_tiles;
        if (d != d_cur) {
            flush(d_cur);
            d_cur = d;
        }
        const double *nh = a.n_hat + 3 * d;
        const int64_t s0 = tile * kSegTile;
        const int nst = (int)((n_seg - s0) < kSegTile ? (n_seg - s0) : kSegTile);
        __syncthreads();
        if (tid < nst) seg_precompute<Real>(segs[tid], a, s0 + tid, nh);
        if constexpr (kLayered) {
            if (tid < nst) esc_precompute<Real>(esc[tid], a, s0 + tid, nh, lay_zt, lay_zb);
        }
        for (int g0 = 0; g0 < n_g; g0 += kRowChunk) {
            const int ng = (n_g - g0) < kRowChunk ? (n_g - g0) : kRowChunk;
            // q / ng for the pass's pair ids q < kSegTile * ng by a multiply-high:
            // magic = floor((2^32 - 1) / ng) + 1 is at least 2^32 / ng and
            // exceeds it by under one, so q magic / 2^32 lies in
            // [q / ng, q / ng + q / 2^32) and its floor is exact for q < 2^32 / ng.
            const unsigned ng_magic = (unsigned)(0xFFFFFFFFull / (unsigned)ng) + 1u;
            __syncthreads();
            for (int j = tid; j < ng; j += blockDim.x) {
                const int g = g0 + j;
                RowPre<Real> &r = rows[j];
                const double *G = a.tables.G + 3 * g;
                const double *ES = a.tables.ES + 3 * ((int64_t)d * n_g + g);
                const double *EP = a.tables.EP + 3 * ((int64_t)d * n_g + g);
                for (int c = 0; c < 3; ++c) {
                    r.G[c] = (Real)G[c];
                    r.ES[c] = (Real)ES[c];
                    r.EP[c] = (Real)EP[c];
                }
                r.g2 = r.G[0] * r.G[0] + r.G[1] * r.G[1] + r.G[2] * r.G[2];
                r.n_dot_g = r.G[0] * (Real)nh[0] + r.G[1] * (Real)nh[1] + r.G[2] * (Real)nh[2];
                r.g_dot_es = r.G[0] * r.ES[0] + r.G[1] * r.ES[1] + r.G[2] * r.ES[2];
                r.g_dot_ep = r.G[0] * r.EP[0] + r.G[1] * r.EP[1] + r.G[2] * r.EP[2];
                r.wm = (Real)a.tables.WM[g];
                r.row = a.tables.row_table[g];
            }
            __syncthreads();
            // ---- A0: prefilter and compact the surviving pairs ----
            const int n_pairs = nst * ng;
            int n_surv;
            if (dtail != nullptr) {
                const int n_it0 = (n_pairs + (int)blockDim.x - 1) / (int)blockDim.x;
                for (int it = 0; it < n_it0; ++it) {
                    const int q = it * blockDim.x + tid;
                    bool ok = false;
                    if (q < n_pairs) {
                        const int si = (int)__umulhi((unsigned)q, ng_magic);
                        ok = pair_may_keep<Real>(segs[si], rows[q - si * ng], E_tab, dtail, n_tab, a.tables, ti);
                    }
                    const unsigned mask = __ballot_sync(0xffffffffu, ok);
                    int base = 0;
                    if (lane == 0 && mask) base = atomicAdd(&p_count, __popc(mask));
                    base = __shfl_sync(0xffffffffu, base, 0);
                    if (ok) pq[base + __popc(mask & ((1u << lane) - 1u))] = q;
                }
                __syncthreads();
                n_surv = p_count;
            } else {
                n_surv = n_pairs;
            }
            // ---- A1: the full chain over the survivors ----
            const int n_it1 = (n_surv + (int)blockDim.x - 1) / (int)blockDim.x;
            for (int it = 0; it < n_it1; ++it) {
                const int k = it * blockDim.x + tid;
                Line<Real> ln;
                ln.good = false;
                if (k < n_surv) {
                    const int q = dtail != nullptr ? pq[k] : k;
                    const int si = (int)__umulhi((unsigned)q, ng_magic);
                    const int gi = q - si * ng;
                    ln = pair_line<Real, kLayered>(segs[si], rows[gi], E_tab, delta_tab, log_mu, n_tab, n_mu,
                                                   a.tables, ti, esc + si, a, lay_t);
                    if (pairs_out) {
                        const int64_t o = ((int64_t)d * n_seg + s0 + si) * n_g + g0 + gi;
                        a.pair_E[o] = (double)ln.E_res;
                        a.pair_a[o] = (double)ln.a_width;
                        a.pair_w[o] = (double)ln.weight;
                        a.pair_good[o] = ln.good ? 1 : 0;
                    }
                    if (ln.good && lines_out) {
                        const unsigned long long slot = atomicAdd(a.line_count, 1ULL);
                        if (slot < (unsigned long long)a.line_capacity) {
                            a.line_E[slot] = (double)ln.E_res;
                            a.line_a[slot] = (double)ln.a_width;
                            a.line_w[slot] = (double)ln.weight;
                            a.line_dir[slot] = d;
                            if (a.line_seg) a.line_seg[slot] = s0 + si;
                        } else {
                            set_status(a.status, PB_DEV_QUEUE_OVERFLOW);
                        }
                    }
                }
                if (binmean) {
                    const unsigned mask = __ballot_sync(0xffffffffu, ln.good);
                    int base = 0;
                    if (lane == 0 && mask) base = atomicAdd(&q_count, __popc(mask));
                    base = __shfl_sync(0xffffffffu, base, 0);
                    if (ln.good) {
                        const int kk = base + __popc(mask & ((1u << lane) - 1u));
                        qE[kk] = ln.E_res;
                        qA[kk] = ln.a_width;
                        qW[kk] = ln.weight;
                    }
                }
            }
            if (!binmean) {
                __syncthreads();
                if (tid == 0) p_count = 0;
                continue;
            }
            __syncthreads();
            // ---- B: windows, scan, spread (line, bin) chunks ----
            const int nq = q_count;
            for (int j = tid; j < nq; j += blockDim.x) {
                const LineWindow lw = line_window((double)qE[j], (double)qA[j], ax, exact_widths, K_far,
                                                  K_far > 0);
                qStart[j] = lw.nb;
                qB0[j] = lw.b0;
                qC[j] = lw.mom ? lw.c : INT_MIN;
                if (lw.mom)
                    line_moments((double)qE[j], (double)qA[j], (double)qW[j], lw, ax,
                                 a.far_moments + (int64_t)d * n_mom * 3);
                // From here on qW holds the line's mass-to-mean scale w pi / a.
                qW[j] = (Real)((double)qW[j] * kPi / (double)qA[j]);
            }
            __syncthreads();
            {
                const int per = (nq + (int)blockDim.x - 1) / (int)blockDim.x;
                const int j0 = tid * per;
                int local = 0;
                for (int j = j0; j < j0 + per && j < nq; ++j) local += qStart[j];
                int incl = local;
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, incl, o);
                    if ((int)lane >= o) incl += v;
                }
                if (lane == 31) scratch[tid >> 5] = incl;
                __syncthreads();
                if (tid == 0) {
                    int run = 0;
                    for (int w = 0; w < n_warps; ++w) { const int v = scratch[w]; scratch[w] = run; run += v; }
                    scratch[41] = run;
                }
                __syncthreads();
                int run = scratch[tid >> 5] + incl - local;
                for (int j = j0; j < j0 + per && j < nq; ++j) { const int v = qStart[j]; qStart[j] = run; run += v; }
                __syncthreads();
                if (tid == 0) qStart[nq] = scratch[41];
                __syncthreads();
            }
            const int n_items = qStart[nq];
            if (a.counters && tid == 0) {
                atomicAdd(&a.counters[0], (unsigned long long)nq);
                atomicAdd(&a.counters[1], (unsigned long long)n_items);
            }
            // Each thread walks one contiguous run of (line, bin) items: one
            // line search per pass, line constants held in registers, and
            // consecutive bins of a line share their edge evaluations.
            {
                const int per = (n_items + (int)blockDim.x - 1) / (int)blockDim.x;
                const int i_begin = min(tid * per, n_items);
                const int i_end = min(i_begin + per, n_items);
                int line = 0;
                if (i_begin < i_end) {
                    int lo = 0, hi = nq;  // last line with qStart[line] <= i_begin
                    while (hi - lo > 1) {
                        const int mid = (lo + hi) >> 1;
                        if (qStart[mid] <= i_begin) lo = mid; else hi = mid;
                    }
                    line = lo - 1;
                }
                int next = i_begin, start = 0;
                LineWindow lw{};
                LineDep L{};
                float Er_f = 0.0f, s_f = 0.0f, scale_f = 0.0f, Ec_f = 0.0f;
                EdgeCache ec;
                ec.valid = false;
                EdgeCacheF ecf;
                ecf.valid = false;
                for (int item = i_begin; item < i_end; ++item) {
                    if (item >= next) {
                        do {
                            ++line;
                            next = qStart[line + 1];
                        } while (item >= next);
                        start = qStart[line];
                        lw.c = qC[line];
                        lw.mom = lw.c != INT_MIN;
                        lw.b0 = qB0[line];
                        L = LineDep{(double)qE[line], (double)qA[line] * kInvPi, (double)qW[line]};
                        if constexpr (kMixed) {
                            Er_f = (float)qE[line];
                            s_f = (float)qA[line] * (float)kInvPi;
                            scale_f = (float)qW[line];
                            Ec_f = lw.mom ? (float)centre_of(ax, lw.c) : 0.0f;
                        }
                        ec.valid = false;
                        ecf.valid = false;
                    }
                    const int b = lw.b0 + (item - start);
                    if constexpr (kMixed) {
                        float vf;
                        bin_fast_f32(Er_f, s_f, scale_f, b, lw.c, Ec_f, edges_f, ax.uniform, (float)ax.inv_w, K_far,
                                     ecf, vf);
                        smem_add(&spec_f[b], vf);
                    } else {
                        double v;
                        const int cls = bin_fast<kMixed>(L, b, lw, ax, K_far, ec, v);
                        if (cls != kBinDone) {
                            const int slot = use_xq ? atomicAdd(&xq_count[cls - 1], 1) : kXQueue;
                            if (slot < kXQueue) {
                                xq[(cls - 1) * kXQueue + slot] = (line << 21) | b;
                                continue;
                            }
                            v = bin_exact<kMixed>(L, b, lw, ax, K_far);  // queue full
                        }
                        smem_add(&spec_s[b], v);
                    }
                }
            }
            // Queued exact bins, one class at a time.
            __syncthreads();
            for (int cls = 0; cls < 2; ++cls) {
                const int nx = min(xq_count[cls], kXQueue);
                for (int k = tid; k < nx; k += blockDim.x) {
                    const int packed = xq[cls * kXQueue + k];
                    const int line = packed >> 21;
                    const int b = packed & ((1 << 21) - 1);
                    LineWindow lw;
                    lw.c = qC[line];
                    lw.mom = lw.c != INT_MIN;
                    lw.b0 = qB0[line];
                    const LineDep L{(double)qE[line], (double)qA[line] * kInvPi, (double)qW[line]};
                    const double v = bin_exact<kMixed>(L, b, lw, ax, K_far);
                    if constexpr (kMixed) smem_add(&spec_f[b], (float)v);
                    else smem_add(&spec_s[b], v);
                }
            }
            if constexpr (kMixed) {
                // Fold the float partials into the FP64 spectrum once per
                // segment tile (after its last row chunk, uniform over the
                // block): a tile's few hundred (line, bin) adds per bin keep
                // float well inside the path's tolerance.
                if (g0 + kRowChunk >= n_g) {
                    __syncthreads();
                    for (int j = tid; j < n_E; j += blockDim.x) {
                        const float v = spec_f[j];
                        if (v != 0.0f) { spec_s[j] += (double)v; spec_f[j] = 0.0f; }
                    }
                }
            }
            __syncthreads();
            if (tid == 0) { q_count = 0; p_count = 0; xq_count[0] = 0; xq_count[1] = 0; }
        }
    }
    flush(d_cur);
}

// Far-field finalize: spec[d][b] += sum_c M[d][c] . envelope(b, c) over the
// (padded, uniform) centre bins c farther than K_far bins from b.
__global__ void far_field_kernel(const double *edges, int n_E, int pad, const double *mom,
                                 double *spec, int K_far) {
    const int d = blockIdx.y;
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n_E) return;
    const int n_mom = n_E + 2 * pad;
    const double *m = mom + (int64_t)d * n_mom * 3;
    const double lo = edges[0];
    const double w = (edges[n_E] - edges[0]) / n_E;
    const double E_lo = edges[b], E_hi = edges[b + 1];
    double acc = 0.0;
    for (int slot = 0; slot < n_mom; ++slot) {
        const int c = slot - pad;
        if (c >= b - K_far && c <= b + K_far) continue;
        const double m0 = m[3 * slot];
        if (m0 == 0.0) continue;
        const double E_c = lo + ((double)c + 0.5) * w;
        const double A = E_lo - E_c, B = E_hi - E_c;
        const double AB = A * B;
        const double f0 = 1.0 / AB;
        const double f1 = (A + B) / (AB * AB);
        const double f2 = (A * A + AB + B * B) / (AB * AB * AB);
        acc += m0 * f0 + m[3 * slot + 1] * f1 + m[3 * slot + 2] * f2;
    }
    spec[(int64_t)d * n_E + b] += acc;
}

// The same far field as a convolution on the uniform axis: with the centre
// bin c and the output bin b a distance D = b - c apart, A = (D - 1/2) w and
// B = (D + 1/2) w, so the three expansion coefficients are
//   f0 = r / w^2, f1 = 2 D r^2 / w^3, f2 = (3 D^2 + 1/4) r^3 / w^4,
//   r = 1 / (D^2 - 1/4),
// and r depends on the integer D alone: one table of r per block replaces a
// division per (bin, centre) pair. A block takes 32 output bins of one
// direction; its 8 warps split the centre bins into 8 contiguous slices (a
// warp's lanes read the same centre bin: broadcast loads) and the slices'
// sums are added in slice order, so the result does not depend on the launch.
constexpr int kFarBins = 32;
constexpr int kFarSlices = 8;

// Acc is the accumulation type: double on the FP64 path, float on the mixed
// one (a bin's far field is a sum of positive envelope terms and two small
// corrections, well inside float over 2,100 centres; the slices' partial sums
// and the spectrum stay FP64).
template <class Acc>
__global__ void __launch_bounds__(kFarBins * kFarSlices) far_field_conv_kernel(const double *edges, int n_E, int pad,
                                                                               const double *mom, double *spec,
                                                                               int K_far) {
    extern __shared__ __align__(16) unsigned char far_smem[];
    Acc *sR = reinterpret_cast<Acc *>(far_smem);  // r(D) for D = -n_mom .. n_mom
    __shared__ double part[3][kFarSlices][kFarBins];
    const int d = blockIdx.y;
    const int n_mom = n_E + 2 * pad;
    const double w = (edges[n_E] - edges[0]) / n_E;
    for (int i = threadIdx.x; i <= 2 * n_mom; i += blockDim.x) {
        const double D = (double)(i - n_mom);
        sR[i] = (Acc)(1.0 / (D * D - 0.25));
    }
    __syncthreads();
    const int lane = threadIdx.x % kFarBins, slice = threadIdx.x / kFarBins;
    const int b = blockIdx.x * kFarBins + lane;
    const double *m = mom + (int64_t)d * n_mom * 3;
    const int per = (n_mom + kFarSlices - 1) / kFarSlices;
    const int s0 = slice * per, s1 = min(s0 + per, n_mom);
    Acc acc0 = 0, acc1 = 0, acc2 = 0;
    if (b < n_E) {
        for (int slot = s0; slot < s1; ++slot) {
            const int c = slot - pad;
            if (c >= b - K_far && c <= b + K_far) continue;
            const double m0 = m[3 * slot];
            if (m0 == 0.0) continue;
            const int D = b - c;
            const Acc r = sR[D + n_mom];
            const Acc Dd = (Acc)D;
            acc0 = fma((Acc)m0, r, acc0);
            acc1 = fma((Acc)m[3 * slot + 1], (Acc)2 * Dd * r * r, acc1);
            acc2 = fma((Acc)m[3 * slot + 2], ((Acc)3 * Dd * Dd + (Acc)0.25) * r * r * r, acc2);
        }
    }
    part[0][slice][lane] = (double)acc0;
    part[1][slice][lane] = (double)acc1;
    part[2][slice][lane] = (double)acc2;
    __syncthreads();
    if (slice == 0 && b < n_E) {
        double t0 = 0.0, t1 = 0.0, t2 = 0.0;
#pragma unroll
        for (int k = 0; k < kFarSlices; ++k) {
            t0 += part[0][k][lane];
            t1 += part[1][k][lane];
            t2 += part[2][k][lane];
        }
        const double iw = 1.0 / w;
        const double iw2 = iw * iw, iw3 = iw2 * iw, iw4 = iw2 * iw2;
        spec[(int64_t)d * n_E + b] += t0 * iw2 + t1 * iw3 + t2 * iw4;
    }
}

// Node reduction of buffered lines: spec[d][e] += sum_j w_j sinc^2(x_je),
// x = a (E_e - E_j) / pi, with the phase a (E_e - E_j) formed in double.
template <class Real>
__global__ void node_reduce_kernel(const double *E_grid, int n_E, const double *line_E,
                                   const double *line_a, const double *line_w, const int32_t *line_dir,
                                   const unsigned long long *line_count, int64_t capacity,
                                   double *spec) {
    constexpr int kTile = 256;
    __shared__ double sE[kTile], sA[kTile], sW[kTile];
    __shared__ int sD[kTile];
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    int64_t n_lines = (int64_t)*line_count;
    if (n_lines > capacity) n_lines = capacity;
    const int64_t per = (n_lines + gridDim.y - 1) / gridDim.y;
    const int64_t j0 = per * blockIdx.y;
    const int64_t j1 = j0 + per < n_lines ? j0 + per : n_lines;
    const double E = e < n_E ? E_grid[e] : 0.0;
    // Accumulate per direction seen in this chunk (directions are few).
    double acc = 0.0;
    int cur_dir = -1;
    for (int64_t t0 = j0; t0 < j1; t0 += kTile) {
        const int nt = (int)((j1 - t0) < kTile ? (j1 - t0) : kTile);
        __syncthreads();
        for (int j = threadIdx.x; j < nt; j += blockDim.x) {
            sE[j] = line_E[t0 + j];
            sA[j] = line_a[t0 + j];
            sW[j] = line_w[t0 + j];
            sD[j] = line_dir[t0 + j];
        }
        __syncthreads();
        if (e < n_E) {
            for (int k = 0; k < nt; ++k) {
                if (sD[k] != cur_dir) {
                    if (cur_dir >= 0 && acc != 0.0) atomicAdd(&spec[(int64_t)cur_dir * n_E + e], acc);
                    acc = 0.0;
                    cur_dir = sD[k];
                }
                double x = sA[k] * (E - sE[k]) / kPi;
                if (x == 0.0) x = 1.0e-20;
                double s;
                if constexpr (sizeof(Real) == 8) {
                    const double y = kPi * x;
                    s = sin(y) / y;
                } else {
                    // y = pi x reduced to [-pi, pi] in double, sine in float.
                    const double y = kPi * x;
                    const double r = y - 2.0 * kPi * rint(y / (2.0 * kPi));
                    s = (double)__sinf((float)r) / y;
                }
                acc += sW[k] * (s * s);
            }
        }
    }
    if (e < n_E && cur_dir >= 0 && acc != 0.0) atomicAdd(&spec[(int64_t)cur_dir * n_E + e], acc);
}

template <class Real>
static size_t cxr_smem_bytes(const pb_cxr_args &a, int far_pad, bool with_moments) {
    constexpr int kRowChunk = row_chunk<Real>();
    constexpr int kQueue = pair_queue<Real>();
    size_t b = sizeof(RowPre<Real>) * kRowChunk + sizeof(SegPre<Real>) * kSegTile + 16;
    b += sizeof(Real) * 3 * kQueue + sizeof(int) * (4 * kQueue + 1 + 64) + 16;
    if (a.tables.n_tab <= kMaxTab) b += sizeof(Real) * (size_t)a.tables.n_tab * (3 + a.tables.n_mu);
    b += 16;
    if (a.quadrature == PB_QUAD_BINMEAN) {
        b += (sizeof(double) + sizeof(float)) * (size_t)a.n_E + (sizeof(Real) == 8 ? sizeof(int) * 2 * kXQueue : 0);
        if (sizeof(Real) == 4) b += sizeof(float) * ((size_t)a.n_E + 1) + 16;
    }
    if (a.n_layer > 0)
        b += 16 + sizeof(EscSeg<Real>) * kSegTile + sizeof(double) * 2 * kMaxEscLayers + sizeof(Real) * kMaxEscLayers;
    return b;
}



template <class Real>
static cudaError_t launch_cxr_t(const pb_cxr_args &a, cudaStream_t s, int sms, int far_pad) {
    const bool binmean = a.quadrature == PB_QUAD_BINMEAN;
    const int K_far = (binmean && a.exact_widths > 0.0 && a.far_moments && far_pad >= 0) ? 2 : 0;
    if (K_far == 0) far_pad = 0;
    if (a.n_layer < 0 || a.n_layer > kMaxEscLayers) return cudaErrorInvalidValue;
    if (a.n_layer > 0 && (!a.z_top || !a.z_bot || !a.mu_off || !a.mu_knot || !a.mu_value || !a.mu_slope))
        return cudaErrorInvalidValue;
    size_t smem = cxr_smem_bytes<Real>(a, far_pad, K_far > 0);
    if (smem > 220 * 1024) return cudaErrorInvalidValue;
    // The float path reads its tables from the shared-memory staging only.
    if (sizeof(Real) == 4 && a.tables.n_tab > kMaxTab) return cudaErrorInvalidValue;
    auto kern = a.n_layer > 0 ? cxr_kernel<Real, true> : cxr_kernel<Real, false>;
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    if (K_far > 0) {
        err = cudaMemsetAsync(a.far_moments, 0,
                              sizeof(double) * (size_t)a.n_dir * (a.n_E + 2 * far_pad) * 3, s);
        if (err != cudaSuccess) return err;
    }
    if (a.line_count) {
        err = cudaMemsetAsync(a.line_count, 0, sizeof(unsigned long long), s);
        if (err != cudaSuccess) return err;
    }
    int per_sm = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kCxrThreads, smem);
    if (err != cudaSuccess) return err;
    if (per_sm < 1) per_sm = 1;
    const int64_t work = (a.n_seg + kSegTile - 1) / kSegTile * (int64_t)a.n_dir;
    int64_t gx = (int64_t)sms * per_sm;
    if (gx > work) gx = work;
    if (gx < 1) gx = 1;
    kern<<<(unsigned)gx, kCxrThreads, smem, s>>>(a, K_far, far_pad);
    err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    if (K_far > 0) {
        dim3 fg((unsigned)((a.n_E + 127) / 128), (unsigned)a.n_dir);
        const size_t tab = sizeof(Real) * (2 * ((size_t)a.n_E + 2 * (size_t)far_pad) + 1);
        if (tab <= 200 * 1024) {
            // the moments sit on a uniform axis (far moments are enabled on uniform edges only)
            auto conv = far_field_conv_kernel<Real>;
            err = cudaFuncSetAttribute(conv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tab);
            if (err != cudaSuccess) return err;
            dim3 cg((unsigned)((a.n_E + kFarBins - 1) / kFarBins), (unsigned)a.n_dir);
            conv<<<cg, kFarBins * kFarSlices, tab, s>>>(a.edges, a.n_E, far_pad, a.far_moments, a.spec, K_far);
        } else {
            far_field_kernel<<<fg, 128, 0, s>>>(a.edges, a.n_E, far_pad, a.far_moments, a.spec, K_far);
        }
        err = cudaGetLastError();
        if (err != cudaSuccess) return err;
    }
    if (a.quadrature == PB_QUAD_NODE && a.line_E != nullptr && a.spec != nullptr) {
        dim3 ng((unsigned)((a.n_E + 127) / 128), 64);
        node_reduce_kernel<Real><<<ng, 128, 0, s>>>(a.E_grid, a.n_E, a.line_E, a.line_a, a.line_w,
                                                    a.line_dir, a.line_count, a.line_capacity, a.spec);
        err = cudaGetLastError();
    }
    return err;
}

cudaError_t launch_cxr(const pb_cxr_args &a, cudaStream_t s, int sms) {
    if (a.precision == PB_MIXED) return launch_cxr_t<float>(a, s, sms, a.far_pad);
    return launch_cxr_t<double>(a, s, sms, a.far_pad);
}

// ---------------------------------------------------------------------------
// Coherent route: per-row line records from the segment list (FP64).
//
// For every (segment, reflection row) pair the chain of pair_amps gives the
// complex PXR+CBS amplitude of both polarisations; the record adds the
// segment's escape-piece ends and formation coefficients, the exact vacuum
// line centre and width with the recoil phase over the electron's age, and
// the phase terms (cxr/_batched.py:561-660, cxr/_formation.py:58-81,
// cxr/_recoil.py:118-147, cxr/_setup.py:1023-1026). Rows hold their kept
// pairs in segment order, row after row (row_off), as the reference's block
// loop lays them out and pb_coherent_reduce reads them: pass 1 flags the kept
// pairs [row][segment], pass 2 scans each row, pass 3 writes the records.
// ---------------------------------------------------------------------------
struct CohRec {
    double f[13];  // E_vac, a_vac, phase_slope, g_phase, cs_re, cs_im, cp_re, cp_im, L_esc, half_dL, apb, bma, q
};

// cxr/_formation.py:58-81
__device__ __forceinline__ void formation_coefficients(double tau_start, double tau_end, double &apb, double &bma,
                                                       double &q) {
    q = 0.25 * (tau_end - tau_start);
    if (fabs(q) < 0.5) {
        const double c0 = exp(-0.25 * (tau_start + tau_end));
        apb = 2.0 * c0 * cosh(q);
        bma = -2.0 * c0 * sinh(q);
    } else {
        const double ea = exp(-0.5 * tau_start), eb = exp(-0.5 * tau_end);
        apb = ea + eb;
        bma = eb - ea;
    }
}

__device__ bool coh_record(const pb_cxr_args &a, const double *t_start, int64_t s, int g, const TabIndex &ti,
                           CohRec *rec) {
    SegPre<double> sp;
    seg_precompute<double>(sp, a, s, a.n_hat);
    RowPre<double> rw;
    const double *nh = a.n_hat;
    for (int c = 0; c < 3; ++c) {
        rw.G[c] = a.tables.G[3 * g + c];
        rw.ES[c] = a.tables.ES[3 * g + c];
        rw.EP[c] = a.tables.EP[3 * g + c];
    }
    rw.g2 = rw.G[0] * rw.G[0] + rw.G[1] * rw.G[1] + rw.G[2] * rw.G[2];
    rw.n_dot_g = rw.G[0] * nh[0] + rw.G[1] * nh[1] + rw.G[2] * nh[2];
    rw.g_dot_es = rw.G[0] * rw.ES[0] + rw.G[1] * rw.ES[1] + rw.G[2] * rw.ES[2];
    rw.g_dot_ep = rw.G[0] * rw.EP[0] + rw.G[1] * rw.EP[1] + rw.G[2] * rw.EP[2];
    rw.wm = a.tables.WM[g];
    rw.row = a.tables.row_table[g];
    const int n_tab = a.tables.n_tab;
    const PairAmps<double> p = pair_amps<double, false>(sp, rw, a.tables.E_tab, a.tables.delta, a.tables.log_mu,
                                                        n_tab, a.tables.n_mu, a.tables, ti);
    double apb, bma, qq;
    formation_coefficients(sp.path0 * p.mu, sp.path1 * p.mu, apb, bma, qq);
    // exact vacuum centre / width and recoil phase over the age, with the
    // vacuum denominator and n.g of the row (cxr/_recoil.py:118-147)
    const double numerator = p.v_dot_g - p.r_num;
    const double den = sp.denom_row + p.r_den;
    const double E_c = kHbarcEvAng * numerator / den;
    const double x = numerator / den * sp.inv_E;
    const double kappa = 1.0 / (1.0 - x);
    const double a_vac = kappa * den * sp.t_L / (2.0 * kHbarcEvAng);
    const double t_mid = (t_start ? t_start[s] : 0.0) + 0.5 * sp.t_L;
    const double rx = a.r_mid[3 * s], ry = a.r_mid[3 * s + 1], rz = a.r_mid[3 * s + 2];
    const double d_geom = t_mid - (rx * nh[0] + ry * nh[1] + rz * nh[2]);
    const double d_shift = kappa * (x * sp.denom_row + p.r_den) * t_mid;
    const double g_shift = kappa * (x * p.v_dot_g - p.r_num) * t_mid;
    const double amp = sqrt(kAlphaFs * p.omega / (4.0 * (kPi * kPi) * kHbarcEvAng));
    const double cs_re = amp * sp.t_L * p.A_re[0], cs_im = amp * sp.t_L * p.A_im[0];
    const double cp_re = amp * sp.t_L * p.A_re[1], cp_im = amp * sp.t_L * p.A_im[1];
    const bool good = p.keep && isfinite(amp) && amp > 0.0 && sp.t_L > 0.0 && isfinite(apb) && apb > 0.0 &&
                      isfinite(bma) && isfinite(cs_re) && isfinite(cs_im) && isfinite(cp_re) && isfinite(cp_im);
    if (rec && good) {
        // record fields (cxr/_batched.py:646-660)
        rec->f[0] = E_c;
        rec->f[1] = a_vac;
        rec->f[2] = (d_geom + d_shift) / kHbarcEvAng;
        rec->f[3] = rx * rw.G[0] + ry * rw.G[1] + rz * rw.G[2] + g_shift;
        rec->f[4] = cs_re;
        rec->f[5] = cs_im;
        rec->f[6] = cp_re;
        rec->f[7] = cp_im;
        rec->f[8] = 0.5 * (sp.path0 + sp.path1);
        rec->f[9] = 0.5 * (sp.path1 - sp.path0);
        rec->f[10] = apb;
        rec->f[11] = bma;
        rec->f[12] = qq;
    }
    return good;
}

__device__ __forceinline__ TabIndex tab_index_of(const pb_cxr_tables &t) {
    TabIndex ti{};
    ti.geometric = t.tab_log_step > 0.0;
    ti.log0 = t.tab_log0;
    ti.inv_h = ti.geometric ? 1.0 / t.tab_log_step : 0.0;
    return ti;
}

// Pass 1: kept flags, row-major [g][s].
__global__ void coh_rec_flags_kernel(const pb_cxr_args a, const double *t_start, int64_t n_seg, uint8_t *flags) {
    const TabIndex ti = tab_index_of(a.tables);
    const int n_g = a.tables.n_g;
    const int64_t n = n_seg * (int64_t)n_g;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = q / n_g;
        const int g = (int)(q - s * n_g);
        flags[(int64_t)g * n_seg + s] = coh_record(a, t_start, s, g, ti, nullptr) ? 1 : 0;
    }
}

// Pass 2: exclusive scan of one row's flags (one block per row) and its count.
__global__ void __launch_bounds__(1024) coh_rec_scan_kernel(int64_t n_seg, const uint8_t *flags, int32_t *pos,
                                                           int64_t *count) {
    __shared__ int64_t warp_sum[32];
    __shared__ int64_t carry;
    const int g = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint8_t *f = flags + (int64_t)g * n_seg;
    int32_t *o = pos + (int64_t)g * n_seg;
    if (tid == 0) carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < n_seg; base += 1024) {
        const int64_t s = base + tid;
        const int v = s < n_seg ? f[s] : 0;
        int incl = v;
        for (int d = 1; d < 32; d <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += u;
        }
        if (lane == 31) warp_sum[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            int64_t w = warp_sum[lane];
            int64_t wi = w;
            for (int d = 1; d < 32; d <<= 1) {
                const int64_t u = __shfl_up_sync(0xffffffffu, wi, d);
                if (lane >= d) wi += u;
            }
            warp_sum[lane] = wi - w;  // exclusive prefix of the warps
        }
        __syncthreads();
        const int64_t excl = carry + warp_sum[warp] + incl - v;
        if (s < n_seg) o[s] = (int32_t)excl;
        __syncthreads();
        if (tid == 1023) carry = excl + v;
        __syncthreads();
    }
    if (tid == 0) count[g] = carry;
}

// Row offsets from the counts (one thread: rows are few).
__global__ void coh_rec_offsets_kernel(int n_g, const int64_t *count, int64_t *row_off) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        int64_t run = 0;
        row_off[0] = 0;
        for (int g = 0; g < n_g; ++g) {
            run += count[g];
            row_off[g + 1] = run;
        }
    }
}

// Pass 3: the records of the kept pairs at their row positions.
__global__ void coh_rec_write_kernel(const pb_coherent_records_args r, const uint8_t *flags, const int32_t *pos) {
    const pb_cxr_args &a = r.cxr;
    const TabIndex ti = tab_index_of(a.tables);
    const int n_g = a.tables.n_g;
    const int64_t n_seg = a.n_seg;
    const int64_t n = n_seg * (int64_t)n_g;
    double *const out[13] = {r.E_vac, r.a_vac, r.phase_slope, r.g_phase, r.cs_re, r.cs_im, r.cp_re,
                             r.cp_im, r.L_esc, r.half_dL, r.apb, r.bma, r.q};
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = q / n_g;
        const int g = (int)(q - s * n_g);
        const int64_t fi = (int64_t)g * n_seg + s;
        if (!flags[fi]) continue;
        CohRec rec;
        if (!coh_record(a, r.t_start, s, g, ti, &rec)) continue;
        const int64_t slot = r.row_off[g] + pos[fi];
        if (slot >= r.capacity) {
            set_status(r.status, PB_DEV_QUEUE_OVERFLOW);
            continue;
        }
#pragma unroll
        for (int k = 0; k < 13; ++k) out[k][slot] = rec.f[k];
        if (r.elec_out) r.elec_out[slot] = a.elec_id[s];
    }
}

uint64_t coherent_records_work_bytes(int64_t n_seg, int n_g) {
    const uint64_t pairs = (uint64_t)n_seg * (uint64_t)n_g;
    const auto al = [](uint64_t b) { return (b + 255) / 256 * 256; };
    return al(pairs) + al(pairs * 4) + al((uint64_t)n_g * 8);
}

cudaError_t launch_coherent_records(const pb_coherent_records_args &r, cudaStream_t s, int sms) {
    const int64_t n_seg = r.cxr.n_seg;
    const int n_g = r.cxr.tables.n_g;
    const uint64_t pairs = (uint64_t)n_seg * (uint64_t)n_g;
    const auto al = [](uint64_t b) { return (b + 255) / 256 * 256; };
    uint8_t *flags = static_cast<uint8_t *>(r.work);
    int32_t *pos = reinterpret_cast<int32_t *>(static_cast<uint8_t *>(r.work) + al(pairs));
    int64_t *count = reinterpret_cast<int64_t *>(static_cast<uint8_t *>(r.work) + al(pairs) + al(pairs * 4));
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((int64_t)((pairs + 255) / 256), (int64_t)sms * 8));
    coh_rec_flags_kernel<<<(unsigned)blocks, 256, 0, s>>>(r.cxr, r.t_start, n_seg, flags);
    coh_rec_scan_kernel<<<(unsigned)n_g, 1024, 0, s>>>(n_seg, flags, pos, count);
    coh_rec_offsets_kernel<<<1, 32, 0, s>>>(n_g, count, r.row_off);
    coh_rec_write_kernel<<<(unsigned)blocks, 256, 0, s>>>(r, flags, pos);
    return cudaGetLastError();
}

// Coarse per-pair binning of a line buffer (surrogate training targets).
__global__ void bin_lines_kernel(int64_t n_lines, const double *line_E, const double *line_a, const double *line_w,
                                 const int32_t *line_dir, const int64_t *line_seg, int dir0, int n_dir_chunk,
                                 int64_t n_seg, double lo, double width, int n_bins, float *target) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_lines;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int dl = line_dir[i] - dir0;
        if (dl < 0 || dl >= n_dir_chunk) continue;
        const int64_t pair = (int64_t)dl * n_seg + line_seg[i];
        const double E_r = line_E[i], a = line_a[i];
        const float s = (float)(a / kPi);
        const float scale = (float)(line_w[i] * kPi / a / width);
        const int c = (int)floor((E_r - lo) / width);
        int K = (int)ceil(64.0 * kPi / (a * width));
        K = K < 1 ? 1 : (K > 64 ? 64 : K);
        const int b0 = max(c - K, 0), b1 = min(c + K, n_bins - 1);
        float r_lo = 0.0f;
        for (int b = b0; b <= b1; ++b) {
            const float x_lo = s * (float)(lo + b * width - E_r);
            const float x_hi = s * (float)(lo + (b + 1) * width - E_r);
            if (b == b0) r_lo = sincsq_tail_f32(x_lo);
            const float r_hi = sincsq_tail_f32(x_hi);
            const float m = r_hi - r_lo + ((x_lo < 0.0f && x_hi >= 0.0f) ? 1.0f : 0.0f);
            r_lo = r_hi;
            if (m != 0.0f) atomicAdd(&target[pair * n_bins + b], scale * m);
        }
    }
}

cudaError_t launch_bin_lines(int64_t n_lines, const double *line_E, const double *line_a, const double *line_w,
                             const int32_t *line_dir, const int64_t *line_seg, int dir0, int n_dir_chunk,
                             int64_t n_seg, double lo, double width, int n_bins, float *target, cudaStream_t st) {
    if (n_lines <= 0) return cudaSuccess;
    const int64_t blocks = std::min<int64_t>((n_lines + 255) / 256, 148 * 16);
    bin_lines_kernel<<<(unsigned)blocks, 256, 0, st>>>(n_lines, line_E, line_a, line_w, line_dir, line_seg, dir0,
                                                        n_dir_chunk, n_seg, lo, width, n_bins, target);
    return cudaGetLastError();
}

}  // namespace pb

// ---------------------------------------------------------------------------
// pb_cxr_score_noalloc: the bin-mean scorer for callers that cannot allocate
// device memory (code running inside a host-side allocator or memory-pool
// callback, an embedding runtime that owns all device memory and forbids
// cudaMalloc, or a static-memory deployment that fixes every allocation at
// load time). Its far-field workspace is this file-scope device array; every
// GPU that loads the library reserves it until the process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocFarDoubles = size_t(1) << 18;  // 2 MiB of FP64 moments
static __device__ __align__(256) double g_noalloc_far[kNoAllocFarDoubles];

// The array's device address differs per CUDA context (a module is loaded
// once per context), so the resolved address is cached per context: keyed by
// the driver's context ID, which stays unique for the life of the process --
// a context re-created after cudaDeviceReset, or one the caller made with the
// driver API, gets a new ID and so a fresh lookup. The two driver functions
// are reached through the runtime (cudaGetDriverEntryPoint), so the library
// does not link the driver library directly.
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

struct NoAllocSlot {
    unsigned long long ctx_id;
    double *ptr;
};
constexpr int kNoAllocSlots = 64;

std::mutex g_noalloc_mu;
NoAllocSlot g_noalloc_cache[kNoAllocSlots] = {};
int g_noalloc_next = 0;
bool g_ctx_fns_tried = false;
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;
thread_local char g_noalloc_err[256] = "";

int noalloc_fail(int code, const char *msg) {
    snprintf(g_noalloc_err, sizeof(g_noalloc_err), "%s", msg);
    pb::set_last_error(g_noalloc_err);
    return code;
}

// ID of this thread's current context, making the device's primary context
// current first if none is (cudaSetDevice initialises it). False when the
// driver functions are unavailable or the query fails: the caller then
// resolves the address without the cache.
bool current_ctx_id(int dev, unsigned long long *id) {
    if (!g_ctx_fns_tried) {
        g_ctx_fns_tried = true;
        void *f0 = nullptr, *f1 = nullptr;
        cudaDriverEntryPointQueryResult q0 = cudaDriverEntryPointSymbolNotFound, q1 = q0;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0) == cudaSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
            q0 == cudaDriverEntryPointSuccess && q1 == cudaDriverEntryPointSuccess) {
            g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f0);
            g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f1);
        }
    }
    if (!g_ctx_get_current || !g_ctx_get_id) return false;
    CUcontext ctx = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS) return false;
    if (!ctx) {
        if (cudaSetDevice(dev) != cudaSuccess || g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
    }
    return g_ctx_get_id(ctx, id) == CUDA_SUCCESS;
}

}  // namespace

extern "C" int pb_cxr_score_noalloc(const pb_cxr_args *args, void *stream) {
    if (!args) return noalloc_fail(PB_ERR_INVALID, "pb_cxr_score_noalloc: args is NULL");
    if (args->quadrature != PB_QUAD_BINMEAN)
        return noalloc_fail(PB_ERR_UNSUPPORTED,
                            "pb_cxr_score_noalloc: only bin-mean quadrature (node sampling needs a line buffer)");
    // The same argument checks as pb_cxr_score (the far-field workspace is
    // this file's array, so far_moments may be NULL).
    const int v = pb::validate_cxr(*args, "pb_cxr_score_noalloc", true);
    if (v != PB_OK || args->n_seg == 0) return v;
    const bool far = args->exact_widths > 0.0 && args->far_pad >= 0;
    if (far) {
        const size_t need = (size_t)args->n_dir * ((size_t)args->n_E + 2 * (size_t)args->far_pad) * 3;
        if (need > kNoAllocFarDoubles) {
            char msg[256];
            snprintf(msg, sizeof(msg),
                     "pb_cxr_score_noalloc: the far field needs %zu FP64 moments (n_dir * (n_E + 2 far_pad) * 3), "
                     "over the fixed workspace of %zu; score fewer directions per call",
                     need, kNoAllocFarDoubles);
            return noalloc_fail(PB_ERR_CAPACITY, msg);
        }
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0)
        return noalloc_fail(PB_ERR_CUDA, "pb_cxr_score_noalloc: no current CUDA device");
    double *ws = nullptr;
    {
        // First call in a context: resolve the array's device address (host
        // code must not use the symbol itself as a pointer).
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        unsigned long long cid = 0;
        const bool keyed = current_ctx_id(dev, &cid);
        if (keyed) {
            for (const NoAllocSlot &e : g_noalloc_cache)
                if (e.ptr && e.ctx_id == cid) ws = e.ptr;
        }
        if (!ws) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_far);
            if (e != cudaSuccess) {
                char msg[256];
                snprintf(msg, sizeof(msg), "pb_cxr_score_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
                return noalloc_fail(PB_ERR_CUDA, msg);
            }
            ws = static_cast<double *>(p);
            if (keyed) {
                g_noalloc_cache[g_noalloc_next] = NoAllocSlot{cid, ws};
                g_noalloc_next = (g_noalloc_next + 1) % kNoAllocSlots;
            }
        }
    }
    pb_cxr_args a = *args;
    a.far_moments = far ? ws : nullptr;
    int sms = 148;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
    const cudaError_t e = pb::launch_cxr(a, (cudaStream_t)stream, sms);
    if (e != cudaSuccess) {
        char msg[256];
        snprintf(msg, sizeof(msg), "pb_cxr_score_noalloc: launch: %s", cudaGetErrorString(e));
        return noalloc_fail(PB_ERR_CUDA, msg);
    }
    return PB_OK;
}
