// Bethe-Heitler + Elwert track-length bremsstrahlung of a segment list
// (sm_100a). spec[d][e] += sum_seg sum_el n_el L dsigma/dk(Z_el, T, k_e)
// * <exp(-mu(k_e) path)>_segment, the estimator of
// src/pyrite/montecarlo/spectrum/brem.py:431-479,1196-1239 before its
// 1/(4 pi Ne) normalisation.
//
// Work split: a block owns 256 photon-energy nodes (one per thread), a chunk
// of segments staged in shared memory with their energy-independent parts
// (incident momentum, beta, Elwert incident factor, escape end paths), and
// one detector direction. Each thread sums its node over the chunk in a
// register; one global atomic per node per block publishes it.
//
// The mixed path forms p_i - p_f without cancellation,
// (p_i^2 - p_f^2)/(p_i + p_f) = k (T_i + T_f + 2 m c^2)/((m c^2)^2 (p_i + p_f)),
// which float needs for MeV electrons and keV photons; FP64 keeps the
// reference's direct difference.
#include <cstdint>

#include "pb_brem_node.cuh"
#include "pb_common.cuh"
#include "pb_internal.h"
#include "pb_layers.cuh"

namespace pb {

constexpr int kBremThreads = 256;
constexpr int kBremChunk = 256;
constexpr int kBremMaxEl = 4;
constexpr int kBremMaxDir = 16;

// A staged segment. FP64 keeps the reference's factors; the float path
// folds the per-segment ones of its cross-section form (brem_nsig):
// beta_i holds beta_i / p_i^2 and nL[el] holds n_el L Z_el^2 den_i[el].
template <class Real>
struct alignas(sizeof(Real) == 4 ? 16 : 8) BremSeg {
    Real T;       // keV
    Real p_i;     // momentum / (m c)
    Real beta_i;
    // Escape geometry: FP64 keeps the clipped end depths (e0, e1); the float
    // path keeps the exit-side depth of the shallower end toward the top (e0)
    // and the bottom (e1), the depth difference |end1 - end0| (e2) and its
    // reciprocal (inv_e2, infinite for a segment parallel to the faces).
    Real e0, e1, e2, inv_e2;
    Real nL[kBremMaxEl];     // n_el * 1e24 * L * 1e-8  [1/cm^2]
    // 1 - exp(-2 pi Z alpha / beta_i); the float path folds it into nL.
    Real den_i[sizeof(Real) == 8 ? kBremMaxEl : 1];
};

__device__ __forceinline__ double b_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float b_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double b_exp(double x) { return exp(x); }
__device__ __forceinline__ float b_exp(float x) { return expf(x); }
__device__ __forceinline__ double b_log(double x) { return log(x); }
__device__ __forceinline__ float b_log(float x) { return logf(x); }
__device__ __forceinline__ double b_expm1(double x) { return expm1(x); }
__device__ __forceinline__ float b_expm1(float x) { return expm1f(x); }

// Base-2 exponential on the SFU (about 2 ulp), for the float path.
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Two floats in one 64-bit register pair, and the packed FP32 arithmetic of
// sm_100 (one instruction for both halves).
__device__ __forceinline__ unsigned long long f2_pack(float lo, float hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2_unpack(unsigned long long v, float &lo, float &hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ unsigned long long f2_fma(unsigned long long a, unsigned long long b,
                                                     unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ unsigned long long f2_mul(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// Reciprocal square root and base-2 logarithm on the SFU, denormals
// flushed (the float path's arguments are normal numbers).
__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float lg2_approx(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Reciprocal on the SFU (about 1 ulp), for the float path.
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// 2^x of both halves.
__device__ __forceinline__ unsigned long long f2_ex2(unsigned long long x) {
    float lo, hi;
    f2_unpack(x, lo, hi);
    return f2_pack(ex2_approx(lo), ex2_approx(hi));
}

template <class Real>
__device__ __forceinline__ Real b_path(Real z, Real thickness, Real nz) {
    const Real inv_nz = (Real)1 / fmax(fabs(nz), (Real)1.0e-12);
    const Real depth = fmin(fmax(z, (Real)0), thickness);
    return nz < (Real)0 ? depth * inv_nz : (thickness - depth) * inv_nz;
}

template <class Real>
__device__ __forceinline__ Real b_mean_transmission(Real t0, Real t1) {
    const Real lo = fmin(t0, t1);
    const Real d = fabs(t1 - t0);
    const Real safe = d > (Real)1.0e-4 ? d : (Real)1;
    const Real ratio = d > (Real)1.0e-4 ? -b_expm1(-safe) / safe : (Real)1 - (Real)0.5 * d + d * d / (Real)6;
    return b_exp(-lo) * ratio;
}

// Stage one segment's energy-independent parts.
template <class Real>
__device__ __forceinline__ void brem_stage(BremSeg<Real> &b, const pb_brem_args &a, int64_t s, Real T_slab,
                                           Real mc2, Real za) {
    const Real T = (Real)a.E_keV[s];
    b.T = T;
    const Real p_i = b_sqrt(T * (T + (Real)2 * mc2)) / mc2;
    b.p_i = p_i;
    b.beta_i = p_i / ((Real)1 + T / mc2);
    const Real half = (Real)0.5 * (Real)a.L[s];
    const Real z = (Real)a.r_mid[3 * s + 2];
    const Real vz = (Real)a.v_hat[3 * s + 2];
    // Depth of each segment end below the top face, clipped to the slab;
    // the escape path toward n is depth/|n_z| (up) or (T - depth)/|n_z|.
    const Real d0 = fmin(fmax(z - half * vz, (Real)0), T_slab);
    const Real d1 = fmin(fmax(z + half * vz, (Real)0), T_slab);
    if constexpr (sizeof(Real) == 8) {
        b.e0 = d0;
        b.e1 = d1;
        b.e2 = 0;
        b.inv_e2 = 0;
    } else {
        b.e0 = fmin(d0, d1);
        b.e1 = fmin(T_slab - d0, T_slab - d1);
        b.e2 = fabs(d1 - d0);
        b.inv_e2 = 1.0f / b.e2;
    }
    const bool rad = a.elec_id[s] < a.Ne && (a.seg_layer == nullptr || a.seg_layer[s] == a.emit_layer);
    const Real path_cm = (Real)a.L[s] * (Real)1e-8;
    for (int el = 0; el < a.n_el; ++el) {
        b.nL[el] = rad ? (Real)(a.n_ang3[el] * 1e24) * (Real)1 * path_cm : (Real)0;
        const Real den_i = (Real)1 - b_exp(-za * (Real)a.Z[el] / b.beta_i);
        if constexpr (sizeof(Real) == 4) {
            const Real Z = (Real)a.Z[el];
            b.nL[el] *= Z * Z * den_i;
        } else {
            b.den_i[el] = den_i;
        }
    }
    if constexpr (sizeof(Real) == 4) b.beta_i = b.beta_i / (p_i * p_i);
}

// Per-thread constants of the float cross-section form.
struct BremKConst {
    float kc;     // k / (m c^2)^2  [1/keV]
    float c2mk;   // 2 m c^2 - k    [keV]
    float c0k;    // c0 ln 2 / k_ev
};

// sum_el n_el L dsigma/dk(Z_el, T, k) of one staged segment (brem.py:396-479).
// The float path evaluates the same expression as
//   rs = 1/sqrt(q), q = T_f (T_f + 2 m c^2):   p_f = q rs / m c^2,
//   1/beta_f = (1 + T_f / m c^2) m c^2 rs,
//   ln((p_i + p_f) / (p_i - p_f)) = ln 2 log2((p_i + p_f)^2 / (k (T + T_f + 2 m c^2) / (m c^2)^2)),
//   (p_i^2 - p_f^2 = k (T + T_f + 2 m c^2) / (m c^2)^2, without cancellation),
// so one (segment, energy) costs five SFU operations (rsqrt, rcp, lg2, and
// ex2 + rcp per element of the Elwert factor).
template <class Real, int NEL = 0>
__device__ __forceinline__ Real brem_nsig(const BremSeg<Real> &b, Real k, Real T_f, const Real *Zs, int n_el_rt,
                                          Real k_ev, Real c0, Real za, Real mc2, const BremKConst &kk,
                                          const float *zl) {
    // NEL > 0: the element count known at compile time (loops unrolled).
    const int n_el = NEL > 0 ? NEL : n_el_rt;
    Real nsig = 0;
    if constexpr (sizeof(Real) == 8) {
        const Real p_f = b_sqrt(T_f * (T_f + (Real)2 * mc2)) / mc2;
        const Real beta_f = p_f / ((Real)1 + T_f / mc2);
        const Real born_log = b_log((b.p_i + p_f) / fmax(b.p_i - p_f, (Real)1e-30));
        for (int el = 0; el < n_el; ++el) {
            const Real Z = Zs[el];
            const Real elwert = b.beta_i / beta_f * b.den_i[el] / ((Real)1 - b_exp(-za * Z / beta_f));
            const Real dsig = c0 * (Z * Z) / k_ev / (b.p_i * b.p_i) * born_log * elwert;
            nsig += b.nL[el] * dsig;
        }
    } else {
        const float inv_mc2 = 1.0f / 510.99895f;
        const float q = T_f * (T_f + 2.0f * mc2);
        const float rs = rsqrt_approx(q);
        const float p_f = q * rs * inv_mc2;
        const float sp = b.p_i + p_f;
        const float dpp = kk.kc * fmaf(2.0f, b.T, kk.c2mk);  // p_i^2 - p_f^2
        const float lg = lg2_approx(fmaxf(sp * sp * rcp_approx(fmaxf(dpp, 1e-30f)), 1e-30f));
        const float inv_beta_f = fmaf(T_f, inv_mc2, 1.0f) * (rs * mc2);
        const float common = kk.c0k * b.beta_i * lg * inv_beta_f;  // beta_i holds beta_i / p_i^2
#pragma unroll
        for (int el = 0; el < (NEL > 0 ? NEL : kBremMaxEl); ++el) {
            if (NEL == 0 && el >= n_el) break;
            const float den_f = 1.0f - ex2_approx(-zl[el] * inv_beta_f);
            nsig = fmaf(b.nL[el] * common, rcp_approx(den_f), nsig);  // nL holds n L Z^2 den_i
        }
    }
    return nsig;
}

// ---------------------------------------------------------------------------
// Direction moments of the segment-mean escape (float path).
//
// A segment's escape toward direction d is its mean transmission
//   Tbar(f) = int_0^1 exp(-(a + b s) f) ds = (exp(-a f) - exp(-c f)) / (b f),
// a = mu e_lo (optical depth of the shallower end below the exit face, along
// the face normal), b = mu e2 (depth extent of the segment), c = a + b, and
// f = 1 / |n_z,d| the direction's path factor. The tiles of one detector
// leave through the same face with path factors f_d = f_c + delta_d inside a
// narrow band |delta_d| <= Delta (0.13 % of f_c for 16 tiles of a 2x2 cm^2
// detector at 1 m). The function g(f) = f Tbar(f) = (exp(-a f) - exp(-c f)) / b
// is a difference of exponentials, so its Taylor series about f_c,
//   g(f_c + Delta h) = sum_n h^n P_n / n!,
//   P_n = (-Delta)^n (a^n exp(-a f_c) - c^n exp(-c f_c)) / b,
// has coefficients that do not depend on the direction. Their sums over the
// segments of a chunk, Q_n = sum_seg nsig_seg P_n,seg, are accumulated per
// photon energy, and every direction is rebuilt once per chunk as
//   sum_seg nsig Tbar(f_d) = (1 / f_d) sum_n h_d^n Q_n / n!,  h_d = delta_d / Delta.
// Two exponentials per (segment, energy) replace two per (segment, energy,
// direction). The P_n follow without cancellation from
//   P_0 = g(f_c),  P_{n+1} = ah P_n + R_n,  R_0 = Delta exp(-c f_c),
//   R_{n+1} = ch R_n,  ah = -Delta a,  ch = -Delta c
// (from a^{n+1} E_a - c^{n+1} E_c = a (a^n E_a - c^n E_c) - b c^n E_c), and
// P_0 = exp(-a f_c) f_c phi(b f_c), phi(x) = (1 - e^-x)/x, takes the series
// of phi below x = 0.1 (degree 5, truncation < x^6/5040 < 2e-10) where the
// difference of the exponentials would cancel.
// Truncation after order N: the remainder of the Taylor series is at most
// about rho^(N+1) / sqrt(2 pi (N+1)) of the unattenuated term, rho = Delta /
// f_min, whatever the optical depths (the attenuation exp(-a f_min) bounds the
// growth of the derivatives); the choice N = 3 for rho <= 0.01 and N = 5 for
// rho <= 0.05 keeps it below 3e-9, and so does N = 2 for rho <= 0.002 (the
// packed kernel's order there).
// ---------------------------------------------------------------------------
struct BremMomentConst {
    float mu_l2fc;  // mu log2(e) f_c
    float mu_fc;    // mu f_c
    float inv_mu;   // 1 / mu
    float mu_dl;    // mu Delta
    float f_c, dl;  // f_c, Delta
};

template <int N, int NEL>
__device__ __forceinline__ void brem_moment_chunk(const BremSeg<float> *segs, int nc, bool up, float k,
                                                  const float *Zs, int n_el, float k_ev, float c0, float za,
                                                  float mc2, const BremKConst &kk, const float *zl,
                                                  const BremMomentConst &m, float (&Q)[N + 1]) {
    for (int j = 0; j < nc; ++j) {
        const BremSeg<float> &b = segs[j];
        const float T_f = b.T - k;
        if (!(T_f > 1e-6f && k > 0.0f)) continue;
        const float nsig = brem_nsig<float, NEL>(b, k, T_f, Zs, n_el, k_ev, c0, za, mc2, kk, zl);
        const float es = up ? b.e0 : b.e1;
        const float ef = es + b.e2;
        const float Ea = ex2_approx(-m.mu_l2fc * es);
        const float Ec = ex2_approx(-m.mu_l2fc * ef);
        const float x = m.mu_fc * b.e2;
        const float phi = fmaf(x, fmaf(x, fmaf(x, fmaf(x, fmaf(x, -1.0f / 720.0f, 1.0f / 120.0f), -1.0f / 24.0f),
                                                   1.0f / 6.0f), -0.5f), 1.0f);
        float P = x > 0.1f ? (Ea - Ec) * (m.inv_mu * b.inv_e2) : Ea * m.f_c * phi;
        Q[0] = fmaf(nsig, P, Q[0]);
        if constexpr (N > 0) {
            const float ah = -m.mu_dl * es, ch = -m.mu_dl * ef;
            float R = m.dl * Ec;
#pragma unroll
            for (int n = 1; n <= N; ++n) {
                P = fmaf(ah, P, R);
                if (n < N) R *= ch;
                Q[n] = fmaf(nsig, P, Q[n]);
            }
        }
    }
}

// sum_n h^n Q_n / n! (Horner).
template <int N>
__device__ __forceinline__ float brem_moment_eval(const float (&Q)[N + 1], float h) {
    constexpr float kInvFact[8] = {1.0f, 1.0f, 0.5f, 1.0f / 6.0f, 1.0f / 24.0f, 1.0f / 120.0f, 1.0f / 720.0f,
                                   1.0f / 5040.0f};
    float r = Q[N] * kInvFact[N];
#pragma unroll
    for (int n = N - 1; n >= 0; --n) r = fmaf(r, h, Q[n] * kInvFact[n]);
    return r;
}

// ---------------------------------------------------------------------------
// Packed moment kernel: the float path for directions on one exit face with
// rho <= 0.01 (order-3 moments, order 2 for rho <= 0.002; a single direction
// is the order-0 case of the same recurrences). Two photon energies per
// thread on packed FP32x2 arithmetic (fma/mul/add.rn.f32x2), so the non-SFU
// instructions of a (segment, energy) pair are issued once per two pairs; the
// moments are summed per chunk in float and then in FP64 shared memory, and
// the directions are rebuilt once at the end (the reconstruction is linear in
// the moments), so no per-direction accumulators are kept. The pair loop
// carries the moments divided by Delta^n (Q_n / Delta^n, rebuilt with
// (f_d - f_c)^n) and, for one element, without the segment factor and c0 / k:
// the segment factor enters the escape exponent as log2 of its ratio to the
// chunk's 2^ref, and c0 2^ref / k scales the chunk's sums. For relativistic final
// states (1/beta_f - 1 < 0.01, T_f > ~3 MeV) the Elwert factor's reciprocal
// 1/(1 - exp(-z/beta_f)) comes from its series in s = z (1/beta_f - 1):
//   G0 [1 - rho s + (rho/2 + rho^2) s^2 - (rho/6 + rho^2 + rho^3) s^3],
//   G0 = 1/(1 - e^-z), rho = e^-z G0, z = 2 pi Z alpha,
// truncation below (rho s)^4 < 1e-8 for Z <= 92; elsewhere the SFU form.
// ---------------------------------------------------------------------------
struct F2 {
    unsigned long long v;
};
__device__ __forceinline__ F2 f2(float lo, float hi) { return F2{f2_pack(lo, hi)}; }
__device__ __forceinline__ F2 f2s(float x) { return F2{f2_pack(x, x)}; }
__device__ __forceinline__ float f2lo(F2 a) { float l, h; f2_unpack(a.v, l, h); return l; }
__device__ __forceinline__ float f2hi(F2 a) { float l, h; f2_unpack(a.v, l, h); return h; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return F2{f2_mul(a.v, b.v)}; }
__device__ __forceinline__ F2 operator+(F2 a, F2 b) {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a.v), "l"(b.v));
    return F2{d};
}
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return F2{f2_fma(a.v, b.v, c.v)}; }
__device__ __forceinline__ F2 neg2(F2 a) { return F2{a.v ^ 0x8000000080000000ull}; }
__device__ __forceinline__ F2 ex2_2(F2 a) { float l, h; f2_unpack(a.v, l, h); return f2(ex2_approx(l), ex2_approx(h)); }
__device__ __forceinline__ F2 rcp_2(F2 a) { float l, h; f2_unpack(a.v, l, h); return f2(rcp_approx(l), rcp_approx(h)); }
__device__ __forceinline__ F2 rsqrt_2(F2 a) {
    float l, h;
    f2_unpack(a.v, l, h);
    return f2(rsqrt_approx(l), rsqrt_approx(h));
}
__device__ __forceinline__ F2 lg2_2(F2 a) { float l, h; f2_unpack(a.v, l, h); return f2(lg2_approx(l), lg2_approx(h)); }

constexpr int kBremPackedThreads = 256;  // x 2 energies

// The packed form's cross section per element without the segment factor
// n L Z^2 den_i and the photon factor c0 ln2 / k:
//   J_el(T) = (beta_i / p_i^2) log2((p_i + p_f)^2 / dpp) / beta_f / (1 - exp(-z / beta_f)),
// for both energies at electron energy T (p_i, bp = beta_i / p_i^2 of T
// given); the Elwert reciprocal from its relativistic series where
// 1/beta_f - 1 < 0.01 in both lanes, else the SFU form. Tf must be > 0.
// With kSum the elements are summed at once, weighted by w (the segment's
// n L Z^2 den_i), into J[0].
template <int NEL, bool kSum = false>
__device__ __forceinline__ void brem_J2(F2 Tf, float T, float p_i, float bp, F2 kc, F2 c2mk, float mc2, float inv_mc2,
                                        const float (&zl)[NEL], const float (&zn)[NEL], const float (&G0)[NEL],
                                        const float (&rh)[NEL], F2 (&J)[NEL], const float *w = nullptr) {
    const F2 q = Tf * (Tf + f2s(2.0f * mc2));
    const F2 rs = rsqrt_2(q);
    const F2 p_f = (q * rs) * f2s(inv_mc2);
    const F2 sp = f2s(p_i) + p_f;
    const F2 dpp = kc * (f2s(2.0f * T) + c2mk);
    const F2 lg = lg2_2((sp * sp) * rcp_2(dpp));
    const F2 inv_bf = fma2(Tf, f2s(inv_mc2), f2s(1.0f)) * (rs * f2s(mc2));
    const F2 base = f2s(bp) * (lg * inv_bf);
    const F2 del = inv_bf + f2s(-1.0f);
    const bool rel = f2lo(del) < 0.01f && f2hi(del) < 0.01f;
#pragma unroll
    for (int el = 0; el < NEL; ++el) {
        F2 ginv;
        if (rel) {
            const F2 sz = del * f2s(zn[el]);
            const float r = rh[el], r2 = r * r;
            const F2 poly = fma2(sz, fma2(sz, fma2(sz, f2s(-(r / 6.0f + r2 + r2 * r)), f2s(0.5f * r + r2)),
                                          f2s(-r)), f2s(1.0f));
            ginv = poly * f2s(G0[el]);
        } else {
            ginv = rcp_2(f2s(1.0f) + neg2(ex2_2(neg2(inv_bf * f2s(zl[el])))));
        }
        if constexpr (kSum) J[0] = fma2(f2s(w[el]) * base, ginv, el == 0 ? f2s(0.0f) : J[0]);
        else J[el] = base * ginv;
    }
}


// Whether the launch's directions take the packed moment kernel: one exit
// face and relative spread rho = Delta / f_min <= 0.01 (the same test both
// brem kernels make, so exactly one of them scores the launch).
__device__ __forceinline__ bool brem_packed_applies(const pb_brem_args &a, int d0, int nd, double &f_c, double &dl) {
    int n_up = 0;
    double f_lo = 1e300, f_hi = 0.0;
    for (int dd = 0; dd < nd; ++dd) {
        const double nz = a.n_hat[3 * (d0 + dd) + 2];
        n_up += nz < 0.0 ? 1 : 0;
        const double f = 1.0 / fmax(fabs(nz), 1.0e-12);
        f_lo = fmin(f_lo, f);
        f_hi = fmax(f_hi, f);
    }
    f_c = 0.5 * (f_lo + f_hi);
    dl = 0.5 * (f_hi - f_lo);
    return (n_up == nd || n_up == 0) && dl <= 0.01 * f_lo;
}

template <int N>
struct MomentOrder {
    static constexpr int value = N;
};

template <int NEL>
__global__ void __launch_bounds__(kBremPackedThreads, 3)
    brem_moment_packed_kernel(const pb_brem_args a, int64_t n_seg, int d0, const BremNodeHdr *nh,
                              const int64_t *nidx) {
    __shared__ BremSeg<float> segs[kBremChunk];
    __shared__ double sQ[8][kBremPackedThreads];  // FP64 moment sums: [energy half * 4 + n][thread]
    __shared__ float sT[3][kBremPackedThreads / 32];  // the chunk's electron energy range, per warp
    // the chunk's per-segment operands already packed for the FP32x2 pair
    // loop (each half holds the same value), so the loop issues no packing
    struct Pk {
        F2 u, lnl, es, ef, e2;
    };
    __shared__ Pk pk[kBremChunk];
    const int nd = (a.n_dir - d0) < kBremMaxDir ? (a.n_dir - d0) : kBremMaxDir;
    double f_c_d, dl_d;
    if (a.precision != PB_MIXED || !brem_packed_applies(a, d0, nd, f_c_d, dl_d)) return;
    const bool up_all = a.n_hat[3 * d0 + 2] < 0.0;
    // Moment order: 2 where rho = Delta / f_min <= 0.002 (truncation below
    // rho^3 / sqrt(6 pi) < 2e-9 of the unattenuated term), else 3.
    const bool order3 = dl_d > 0.002 * (f_c_d - dl_d);
    const float T_slab = (float)a.thickness;
    const float mc2 = 510.99895f, inv_mc2 = 1.0f / 510.99895f;
    const float za = (float)(2.0 * kPi * kAlphaFs);
    const int e0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    const bool on_a = e0 < a.n_E, on_b = e0 + 1 < a.n_E;
    // per-energy constants, packed (energy e0 low, e0 + 1 high)
    double kd[2], mud[2];
    for (int h = 0; h < 2; ++h) {
        const int e = e0 + h;
        const bool on = e < a.n_E;
        kd[h] = on ? a.E_grid[e] / 1e3 : 0.0;  // k = 0 marks an idle lane: no pair is valid
        mud[h] = on ? a.mu[e] : 0.0;
    }
    const F2 k2 = f2((float)kd[0], (float)kd[1]);
    const F2 kc = f2((float)(kd[0] / (510.99895 * 510.99895)), (float)(kd[1] / (510.99895 * 510.99895)));
    const F2 c2mk = f2((float)(2.0 * 510.99895 - kd[0]), (float)(2.0 * 510.99895 - kd[1]));
    const double c0 = 16.0 / 3.0 * kAlphaFs * kReCm2 * 0.6931471805599453;
    const F2 nmu_l2fc = f2((float)(-mud[0] * 1.4426950408889634 * f_c_d), (float)(-mud[1] * 1.4426950408889634 * f_c_d));
    const F2 inv_mu = f2(mud[0] > 0.0 ? (float)(1.0 / mud[0]) : 0.0f, mud[1] > 0.0 ? (float)(1.0 / mud[1]) : 0.0f);
    const F2 nmu = f2((float)-mud[0], (float)-mud[1]);
    const F2 nmu_fc = f2((float)(-mud[0] * f_c_d), (float)(-mud[1] * f_c_d));
    const F2 fc2 = f2s((float)f_c_d);
    // Depth extent below which x = mu f_c e2 <= 0.1 in every lane of this
    // warp (the largest mu of its 64 energies): the pair loop's branch on it
    // is warp-uniform, since all lanes take the same segment.
    float e2_series;
    {
        float mm = (float)(fmax(mud[0], mud[1]) * f_c_d);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mm = fmaxf(mm, __shfl_xor_sync(0xffffffffu, mm, o));
        e2_series = mm > 0.0f ? 0.1f / mm : 3.4e38f;
    }
    // Elwert constants per element: z log2(e) for the SFU form; G0 and rho
    // of the relativistic series.
    float zl[NEL], zn[NEL], G0[NEL], rh[NEL];
#pragma unroll
    for (int el = 0; el < NEL; ++el) {
        const double z = 2.0 * kPi * kAlphaFs * a.Z[el];
        const double ez = exp(-z);
        zl[el] = (float)(z * 1.4426950408889634);
        zn[el] = (float)z;
        G0[el] = (float)(1.0 / (1.0 - ez));
        rh[el] = (float)(ez / (1.0 - ez));
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) sQ[i][threadIdx.x] = 0.0;
    const bool act_a = kd[0] > 0.0, act_b = kd[1] > 0.0;
    int64_t live = n_seg;
    if (a.n_seg_device && (int64_t)*a.n_seg_device < live) live = (int64_t)*a.n_seg_device;
    // With the depth-node form active, only the segments it left out.
    const int64_t *sidx = nullptr;
    if (nh != nullptr && nh->ok) {
        live = (int64_t)nh->n_out;
        sidx = nidx;
    }
    const int64_t per = (live + gridDim.y - 1) / gridDim.y;
    const int64_t s_begin = per * blockIdx.y;
    int64_t s_end = s_begin + per < live ? s_begin + per : live;
    if (s_end < s_begin) s_end = s_begin;
    for (int64_t c0s = s_begin; c0s < s_end; c0s += kBremChunk) {
        const int nc = (int)((s_end - c0s) < kBremChunk ? (s_end - c0s) : kBremChunk);
        __syncthreads();
        float tlo = 3.4e38f, thi = -3.4e38f, nmax = 0.0f;
        for (int j = threadIdx.x; j < nc; j += blockDim.x) {
            brem_stage<float>(segs[j], a, sidx ? sidx[c0s + j] : c0s + j, T_slab, mc2, za);
            tlo = fminf(tlo, segs[j].T);
            thi = fmaxf(thi, segs[j].T);
            nmax = fmaxf(nmax, segs[j].nL[0]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            tlo = fminf(tlo, __shfl_xor_sync(0xffffffffu, tlo, o));
            thi = fmaxf(thi, __shfl_xor_sync(0xffffffffu, thi, o));
            nmax = fmaxf(nmax, __shfl_xor_sync(0xffffffffu, nmax, o));
        }
        if ((threadIdx.x & 31) == 0) {
            sT[0][threadIdx.x >> 5] = tlo;
            sT[1][threadIdx.x >> 5] = thi;
            sT[2][threadIdx.x >> 5] = nmax;
        }
        __syncthreads();
        tlo = sT[0][0];
        thi = sT[1][0];
        nmax = sT[2][0];
#pragma unroll
        for (int w = 1; w < kBremPackedThreads / 32; ++w) {
            tlo = fminf(tlo, sT[0][w]);
            thi = fmaxf(thi, sT[1][w]);
            nmax = fmaxf(nmax, sT[2][w]);
        }
        // One element: the segment factor n L Z^2 den_i rides in the escape
        // exponent as log2 of its ratio to 2^ref (ref the chunk's largest,
        // rounded down), so the pair loop multiplies by neither it nor c0 / k;
        // both come back once per chunk. Several elements weight the cross
        // section itself (ref = 0, exponent offset 0).
        const int ref = (NEL == 1 && nmax > 0.0f) ? (int)floorf(log2f(nmax)) : 0;
        {
            const float tc = 0.5f * (tlo + thi), th = 0.5f * (thi - tlo);
            const float ith = th > 0.0f ? 1.0f / th : 0.0f;
            for (int j = threadIdx.x; j < nc; j += blockDim.x) {
                const BremSeg<float> &b = segs[j];
                const float es = up_all ? b.e0 : b.e1;
                const float lnl = NEL == 1 ? log2f(b.nL[0]) - (float)ref : 0.0f;  // log2(0) = -inf: no emission
                pk[j] = Pk{f2s((b.T - tc) * ith), f2s(lnl), f2s(es), f2s(es + b.e2), f2s(b.e2)};
            }
        }
        __syncthreads();
        if (!on_a) continue;
        // The chunk's electrons span [tlo, thi]. Where that range is narrow
        // (at most 10 % of tlo) and clear of the spectrum's tip, J_el(T) of
        // this thread's two energies is the cubic through four Chebyshev
        // nodes of the range, accepted only if it matches J at both ends and
        // the middle to 1e-6: the pair loop then costs a cubic per element
        // instead of five SFU operations.
        // Chebyshev nodes cos((2j + 1) pi / 8)
        constexpr float kCheb4[4] = {0.92387953251128676f, 0.38268343236508977f, -0.38268343236508977f,
                                     -0.92387953251128676f};
        const float t_c = 0.5f * (tlo + thi), t_h = 0.5f * (thi - tlo);
        // (single-element targets: more elements would spill the coefficients)
        bool cub = NEL == 1 && t_h <= 0.05f * tlo && tlo - fmaxf(f2lo(k2), f2hi(k2)) > 0.01f * tlo;
        F2 A0[NEL], A1[NEL], A2[NEL], A3[NEL];
        if (NEL == 1 && cub) {
            F2 fj[4][NEL];
#pragma unroll
            for (int jn = 0; jn < 4; ++jn) {
                const float T = fmaf(t_h, kCheb4[jn], t_c);
                const float p_i = sqrtf(T * (T + 2.0f * mc2)) * inv_mc2;
                const float bi = p_i / (1.0f + T * inv_mc2);
                brem_J2<NEL>(f2s(T) + neg2(k2), T, p_i, bi / (p_i * p_i), kc, c2mk, mc2, inv_mc2, zl, zn, G0, rh,
                             fj[jn]);
            }
#pragma unroll
            for (int el = 0; el < NEL; ++el) {
                // Chebyshev coefficients c_m = (2 / 4) sum_j f_j T_m(x_j), c_0 halved,
                // then the monomial form in u: a0 = c0 - c2, a1 = c1 - 3 c3, a2 = 2 c2, a3 = 4 c3.
                F2 c[4];
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    F2 acc = f2s(0.0f);
#pragma unroll
                    for (int jn = 0; jn < 4; ++jn) {
                        const float x = kCheb4[jn];
                        const float Tm = m == 0 ? 1.0f : m == 1 ? x : m == 2 ? 2.0f * x * x - 1.0f : x * (4.0f * x * x - 3.0f);
                        acc = fma2(fj[jn][el], f2s(Tm), acc);
                    }
                    c[m] = acc * f2s(m == 0 ? 0.25f : 0.5f);
                }
                A0[el] = c[0] + neg2(c[2]);
                A1[el] = c[1] + neg2(c[3] * f2s(3.0f));
                A2[el] = c[2] * f2s(2.0f);
                A3[el] = c[3] * f2s(4.0f);
            }
#pragma unroll
            for (int jc = 0; jc < 3; ++jc) {
                const float u = jc == 0 ? -1.0f : jc == 1 ? 0.0f : 1.0f;
                const float T = fmaf(t_h, u, t_c);
                const float p_i = sqrtf(T * (T + 2.0f * mc2)) * inv_mc2;
                const float bi = p_i / (1.0f + T * inv_mc2);
                F2 ex[NEL];
                brem_J2<NEL>(f2s(T) + neg2(k2), T, p_i, bi / (p_i * p_i), kc, c2mk, mc2, inv_mc2, zl, zn, G0, rh, ex);
#pragma unroll
                for (int el = 0; el < NEL; ++el) {
                    const F2 pv = fma2(fma2(fma2(A3[el], f2s(u), A2[el]), f2s(u), A1[el]), f2s(u), A0[el]);
                    const F2 d = pv + neg2(ex[el]);
                    cub = cub && fabsf(f2lo(d)) <= 1e-6f * fabsf(f2lo(ex[el])) &&
                          fabsf(f2hi(d)) <= 1e-6f * fabsf(f2hi(ex[el]));
                }
            }
        }
        F2 Q0 = f2s(0.0f), Q1 = f2s(0.0f), Q2 = f2s(0.0f), Q3 = f2s(0.0f);
        // The pair loop for moment order 2 or 3 (the order is uniform over the launch).
        auto pairs = [&](auto order) {
            constexpr int kOrd = decltype(order)::value;
            for (int j = 0; j < nc; ++j) {
                const BremSeg<float> &b = segs[j];
                F2 nsig = f2s(0.0f);
                const Pk &q = pk[j];
                if (NEL == 1 && cub) {  // uniform over the thread's chunk
                    nsig = fma2(fma2(fma2(A3[0], q.u, A2[0]), q.u, A1[0]), q.u, A0[0]);
                } else {
                    F2 Tf = f2s(b.T) + neg2(k2);
                    const float tfl = f2lo(Tf), tfh = f2hi(Tf);
                    const bool va = tfl > 1e-6f && act_a, vb = tfh > 1e-6f && act_b;
                    if (!va && !vb) continue;
                    Tf = f2(va ? tfl : 1.0f, vb ? tfh : 1.0f);  // keep idle halves finite
                    F2 J[NEL];
                    // beta_i holds beta_i / p_i^2, nL holds n L Z^2 den_i
                    const float one[1] = {1.0f};
                    brem_J2<NEL, true>(Tf, b.T, b.p_i, b.beta_i, kc, c2mk, mc2, inv_mc2, zl, zn, G0, rh, J,
                                       NEL == 1 ? one : b.nL);
                    nsig = J[0];
                    nsig = f2(va ? f2lo(nsig) : 0.0f, vb ? f2hi(nsig) : 0.0f);
                }
                // escape moments (brem_moment_chunk, order kOrd, both energies)
                const F2 Ea = ex2_2(fma2(nmu_l2fc, q.es, q.lnl));
                // y = -x = -mu f_c e2; phi(x) = (1 - e^-x)/x = sum_n y^n / (n + 1)!
                const F2 y = nmu_fc * q.e2;
                const F2 phi = fma2(y, fma2(y, fma2(y, fma2(y, fma2(y, f2s(1.0f / 720.0f), f2s(1.0f / 120.0f)),
                                                              f2s(1.0f / 24.0f)), f2s(1.0f / 6.0f)), f2s(0.5f)),
                                    f2s(1.0f));
                const F2 A = Ea * phi;
                F2 P = A * fc2, Ec;
                if (f2lo(q.e2) <= e2_series) {
                    // x <= 0.1 in both lanes: P_0 = E_a f_c phi(x) from the series,
                    // and E_c = E_a e^-x = E_a (1 - x phi(x)) (no second exponential).
                    Ec = fma2(A, y, Ea);
                } else {
                    Ec = ex2_2(fma2(nmu_l2fc, q.ef, q.lnl));
                    const F2 dif = (Ea + neg2(Ec)) * (inv_mu * f2s(b.inv_e2));
                    P = f2(f2lo(y) < -0.1f ? f2lo(dif) : f2lo(P), f2hi(y) < -0.1f ? f2hi(dif) : f2hi(P));
                }
                Q0 = fma2(nsig, P, Q0);
                // P_n / Delta^n: the recurrence without Delta (it returns as
                // (f - f_c)^n at the reconstruction)
                const F2 ah = nmu * q.es, ch = nmu * q.ef;
                P = fma2(ah, P, Ec);
                Q1 = fma2(nsig, P, Q1);
                F2 R = Ec * ch;
                P = fma2(ah, P, R);
                Q2 = fma2(nsig, P, Q2);
                if constexpr (kOrd >= 3) {
                    R = R * ch;
                    P = fma2(ah, P, R);
                    Q3 = fma2(nsig, P, Q3);
                }
            }
        };
        if (order3) pairs(MomentOrder<3>{});
        else pairs(MomentOrder<2>{});
        const int t = threadIdx.x;
        const double sc = ldexp(c0, ref);
        const double s_lo = sc / fmax(a.E_grid[e0], 1e-30), s_hi = on_b ? sc / fmax(a.E_grid[e0 + 1], 1e-30) : 0.0;
        sQ[0][t] += f2lo(Q0) * s_lo; sQ[4][t] += f2hi(Q0) * s_hi;
        sQ[1][t] += f2lo(Q1) * s_lo; sQ[5][t] += f2hi(Q1) * s_hi;
        sQ[2][t] += f2lo(Q2) * s_lo; sQ[6][t] += f2hi(Q2) * s_hi;
        sQ[3][t] += f2lo(Q3) * s_lo; sQ[7][t] += f2hi(Q3) * s_hi;
    }
    // Every direction of the launch from the summed moments:
    // (1/f_d) sum_n (f_d - f_c)^n (Q_n / Delta^n) / n!.
    for (int dd = 0; dd < nd; ++dd) {
        const double f = 1.0 / fmax(fabs(a.n_hat[3 * (d0 + dd) + 2]), 1.0e-12);
        const double hh = f - f_c_d;
        for (int h = 0; h < 2; ++h) {
            if (!(h == 0 ? on_a : on_b)) continue;
            const double *Qh[4] = {&sQ[4 * h][threadIdx.x], &sQ[4 * h + 1][threadIdx.x], &sQ[4 * h + 2][threadIdx.x],
                                   &sQ[4 * h + 3][threadIdx.x]};
            const double v = (((*Qh[3] * (1.0 / 6.0)) * hh + *Qh[2] * 0.5) * hh + *Qh[1]) * hh + *Qh[0];
            if (v != 0.0) atomicAdd(&a.spec[(int64_t)(d0 + dd) * a.n_E + e0 + h], v / f);
        }
    }
}

template <class Real, int NEL>
__global__ void __launch_bounds__(kBremThreads, sizeof(Real) == 4 ? 4 : 2)
    brem_kernel(const pb_brem_args a, int64_t n_seg, int d0, const BremNodeHdr *nh, const int64_t *nidx) {
    // Segment chunk staged in shared memory (half as many FP64 segments, to
    // stay within the static shared-memory limit next to the accumulators).
    constexpr int kChunk = sizeof(Real) == 4 ? kBremChunk : kBremChunk / 2;
    __shared__ BremSeg<Real> segs[kChunk];
    // Per-thread FP64 sums over the block's segments, one per direction, in
    // shared memory (keeps the registers for the per-chunk partials).
    __shared__ double acc[kBremMaxDir][kBremThreads];
    __shared__ Real Zs[kBremMaxEl];
    __shared__ float zl[kBremMaxEl];  // 2 pi alpha Z log2(e)
    __shared__ Real inv_nz[kBremMaxDir];
    __shared__ int up[kBremMaxDir];
    __shared__ float inv_f_ln2[kBremMaxDir];
    const int nd = (a.n_dir - d0) < kBremMaxDir ? (a.n_dir - d0) : kBremMaxDir;
    const Real T_slab = (Real)a.thickness;
    const int n_el = a.n_el;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const bool on = e < a.n_E;
    const Real mc2 = (Real)510.99895;
    const Real za = (Real)(2.0 * kPi * kAlphaFs);
    if (threadIdx.x < n_el) {
        Zs[threadIdx.x] = (Real)a.Z[threadIdx.x];
        zl[threadIdx.x] = (float)(2.0 * kPi * kAlphaFs * a.Z[threadIdx.x] * 1.4426950408889634);
    }
    if (threadIdx.x < nd) {
        const Real nz = (Real)a.n_hat[3 * (d0 + threadIdx.x) + 2];
        inv_nz[threadIdx.x] = (Real)1 / fmax(fabs(nz), (Real)1.0e-12);
        up[threadIdx.x] = nz < (Real)0;
        inv_f_ln2[threadIdx.x] = (float)(fmax(fabs((double)nz), 1.0e-12) / 0.6931471805599453);
    }
    // Whether every direction of this launch leaves through the same face
    // (+1 top, -1 bottom, 0 mixed), read from the directions themselves.
    int side_all = 0;
    {
        int n_up = 0;
        for (int dd = 0; dd < nd; ++dd) n_up += a.n_hat[3 * (d0 + dd) + 2] < 0.0 ? 1 : 0;
        side_all = n_up == nd ? 1 : (n_up == 0 ? -1 : 0);
    }
    // Directions on one face within rho <= 0.01: the packed moment kernel
    // (brem_moment_packed_kernel) scores this launch.
    if constexpr (sizeof(Real) == 4) {
        double fc_p, dl_p;
        if (brem_packed_applies(a, d0, nd, fc_p, dl_p)) return;
    }
    // Moment form (see brem_moment_chunk): float, one exit face, and the
    // path factors within rho = Delta / f_min <= 0.05 of their centre.
    __shared__ float mom_h[kBremMaxDir];     // (f_d - f_c) / Delta
    __shared__ float mom_invf[kBremMaxDir];  // 1 / f_d
    int order = -1;
    double f_c = 1.0, dl = 0.0;
    if (sizeof(Real) == 4 && side_all != 0) {
        double f_lo = 1e300, f_hi = 0.0;
        for (int dd = 0; dd < nd; ++dd) {
            const double f = 1.0 / fmax(fabs(a.n_hat[3 * (d0 + dd) + 2]), 1.0e-12);
            f_lo = fmin(f_lo, f);
            f_hi = fmax(f_hi, f);
        }
        f_c = 0.5 * (f_lo + f_hi);
        dl = 0.5 * (f_hi - f_lo);
        const double rho = dl / f_lo;
        order = dl == 0.0 ? 0 : (rho <= 0.01 ? 3 : (rho <= 0.05 ? 5 : -1));
        if (threadIdx.x < nd) {
            const double f = 1.0 / fmax(fabs(a.n_hat[3 * (d0 + threadIdx.x) + 2]), 1.0e-12);
            mom_h[threadIdx.x] = dl > 0.0 ? (float)((f - f_c) / dl) : 0.0f;
            mom_invf[threadIdx.x] = (float)(1.0 / f);
        }
    }
    const double k_kev_d = on ? a.E_grid[e] / 1e3 : 1.0;
    const Real k = (Real)k_kev_d;
    const Real mu = on ? (Real)a.mu[e] : (Real)0;
    const Real k_ev = fmax((Real)(k_kev_d * 1e3), (Real)1e-30);
    const Real c0 = (Real)(16.0 / 3.0 * kAlphaFs * kReCm2);
    BremKConst kk;
    kk.kc = (float)(k_kev_d / (510.99895 * 510.99895));
    kk.c2mk = (float)(2.0 * 510.99895 - k_kev_d);
    kk.c0k = (float)(16.0 / 3.0 * kAlphaFs * kReCm2 * 0.6931471805599453 / fmax(k_kev_d * 1e3, 1e-30));
#pragma unroll
    for (int j = 0; j < kBremMaxDir; ++j) acc[j][threadIdx.x] = 0.0;
    if (a.n_seg_device) {
        const int64_t live = (int64_t)*a.n_seg_device;
        if (live < n_seg) n_seg = live;
    }
    // With the depth-node form active, only the segments it left out.
    const int64_t *sidx = nullptr;
    if (nh != nullptr && nh->ok) {
        n_seg = (int64_t)nh->n_out;
        sidx = nidx;
    }
    // Slices of the live segments (the count read on the device), so every
    // block of the wave has work.
    const int64_t per = (n_seg + gridDim.y - 1) / gridDim.y;
    const int64_t s_begin = per * blockIdx.y;
    int64_t s_end = s_begin + per < n_seg ? s_begin + per : n_seg;
    if (s_end < s_begin) s_end = s_begin;
    for (int64_t c0s = s_begin; c0s < s_end; c0s += kChunk) {
        const int nc = (int)((s_end - c0s) < kChunk ? (s_end - c0s) : kChunk);
        __syncthreads();
        for (int j = threadIdx.x; j < nc; j += blockDim.x) {
            brem_stage<Real>(segs[j], a, sidx ? sidx[c0s + j] : c0s + j, T_slab, mc2, za);
        }
        __syncthreads();
        if (!on) continue;
        if constexpr (sizeof(Real) == 4) {
            if (order >= 0) {
                BremMomentConst m;
                m.mu_l2fc = (float)((double)mu * 1.4426950408889634 * f_c);
                m.mu_fc = (float)((double)mu * f_c);
                m.inv_mu = mu > 0.0f ? 1.0f / mu : 0.0f;
                m.mu_dl = (float)((double)mu * dl);
                m.f_c = (float)f_c;
                m.dl = (float)dl;
                const bool up_all = side_all > 0;
                if (order == 0) {
                    float Q[1] = {0.0f};
                    brem_moment_chunk<0, NEL>(segs, nc, up_all, k, Zs, n_el, k_ev, c0, za, mc2, kk, zl, m, Q);
                    for (int dd = 0; dd < nd; ++dd)
                        acc[dd][threadIdx.x] += (double)Q[0] * (double)mom_invf[dd];
                } else if (order == 3) {
                    float Q[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                    brem_moment_chunk<3, NEL>(segs, nc, up_all, k, Zs, n_el, k_ev, c0, za, mc2, kk, zl, m, Q);
                    for (int dd = 0; dd < nd; ++dd)
                        acc[dd][threadIdx.x] += (double)brem_moment_eval<3>(Q, mom_h[dd]) * (double)mom_invf[dd];
                } else {
                    float Q[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
                    brem_moment_chunk<5, NEL>(segs, nc, up_all, k, Zs, n_el, k_ev, c0, za, mc2, kk, zl, m, Q);
                    for (int dd = 0; dd < nd; ++dd)
                        acc[dd][threadIdx.x] += (double)brem_moment_eval<5>(Q, mom_h[dd]) * (double)mom_invf[dd];
                }
                continue;
            }
        }
        // Partial sums per chunk (float on the mixed path), folded into the
        // FP64 accumulators once per chunk.
        Real part[kBremMaxDir];
#pragma unroll
        for (int dd = 0; dd < kBremMaxDir; ++dd) part[dd] = 0;
        for (int j = 0; j < nc; ++j) {
            const BremSeg<Real> &b = segs[j];
            const Real T_f = b.T - k;
            if (!(T_f > (Real)1e-6 && k > (Real)0)) continue;
            const Real nsig = brem_nsig<Real, NEL>(b, k, T_f, Zs, n_el, k_ev, c0, za, mc2, kk, zl);
            if constexpr (sizeof(Real) == 8) {
#pragma unroll
                for (int dd = 0; dd < kBremMaxDir; ++dd) {
                    if (dd < nd) {
                        const Real f = inv_nz[dd];
                        const Real p0 = up[dd] ? b.e0 * f : (T_slab - b.e0) * f;
                        const Real p1 = up[dd] ? b.e1 * f : (T_slab - b.e1) * f;
                        part[dd] += nsig * b_mean_transmission<Real>(p0 * mu, p1 * mu);
                    }
                }
            } else {
                // Escape mean exp(-lo) (1 - e^-D)/D per direction, with base-2
                // optical depths A f (lower end) and B f (depth difference),
                // D = B f ln 2. Sums are kept without the factor 1/(f ln 2),
                // applied once per chunk:
                //   D > 0.01: [nsig / B] 2^(-A f) (1 - 2^(-B f));
                //   otherwise: nsig 2^(-A f) (1 - D/2 + D^2/6 - D^3/24) f ln 2,
                // the series where the difference would cancel (D^4/120 < 1e-10).
                // This per-direction form serves directions that leave through
                // both faces or spread too widely for the moment form.
                const float mu2 = mu * 1.44269504f;
                const float A_dn = mu2 * b.e1;
                const float A_up = mu2 * b.e0;
                const float B = mu2 * b.e2;
                {
                    const float w = B > 0.0f ? __fdividef(nsig, B) : 0.0f;
#pragma unroll
                    for (int dd = 0; dd < kBremMaxDir; ++dd) {
                        if (dd < nd) {
                            const float f = inv_nz[dd];
                            const float fl = f * 0.69314718f;
                            const float D = B * fl;
                            const float A = up[dd] ? A_up : A_dn;
                            const float e_lo = ex2_approx(-A * f);
                            const float t = D > 0.01f
                                                ? w * (1.0f - ex2_approx(-B * f))
                                                : nsig * fl * fmaf(D, fmaf(D, fmaf(D, -1.0f / 24.0f, 1.0f / 6.0f), -0.5f), 1.0f);
                            part[dd] = fmaf(t, e_lo, part[dd]);
                        }
                    }
                }
            }
        }
        if constexpr (sizeof(Real) == 4) {
#pragma unroll
            for (int dd = 0; dd < kBremMaxDir; ++dd) acc[dd][threadIdx.x] += (double)part[dd] * (double)inv_f_ln2[dd];
        } else {
#pragma unroll
            for (int dd = 0; dd < kBremMaxDir; ++dd) acc[dd][threadIdx.x] += (double)part[dd];
        }
    }
    if (on) {
#pragma unroll
        for (int dd = 0; dd < kBremMaxDir; ++dd)
            if (dd < nd && acc[dd][threadIdx.x] != 0.0)
                atomicAdd(&a.spec[(int64_t)(d0 + dd) * a.n_E + e], acc[dd][threadIdx.x]);
    }
}

// Layered absorber: each staged segment also carries its escape pieces
// (pb_layers.cuh); per photon energy a thread holds every layer's mu and the
// whole-layer optical depths above and below each layer, so a piece's end
// depths cost one FMA each and its transmission the reference's closed form
// (brem.py:1195-1200, segment_escape.py:276-289), weighted by its fraction.
template <class Real>
struct BremPieces {
    int np;
    int m[kMaxEscLayers];
    Real f[kMaxEscLayers], u0[kMaxEscLayers], u1[kMaxEscLayers];
};

constexpr int kBremChunkLayered = 64;

template <class Real>
__global__ void __launch_bounds__(kBremThreads) brem_layered_kernel(const pb_brem_args a, int64_t n_seg, int d0) {
    constexpr int kChunk = kBremChunkLayered;
    __shared__ BremSeg<Real> segs[kChunk];
    __shared__ BremPieces<Real> pcs[kChunk];
    __shared__ double acc[kBremMaxDir][kBremThreads];
    __shared__ Real Zs[kBremMaxEl];
    __shared__ float zl[kBremMaxEl];  // 2 pi alpha Z log2(e)
    __shared__ Real inv_nz[kBremMaxDir];
    __shared__ int up[kBremMaxDir];
    __shared__ double zt_s[kMaxEscLayers], zb_s[kMaxEscLayers];
    __shared__ int bad;
    const int nd = (a.n_dir - d0) < kBremMaxDir ? (a.n_dir - d0) : kBremMaxDir;
    const int n_el = a.n_el;
    const int nl = a.n_layer;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const bool on = e < a.n_E;
    const Real mc2 = (Real)510.99895;
    const Real za = (Real)(2.0 * kPi * kAlphaFs);
    if (threadIdx.x < n_el) {
        Zs[threadIdx.x] = (Real)a.Z[threadIdx.x];
        zl[threadIdx.x] = (float)(2.0 * kPi * kAlphaFs * a.Z[threadIdx.x] * 1.4426950408889634);
    }
    if (threadIdx.x < nd) {
        const Real nz = (Real)a.n_hat[3 * (d0 + threadIdx.x) + 2];
        inv_nz[threadIdx.x] = (Real)1 / fmax(fabs(nz), (Real)1.0e-12);
        up[threadIdx.x] = nz < (Real)0;
    }
    if (threadIdx.x < nl) {
        zt_s[threadIdx.x] = a.z_top[threadIdx.x];
        zb_s[threadIdx.x] = a.z_bot[threadIdx.x];
    }
    if (threadIdx.x == 0) {
        // Contiguous layers in depth order, as the pieces assume.
        int b = 0;
        for (int k = 0; k < nl; ++k) {
            if (!(a.z_bot[k] > a.z_top[k])) b = 1;
            if (k + 1 < nl && fabs(a.z_bot[k] - a.z_top[k + 1]) > 1e-9 * fmax(1.0, fabs(a.z_bot[k]))) b = 1;
        }
        bad = b;
        if (b && a.status) atomicOr(a.status, PB_DEV_BAD_INPUT);
    }
    __syncthreads();
    if (bad) return;
    // Per-energy layer attenuation and whole-layer depths above / below.
    Real mu_l[kMaxEscLayers], t_l[kMaxEscLayers], c_up[kMaxEscLayers], c_dn[kMaxEscLayers];
#pragma unroll
    for (int k = 0; k < kMaxEscLayers; ++k) {
        mu_l[k] = (k < nl && on) ? (Real)a.mu_layer[(int64_t)k * a.n_E + e] : (Real)0;
        t_l[k] = k < nl ? (Real)(zb_s[k] - zt_s[k]) : (Real)0;
    }
    {
        Real run = 0;
#pragma unroll
        for (int k = 0; k < kMaxEscLayers; ++k) {
            c_up[k] = run;
            run += mu_l[k] * t_l[k];
        }
        run = 0;
#pragma unroll
        for (int k = kMaxEscLayers - 1; k >= 0; --k) {
            c_dn[k] = run;
            run += mu_l[k] * t_l[k];
        }
    }
    const double k_kev_d = on ? a.E_grid[e] / 1e3 : 1.0;
    const Real k = (Real)k_kev_d;
    const Real k_ev = fmax((Real)(k_kev_d * 1e3), (Real)1e-30);
    const Real c0 = (Real)(16.0 / 3.0 * kAlphaFs * kReCm2);
    BremKConst kk;
    kk.kc = (float)(k_kev_d / (510.99895 * 510.99895));
    kk.c2mk = (float)(2.0 * 510.99895 - k_kev_d);
    kk.c0k = (float)(16.0 / 3.0 * kAlphaFs * kReCm2 * 0.6931471805599453 / fmax(k_kev_d * 1e3, 1e-30));
#pragma unroll
    for (int j = 0; j < kBremMaxDir; ++j) acc[j][threadIdx.x] = 0.0;
    if (a.n_seg_device) {
        const int64_t live = (int64_t)*a.n_seg_device;
        if (live < n_seg) n_seg = live;
    }
    // Slices of the live segments (the count read on the device), so every
    // block of the wave has work.
    const int64_t per = (n_seg + gridDim.y - 1) / gridDim.y;
    const int64_t s_begin = per * blockIdx.y;
    int64_t s_end = s_begin + per < n_seg ? s_begin + per : n_seg;
    if (s_end < s_begin) s_end = s_begin;
    const Real T_stack = (Real)zb_s[nl - 1];
    for (int64_t c0s = s_begin; c0s < s_end; c0s += kChunk) {
        const int nc = (int)((s_end - c0s) < kChunk ? (s_end - c0s) : kChunk);
        __syncthreads();
        for (int j = threadIdx.x; j < nc; j += blockDim.x) {
            const int64_t s = c0s + j;
            brem_stage<Real>(segs[j], a, s, T_stack, mc2, za);
            const double half = 0.5 * a.L[s];
            const double z = a.r_mid[3 * s + 2], vz = a.v_hat[3 * s + 2];
            EscPiece pp[kMaxEscLayers];
            const int np = esc_pieces(z - half * vz, z + half * vz, nl, zt_s, zb_s, pp);
            BremPieces<Real> &P = pcs[j];
            P.np = np;
            for (int p = 0; p < np; ++p) {
                P.m[p] = pp[p].m;
                P.f[p] = (Real)pp[p].f;
                P.u0[p] = (Real)pp[p].u0;
                P.u1[p] = (Real)pp[p].u1;
            }
        }
        __syncthreads();
        if (!on) continue;
        Real part[kBremMaxDir];
#pragma unroll
        for (int dd = 0; dd < kBremMaxDir; ++dd) part[dd] = 0;
        for (int j = 0; j < nc; ++j) {
            const BremSeg<Real> &b = segs[j];
            const Real T_f = b.T - k;
            if (!(T_f > (Real)1e-6 && k > (Real)0)) continue;
            const Real nsig = brem_nsig<Real>(b, k, T_f, Zs, n_el, k_ev, c0, za, mc2, kk, zl);
            const BremPieces<Real> &P = pcs[j];
            for (int p = 0; p < P.np; ++p) {
                const int m = P.m[p];
                const Real mum = esc_pick<Real>(mu_l, m), tm = esc_pick<Real>(t_l, m);
                const Real cu = esc_pick<Real>(c_up, m), cd = esc_pick<Real>(c_dn, m);
                const Real up0 = cu + mum * P.u0[p], up1 = cu + mum * P.u1[p];
                const Real dn0 = cd + mum * (tm - P.u0[p]), dn1 = cd + mum * (tm - P.u1[p]);
                const Real w = nsig * P.f[p];
#pragma unroll
                for (int dd = 0; dd < kBremMaxDir; ++dd) {
                    if (dd < nd) {
                        const Real f = inv_nz[dd];
                        const Real t0 = (up[dd] ? up0 : dn0) * f;
                        const Real t1 = (up[dd] ? up1 : dn1) * f;
                        part[dd] += w * b_mean_transmission<Real>(t0, t1);
                    }
                }
            }
        }
#pragma unroll
        for (int dd = 0; dd < kBremMaxDir; ++dd) acc[dd][threadIdx.x] += (double)part[dd];
    }
    if (on) {
#pragma unroll
        for (int dd = 0; dd < kBremMaxDir; ++dd)
            if (dd < nd && acc[dd][threadIdx.x] != 0.0)
                atomicAdd(&a.spec[(int64_t)(d0 + dd) * a.n_E + e], acc[dd][threadIdx.x]);
    }
}

cudaError_t launch_brem(const pb_brem_args &a, cudaStream_t s, int sms) {
    if (a.n_el > kBremMaxEl || a.n_el < 1) return cudaErrorInvalidValue;
    if (a.n_layer > 0) {
        if (a.n_layer > kMaxEscLayers) return cudaErrorInvalidValue;
        const unsigned gx = (unsigned)((a.n_E + kBremThreads - 1) / kBremThreads);
        int per_sm = 0;
        cudaError_t oe = a.precision == PB_MIXED
                             ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, brem_layered_kernel<float>,
                                                                             kBremThreads, 0)
                             : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, brem_layered_kernel<double>,
                                                                             kBremThreads, 0);
        if (oe != cudaSuccess) return oe;
        if (per_sm < 1) per_sm = 1;
        int64_t gy = (int64_t)sms * per_sm / (int64_t)gx;
        const int64_t max_y = (a.n_seg + kBremChunkLayered - 1) / kBremChunkLayered;
        if (gy > max_y) gy = max_y;
        if (gy < 1) gy = 1;
        dim3 grid(gx, (unsigned)gy, 1);
        for (int d0 = 0; d0 < a.n_dir; d0 += kBremMaxDir) {
            if (a.precision == PB_MIXED) brem_layered_kernel<float><<<grid, kBremThreads, 0, s>>>(a, a.n_seg, d0);
            else brem_layered_kernel<double><<<grid, kBremThreads, 0, s>>>(a, a.n_seg, d0);
            cudaError_t err = cudaGetLastError();
            if (err != cudaSuccess) return err;
        }
        return cudaSuccess;
    }
    int64_t n_seg = a.n_seg;
    // Mixed precision with a workspace: the depth-node form first; the
    // per-(segment, energy) kernels below then take only the segments it left
    // out (all of them where it does not apply on the device).
    const BremNodeHdr *nh = nullptr;
    const int64_t *nidx = nullptr;
    if (a.precision == PB_MIXED) {
        const cudaError_t ne = launch_brem_node(a, s, sms, &nh, &nidx);
        if (ne != cudaSuccess) return ne;
    }
    const unsigned gx = (unsigned)((a.n_E + kBremThreads - 1) / kBremThreads);
    // One wave: as many segment slices as keep every SM at its resident limit.
    // The kernel instance for this element count (loops over elements unrolled).
    using Kern = void (*)(const pb_brem_args, int64_t, int, const BremNodeHdr *, const int64_t *);
    Kern kern = nullptr;
    if (a.precision == PB_MIXED) {
        const Kern t[kBremMaxEl] = {brem_kernel<float, 1>, brem_kernel<float, 2>, brem_kernel<float, 3>,
                                    brem_kernel<float, 4>};
        kern = t[a.n_el - 1];
    } else {
        const Kern t[kBremMaxEl] = {brem_kernel<double, 1>, brem_kernel<double, 2>, brem_kernel<double, 3>,
                                    brem_kernel<double, 4>};
        kern = t[a.n_el - 1];
    }
    int per_sm = 0;
    cudaError_t oe = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBremThreads, 0);
    if (oe != cudaSuccess) return oe;
    if (per_sm < 1) per_sm = 1;
    int64_t gy = (int64_t)sms * per_sm / (int64_t)gx;
    const int64_t max_y = (n_seg + kBremChunk - 1) / kBremChunk;
    if (gy > max_y) gy = max_y;
    if (gy < 1) gy = 1;
    dim3 grid(gx, (unsigned)gy, 1);
    // Mixed precision: the packed two-energy moment kernel takes the launches
    // whose directions share an exit face within rho <= 0.01; for the others
    // it returns at once and brem_kernel scores them (each kernel makes the
    // same test on the device, so exactly one of the two does the work).
    Kern packed = nullptr;
    dim3 pgrid(1, 1, 1);
    if (a.precision == PB_MIXED) {
        const Kern t[kBremMaxEl] = {brem_moment_packed_kernel<1>, brem_moment_packed_kernel<2>,
                                    brem_moment_packed_kernel<3>, brem_moment_packed_kernel<4>};
        packed = t[a.n_el - 1];
        int pp = 0;
        oe = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pp, packed, kBremPackedThreads, 0);
        if (oe != cudaSuccess) return oe;
        if (pp < 1) pp = 1;
        const unsigned px = (unsigned)((a.n_E + 2 * kBremPackedThreads - 1) / (2 * kBremPackedThreads));
        int64_t py = (int64_t)sms * pp / (int64_t)px;
        if (py > max_y) py = max_y;
        if (py < 1) py = 1;
        pgrid = dim3(px, (unsigned)py, 1);
    }
    for (int d0 = 0; d0 < a.n_dir; d0 += kBremMaxDir) {
        if (packed) {
            packed<<<pgrid, kBremPackedThreads, 0, s>>>(a, n_seg, d0, nh, nidx);
            cudaError_t err = cudaGetLastError();
            if (err != cudaSuccess) return err;
        }
        kern<<<grid, kBremThreads, 0, s>>>(a, n_seg, d0, nh, nidx);
        cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) return err;
    }
    return cudaSuccess;
}

}  // namespace pb
