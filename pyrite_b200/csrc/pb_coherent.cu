// Coherent (field-sum) CXR reduction of per-row line records, sm_100a.
//
// The reference reduces each row (one reflection x mosaic orientation) by
// building the dense complex matrix SP[line, E] = F_j(E) exp(i phi_j(E)) in
// chunks and contracting it with the line coefficients, two complex GEMVs per
// chunk (cxr/_batched_finalize.py:209-243); its CUDA form gives one block per
// energy and strides the lines over threads (coherent_jit_kernel.py:118-240).
// Here the work is a line-chunk x energy-tile grid: a CTA stages up to
// kStage line records into shared memory (96 bytes each, read back as
// broadcasts), every thread owns kEPT energies and sums the four field
// components of both polarisations in registers, and writes them once per
// work item (row, chunk of lines). A second kernel adds a row's chunks in
// FP64, in item order, squares, weights and sums the rows -- deterministic,
// with no atomics.
//
// Precision: the propagation phase phi = phase_slope E - g_phase - L_esc
// delta_omega(E) reaches 1e8 rad (emission time over hbar c times E), and the
// formation argument v = a_vac (E - E_vac) - half_dL delta_omega reaches
// 1e5 rad. Both are formed in FP64, in turns, as a chain of FMAs that
// carries the constant 1.5 * 2^29: the sum then lies in [2^29, 2^30), whose
// unit in the last place is 2^-23 turn, so the low 23 bits of its mantissa
// are the fractional turn -- one bit mask instead of a rounding, a
// subtraction and a conversion. A line whose terms could leave that binade
// (checked per line against the CTA's energies) takes the plain FP64 path
// instead: turns reduced by adding and subtracting 1.5 * 2^52, converted to
// FP32. The fractions go to the SFU sine and cosine (absolute error about
// 2^-21 on [-pi, pi]). Near resonance, |v| <= 1, sin v and cos v come from
// their Taylor series about 0 (Horner form in v^2, to the v^11 and v^12
// terms: truncation below 2e-10), since the formation factor divides sin v
// by v there.
#include <cstdint>

#include "pb_internal.h"

namespace pb {
namespace {

constexpr int kThreads = 256;
constexpr int kEPT = 4;                        // energies per thread
constexpr int kETile = kThreads * kEPT;        // energies per CTA
constexpr int kStage = 128;                    // lines per shared-memory stage
constexpr int64_t kMinChunk = 256;             // lines per work item, lower bound
constexpr int64_t kTargetItemsTimesTiles = 148 * 3 * 4;  // ~4 waves of 3 CTAs per SM
constexpr float kSeriesW2 = 1.0e-6f;           // _formation.py:55 FORMATION_SERIES_W2

// One line record as the field loop reads it, phases in turns. ``fast``
// lines hold the offset forms Gx = 1.5 * 2^29 - g_phase / 2 pi and
// Vx = 1.5 * 2^29 - a_vac E_vac / 2 pi; the others hold g_phase / 2 pi and
// E_vac.
struct alignas(16) CohLine {
    double ps_t, L_t, a_t, h_t;  // phase_slope, L_esc, a_vac, half_dL over 2 pi
    double Gx, Vx;
    float apb, bma, q, qapb, qbma, csr, csi, cpr, cpi;
    int fast;
    float pad[2];
};
static_assert(sizeof(CohLine) == 96, "CohLine packs into six 16-byte words");

constexpr double kInv2Pi = 0.15915494309189535;
constexpr double kRound64 = 6755399441055744.0;  // 1.5 * 2^52: x + c - c rounds |x| < 2^51 to an integer
constexpr float kTwoPiF = 6.2831853071795865f;
constexpr double kTurnBase = 805306368.0;        // 1.5 * 2^29
constexpr double kFastLimit = 134217728.0;       // 2^27 turns: offset sums stay in [2^29, 2^30)

// (sin, cos) of 2 pi f, f the fraction of x - kTurnBase, for x in [2^29, 2^30).
__device__ __forceinline__ void sincos_turns_offset(double x, float &s, float &c) {
    const unsigned lo = (unsigned)__double2loint(x);
    const float g = __uint_as_float((lo & 0x7FFFFFu) | 0x3F800000u) - 1.5f;  // f - 1/2 in [-1/2, 1/2)
    float sg, cg;
    __sincosf(g * kTwoPiF, &sg, &cg);
    s = -sg;  // sin(2 pi f) = -sin(2 pi (f - 1/2))
    c = -cg;
}

// (sin, cos) of 2 pi t for any FP64 t with |t| < 2^51.
__device__ __forceinline__ void sincos_turns(double t, float &s, float &c) {
    __sincosf((float)(t - ((t + kRound64) - kRound64)) * kTwoPiF, &s, &c);
}

__host__ __device__ __forceinline__ int64_t imin(int64_t x, int64_t y) { return x < y ? x : y; }
__host__ __device__ __forceinline__ int64_t imax(int64_t x, int64_t y) { return x > y ? x : y; }

__host__ __device__ inline int64_t n_etiles(int n_E) { return (n_E + kETile - 1) / kETile; }

// Lines per work item: enough items for ~4 waves over the energy tiles,
// never below kMinChunk, a multiple of kStage.
__host__ inline int64_t chunk_lines(int64_t n_line, int n_E) {
    int64_t items = kTargetItemsTimesTiles / n_etiles(n_E);
    if (items < 1) items = 1;
    int64_t k = (n_line + items - 1) / items;
    if (k < kMinChunk) k = kMinChunk;
    return (k + kStage - 1) / kStage * kStage;
}

// sum_r ceil(count_r / K) <= floor(n_line / K) + n_row for any partition.
__host__ inline int64_t max_items(int n_row, int64_t n_line, int64_t K) { return n_row + n_line / K; }

__host__ inline size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// One block: item_off[r] = sum_{s<r} ceil(count_s / K), clamped to n_item_max.
// Row bounds are clamped into [0, n_line] and made nondecreasing, so a bad
// row_off never sends the field kernel outside the record arrays; it is
// flagged in ``status``.
__global__ void __launch_bounds__(1024) coh_items_kernel(const int64_t *__restrict__ row_off, int n_row,
                                                         int64_t n_line, int64_t K, int64_t n_item_max,
                                                         int64_t *__restrict__ item_off,
                                                         unsigned int *__restrict__ status) {
    __shared__ int64_t part[1024];
    const int tid = threadIdx.x;
    const int per = (n_row + 1023) / 1024;
    const int r0 = min(n_row, tid * per), r1 = min(n_row, r0 + per);
    bool bad = false;
    int64_t s = 0;
    for (int r = r0; r < r1; ++r) {
        const int64_t a = row_off[r], b = row_off[r + 1];
        if (a < 0 || b < a || b > n_line) bad = true;
        const int64_t cnt = imax(0, imin(b, n_line) - imax(a, 0));
        s += (cnt + K - 1) / K;
    }
    if (tid == 0 && (row_off[0] != 0 || row_off[n_row] != n_line)) bad = true;
    part[tid] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int64_t v = tid >= off ? part[tid - off] : 0;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    int64_t base = part[tid] - s;
    for (int r = r0; r < r1; ++r) {
        const int64_t a = row_off[r], b = row_off[r + 1];
        const int64_t cnt = imax(0, imin(b, n_line) - imax(a, 0));
        item_off[r] = imin(base, n_item_max);
        base += (cnt + K - 1) / K;
    }
    if (tid == 1023) item_off[n_row] = imin(part[1023], n_item_max);
    if (bad && status) atomicOr(status, PB_DEV_BAD_INPUT);
}

// sin v and cos v for |v| <= 1 from their Taylor series (Horner in v^2).
__device__ __forceinline__ void sincos_taylor(float v, float &sv, float &cv) {
    const float z = v * v;
    float ps = fmaf(z, -1.f / 39916800.f, 1.f / 362880.f);
    ps = fmaf(z, ps, -1.f / 5040.f);
    ps = fmaf(z, ps, 1.f / 120.f);
    ps = fmaf(z, ps, -1.f / 6.f);
    sv = fmaf(v * z, ps, v);
    float pc = fmaf(z, 1.f / 479001600.f, -1.f / 3628800.f);
    pc = fmaf(z, pc, 1.f / 40320.f);
    pc = fmaf(z, pc, -1.f / 720.f);
    pc = fmaf(z, pc, 1.f / 24.f);
    pc = fmaf(z, pc, -0.5f);
    cv = fmaf(z, pc, 1.f);
}

// acc += (c_sigma, c_pi) F(v) exp(i phi): the formation factor of the
// absorbed piece (_formation.py:84-110, series below |w|^2 < 1e-6) rotated by
// the propagation phase (_batched_finalize.py:213-218).
__device__ __forceinline__ void add_line_field(const CohLine &l, float vf, float sv, float cv, float sp, float cp,
                                               float acc[4]) {
    const float w2 = fmaf(l.q, l.q, vf * vf);
    float fr, fi;
    if (w2 < kSeriesW2) {
        const float half = 0.5f * l.apb;
        fr = half * (1.f - l.q * l.q * (1.f / 3.f) - vf * vf * (1.f / 6.f));
        fi = -half * l.q * vf * (1.f / 3.f);
    } else {
        const float inv = __fdividef(0.5f, w2);
        fr = fmaf(vf * l.apb, sv, -l.qbma * cv) * inv;
        fi = -fmaf(vf * l.bma, cv, l.qapb * sv) * inv;
    }
    const float pr = fmaf(fr, cp, -fi * sp);
    const float pi = fmaf(fr, sp, fi * cp);
    acc[0] = fmaf(l.csr, pr, fmaf(-l.csi, pi, acc[0]));
    acc[1] = fmaf(l.csr, pi, fmaf(l.csi, pr, acc[1]));
    acc[2] = fmaf(l.cpr, pr, fmaf(-l.cpi, pi, acc[2]));
    acc[3] = fmaf(l.cpr, pi, fmaf(l.cpi, pr, acc[3]));
}

// The same term added to the row's field and to the current electron's.
__device__ __forceinline__ void add_line_field2(const CohLine &l, float vf, float sv, float cv, float sp, float cp,
                                                float acc[4], float acc_e[4]) {
    float t[4] = {0.f, 0.f, 0.f, 0.f};
    add_line_field(l, vf, sv, cv, sp, cp, t);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        acc[c] += t[c];
        acc_e[c] += t[c];
    }
}

struct CohArgs {
    const int64_t *row_off;
    const double *E, *dom;
    const double *E_vac, *a_vac, *ps, *gp, *csr, *csi, *cpr, *cpi, *L, *h, *apb, *bma, *q;
    int n_row, n_E;
    float cutoff;  // > 0: |v| window
    int64_t n_line, K, n_item_max;
    const int64_t *item_off;
    float *partial;  // [n_item_max][4][n_E]
    // Decoherence blend only: electron of every line (nondecreasing inside a
    // row), the per-item sum over electrons of each electron's own squared
    // field [n_item_max][n_E], and the status word for unordered electrons.
    const int64_t *elec;
    float *power;
    unsigned int *status;
};

// kGrouped: items start and end on electron boundaries (the nominal bounds
// moved forward past lines of the electron that straddles them; adjacent
// items move a shared bound alike, so the items still partition the row),
// and besides the row's field the kernel sums every electron's own field,
// squares it where the electron ends and adds the squares up per item.
template <bool kGrouped>
__global__ void __launch_bounds__(kThreads, kGrouped ? 2 : 3) coh_field_kernel(const CohArgs a) {
    __shared__ CohLine sm[kStage];
    const int64_t item = blockIdx.x;
    const int64_t n_item = a.item_off[a.n_row];
    if (item >= n_item) return;  // uniform over the block
    // Row of this item: the largest r with item_off[r] <= item.
    int lo = 0, hi = a.n_row;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (a.item_off[mid] <= item) lo = mid;
        else hi = mid;
    }
    const int64_t rb = imin(imax(a.row_off[lo], 0), a.n_line);
    const int64_t re = imin(imax(a.row_off[lo + 1], rb), a.n_line);
    int64_t j0 = imin(rb + (item - a.item_off[lo]) * a.K, re);
    int64_t j1 = imin(j0 + a.K, re);
    if constexpr (kGrouped) {
        while (j0 > rb && j0 < re && a.elec[j0] == a.elec[j0 - 1]) ++j0;
        while (j1 > rb && j1 < re && a.elec[j1] == a.elec[j1 - 1]) ++j1;
    }

    const int tid = threadIdx.x;
    const int e_base = blockIdx.y * kETile + tid;
    double E[kEPT], D[kEPT];
#pragma unroll
    for (int m = 0; m < kEPT; ++m) {
        const int e = e_base + m * kThreads;
        E[m] = e < a.n_E ? a.E[e] : 0.0;
        D[m] = e < a.n_E ? a.dom[e] : 0.0;
    }
    float acc[kEPT][4];
#pragma unroll
    for (int m = 0; m < kEPT; ++m) acc[m][0] = acc[m][1] = acc[m][2] = acc[m][3] = 0.f;
    // kGrouped: the current electron's field and the item's sum of squares
    float acc_e[kGrouped ? kEPT : 1][4], pw[kGrouped ? kEPT : 1];
#pragma unroll
    for (int m = 0; m < (kGrouped ? kEPT : 1); ++m) acc_e[m][0] = acc_e[m][1] = acc_e[m][2] = acc_e[m][3] = pw[m] = 0.f;

    // largest |E| and |delta_omega| of this CTA's energies (for the fast-path check)
    __shared__ double red[2][kThreads / 32];
    double em = 0.0, dm = 0.0;
#pragma unroll
    for (int m = 0; m < kEPT; ++m) {
        em = fmax(em, fabs(E[m]));
        dm = fmax(dm, fabs(D[m]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        em = fmax(em, __shfl_xor_sync(0xffffffffu, em, o));
        dm = fmax(dm, __shfl_xor_sync(0xffffffffu, dm, o));
    }
    if ((tid & 31) == 0) {
        red[0][tid >> 5] = em;
        red[1][tid >> 5] = dm;
    }
    __syncthreads();
    double Emax = 0.0, Dmax = 0.0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) {
        Emax = fmax(Emax, red[0][w]);
        Dmax = fmax(Dmax, red[1][w]);
    }

    for (int64_t s0 = j0; s0 < j1; s0 += kStage) {
        const int n = (int)imin(kStage, j1 - s0);
        __syncthreads();  // the previous stage has been read
        if (tid < n) {
            const int64_t j = s0 + tid;
            CohLine l;
            l.ps_t = a.ps[j] * kInv2Pi;
            l.L_t = a.L[j] * kInv2Pi;
            l.a_t = a.a_vac[j] * kInv2Pi;
            l.h_t = a.h[j] * kInv2Pi;
            const double gt = a.gp[j] * kInv2Pi, Ev = a.E_vac[j];
            const double phase_span = fabs(l.ps_t) * Emax + fabs(gt) + fabs(l.L_t) * Dmax;
            const double v_span = fabs(l.a_t) * (Emax + fabs(Ev)) + fabs(l.h_t) * Dmax;
            l.fast = phase_span < kFastLimit && v_span < kFastLimit;  // false for NaN too
            l.Gx = l.fast ? kTurnBase - gt : gt;
            l.Vx = l.fast ? kTurnBase - l.a_t * Ev : Ev;
            l.apb = (float)a.apb[j];
            l.bma = (float)a.bma[j];
            l.q = (float)a.q[j];
            l.qapb = l.q * l.apb;
            l.qbma = l.q * l.bma;
            l.csr = (float)a.csr[j];
            l.csi = (float)a.csi[j];
            l.cpr = (float)a.cpr[j];
            l.cpi = (float)a.cpi[j];
            l.pad[0] = l.pad[1] = 0.f;
            if constexpr (kGrouped) {
                if (j > j0) {
                    const int64_t ep = a.elec[j - 1], ej = a.elec[j];
                    l.pad[0] = ej != ep ? 1.f : 0.f;  // an electron starts here
                    if (ej < ep && a.status) atomicOr(a.status, PB_DEV_BAD_INPUT);
                }
            }
            sm[tid] = l;
        }
        __syncthreads();
        for (int i = 0; i < n; ++i) {
            const CohLine l = sm[i];
            if constexpr (kGrouped) {
                if (l.pad[0] != 0.f) {  // uniform: close the previous electron
#pragma unroll
                    for (int m = 0; m < kEPT; ++m) {
                        pw[m] += acc_e[m][0] * acc_e[m][0] + acc_e[m][1] * acc_e[m][1] +
                                 acc_e[m][2] * acc_e[m][2] + acc_e[m][3] * acc_e[m][3];
                        acc_e[m][0] = acc_e[m][1] = acc_e[m][2] = acc_e[m][3] = 0.f;
                    }
                }
            }
            if (l.fast) {  // uniform over the block: one line at a time
#pragma unroll
                for (int m = 0; m < kEPT; ++m) {
                    const double vx = fma(l.a_t, E[m], fma(-l.h_t, D[m], l.Vx));
                    const float vf = (float)(vx - kTurnBase) * kTwoPiF;
                    if (a.cutoff > 0.f && fabsf(vf) > a.cutoff) continue;
                    float sv, cv, sp, cp;
                    if (fabsf(vf) <= 1.f) sincos_taylor(vf, sv, cv);
                    else sincos_turns_offset(vx, sv, cv);
                    sincos_turns_offset(fma(l.ps_t, E[m], fma(-l.L_t, D[m], l.Gx)), sp, cp);
                    if constexpr (kGrouped) add_line_field2(l, vf, sv, cv, sp, cp, acc[m], acc_e[m]);
                    else add_line_field(l, vf, sv, cv, sp, cp, acc[m]);
                }
            } else {
#pragma unroll
                for (int m = 0; m < kEPT; ++m) {
                    const double vt = fma(l.a_t, E[m] - l.Vx, -l.h_t * D[m]);
                    const float vf = (float)vt * kTwoPiF;
                    if (a.cutoff > 0.f && fabsf(vf) > a.cutoff) continue;
                    float sv, cv, sp, cp;
                    if (fabsf(vf) <= 1.f) sincos_taylor(vf, sv, cv);
                    else sincos_turns(vt, sv, cv);
                    sincos_turns(fma(l.ps_t, E[m], -fma(l.L_t, D[m], l.Gx)), sp, cp);
                    if constexpr (kGrouped) add_line_field2(l, vf, sv, cv, sp, cp, acc[m], acc_e[m]);
                    else add_line_field(l, vf, sv, cv, sp, cp, acc[m]);
                }
            }
        }
    }
#pragma unroll
    for (int m = 0; m < kEPT; ++m) {
        const int e = e_base + m * kThreads;
        if (e < a.n_E) {
#pragma unroll
            for (int c = 0; c < 4; ++c) a.partial[((size_t)item * 4 + c) * a.n_E + e] = acc[m][c];
            if constexpr (kGrouped)
                a.power[(size_t)item * a.n_E + e] = pw[m] + acc_e[m][0] * acc_e[m][0] + acc_e[m][1] * acc_e[m][1] +
                                                    acc_e[m][2] * acc_e[m][2] + acc_e[m][3] * acc_e[m][3];
        }
    }
}

// spec[e] += scale * sum_r w_r (|sum_items F_sigma|^2 + |sum_items F_pi|^2).
// One thread per energy walks every item of every row in order, so the loop
// is unrolled to keep several partial loads in flight (the adds stay in item
// order: the result does not change) and blocks are small, spreading the
// energies over more SMs.
constexpr int kFinalizeThreads = 64;

__global__ void __launch_bounds__(kFinalizeThreads)
    coh_finalize_kernel(int n_row, int n_E, const int64_t *__restrict__ item_off, const double *__restrict__ w_row,
                        const float *__restrict__ partial, double scale, double *__restrict__ spec) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_E) return;
    double total = 0.0;
    int64_t i0 = item_off[0];
    for (int r = 0; r < n_row; ++r) {
        const int64_t i1 = item_off[r + 1];
        if (i1 > i0) {
            double f[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 4
            for (int64_t i = i0; i < i1; ++i) {
#pragma unroll
                for (int c = 0; c < 4; ++c) f[c] += (double)partial[((size_t)i * 4 + c) * n_E + e];
            }
            total += w_row[r] * (f[0] * f[0] + f[1] * f[1] + f[2] * f[2] + f[3] * f[3]);
        }
        i0 = i1;
    }
    spec[e] += scale * total;
}

// The sampled-bunch blend (_batched_finalize.py:163-243):
// spec[e] += scale * sum_r w_r (F_r(e) |sum_items F|^2 + (1 - F_r(e)) sum_items power),
// rows and items in order, as coh_finalize_kernel.
__global__ void __launch_bounds__(kFinalizeThreads)
    coh_finalize_blend_kernel(int n_row, int n_E, const int64_t *__restrict__ item_off,
                              const double *__restrict__ w_row, const double *__restrict__ F_row,
                              const float *__restrict__ partial, const float *__restrict__ power, double scale,
                              double *__restrict__ spec) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_E) return;
    double total = 0.0;
    int64_t i0 = item_off[0];
    for (int r = 0; r < n_row; ++r) {
        const int64_t i1 = item_off[r + 1];
        if (i1 > i0) {
            double f[4] = {0.0, 0.0, 0.0, 0.0}, g = 0.0;
#pragma unroll 4
            for (int64_t i = i0; i < i1; ++i) {
#pragma unroll
                for (int c = 0; c < 4; ++c) f[c] += (double)partial[((size_t)i * 4 + c) * n_E + e];
                g += (double)power[(size_t)i * n_E + e];
            }
            const double F = F_row[(size_t)r * n_E + e];
            const double flat = f[0] * f[0] + f[1] * f[1] + f[2] * f[2] + f[3] * f[3];
            total += w_row[r] * (F * flat + (1.0 - F) * g);
        }
        i0 = i1;
    }
    spec[e] += scale * total;
}

// Streamed route: fold this call's item partials into the persistent FP64
// field planes of every row (and the per-electron power planes), one thread
// per (row, energy), items in order -- one writer per cell, no atomics.
__global__ void coh_fold_kernel(int n_row, int n_E, const int64_t *__restrict__ item_off,
                                const float *__restrict__ partial, const float *__restrict__ power,
                                double *__restrict__ fields, double *__restrict__ pw_planes) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_E) return;
    for (int r = blockIdx.y; r < n_row; r += gridDim.y) {  // grid.y <= 65535 rows at a time
        const int64_t i0 = item_off[r], i1 = item_off[r + 1];
        if (i1 <= i0) continue;
        double f[4] = {0.0, 0.0, 0.0, 0.0}, g = 0.0;
        for (int64_t i = i0; i < i1; ++i) {
#pragma unroll
            for (int c = 0; c < 4; ++c) f[c] += (double)partial[((size_t)i * 4 + c) * n_E + e];
            if (power) g += (double)power[(size_t)i * n_E + e];
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) fields[((size_t)r * 4 + c) * n_E + e] += f[c];
        if (power) pw_planes[(size_t)r * n_E + e] += g;
    }
}

// spec[e] += scale sum_r w_r (F |field|^2 + (1 - F) power), F = 1 without
// row factors; rows in order.
__global__ void coh_stream_finalize_kernel(int n_row, int n_E, const double *__restrict__ w_row,
                                           const double *__restrict__ fields, const double *__restrict__ pw_planes,
                                           const double *__restrict__ F_row, double scale,
                                           double *__restrict__ spec) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_E) return;
    double total = 0.0;
    for (int r = 0; r < n_row; ++r) {
        const double *f = fields + (size_t)r * 4 * n_E + e;
        const double flat = f[0] * f[0] + f[(size_t)n_E] * f[(size_t)n_E] + f[2 * (size_t)n_E] * f[2 * (size_t)n_E] +
                            f[3 * (size_t)n_E] * f[3 * (size_t)n_E];
        if (F_row) {
            const double F = F_row[(size_t)r * n_E + e];
            total += w_row[r] * (F * flat + (1.0 - F) * pw_planes[(size_t)r * n_E + e]);
        } else {
            total += w_row[r] * flat;
        }
    }
    spec[e] += scale * total;
}

// F_r(e) = |(1/N) sum_p exp(i (omega_e A_p - g_r,perp . xy0_p))|^2
// (cxr/_per_hkl.py:121-160, cxr/_setup.py:745-760), FP64 throughout: one
// thread per (row, energy), the population staged in shared memory.
constexpr int kDecohThreads = 256;
constexpr int kDecohStage = 512;

__global__ void __launch_bounds__(kDecohThreads)
    decoherence_kernel(int n_row, int n_pop, int n_E, const double *__restrict__ G, const double *__restrict__ A,
                       const double *__restrict__ xy0, const double *__restrict__ omega, double *__restrict__ F) {
    __shared__ double sA[kDecohStage], sB[kDecohStage];
    const int r = blockIdx.y;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const double gx = G[3 * r], gy = G[3 * r + 1];
    const double w = e < n_E ? omega[e] : 0.0;
    double cr = 0.0, ci = 0.0;
    for (int p0 = 0; p0 < n_pop; p0 += kDecohStage) {
        const int n = min(kDecohStage, n_pop - p0);
        __syncthreads();
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            sA[k] = A[p0 + k];
            sB[k] = __dadd_rn(__dmul_rn(xy0[2 * (p0 + k)], gx), __dmul_rn(xy0[2 * (p0 + k) + 1], gy));
        }
        __syncthreads();
        for (int k = 0; k < n; ++k) {
            double sn, cs;
            sincos(__dsub_rn(__dmul_rn(w, sA[k]), sB[k]), &sn, &cs);
            cr += cs;
            ci += sn;
        }
    }
    if (e < n_E) {
        cr /= n_pop;
        ci /= n_pop;
        F[(size_t)r * n_E + e] = cr * cr + ci * ci;
    }
}

}  // namespace

cudaError_t launch_decoherence(const pb_decoherence_args &p, cudaStream_t s) {
    dim3 grid((unsigned)((p.n_E + kDecohThreads - 1) / kDecohThreads), (unsigned)p.n_row);
    decoherence_kernel<<<grid, kDecohThreads, 0, s>>>(p.n_row, p.n_pop, p.n_E, p.G, p.A_pop, p.xy0_pop, p.omega,
                                                      p.F);
    return cudaGetLastError();
}

uint64_t coherent_blend_work_bytes(int n_row, int64_t n_line, int n_E) {
    const int64_t K = chunk_lines(n_line, n_E);
    const int64_t items = max_items(n_row, n_line, K);
    return coherent_work_bytes(n_row, n_line, n_E) + align256((size_t)items * (size_t)n_E * sizeof(float));
}

uint64_t coherent_work_bytes(int n_row, int64_t n_line, int n_E) {
    const int64_t K = chunk_lines(n_line, n_E);
    const int64_t items = max_items(n_row, n_line, K);
    return align256((size_t)(n_row + 1) * sizeof(int64_t)) + (size_t)items * 4 * (size_t)n_E * sizeof(float);
}

int64_t coherent_items(int n_row, int64_t n_line, int n_E) {
    return max_items(n_row, n_line, chunk_lines(n_line, n_E));
}

cudaError_t launch_coherent_impl(const pb_coherent_args &p, const int64_t *elec, const double *F_row,
                                 cudaStream_t s, double *fields = nullptr, double *pw_planes = nullptr) {
    const int64_t K = chunk_lines(p.n_line, p.n_E);
    const int64_t n_item_max = max_items(p.n_row, p.n_line, K);
    auto *item_off = static_cast<int64_t *>(p.work);
    auto *partial = reinterpret_cast<float *>(static_cast<char *>(p.work) +
                                              align256((size_t)(p.n_row + 1) * sizeof(int64_t)));
    coh_items_kernel<<<1, 1024, 0, s>>>(p.row_off, p.n_row, p.n_line, K, n_item_max, item_off, p.status);
    CohArgs a;
    a.row_off = p.row_off;
    a.E = p.E;
    a.dom = p.delta_omega;
    a.E_vac = p.E_vac;
    a.a_vac = p.a_vac;
    a.ps = p.phase_slope;
    a.gp = p.g_phase;
    a.csr = p.cs_re;
    a.csi = p.cs_im;
    a.cpr = p.cp_re;
    a.cpi = p.cp_im;
    a.L = p.L_esc;
    a.h = p.half_dL;
    a.apb = p.apb;
    a.bma = p.bma;
    a.q = p.q;
    a.n_row = p.n_row;
    a.n_E = p.n_E;
    a.cutoff = (float)p.sinc_cutoff;
    a.n_line = p.n_line;
    a.K = K;
    a.n_item_max = n_item_max;
    a.item_off = item_off;
    a.partial = partial;
    a.elec = elec;
    a.power = elec ? reinterpret_cast<float *>(reinterpret_cast<char *>(partial) +
                                               (size_t)n_item_max * 4 * (size_t)p.n_E * sizeof(float))
                   : nullptr;
    a.status = p.status;
    dim3 grid((unsigned)n_item_max, (unsigned)n_etiles(p.n_E));
    const unsigned fin_blocks = (unsigned)((p.n_E + kFinalizeThreads - 1) / kFinalizeThreads);
    if (fields) {  // streamed: fold into the persistent planes, no squaring yet
        if (elec) coh_field_kernel<true><<<grid, kThreads, 0, s>>>(a);
        else coh_field_kernel<false><<<grid, kThreads, 0, s>>>(a);
        dim3 fgrid((unsigned)((p.n_E + kFinalizeThreads - 1) / kFinalizeThreads),
                   (unsigned)(p.n_row < 65535 ? p.n_row : 65535));
        coh_fold_kernel<<<fgrid, kFinalizeThreads, 0, s>>>(p.n_row, p.n_E, item_off, partial, elec ? a.power : nullptr,
                                                           fields, pw_planes);
    } else if (elec) {
        coh_field_kernel<true><<<grid, kThreads, 0, s>>>(a);
        coh_finalize_blend_kernel<<<fin_blocks, kFinalizeThreads, 0, s>>>(p.n_row, p.n_E, item_off, p.row_weight,
                                                                          F_row, partial, a.power, p.scale, p.spec);
    } else {
        coh_field_kernel<false><<<grid, kThreads, 0, s>>>(a);
        coh_finalize_kernel<<<fin_blocks, kFinalizeThreads, 0, s>>>(p.n_row, p.n_E, item_off, p.row_weight, partial,
                                                                    p.scale, p.spec);
    }
    return cudaGetLastError();
}

cudaError_t launch_coherent(const pb_coherent_args &p, cudaStream_t s) {
    return launch_coherent_impl(p, nullptr, nullptr, s);
}

cudaError_t launch_coherent_blend(const pb_coherent_blend_args &p, cudaStream_t s) {
    return launch_coherent_impl(p.base, p.elec_id, p.F_row, s);
}

cudaError_t launch_coherent_accumulate(const pb_coherent_stream_args &p, cudaStream_t s) {
    return launch_coherent_impl(p.base, p.elec_id, nullptr, s, p.fields, p.power);
}

cudaError_t launch_coherent_stream_finalize(int n_row, int n_E, const double *w_row, const double *fields,
                                            const double *power, const double *F_row, double scale, double *spec,
                                            cudaStream_t s) {
    coh_stream_finalize_kernel<<<(unsigned)((n_E + kFinalizeThreads - 1) / kFinalizeThreads), kFinalizeThreads, 0,
                                 s>>>(n_row, n_E, w_row, fields, power, F_row, scale, spec);
    return cudaGetLastError();
}

}  // namespace pb
