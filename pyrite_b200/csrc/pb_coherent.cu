// Coherent (field-sum) CXR reduction of per-row line records, sm_100a.
//
// The reference reduces each row (one reflection x mosaic orientation) by
// building the dense complex matrix SP[line, E] = F_j(E) exp(i phi_j(E)) in
// chunks and contracting it with the line coefficients, two complex GEMVs per
// chunk (cxr/_batched_finalize.py:209-243); its CUDA form gives one block per
// energy and strides the lines over threads (coherent_jit_kernel.py:118-240).
// Here the work is a line-chunk x energy-tile grid: a CTA stages up to
// kStage line records into shared memory (80 bytes each, read back as
// broadcasts), every thread owns kEPT energies and sums the four field
// components of both polarisations in registers, and writes them once per
// work item (row, chunk of lines). A second kernel adds a row's chunks in
// FP64, in item order, squares, weights and sums the rows -- deterministic,
// with no atomics.
//
// Precision: the propagation phase phi = phase_slope E - g_phase - L_esc
// delta_omega(E) reaches 1e8 rad (emission time over hbar c times E), and the
// formation argument v = a_vac (E - E_vac) - half_dL delta_omega reaches
// 1e5 rad. Both are formed in FP64, in turns, and their integer parts removed
// there (round to nearest by adding and subtracting 1.5 * 2^52); g_phase is
// reduced once per line. The remaining fractions go to the SFU sine and
// cosine in FP32 (absolute error about 2^-21 on [-pi, pi]). Near resonance,
// |v| <= 1, sin v and cos v come instead from their Taylor series about 0
// (Horner form in v^2, to the v^11 and v^12 terms: truncation below 2e-10),
// since the formation factor divides sin v by v there.
#include <cstdint>

#include "pb_internal.h"

namespace pb {
namespace {

constexpr int kThreads = 256;
constexpr int kEPT = 2;                        // energies per thread
constexpr int kETile = kThreads * kEPT;        // energies per CTA
constexpr int kStage = 128;                    // lines per shared-memory stage
constexpr int64_t kMinChunk = 256;             // lines per work item, lower bound
constexpr int64_t kTargetItemsTimesTiles = 148 * 8;
constexpr float kSeriesW2 = 1.0e-6f;           // _formation.py:55 FORMATION_SERIES_W2

// One line record as the field loop reads it: phase terms in turns.
struct alignas(16) CohLine {
    double ps_t;    // phase_slope / 2 pi
    double L_t;     // L_esc / 2 pi
    double Ev;      // E_vac
    double a, h;    // a_vac, half_dL
    float gp_frac;  // g_phase / 2 pi minus its nearest integer
    float apb, bma, q, csr, csi, cpr, cpi;
    float pad[2];
};
static_assert(sizeof(CohLine) == 80, "CohLine packs into five 16-byte words");

constexpr double kInv2Pi = 0.15915494309189535;
constexpr double kRound64 = 6755399441055744.0;  // 1.5 * 2^52: x + c - c rounds |x| < 2^51 to an integer
constexpr float kRound32 = 12582912.0f;          // 1.5 * 2^23, for |x| < 2^22
constexpr float kTwoPiF = 6.2831853071795865f;

__host__ __device__ __forceinline__ int64_t imin(int64_t x, int64_t y) { return x < y ? x : y; }
__host__ __device__ __forceinline__ int64_t imax(int64_t x, int64_t y) { return x > y ? x : y; }

__host__ __device__ inline int64_t n_etiles(int n_E) { return (n_E + kETile - 1) / kETile; }

// Lines per work item: enough items for ~8 CTAs per SM over the energy tiles,
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

struct CohArgs {
    const int64_t *row_off;
    const double *E, *dom;
    const double *E_vac, *a_vac, *ps, *gp, *csr, *csi, *cpr, *cpi, *L, *h, *apb, *bma, *q;
    int n_row, n_E;
    float cutoff;  // > 0: |v| window
    int64_t n_line, K, n_item_max;
    const int64_t *item_off;
    float *partial;  // [n_item_max][4][n_E]
};

__global__ void __launch_bounds__(kThreads, 4) coh_field_kernel(const CohArgs a) {
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
    const int64_t j0 = rb + (item - a.item_off[lo]) * a.K;
    const int64_t j1 = imin(j0 + a.K, re);

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

    for (int64_t s0 = j0; s0 < j1; s0 += kStage) {
        const int n = (int)imin(kStage, j1 - s0);
        __syncthreads();  // the previous stage has been read
        if (tid < n) {
            const int64_t j = s0 + tid;
            CohLine l;
            l.ps_t = a.ps[j] * kInv2Pi;
            l.L_t = a.L[j] * kInv2Pi;
            l.Ev = a.E_vac[j];
            const double gt = a.gp[j] * kInv2Pi;
            l.gp_frac = (float)(gt - ((gt + kRound64) - kRound64));
            l.a = a.a_vac[j];
            l.h = a.h[j];
            l.apb = (float)a.apb[j];
            l.bma = (float)a.bma[j];
            l.q = (float)a.q[j];
            l.csr = (float)a.csr[j];
            l.csi = (float)a.csi[j];
            l.cpr = (float)a.cpr[j];
            l.cpi = (float)a.cpi[j];
            l.pad[0] = l.pad[1] = 0.f;
            sm[tid] = l;
        }
        __syncthreads();
        for (int i = 0; i < n; ++i) {
            const CohLine l = sm[i];
#pragma unroll
            for (int m = 0; m < kEPT; ++m) {
                // formation factor of the absorbed piece (_formation.py:84-110)
                const double v = fma(l.a, E[m] - l.Ev, -l.h * D[m]);
                const float vf = (float)v;
                if (a.cutoff > 0.f && fabsf(vf) > a.cutoff) continue;
                const float w2 = fmaf(l.q, l.q, vf * vf);
                float fr, fi;
                if (w2 < kSeriesW2) {
                    const float half = 0.5f * l.apb;
                    fr = half * (1.f - l.q * l.q * (1.f / 3.f) - vf * vf * (1.f / 6.f));
                    fi = -half * l.q * vf * (1.f / 3.f);
                } else {
                    float sv, cv;
                    if (fabsf(vf) <= 1.f) {
                        sincos_taylor(vf, sv, cv);
                    } else {
                        const double tv = v * kInv2Pi;
                        __sincosf((float)(tv - ((tv + kRound64) - kRound64)) * kTwoPiF, &sv, &cv);
                    }
                    const float inv = __fdividef(1.f, 2.f * w2);
                    fr = (vf * l.apb * sv - l.q * l.bma * cv) * inv;
                    fi = -(vf * l.bma * cv + l.q * l.apb * sv) * inv;
                }
                // propagation phase (_batched_finalize.py:213-215), in turns
                const double t = fma(l.ps_t, E[m], -l.L_t * D[m]);
                float x = (float)(t - ((t + kRound64) - kRound64)) - l.gp_frac;
                x -= (x + kRound32) - kRound32;
                float sp, cp;
                __sincosf(x * kTwoPiF, &sp, &cp);
                const float pr = fr * cp - fi * sp;
                const float pi = fr * sp + fi * cp;
                acc[m][0] += l.csr * pr - l.csi * pi;
                acc[m][1] += l.csr * pi + l.csi * pr;
                acc[m][2] += l.cpr * pr - l.cpi * pi;
                acc[m][3] += l.cpr * pi + l.cpi * pr;
            }
        }
    }
#pragma unroll
    for (int m = 0; m < kEPT; ++m) {
        const int e = e_base + m * kThreads;
        if (e < a.n_E) {
#pragma unroll
            for (int c = 0; c < 4; ++c) a.partial[((size_t)item * 4 + c) * a.n_E + e] = acc[m][c];
        }
    }
}

// spec[e] += scale * sum_r w_r (|sum_items F_sigma|^2 + |sum_items F_pi|^2).
__global__ void __launch_bounds__(256) coh_finalize_kernel(int n_row, int n_E, const int64_t *__restrict__ item_off,
                                                           const double *__restrict__ w_row,
                                                           const float *__restrict__ partial, double scale,
                                                           double *__restrict__ spec) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_E) return;
    double total = 0.0;
    int64_t i0 = item_off[0];
    for (int r = 0; r < n_row; ++r) {
        const int64_t i1 = item_off[r + 1];
        if (i1 > i0) {
            double f[4] = {0.0, 0.0, 0.0, 0.0};
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

}  // namespace

uint64_t coherent_work_bytes(int n_row, int64_t n_line, int n_E) {
    const int64_t K = chunk_lines(n_line, n_E);
    const int64_t items = max_items(n_row, n_line, K);
    return align256((size_t)(n_row + 1) * sizeof(int64_t)) + (size_t)items * 4 * (size_t)n_E * sizeof(float);
}

cudaError_t launch_coherent(const pb_coherent_args &p, cudaStream_t s) {
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
    dim3 grid((unsigned)n_item_max, (unsigned)n_etiles(p.n_E));
    coh_field_kernel<<<grid, kThreads, 0, s>>>(a);
    coh_finalize_kernel<<<(p.n_E + 255) / 256, 256, 0, s>>>(p.n_row, p.n_E, item_off, p.row_weight, partial,
                                                            p.scale, p.spec);
    return cudaGetLastError();
}

}  // namespace pb
