// Characteristic-line yields of a segment list (sm_100a).
//
// Per segment row r and direction d, for every line j of one emitting
// element (src/pyrite/montecarlo/spectrum/characteristic.py:837-900 and the
// fused chunk kernel _characteristic_chunk_kernel.py:120-190):
//   sigma_s  = masked linear interpolation of shell s's ionisation table at
//              the row's energy (characteristic.py:760-801, numpy interp);
//   sigma_j  = sum_s sigma_s response[s][j]                (shells in order);
//   per linear escape piece p of the row (segment_escape.py:191-268):
//     tau0/1 = sum_k path_start/end[p][k] mu[k][j]         (layers in order),
//     y     += n 1e24 (L f_p 1e-8) sigma_j <exp(-tau)>(tau0, tau1);
// and line_yield[d][j] += sum over rows.
//
// Work split: a persistent grid strides over segments, one per thread. The
// escape pieces of a row depend on the direction only through n_z, so each
// thread forms them once per direction; the per-line sums are reduced over
// the warp by shuffles and added to a block-shared [n_dir][n_line] FP64
// accumulator, published with one global atomic per entry per block.
#include <cstdint>

#include "pb_common.cuh"
#include "pb_internal.h"

namespace pb {

constexpr int kCharThreads = 256;
constexpr int kCharMaxShell = 40;
constexpr int kCharMaxLine = 256;
constexpr int kCharMaxLayer = 8;

// numpy.interp at q on one shell table, with the scorer's in-range mask.
__device__ __forceinline__ double shell_interp(double q, const double *e, const double *v, int64_t n) {
    if (!(q >= e[0] && q <= e[n - 1])) return 0.0;
    int64_t lo = 0, hi = n - 1;  // e[lo] <= q < e[hi] (or q == e[n-1])
    if (q == e[n - 1]) return v[n - 1];
    while (hi - lo > 1) {
        const int64_t m = (lo + hi) >> 1;
        if (e[m] <= q) lo = m; else hi = m;
    }
    const double slope = (v[hi] - v[lo]) / (e[hi] - e[lo]);
    return slope * (q - e[lo]) + v[lo];
}

// Segment mean of exp(-tau) for tau linear between t0 and t1
// (segment_escape.py:291-303): exp(-min) (1 - exp(-d))/d, series below 1e-4.
template <bool kMixed>
__device__ __forceinline__ double mean_transmission_d(double t0, double t1) {
    const double lo = fmin(t0, t1);
    const double d = fabs(t1 - t0);
    if constexpr (kMixed) {
        const float df = (float)d;
        const float ratio = d > 1.0e-4 ? -expm1f(-df) / df : (1.0f - 0.5f * df) + (df * df) * (1.0f / 6.0f);
        return (double)(__expf(-(float)lo) * ratio);
    } else {
        const double ratio = d > 1.0e-4 ? -expm1(-d) / d : (1.0 - 0.5 * d) + (d * d) / 6.0;
        return exp(-lo) * ratio;
    }
}

// Escape path per layer from depth z along a direction with z-component n_z
// (segment_escape.py:33-76 for the laterally infinite slab / layer stack).
__device__ __forceinline__ void paths_at(double z, double n_z, double thickness, int n_layer, const double *z_top,
                                         const double *z_bot, double *out) {
    const double inv = 1.0 / fmax(fabs(n_z), 1.0e-12);
    if (n_layer == 0) {
        const double depth = fmin(fmax(z, 0.0), thickness);
        out[0] = n_z < 0.0 ? depth * inv : (thickness - depth) * inv;
        return;
    }
    for (int k = 0; k < n_layer; ++k) {
        const double dz = n_z < 0.0 ? fmax(fmin(z, z_bot[k]) - z_top[k], 0.0)
                                    : fmax(z_bot[k] - fmax(z, z_top[k]), 0.0);
        out[k] = dz * inv;
    }
}

template <bool kMixed>
__global__ void __launch_bounds__(kCharThreads) char_yield_kernel(const pb_char_args a) {
    extern __shared__ __align__(16) double acc[];  // [n_dir][n_line]
    int64_t n_seg = a.n_seg;
    if (a.n_seg_device && (int64_t)*a.n_seg_device < n_seg) n_seg = (int64_t)*a.n_seg_device;
    const int n_dir = a.n_dir, n_line = a.n_line, n_shell = a.n_shell;
    const int n_k = a.n_layer > 0 ? a.n_layer : 1;
    const int tid = threadIdx.x, lane = tid & 31;
    for (int i = tid; i < n_dir * n_line; i += blockDim.x) acc[i] = 0.0;
    __syncthreads();

    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    // Every thread of a warp runs the same number of iterations so the
    // shuffles below see the full warp.
    const int64_t n_iter = (n_seg + stride - 1) / stride;
    for (int64_t it = 0; it < n_iter; ++it) {
        const int64_t s = it * stride + (int64_t)blockIdx.x * blockDim.x + tid;
        const bool valid = s < n_seg && a.elec_id[s] < a.Ne && (a.seg_layer == nullptr || a.seg_layer[s] == a.emit_layer);
        double sig[kCharMaxShell];
        double r0z = 0.0, r1z = 0.0, path_cm = 0.0;
        // Pieces: cut fractions at the interior layer boundaries, sorted.
        double cuts[kCharMaxLayer + 1];
        int n_cut = 0;
        if (valid) {
            const double L = a.L[s];
            const double vz = a.v_hat[3 * s + 2];
            r0z = a.r_mid[3 * s + 2] - 0.5 * L * vz;
            r1z = a.r_mid[3 * s + 2] + 0.5 * L * vz;
            path_cm = a.n_atoms * 1.0e24 * (L * 1.0e-8);
            const double q = a.E_keV[s] * 1.0e3;
            for (int sh = 0; sh < n_shell; ++sh) {
                const int64_t o = a.shell_offset[sh];
                sig[sh] = shell_interp(q, a.shell_E + o, a.shell_sigma + o, a.shell_offset[sh + 1] - o);
            }
            cuts[n_cut++] = 0.0;
            cuts[n_cut++] = 1.0;
            for (int k = 1; k < a.n_layer; ++k) {
                const double st = r0z - a.z_top[k], en = r1z - a.z_top[k];
                const double den = st - en;
                const double f = st / (den == 0.0 ? 1.0 : den);
                cuts[n_cut++] = (f > 0.0 && f < 1.0) ? f : 1.0;
            }
            for (int i = 1; i < n_cut; ++i) {  // insertion sort
                const double v = cuts[i];
                int j = i - 1;
                while (j >= 0 && cuts[j] > v) { cuts[j + 1] = cuts[j]; --j; }
                cuts[j + 1] = v;
            }
        }
        for (int d = 0; d < n_dir; ++d) {
            const double n_z = a.n_hat[3 * d + 2];
            for (int j = 0; j < n_line; ++j) {
                double y = 0.0;
                if (valid) {
                    double sj = 0.0;
                    for (int sh = 0; sh < n_shell; ++sh) sj = sj + sig[sh] * a.response[(int64_t)sh * n_line + j];
                    if (sj != 0.0) {
                        double p0[kCharMaxLayer], p1[kCharMaxLayer];
                        for (int c = 0; c + 1 < n_cut; ++c) {
                            const double frac = cuts[c + 1] - cuts[c];
                            if (!(frac > 1.0e-12)) continue;
                            if (a.n_layer == 0) {
                                paths_at(r0z, n_z, a.thickness, 0, nullptr, nullptr, p0);
                                paths_at(r1z, n_z, a.thickness, 0, nullptr, nullptr, p1);
                            } else {
                                // Sample the affine piece at 1/4 and 3/4 and extrapolate
                                // to its ends (segment_escape.py:256-268).
                                const double dz = r1z - r0z;
                                const double zq = r0z + (cuts[c] + 0.25 * frac) * dz;
                                const double z3 = r0z + (cuts[c] + 0.75 * frac) * dz;
                                double q1[kCharMaxLayer], q3[kCharMaxLayer];
                                paths_at(zq, n_z, a.thickness, a.n_layer, a.z_top, a.z_bot, q1);
                                paths_at(z3, n_z, a.thickness, a.n_layer, a.z_top, a.z_bot, q3);
                                for (int k = 0; k < n_k; ++k) {
                                    p0[k] = fmax(1.5 * q1[k] - 0.5 * q3[k], 0.0);
                                    p1[k] = fmax(1.5 * q3[k] - 0.5 * q1[k], 0.0);
                                }
                            }
                            double t0 = 0.0, t1 = 0.0;
                            for (int k = 0; k < n_k; ++k) {
                                const double m = a.mu[(int64_t)k * n_line + j];
                                t0 = t0 + p0[k] * m;
                                t1 = t1 + p1[k] * m;
                            }
                            const double pc = a.n_layer == 0 ? path_cm : path_cm * frac;
                            y += (pc * sj) * mean_transmission_d<kMixed>(t0, t1);
                        }
                    }
                }
                for (int o = 16; o > 0; o >>= 1) y += __shfl_down_sync(0xffffffffu, y, o);
                if (lane == 0 && y != 0.0) atomicAdd(&acc[d * n_line + j], y);
            }
        }
    }
    __syncthreads();
    for (int i = tid; i < n_dir * n_line; i += blockDim.x)
        if (acc[i] != 0.0) atomicAdd(&a.line_yield[i], acc[i]);
}

__global__ void char_spectrum_kernel(int n_line, int n_E, const double *yield, const double *profiles,
                                     double *spec) {
    const int d = blockIdx.y;
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n_E) return;
    double acc = 0.0;
    for (int j = 0; j < n_line; ++j) acc += yield[(int64_t)d * n_line + j] * profiles[(int64_t)j * n_E + b];
    spec[(int64_t)d * n_E + b] += acc;
}

cudaError_t launch_char(const pb_char_args &a, cudaStream_t s, int sms) {
    if (a.n_shell > kCharMaxShell || a.n_line > kCharMaxLine || a.n_layer > kCharMaxLayer)
        return cudaErrorInvalidValue;
    const int64_t n_seg = a.n_seg;  // capacity; the kernel reads n_seg_device itself
    if (n_seg <= 0) return cudaSuccess;
    const size_t smem = sizeof(double) * (size_t)a.n_dir * a.n_line;
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    auto kern = a.precision == PB_MIXED ? char_yield_kernel<true> : char_yield_kernel<false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kCharThreads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    int64_t blocks = (n_seg + kCharThreads - 1) / kCharThreads;
    if (blocks > (int64_t)sms * per_sm) blocks = (int64_t)sms * per_sm;
    kern<<<(unsigned)blocks, kCharThreads, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_char_spectrum(int n_dir, int n_line, int n_E, const double *yield, const double *profiles,
                                 double *spec, cudaStream_t s) {
    dim3 grid((unsigned)((n_E + 127) / 128), (unsigned)n_dir);
    char_spectrum_kernel<<<grid, 128, 0, s>>>(n_line, n_E, yield, profiles, spec);
    return cudaGetLastError();
}

}  // namespace pb
