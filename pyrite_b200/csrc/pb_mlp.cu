// BF16 MLP surrogate of the per-segment PXR+CBS spectrum: tcgen05 GEMM with
// fused epilogues (training forward and backward), and the elementwise
// training kernels (MSE gradient, bias gradient, Adam, weight packing).
//
// GEMM: D[M x N] = A[M x K] . B[N x K]^T, A and B bf16 with K contiguous in
// global memory. A block of 128 threads owns a 128 x 256 output tile in
// tensor memory (256 FP32 columns); K advances in 64-wide chunks staged into
// shared memory in the interleaved core-matrix layout (pb_umma.cuh) by
// 16-byte cp.async, double-buffered so the next chunk loads while the tensor
// core consumes this one. One thread issues the MMAs and commits each chunk
// to that stage's mbarrier; every wait is bounded and a timeout is reported
// through the status word. The epilogue reads the accumulator with
// tcgen05.ld (warp w owns rows 32w..32w+31) and applies, in order: bias,
// multiplication by silu'(z) (backward), storage of the pre-activation in
// FP32, SiLU, storage in bf16 row-major and/or transposed. SiLU is the tanh
// form of silu_fast, the one the inference kernel evaluates.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>

#include "pb_common.cuh"
#include "pb_internal.h"
#include "pb_umma.cuh"

namespace pb {

constexpr int kGemmThreads = 128;
constexpr int kGemmBM = 128;
constexpr int kGemmBN = 256;
constexpr int kGemmBK = 64;
constexpr int kGemmStages = 2;
constexpr uint32_t kGemmSboA = (kGemmBK / 8) * 128;  // 1024 B between 8-row groups
constexpr uint32_t kGemmTileA = kGemmBM * kGemmBK * 2;   // 16 KB
constexpr uint32_t kGemmTileB = kGemmBN * kGemmBK * 2;   // 32 KB
constexpr uint32_t kGemmSmem = kGemmStages * (kGemmTileA + kGemmTileB) + 64;

// SiLU as x (1 + tanh(x / 2)) / 2 with the hardware tanh approximation; the
// training and inference kernels use this same form (and its derivative), so
// the trained function is the one inference evaluates.
__device__ __forceinline__ float tanh_fast(float x) {
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(x));
    return t;
}
__device__ __forceinline__ float silu_fast(float x) { return 0.5f * x * (1.0f + tanh_fast(0.5f * x)); }
__device__ __forceinline__ float dsilu_fast(float z) {
    const float t = tanh_fast(0.5f * z);
    return 0.5f * (1.0f + t) + 0.25f * z * (1.0f - t * t);
}

// Stage one K chunk of A (128 rows) and B (256 rows) into shared memory;
// rows or columns outside the matrices are zero-filled.
__device__ __forceinline__ void gemm_load_chunk(const pb_mlp_gemm_args &g, int m0, int n0, int k0, int kc,
                                                uint8_t *sA, uint8_t *sB) {
    const int tid = threadIdx.x;
    const uint32_t a_base = smem_addr(sA), b_base = smem_addr(sB);
    for (int p = tid; p < kGemmBM * (kGemmBK / 8); p += kGemmThreads) {
        const int r = p >> 3, c = p & 7;
        const uint32_t off = umma::core_offset((uint32_t)r, (uint32_t)(c * 8), kGemmSboA);
        if (m0 + r < g.M && c * 8 < kc) {
            umma::cp_async16(a_base + off, reinterpret_cast<const __nv_bfloat16 *>(g.A) + (int64_t)(m0 + r) * g.lda + k0 + c * 8);
        } else {
            *reinterpret_cast<uint4 *>(sA + off) = make_uint4(0u, 0u, 0u, 0u);
        }
    }
    for (int p = tid; p < kGemmBN * (kGemmBK / 8); p += kGemmThreads) {
        const int r = p >> 3, c = p & 7;
        const uint32_t off = umma::core_offset((uint32_t)r, (uint32_t)(c * 8), kGemmSboA);
        if (n0 + r < g.N && c * 8 < kc) {
            umma::cp_async16(b_base + off, reinterpret_cast<const __nv_bfloat16 *>(g.B) + (int64_t)(n0 + r) * g.ldb + k0 + c * 8);
        } else {
            *reinterpret_cast<uint4 *>(sB + off) = make_uint4(0u, 0u, 0u, 0u);
        }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

__global__ void __launch_bounds__(kGemmThreads) mlp_gemm_kernel(const pb_mlp_gemm_args g) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *sA[kGemmStages], *sB[kGemmStages];
    for (int s = 0; s < kGemmStages; ++s) {
        sA[s] = smem + s * (kGemmTileA + kGemmTileB);
        sB[s] = sA[s] + kGemmTileA;
    }
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + kGemmStages * (kGemmTileA + kGemmTileB));
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + kGemmStages);
    volatile int *s_ok = reinterpret_cast<volatile int *>(tslot + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * kGemmBM, n0 = blockIdx.y * kGemmBN;
    const int nt = min(kGemmBN, g.N - n0);
    const int nt16 = (nt + 15) & ~15;

    if (warp == 0) {
        umma::tmem_alloc(tslot, 256);
        umma::tmem_relinquish();
    }
    if (tid == 0) {
        for (int s = 0; s < kGemmStages; ++s) mbar_init(&mbar[s], 1);
        *s_ok = 1;
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t taddr = *tslot;
    const uint32_t idesc = umma::idesc_bf16_f32(128, (uint32_t)nt16);
    const int n_chunks = (g.K + kGemmBK - 1) / kGemmBK;
    // Only thread 0 issues MMAs and waits on their mbarriers; the outcome of
    // each wait reaches the block through *s_ok after a barrier.
    uint32_t phase[kGemmStages] = {0u, 0u};

    gemm_load_chunk(g, m0, n0, 0, min(kGemmBK, g.K), sA[0], sB[0]);
    for (int ch = 0; ch < n_chunks; ++ch) {
        const int s = ch % kGemmStages;
        const int k0 = ch * kGemmBK;
        const int kc = min(kGemmBK, g.K - k0);
        if (ch + 1 < n_chunks) {
            const int s1 = (ch + 1) % kGemmStages;
            if (ch + 1 >= kGemmStages && tid == 0) {
                // The stage's previous MMAs must finish before it is refilled.
                if (!mbar_wait(&mbar[s1], phase[s1])) *s_ok = 0;
                phase[s1] ^= 1u;
            }
            __syncthreads();
            if (!*s_ok) break;
            gemm_load_chunk(g, m0, n0, k0 + kGemmBK, min(kGemmBK, g.K - k0 - kGemmBK), sA[s1], sB[s1]);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        umma::fence_smem_to_async();
        __syncthreads();
        if (tid == 0) {
            umma::fence_after_sync();
            const uint32_t a0 = smem_addr(sA[s]), b0 = smem_addr(sB[s]);
            for (int ks = 0; ks < kc / 16; ++ks) {
                const uint64_t ad = umma::smem_desc(a0 + ks * 256u, 128u, kGemmSboA);
                const uint64_t bd = umma::smem_desc(b0 + ks * 256u, 128u, kGemmSboA);
                umma::mma_bf16(taddr, ad, bd, idesc, (ch > 0 || ks > 0) ? 1u : 0u);
            }
            umma::commit(&mbar[s]);
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    if (tid == 0) {
        // The last chunk's commit covers every MMA issued before it.
        const int s_last = (n_chunks - 1) % kGemmStages;
        if (*s_ok) {
            if (!mbar_wait(&mbar[s_last], phase[s_last])) *s_ok = 0;
        }
        if (!*s_ok) {
            set_status(g.status, PB_DEV_WAIT_TIMEOUT);
            for (int st = 0; st < kGemmStages; ++st) mbar_wait(&mbar[st], phase[st]);  // bounded drain
        }
    }
    __syncthreads();
    const bool ok = *s_ok != 0;
    umma::fence_after_sync();

    if (ok) {
        const int m = m0 + warp * 32 + lane;
        for (int c0 = 0; c0 < nt16; c0 += 16) {
            float v[16];
            umma::tmem_ld16(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (m >= g.M) continue;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int n = n0 + c0 + i;
                if (n >= g.N) break;
                float x = v[i];
                if (g.bias) x += g.bias[n];
                if (g.dsilu_z) {
                    x *= dsilu_fast(g.dsilu_z[(int64_t)m * g.ldz + n]);
                }
                if (g.out_f32) {
                    float *o = g.out_f32 + (int64_t)m * g.ldc + n;
                    *o = g.beta != 0.0f ? x + g.beta * *o : x;
                }
                const float h = g.act == 1 ? silu_fast(x) : x;
                if (g.out_bf16) reinterpret_cast<__nv_bfloat16 *>(g.out_bf16)[(int64_t)m * g.ldh + n] = __float2bfloat16_rn(h);
                if (g.out_bf16_t) reinterpret_cast<__nv_bfloat16 *>(g.out_bf16_t)[(int64_t)n * g.ldt + m] = __float2bfloat16_rn(h);
            }
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(taddr, 256);
}

cudaError_t launch_mlp_gemm(const pb_mlp_gemm_args &g, cudaStream_t s) {
    cudaError_t e = cudaFuncSetAttribute(mlp_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem);
    if (e != cudaSuccess) return e;
    dim3 grid((unsigned)((g.M + kGemmBM - 1) / kGemmBM), (unsigned)((g.N + kGemmBN - 1) / kGemmBN));
    mlp_gemm_kernel<<<grid, kGemmThreads, kGemmSmem, s>>>(g);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Elementwise training kernels
// ---------------------------------------------------------------------------

// dY = scale (Y - T) in bf16, row-major and transposed; loss += sum (Y - T)^2.
__global__ void mse_grad_kernel(int rows, int cols, const float *Y, const __nv_bfloat16 *T, int64_t ldt_in,
                                float t_scale, float g_scale, __nv_bfloat16 *dY, __nv_bfloat16 *dYt, int64_t ld_t,
                                float *loss) {
    float acc = 0.0f;
    const int64_t n = (int64_t)rows * cols;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(i / cols), c = (int)(i - (int64_t)r * cols);
        const float d = Y[i] - t_scale * __bfloat162float(T[(int64_t)r * ldt_in + c]);
        acc += d * d;
        const __nv_bfloat16 g = __float2bfloat16_rn(g_scale * d);
        dY[i] = g;
        dYt[(int64_t)c * ld_t + r] = g;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc != 0.0f) atomicAdd(loss, acc);
}

// Group-aggregate loss: rows come in groups of S (one detector direction and
// S segments each); with w the rows' normalised weights, per group and output
//   A_hat = sum_s w_s Y_s,  A = t_scale sum_s w_s T_s,  d = A_hat - A,
// loss += d^2 and dY_s = g_scale w_s d (bf16, row-major and transposed).
__global__ void group_mse_grad_kernel(int groups, int S, int cols, const float *Y, const __nv_bfloat16 *T,
                                      int64_t ldt_in, const float *w, float t_scale, float g_scale, __nv_bfloat16 *dY,
                                      __nv_bfloat16 *dYt, int64_t ld_t, float *loss) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    const int g = blockIdx.y;
    float acc = 0.0f;
    if (o < cols) {
        float ah = 0.0f, at = 0.0f;
        for (int s = 0; s < S; ++s) {
            const int64_t r = (int64_t)g * S + s;
            ah += w[r] * Y[r * cols + o];
            at += w[r] * __bfloat162float(T[r * ldt_in + o]);
        }
        const float d = ah - t_scale * at;
        acc = d * d;
        for (int s = 0; s < S; ++s) {
            const int64_t r = (int64_t)g * S + s;
            const __nv_bfloat16 v = __float2bfloat16_rn(g_scale * w[r] * d);
            dY[r * cols + o] = v;
            dYt[(int64_t)o * ld_t + r] = v;
        }
    }
    for (int k = 16; k > 0; k >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, k);
    if ((threadIdx.x & 31) == 0 && acc != 0.0f) atomicAdd(loss, acc);
}

cudaError_t launch_mlp_group_mse_grad(int groups, int S, int cols, const float *Y, const void *T, int64_t ldt_in,
                                      const float *w, float t_scale, float g_scale, void *dY, void *dYt, int64_t ld_t,
                                      float *loss, cudaStream_t s) {
    dim3 grid((unsigned)((cols + 127) / 128), (unsigned)groups);
    group_mse_grad_kernel<<<grid, 128, 0, s>>>(groups, S, cols, Y, (const __nv_bfloat16 *)T, ldt_in, w, t_scale,
                                               g_scale, (__nv_bfloat16 *)dY, (__nv_bfloat16 *)dYt, ld_t, loss);
    return cudaGetLastError();
}

// out[c] += sum_r X[r][c] (FP32).
__global__ void colsum_kernel(int rows, int cols, const float *X, int64_t ld, float *out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    const int r0 = blockIdx.y * 256, r1 = min(rows, r0 + 256);
    float acc = 0.0f;
    for (int r = r0; r < r1; ++r) acc += X[(int64_t)r * ld + c];
    atomicAdd(&out[c], acc);
}

// Adam with decoupled weight decay on a packed FP32 parameter vector.
__global__ void adam_kernel(int64_t n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2,
                            float eps, float wd, float bc1, float bc2) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float mh = mi / bc1, vh = vi / bc2;
        p[i] -= lr * (mh / (sqrtf(vh) + eps) + wd * p[i]);
    }
}

// W [rows][cols] FP32 -> Wb [rows][ldb] bf16 (zero padded to ldb) and
// Wt [cols][ldt] bf16 (transposed, zero padded rows up to pad_cols).
__global__ void pack_weights_kernel(int rows, int cols, const float *W, __nv_bfloat16 *Wb, int ldb,
                                    __nv_bfloat16 *Wt, int ldt, int pad_cols) {
    const int64_t n = (int64_t)rows * ldb;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(i / ldb), c = (int)(i - (int64_t)r * ldb);
        const float w = c < cols ? W[(int64_t)r * cols + c] : 0.0f;
        const __nv_bfloat16 b = __float2bfloat16_rn(w);
        Wb[i] = b;
        if (Wt && c < pad_cols) Wt[(int64_t)c * ldt + r] = b;
    }
}

cudaError_t launch_mlp_mse_grad(int rows, int cols, const float *Y, const void *T, int64_t ldt_in, float t_scale,
                                float g_scale, void *dY, void *dYt, int64_t ld_t, float *loss, cudaStream_t s) {
    const int64_t n = (int64_t)rows * cols;
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
    mse_grad_kernel<<<blocks, 256, 0, s>>>(rows, cols, Y, (const __nv_bfloat16 *)T, ldt_in, t_scale, g_scale,
                                           (__nv_bfloat16 *)dY, (__nv_bfloat16 *)dYt, ld_t, loss);
    return cudaGetLastError();
}

cudaError_t launch_mlp_colsum(int rows, int cols, const float *X, int64_t ld, float *out, cudaStream_t s) {
    dim3 grid((unsigned)((cols + 127) / 128), (unsigned)((rows + 255) / 256));
    colsum_kernel<<<grid, 128, 0, s>>>(rows, cols, X, ld, out);
    return cudaGetLastError();
}

cudaError_t launch_mlp_adam(int64_t n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2,
                            float eps, float wd, float bc1, float bc2, cudaStream_t s) {
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
    adam_kernel<<<blocks, 256, 0, s>>>(n, p, g, m, v, lr, b1, b2, eps, wd, bc1, bc2);
    return cudaGetLastError();
}

cudaError_t launch_mlp_pack(int rows, int cols, const float *W, void *Wb, int ldb, void *Wt, int ldt, int pad_cols,
                            cudaStream_t s) {
    const int64_t n = (int64_t)rows * ldb;
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
    pack_weights_kernel<<<blocks, 256, 0, s>>>(rows, cols, W, (__nv_bfloat16 *)Wb, ldb, (__nv_bfloat16 *)Wt, ldt,
                                               pad_cols);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Fused surrogate inference: features -> 4 x (256, SiLU) -> length-weighted
// per-direction sums of the last hidden layer.
//
// The output layer is linear, so for every direction d
//   sum_s L_s (W5 h4(x_sd) + b5) = W5 (sum_s L_s h4(x_sd)) + b5 sum_s L_s,
// and the kernel only accumulates hsum[d] = sum_s L_s h4 and lsum[d] =
// sum_s L_s; mlp_head_kernel applies W5 and b5 once per direction.
//
// A persistent block (one per SM, 128 threads, thread = row) walks
// contiguous (direction, 128-segment tile) work. Per tile: features -> X
// (128 x 16 bf16) in shared memory; layer 1 is one K=16 MMA against W1 held
// in shared memory; layers 2-4 stream their weights from global memory (L2)
// in four 32 KB K-chunks, pre-packed in the interleaved layout so each chunk
// is one bulk copy, with three chunks kept in flight ahead of the MMAs. Each epilogue reads the
// 128 x 256 FP32 accumulator from tensor memory, adds the bias, applies SiLU
// (x (1 + tanh(x/2)) / 2) and writes bf16 activations back over the layer's
// input in shared memory; the last one weights each row by its segment
// length and reduces the tile's rows with a 16-shuffle transpose-reduce
// into the block's per-direction sum.
// ---------------------------------------------------------------------------
constexpr int kInfThreads = 128;
constexpr uint32_t kInfSboX = 256;    // X: 128 x 16, 2 core matrices along K
constexpr uint32_t kInfSboH = 4096;   // H: 128 x 256
constexpr uint32_t kInfSboW = 1024;   // W chunk: 256 x 64
constexpr uint32_t kInfChunk = 256 * 64 * 2;  // 32 KB
constexpr uint32_t kInfW1 = 256 * 16 * 2;     // 8 KB
constexpr int kInfStages = 4;                 // weight chunk stages: one whole layer in flight
constexpr uint32_t kInfSmem = kInfW1 + 128 * 16 * 2 + 128 * 256 * 2 + kInfStages * kInfChunk + 4 * 256 * 4 + 257 * 4 + 160;


__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&v);
}

// Feature vector of segment s seen from direction d (pb_mlp_infer_args);
// returns the segment's weight (its length, 0 when it does not count).
struct FeatureMap {
    float Ex, Ey, Ez, Fx, Fy, Fz, inv_th, lnElo, inv_lnE, inv_thick;
    __device__ explicit FeatureMap(const pb_mlp_infer_args &a)
        : Ex((float)a.e_x[0]), Ey((float)a.e_x[1]), Ez((float)a.e_x[2]), Fx((float)a.e_y[0]),
          Fy((float)a.e_y[1]), Fz((float)a.e_y[2]), inv_th(1.0f / (float)a.theta_max),
          lnElo(logf((float)a.E_lo_MeV)), inv_lnE(1.0f / (logf((float)a.E_hi_MeV) - logf((float)a.E_lo_MeV))),
          inv_thick(1.0f / (float)a.thickness) {}
    __device__ float operator()(const pb_mlp_infer_args &a, int64_t s, int64_t n_seg, int d, float *x) const {
#pragma unroll
        for (int i = 0; i < 6; ++i) x[i] = 0.0f;
        if (s >= n_seg || a.elec_id[s] >= a.Ne) return 0.0f;
        const float vx = (float)a.v_hat[3 * s], vy = (float)a.v_hat[3 * s + 1], vz = (float)a.v_hat[3 * s + 2];
        x[0] = 2.0f * (logf((float)a.E_keV[s] * 1.0e-3f) - lnElo) * inv_lnE - 1.0f;
        x[1] = (vx * Ex + vy * Ey + vz * Ez) * inv_th;
        x[2] = (vx * Fx + vy * Fy + vz * Fz) * inv_th;
        x[3] = 2.0f * fminf(fmaxf((float)a.r_mid[3 * s + 2] * inv_thick, 0.0f), 1.0f) - 1.0f;
        x[4] = a.dir_uv[2 * d];
        x[5] = a.dir_uv[2 * d + 1];
        return (float)a.L[s];
    }
};

// Training inputs: X[(d n_seg + s)][16] bf16 (features, zero padded) and
// weight[d n_seg + s], exactly the inference kernel's rows.
__global__ void mlp_features_kernel(const pb_mlp_infer_args a, __nv_bfloat16 *X, float *weight) {
    const FeatureMap fm(a);
    const int64_t n = (int64_t)a.n_dir * a.n_seg;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int d = (int)(i / a.n_seg);
        const int64_t s = i - (int64_t)d * a.n_seg;
        float x[6];
        const float w = fm(a, s, a.n_seg, d, x);
        for (int k = 0; k < 16; ++k) X[i * 16 + k] = __float2bfloat16_rn(k < 6 ? x[k] : 0.0f);
        if (weight) weight[i] = w;
    }
}

cudaError_t launch_mlp_features(const pb_mlp_infer_args &a, void *X, float *weight, cudaStream_t s) {
    const int64_t n = (int64_t)a.n_dir * a.n_seg;
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
    mlp_features_kernel<<<blocks, 256, 0, s>>>(a, (__nv_bfloat16 *)X, weight);
    return cudaGetLastError();
}

__global__ void __launch_bounds__(kInfThreads, 1) mlp_infer_kernel(const pb_mlp_infer_args a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *sW1 = smem;
    uint8_t *sX = sW1 + kInfW1;
    uint8_t *sH = sX + 128 * 16 * 2;
    uint8_t *sW = sH + 128 * 256 * 2;  // kInfStages chunk stages
    float *sBias = reinterpret_cast<float *>(sW + kInfStages * kInfChunk);  // [4][256]
    float *sHsum = sBias + 4 * 256;                                          // [256] + lsum
    uint64_t *bar = reinterpret_cast<uint64_t *>(sHsum + 257 + 3);           // 8-byte aligned
    uint64_t *full = bar;                      // [kInfStages] weight chunk landed
    uint64_t *empty = bar + kInfStages;        // [kInfStages] MMAs of the chunk done
    uint64_t *mma_done = bar + 2 * kInfStages;
    uint64_t *w1_bar = mma_done + 1;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(w1_bar + 1);
    volatile int *s_ok = reinterpret_cast<volatile int *>(tslot + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    int64_t n_seg = a.n_seg;
    if (a.n_seg_device && (int64_t)*a.n_seg_device < n_seg) n_seg = (int64_t)*a.n_seg_device;
    const int64_t n_tiles = (n_seg + 127) / 128;
    const int64_t n_work = n_tiles * a.n_dir;
    const int64_t w_begin = n_work * blockIdx.x / gridDim.x;
    const int64_t w_end = n_work * (blockIdx.x + 1) / gridDim.x;

    if (warp == 0) {
        umma::tmem_alloc(tslot, 256);
        umma::tmem_relinquish();
    }
    for (int i = tid; i < 4 * 256; i += kInfThreads) sBias[i] = a.bias[i / 256][i % 256];
    for (int i = tid; i < 257; i += kInfThreads) sHsum[i] = 0.0f;
    if (tid == 0) {
        for (int i = 0; i < 2 * kInfStages + 2; ++i) mbar_init(&bar[i], 1);
        *s_ok = 1;
        mbar_expect_tx(w1_bar, kInfW1);
        bulk_g2s(sW1, a.w1_packed, kInfW1, w1_bar);
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t taddr = *tslot;
    const uint32_t lane_off = (uint32_t)(warp * 32) << 16;
    const uint32_t idesc = umma::idesc_bf16_f32(128, 256);
    // Thread 0's pipeline state.
    uint32_t q_load = 0, q_mma = 0, mma_phase = 0;
    bool w1_ready = false;
    const uint8_t *wsrc[3] = {static_cast<const uint8_t *>(a.w_packed[0]), static_cast<const uint8_t *>(a.w_packed[1]),
                              static_cast<const uint8_t *>(a.w_packed[2])};

    // Issue the bulk copy of chunk q (layer 2 + (q / 4) % 3, K-chunk q % 4)
    // into stage q % kInfStages, once the MMAs of chunk q - kInfStages left it.
    auto load_chunk = [&](uint32_t q) -> bool {
        const uint32_t s = q % kInfStages;
        if (q >= kInfStages && !mbar_wait(&empty[s], (q / kInfStages - 1u) & 1u)) return false;
        const uint32_t layer = (q >> 2) % 3u, kc = q & 3u;
        mbar_expect_tx(&full[s], kInfChunk);
        bulk_g2s(sW + s * kInfChunk, wsrc[layer] + (size_t)kc * kInfChunk, kInfChunk, &full[s]);
        return true;
    };
    if (tid == 0 && w_begin < w_end) {
        for (uint32_t q = 0; q + 1 < (uint32_t)kInfStages; ++q)
            if (!load_chunk(q)) *s_ok = 0;
        q_load = kInfStages - 1;
    }

    const FeatureMap fm(a);
    int d_cur = -1;

    auto flush = [&](int d) {
        __syncthreads();
        if (d >= 0) {
            for (int i = tid; i < 257; i += kInfThreads) {
                const float v = sHsum[i];
                if (v != 0.0f) {
                    if (i < 256) atomicAdd(&a.hsum[(int64_t)d * 256 + i], (double)v);
                    else atomicAdd(&a.lsum[d], (double)v);
                }
                sHsum[i] = 0.0f;
            }
        }
        __syncthreads();
    };

    for (int64_t wk = w_begin; wk < w_end; ++wk) {
        const int d = (int)(wk / n_tiles);
        const int64_t t = wk - (int64_t)d * n_tiles;
        if (d != d_cur) {
            flush(d_cur);
            d_cur = d;
        }
        // ---- features of this thread's row ----
        const int64_t sidx = t * 128 + tid;
        float x[6];
        const float wrow = fm(a, sidx, n_seg, d, x);
        {
            uint4 lo = make_uint4(pack_bf16x2(x[0], x[1]), pack_bf16x2(x[2], x[3]), pack_bf16x2(x[4], x[5]), 0u);
            *reinterpret_cast<uint4 *>(sX + umma::core_offset((uint32_t)tid, 0u, kInfSboX)) = lo;
            *reinterpret_cast<uint4 *>(sX + umma::core_offset((uint32_t)tid, 8u, kInfSboX)) =
                make_uint4(0u, 0u, 0u, 0u);
        }
        umma::fence_smem_to_async();
        __syncthreads();
        if (!*s_ok) break;

        for (int layer = 0; layer < 4; ++layer) {
            // ---- MMAs of this layer (thread 0) ----
            if (tid == 0) {
                umma::fence_after_sync();
                bool good = true;
                if (layer == 0) {
                    if (!w1_ready) {
                        good = mbar_wait(w1_bar, 0u);
                        w1_ready = good;
                    }
                    if (good)
                        umma::mma_bf16(taddr, umma::smem_desc(smem_addr(sX), 128u, kInfSboX),
                                       umma::smem_desc(smem_addr(sW1), 128u, kInfSboX), idesc, 0u);
                } else {
                    for (int kc = 0; kc < 4 && good; ++kc) {
                        const uint32_t s = q_mma % kInfStages;
                        good = mbar_wait(&full[s], (q_mma / kInfStages) & 1u);
                        if (!good) break;
                        const uint32_t w0 = smem_addr(sW + s * kInfChunk);
                        const uint32_t h0 = smem_addr(sH) + (uint32_t)kc * 1024u;  // K offset 64 = 8 core matrices
                        for (int ks = 0; ks < 4; ++ks)
                            umma::mma_bf16(taddr, umma::smem_desc(h0 + ks * 256u, 128u, kInfSboH),
                                           umma::smem_desc(w0 + ks * 256u, 128u, kInfSboW), idesc,
                                           (kc > 0 || ks > 0) ? 1u : 0u);
                        umma::commit(&empty[s]);
                        ++q_mma;
                        // Keep kInfStages - 1 chunks ahead (weights are the same every
                        // tile): the next load reuses the stage of the chunk issued one
                        // step earlier, while the MMAs just issued keep the core busy.
                        if (q_load < q_mma + kInfStages - 1) {
                            good = load_chunk(q_load);
                            ++q_load;
                        }
                    }
                }
                umma::commit(mma_done);
                if (good) good = mbar_wait(mma_done, mma_phase);
                mma_phase ^= 1u;
                if (!good) {
                    *s_ok = 0;
                    set_status(a.status, PB_DEV_WAIT_TIMEOUT);
                }
            }
            __syncthreads();
            if (!*s_ok) break;
            umma::fence_after_sync();
            // ---- epilogue ----
            const float *bias = sBias + layer * 256;
            if (layer < 3) {
                for (int c0 = 0; c0 < 256; c0 += 16) {
                    float v[16];
                    umma::tmem_ld16(taddr + lane_off + (uint32_t)c0, v);
                    uint32_t p[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        p[i] = pack_bf16x2(silu_fast(v[2 * i] + bias[c0 + 2 * i]),
                                           silu_fast(v[2 * i + 1] + bias[c0 + 2 * i + 1]));
                    *reinterpret_cast<uint4 *>(sH + umma::core_offset((uint32_t)tid, (uint32_t)c0, kInfSboH)) =
                        make_uint4(p[0], p[1], p[2], p[3]);
                    *reinterpret_cast<uint4 *>(sH + umma::core_offset((uint32_t)tid, (uint32_t)c0 + 8u, kInfSboH)) =
                        make_uint4(p[4], p[5], p[6], p[7]);
                }
                umma::fence_before_sync();
                umma::fence_smem_to_async();
                __syncthreads();
            } else {
                for (int c0 = 0; c0 < 256; c0 += 16) {
                    float v[16];
                    umma::tmem_ld16(taddr + lane_off + (uint32_t)c0, v);
#pragma unroll
                    for (int i = 0; i < 16; ++i) v[i] = wrow * silu_fast(v[i] + bias[c0 + i]);
                    // Transpose-reduce: after the four halving steps lane l holds
                    // the partial sum of column (l >> 1); the last step adds the pair.
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const bool up = lane & 16;
                        const float send = up ? v[i] : v[i + 8], keep = up ? v[i + 8] : v[i];
                        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const bool up = lane & 8;
                        const float send = up ? v[i] : v[i + 4], keep = up ? v[i + 4] : v[i];
                        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
                    }
#pragma unroll
                    for (int i = 0; i < 2; ++i) {
                        const bool up = lane & 4;
                        const float send = up ? v[i] : v[i + 2], keep = up ? v[i + 2] : v[i];
                        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
                    }
                    {
                        const bool up = lane & 2;
                        const float send = up ? v[0] : v[1], keep = up ? v[1] : v[0];
                        v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
                    }
                    v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
                    if ((lane & 1) == 0) atomicAdd(&sHsum[c0 + (lane >> 1)], v[0]);
                }
                float wsum = wrow;
                for (int o = 16; o > 0; o >>= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
                if (lane == 0 && wsum != 0.0f) atomicAdd(&sHsum[256], wsum);
                umma::fence_before_sync();
                __syncthreads();
            }
        }
        if (!*s_ok) break;
    }
    flush(d_cur);
    if (tid == 0) {
        // Drain weight copies still in flight before the block exits.
        for (uint32_t q = q_mma; q < q_load; ++q) mbar_wait(&full[q % kInfStages], (q / kInfStages) & 1u);
        if (!w1_ready) mbar_wait(w1_bar, 0u);
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(taddr, 256);
}

// ---------------------------------------------------------------------------
// Two-tile ping-pong variant: the epilogues of one tile overlap the MMAs of
// the other.
//
// 576 threads: warps 0-7 and warps 8-15 each own a tile slot -- 256
// tensor-memory columns, an X and an H buffer -- as two warpgroups, one per
// 128-column half of every layer's epilogue; warp 17's lane 0 streams the
// weight chunks through the stages and warp 16's lane 0 issues the MMAs of
// the two slots in the order (layer 1: slot 0, slot 1), (layer 2: slot 0,
// slot 1), ..., so the tensor core works on one slot while the other slot's
// warps run its epilogue, and a weight copy never waits behind an MMA issue. A slot's 256 threads hand it to the producer through in_ready[s]
// (one arrival by its leader after a named-barrier sync of the slot) and get
// the accumulator back through acc_full[s] (tcgen05.commit).
// Blocks own an even number of tiles (an odd range gets one empty tile, all
// of whose rows weigh 0). Every wait is bounded; a timeout sets the status
// word and an abort flag that every role checks after its waits.
// ---------------------------------------------------------------------------
// PB_MLP_INFER=serial selects the single-tile kernel above (the reference
// point for the ping-pong one); the default is the ping-pong kernel.
static int infer_variant() {
    static int v = -1;
    if (v < 0) {
        const char *e = getenv("PB_MLP_INFER");
        v = (e && e[0] == 's') ? 1 : 2;
    }
    return v;
}

constexpr int kPPThreads = 576;
constexpr int kPPProducerWarp = 16;  // MMA issue
constexpr int kPPLoaderWarp = 17;    // weight streaming
constexpr int kPPStages = 2;
constexpr uint32_t kPPChunk = kInfChunk;
constexpr uint32_t kPPSmem = kInfW1 + 2 * (128 * 16 * 2) + 2 * (128 * 256 * 2) + kPPStages * kPPChunk +
                             4 * 256 * 4 + 2 * 257 * 4 + 256;

__device__ __forceinline__ void wg_sync(int slot) {
    asm volatile("bar.sync %0, 256;" ::"r"(1 + slot) : "memory");
}

__global__ void __launch_bounds__(kPPThreads, 1) mlp_infer_pp_kernel(const pb_mlp_infer_args a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *sW1 = smem;
    uint8_t *sX = sW1 + kInfW1;                 // [2] x 4 KB
    uint8_t *sH = sX + 2 * (128 * 16 * 2);      // [2] x 64 KB
    uint8_t *sW = sH + 2 * (128 * 256 * 2);     // kPPStages x 32 KB
    float *sBias = reinterpret_cast<float *>(sW + kPPStages * kPPChunk);   // [4][256]
    float *sHsum = sBias + 4 * 256;                                         // [2][257]
    uint64_t *bar = reinterpret_cast<uint64_t *>(
        (reinterpret_cast<uintptr_t>(sHsum + 2 * 257) + 15) & ~static_cast<uintptr_t>(15));
    uint64_t *full = bar;                        // [kPPStages]
    uint64_t *empty = bar + kPPStages;           // [kPPStages]
    uint64_t *in_ready = bar + 2 * kPPStages;    // [2]
    uint64_t *acc_full = in_ready + 2;           // [2]
    uint64_t *w1_bar = acc_full + 2;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(w1_bar + 1);
    volatile int *s_abort = reinterpret_cast<volatile int *>(tslot + 1);
    volatile int *s_ok = s_abort + 1;  // [2] per-slot result of the leader's last wait

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    int64_t n_seg = a.n_seg;
    if (a.n_seg_device && (int64_t)*a.n_seg_device < n_seg) n_seg = (int64_t)*a.n_seg_device;
    const int64_t n_tiles = (n_seg + 127) / 128;
    const int64_t n_work = n_tiles * a.n_dir;
    const int64_t w_begin = n_work * blockIdx.x / gridDim.x;
    const int64_t w_end = n_work * (blockIdx.x + 1) / gridDim.x;
    const int64_t T = w_end - w_begin;
    const int64_t n_pairs = (T + 1) / 2;

    if (warp == 0) {
        umma::tmem_alloc(tslot, 512);
        umma::tmem_relinquish();
    }
    for (int i = tid; i < 4 * 256; i += kPPThreads) sBias[i] = a.bias[i / 256][i % 256];
    for (int i = tid; i < 2 * 257; i += kPPThreads) sHsum[i] = 0.0f;
    if (tid == 0) {
        for (int i = 0; i < 2 * kPPStages + 5; ++i) mbar_init(&bar[i], 1);
        *s_abort = 0;
        s_ok[0] = s_ok[1] = 1;
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t taddr = *tslot;

    if (warp == kPPLoaderWarp) {
        // -------------------------- loader --------------------------
        // Streams the weight chunks into the stages as soon as the MMAs of a
        // stage's previous chunk are done, independently of the MMA issue.
        if (lane == 0 && n_pairs > 0) {
            const uint8_t *wsrc[3] = {static_cast<const uint8_t *>(a.w_packed[0]),
                                      static_cast<const uint8_t *>(a.w_packed[1]),
                                      static_cast<const uint8_t *>(a.w_packed[2])};
            mbar_expect_tx(w1_bar, kInfW1);
            bulk_g2s(sW1, a.w1_packed, kInfW1, w1_bar);
            // Chunk q of the stream: per tile pair 24 chunks, layer (q % 24) / 8
            // of W2..W4, K-chunk q % 4 (each layer's four chunks twice, once
            // per slot).
            const uint32_t q_total = (uint32_t)n_pairs * 24u;
            bool good = true;
            uint32_t q = 0;
            for (; q < q_total; ++q) {
                const uint32_t st = q % kPPStages;
                if (q >= kPPStages) good = mbar_wait(&empty[st], (q / kPPStages - 1u) & 1u);
                if (!good || *s_abort) break;
                const uint32_t layer = (q % 24u) / 8u, kc = q & 3u;
                mbar_expect_tx(&full[st], kPPChunk);
                bulk_g2s(sW + st * kPPChunk, wsrc[layer] + (size_t)kc * kPPChunk, kPPChunk, &full[st]);
            }
            if (!good) {
                *s_abort = 1;
                set_status(a.status, PB_DEV_WAIT_TIMEOUT);
            }
            // Drain the copies still in flight (bounded) before the block exits:
            // the last kPPStages issued chunks, whose stages nothing reuses.
            for (uint32_t k = q > (uint32_t)kPPStages ? q - kPPStages : 0u; k < q; ++k)
                mbar_wait(&full[k % kPPStages], (k / kPPStages) & 1u);
            mbar_wait(w1_bar, 0u);
        }
    } else if (warp == kPPProducerWarp) {
        // ------------------------- MMA issue -------------------------
        if (lane == 0 && n_pairs > 0) {
            const uint32_t idesc = umma::idesc_bf16_f32(128, 256);
            uint32_t q_mma = 0;
            uint32_t in_phase[2] = {0u, 0u};
            bool good = mbar_wait(w1_bar, 0u);
            for (int64_t p = 0; p < n_pairs && good; ++p) {
                for (int layer = 0; layer < 4 && good; ++layer) {
                    for (int slot = 0; slot < 2 && good; ++slot) {
                        good = mbar_wait(&in_ready[slot], in_phase[slot]);
                        in_phase[slot] ^= 1u;
                        if (!good || *s_abort) { good = false; break; }
                        umma::fence_after_sync();
                        const uint32_t d_tmem = taddr + (uint32_t)(slot * 256);
                        if (layer == 0) {
                            umma::mma_bf16(d_tmem, umma::smem_desc(smem_addr(sX + slot * 4096), 128u, kInfSboX),
                                           umma::smem_desc(smem_addr(sW1), 128u, kInfSboX), idesc, 0u);
                        } else {
                            const uint32_t h0 = smem_addr(sH + slot * 65536);
                            for (int kc = 0; kc < 4 && good; ++kc) {
                                const uint32_t st = q_mma % kPPStages;
                                good = mbar_wait(&full[st], (q_mma / kPPStages) & 1u);
                                if (!good) break;
                                const uint32_t w0 = smem_addr(sW + st * kPPChunk);
                                for (int ks = 0; ks < 4; ++ks)
                                    umma::mma_bf16(d_tmem,
                                                   umma::smem_desc(h0 + (uint32_t)kc * 1024u + ks * 256u, 128u,
                                                                   kInfSboH),
                                                   umma::smem_desc(w0 + ks * 256u, 128u, kInfSboW), idesc,
                                                   (kc > 0 || ks > 0) ? 1u : 0u);
                                umma::commit(&empty[st]);
                                ++q_mma;
                            }
                        }
                        umma::commit(&acc_full[slot]);
                    }
                }
            }
            if (!good) {
                *s_abort = 1;
                set_status(a.status, PB_DEV_WAIT_TIMEOUT);
            }
        }
    } else {
        // --------------------- epilogue warpgroups ---------------------
        const int slot = warp >> 3;
        const int half = (warp >> 2) & 1;     // columns [128 half, 128 half + 128)
        const int rs = tid - 256 * slot;      // thread within the slot
        const int r = rs & 127;               // row of the tile
        const int wq = warp & 3;              // TMEM lanes 32 wq.. (the warp's quadrant)
        const bool leader = rs == 0;
        const int col0 = 128 * half;
        uint8_t *mX = sX + slot * 4096;
        uint8_t *mH = sH + slot * 65536;
        float *hs = sHsum + slot * 257;
        const uint32_t t_base = taddr + (uint32_t)(slot * 256) + ((uint32_t)(wq * 32) << 16);
        const FeatureMap fm(a);
        uint32_t acc_phase = 0;
        int d_cur = -1;
        auto flush = [&](int d) {
            wg_sync(slot);
            if (d >= 0) {
                for (int i = rs; i < 257; i += 256) {
                    const float v = hs[i];
                    if (v != 0.0f) {
                        if (i < 256) atomicAdd(&a.hsum[(int64_t)d * 256 + i], (double)v);
                        else atomicAdd(&a.lsum[d], (double)v);
                    }
                    hs[i] = 0.0f;
                }
            }
            wg_sync(slot);
        };
        // Hand the slot to the producer: every thread's shared-memory writes
        // and tensor-memory reads are done, then one arrival.
        auto hand_over = [&]() {
            umma::fence_smem_to_async();
            umma::fence_before_sync();
            wg_sync(slot);
            if (leader) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&in_ready[slot])) : "memory");
        };
        // Wait for this slot's accumulator; false (for the whole group) on abort.
        auto wait_acc = [&]() -> bool {
            if (leader) {
                const bool ok = mbar_wait(&acc_full[slot], acc_phase) && !*s_abort;
                if (!ok) *s_abort = 1;
                s_ok[slot] = ok ? 1 : 0;
            }
            acc_phase ^= 1u;
            wg_sync(slot);
            const bool ok = s_ok[slot] != 0;
            umma::fence_after_sync();
            return ok;
        };
        for (int64_t p = 0; p < n_pairs; ++p) {
            const int64_t t = 2 * p + slot;
            const bool real = t < T;
            const int64_t wk = w_begin + (real ? t : T - 1);
            const int d = (int)(wk / n_tiles);
            const int64_t tile = wk - (int64_t)d * n_tiles;
            if (real && d != d_cur) {
                flush(d_cur);
                d_cur = d;
            }
            float x[6];
            const float wrow = real ? fm(a, tile * 128 + r, n_seg, d, x) : (fm(a, n_seg, n_seg, d, x), 0.0f);
            if (half == 0) {
                *reinterpret_cast<uint4 *>(mX + umma::core_offset((uint32_t)r, 0u, kInfSboX)) =
                    make_uint4(pack_bf16x2(x[0], x[1]), pack_bf16x2(x[2], x[3]), pack_bf16x2(x[4], x[5]), 0u);
                *reinterpret_cast<uint4 *>(mX + umma::core_offset((uint32_t)r, 8u, kInfSboX)) =
                    make_uint4(0u, 0u, 0u, 0u);
            }
            hand_over();
            bool ok = true;
            for (int layer = 0; layer < 4 && ok; ++layer) {
                ok = wait_acc();
                if (!ok) break;
                const float *bias = sBias + layer * 256;
                if (layer < 3) {
                    for (int c0 = col0; c0 < col0 + 128; c0 += 16) {
                        float v[16];
                        umma::tmem_ld16(t_base + (uint32_t)c0, v);
                        uint32_t pk[8];
#pragma unroll
                        for (int i = 0; i < 8; ++i)
                            pk[i] = pack_bf16x2(silu_fast(v[2 * i] + bias[c0 + 2 * i]),
                                                silu_fast(v[2 * i + 1] + bias[c0 + 2 * i + 1]));
                        *reinterpret_cast<uint4 *>(mH + umma::core_offset((uint32_t)r, (uint32_t)c0, kInfSboH)) =
                            make_uint4(pk[0], pk[1], pk[2], pk[3]);
                        *reinterpret_cast<uint4 *>(mH + umma::core_offset((uint32_t)r, (uint32_t)c0 + 8u, kInfSboH)) =
                            make_uint4(pk[4], pk[5], pk[6], pk[7]);
                    }
                    hand_over();
                } else {
                    for (int c0 = col0; c0 < col0 + 128; c0 += 16) {
                        float v[16];
                        umma::tmem_ld16(t_base + (uint32_t)c0, v);
#pragma unroll
                        for (int i = 0; i < 16; ++i) v[i] = wrow * silu_fast(v[i] + bias[c0 + i]);
#pragma unroll
                        for (int i = 0; i < 8; ++i) {
                            const bool up = lane & 16;
                            const float send = up ? v[i] : v[i + 8], keep = up ? v[i + 8] : v[i];
                            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
                        }
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const bool up = lane & 8;
                            const float send = up ? v[i] : v[i + 4], keep = up ? v[i + 4] : v[i];
                            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
                        }
#pragma unroll
                        for (int i = 0; i < 2; ++i) {
                            const bool up = lane & 4;
                            const float send = up ? v[i] : v[i + 2], keep = up ? v[i + 2] : v[i];
                            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
                        }
                        {
                            const bool up = lane & 2;
                            const float send = up ? v[0] : v[1], keep = up ? v[1] : v[0];
                            v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
                        }
                        v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
                        if ((lane & 1) == 0 && v[0] != 0.0f) atomicAdd(&hs[c0 + (lane >> 1)], v[0]);
                    }
                    float wsum = wrow;
                    for (int o = 16; o > 0; o >>= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
                    if (half == 0 && lane == 0 && wsum != 0.0f) atomicAdd(&hs[256], wsum);
                    // Tensor-memory reads of this slot are complete before the
                    // next tile's features are handed over (hand_over fences).
                }
            }
            if (!ok) break;
        }
        flush(d_cur);
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(taddr, 512);
}

// spec[d][o] += t_scale (sum_k W5[o][k] hsum[d][k] + b5[o] lsum[d]).
__global__ void mlp_head_kernel(int n_dir, int n_out, const float *W5, const float *b5, const double *hsum,
                                const double *lsum, double t_scale, double *spec) {
    const int d = blockIdx.y;
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n_out) return;
    double acc = (double)b5[o] * lsum[d];
    for (int k = 0; k < 256; ++k) acc += (double)W5[(int64_t)o * 256 + k] * hsum[(int64_t)d * 256 + k];
    spec[(int64_t)d * n_out + o] += t_scale * acc;
}

// Segments of every stride-th history (elec_id % stride == 0), appended to
// dst with one atomic per warp; the exact sub-sample of the surrogate's
// control-variate correction.
__global__ void segments_sample_kernel(const pb_segments src, int64_t stride, pb_segments dst, unsigned int *status) {
    const int64_t n = (int64_t)*src.count < src.capacity ? (int64_t)*src.count : src.capacity;
    const int lane = threadIdx.x & 31;
    const int64_t n_iter = (n + (int64_t)gridDim.x * blockDim.x - 1) / ((int64_t)gridDim.x * blockDim.x);
    for (int64_t it = 0; it < n_iter; ++it) {
        const int64_t i = (it * gridDim.x + blockIdx.x) * (int64_t)blockDim.x + threadIdx.x;
        const bool take = i < n && src.elec_id[i] % stride == 0;
        const unsigned mask = __ballot_sync(0xffffffffu, take);
        unsigned long long base = 0;
        if (lane == 0 && mask) base = atomicAdd(dst.count, (unsigned long long)__popc(mask));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (!take) continue;
        const int64_t j = (int64_t)base + __popc(mask & ((1u << lane) - 1u));
        if (j >= dst.capacity) {
            set_status(status, PB_DEV_QUEUE_OVERFLOW);
            continue;
        }
        for (int c = 0; c < 3; ++c) {
            dst.r_mid[3 * j + c] = src.r_mid[3 * i + c];
            dst.v_hat[3 * j + c] = src.v_hat[3 * i + c];
        }
        dst.L[j] = src.L[i];
        dst.E_repr[j] = src.E_repr[i];
        dst.elec_id[j] = src.elec_id[i];
        if (dst.layer && src.layer) dst.layer[j] = src.layer[i];
    }
}

cudaError_t launch_segments_sample(const pb_segments &src, int64_t stride, const pb_segments &dst,
                                   unsigned int *status, cudaStream_t s, int sms) {
    cudaError_t e = cudaMemsetAsync(dst.count, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    int64_t blocks = (src.capacity + 255) / 256;
    if (blocks > (int64_t)sms * 8) blocks = (int64_t)sms * 8;
    if (blocks < 1) blocks = 1;
    segments_sample_kernel<<<(unsigned)blocks, 256, 0, s>>>(src, stride, dst, status);
    return cudaGetLastError();
}

// W FP32 [256][cols] -> interleaved bf16 chunks of kc columns (zero padded).
__global__ void pack_umma_kernel(int cols, int kc, const float *W, __nv_bfloat16 *out) {
    const int n_chunks = (cols + kc - 1) / kc;
    const int64_t n = (int64_t)256 * n_chunks * kc;
    const uint32_t sbo = (uint32_t)(kc / 8) * 128u;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(i / (n_chunks * kc));
        const int k = (int)(i - (int64_t)r * n_chunks * kc);
        const int c = k / kc, kk = k - c * kc;
        const float w = k < cols ? W[(int64_t)r * cols + k] : 0.0f;
        const size_t byte = (size_t)c * 256 * kc * 2 + umma::core_offset((uint32_t)r, (uint32_t)kk, sbo);
        out[byte / 2] = __float2bfloat16_rn(w);
    }
}

cudaError_t launch_mlp_infer(const pb_mlp_infer_args &a, cudaStream_t s, int sms) {
    const int64_t work = (a.n_seg + 127) / 128 * (int64_t)a.n_dir;
    int64_t grid = sms;
    if (grid > work) grid = work;
    if (grid < 1) return cudaSuccess;
    if (infer_variant() == 1) {
        cudaError_t e = cudaFuncSetAttribute(mlp_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kInfSmem);
        if (e != cudaSuccess) return e;
        mlp_infer_kernel<<<(unsigned)grid, kInfThreads, kInfSmem, s>>>(a);
    } else {
        cudaError_t e = cudaFuncSetAttribute(mlp_infer_pp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kPPSmem);
        if (e != cudaSuccess) return e;
        mlp_infer_pp_kernel<<<(unsigned)grid, kPPThreads, kPPSmem, s>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t launch_mlp_head(int n_dir, int n_out, const float *W5, const float *b5, const double *hsum,
                            const double *lsum, double t_scale, double *spec, cudaStream_t s) {
    dim3 grid((unsigned)((n_out + 127) / 128), (unsigned)n_dir);
    mlp_head_kernel<<<grid, 128, 0, s>>>(n_dir, n_out, W5, b5, hsum, lsum, t_scale, spec);
    return cudaGetLastError();
}

cudaError_t launch_mlp_pack_umma(int cols, int kc, const float *W, void *out, cudaStream_t s) {
    const int n_chunks = (cols + kc - 1) / kc;
    const int64_t n = (int64_t)256 * n_chunks * kc;
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
    pack_umma_kernel<<<blocks, 256, 0, s>>>(cols, kc, W, (__nv_bfloat16 *)out);
    return cudaGetLastError();
}

}  // namespace pb
