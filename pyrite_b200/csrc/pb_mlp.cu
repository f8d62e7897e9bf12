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
// FP32, SiLU, storage in bf16 row-major and/or transposed.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

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

__device__ __forceinline__ float sigmoidf_(float x) { return 1.0f / (1.0f + __expf(-x)); }

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
                    const float z = g.dsilu_z[(int64_t)m * g.ldz + n];
                    const float sg = sigmoidf_(z);
                    x *= sg * (1.0f + z * (1.0f - sg));
                }
                if (g.out_f32) {
                    float *o = g.out_f32 + (int64_t)m * g.ldc + n;
                    *o = g.beta != 0.0f ? x + g.beta * *o : x;
                }
                const float h = g.act == 1 ? x * sigmoidf_(x) : x;
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

}  // namespace pb
