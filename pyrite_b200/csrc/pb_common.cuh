// Shared device helpers of the pyrite_b200 kernels (sm_100a).
//
// Counter RNGs, physical constants and small numerics. The transport and
// scoring kernels include this header; nothing here holds state.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pyrite_b200.h"

namespace pb {

// Physical constants of the reference (src/pyrite/materials/crystal.py:47-52,
// transport/stopping.py:193-196, spectrum/brem.py:63-64).
constexpr double kHbarcEvAng = 1973.269804;
constexpr double kMeEv = 510998.95;
constexpr double kMc2Kev = 510.99895;
constexpr double kAlphaFs = 1.0 / 137.035999;
constexpr double kLn2 = 0.6931471805599453;
constexpr double kBsPrefactor = 1.535e-6;
constexpr double kReCm2 = 7.9407877e-26;
constexpr double kPi = 3.14159265358979323846;

constexpr uint64_t kPhi = 0x9E3779B97F4A7C15ULL;

// SplitMix64 finalizer used as a counter hash (transport/kinematics.py:205-229).
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

__host__ __device__ __forceinline__ uint64_t stream_key(uint64_t seed, uint64_t elec) {
    return splitmix64(seed + kPhi * (elec + 1ULL));
}

// Draw ``c`` of a SplitMix64 counter stream in [0, 1), 53-bit mantissa.
__device__ __forceinline__ double splitmix_uniform(uint64_t key, uint64_t c) {
    uint64_t z = splitmix64(key + kPhi * (c + 1ULL));
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// Open-interval uniform with a 52-bit mantissa (kinematics.py:270-299).
__device__ __forceinline__ double splitmix_open_uniform(uint64_t key, uint64_t c) {
    uint64_t z = splitmix64(key + kPhi * (c + 1ULL));
    return ((double)(z >> 12) + 0.5) * (1.0 / 4503599627370496.0);
}

// Philox4x32-10 (Salmon et al., SC11): ten rounds on a 128-bit counter with a
// 64-bit key. Multiplier and Weyl constants are the published ones.
__device__ __forceinline__ void philox4x32_10(uint32_t &c0, uint32_t &c1, uint32_t &c2,
                                              uint32_t &c3, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// Draw ``d`` of the Philox stream keyed by ``key``: block d/2 is the counter,
// even draws take words (0,1), odd draws (2,3); 53-bit mantissa in [0, 1).
__device__ __forceinline__ double philox_uniform(uint64_t key, uint64_t d) {
    uint64_t block = d >> 1;
    uint32_t c0 = (uint32_t)block, c1 = (uint32_t)(block >> 32), c2 = 0u, c3 = 0u;
    philox4x32_10(c0, c1, c2, c3, (uint32_t)key, (uint32_t)(key >> 32));
    uint32_t a = (d & 1ULL) ? c2 : c0;
    uint32_t b = (d & 1ULL) ? c3 : c1;
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

template <int kRng>
__device__ __forceinline__ double uniform(uint64_t key, uint64_t c) {
    if constexpr (kRng == PB_RNG_PHILOX) return philox_uniform(key, c);
    else return splitmix_uniform(key, c);
}

// Bounded-wait budget of every mbarrier poll in this library.
constexpr uint32_t kWaitLimit = 1u << 26;

__device__ __forceinline__ void set_status(unsigned int *status, unsigned int bits) {
    if (status) atomicOr(status, bits);
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// One non-multicast bulk copy global -> shared completing on ``mbar``.
// Source and destination 16-byte aligned, ``bytes`` a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *mbar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
        :
        : "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(mbar))
        : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(mbar)), "r"(count)
                 : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(mbar)),
                 "r"(bytes)
                 : "memory");
}

// Bounded parity wait; returns false when the budget ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity) {
    for (uint32_t it = 0; it < kWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_addr(mbar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

}  // namespace pb
