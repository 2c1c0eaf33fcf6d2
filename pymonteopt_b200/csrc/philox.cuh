// philox.cuh — Philox4x32-10 on the device.
//
// Written from the published algorithm (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11).  Counter and key
// layout of this engine: key = (seed_lo, seed_hi); counter = (n, stream,
// photon_lo, photon_hi), which is also cuRAND's Philox4_32_10 layout for
// curand_init(seed, subsequence = photon, offset = 4 * n) when stream == 0.
#pragma once
#include <cstdint>

namespace pmo {

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c.x;
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

// 32-bit word -> uniform in (0, 1]: ((x >> 8) + 1) * 2^-24, exact in float
// and in double, so the FP32 and FP64 builds consume identical draws.
template <typename R>
__device__ __forceinline__ R u01(uint32_t x) {
    return (R)((x >> 8) + 1u) * (R)5.9604644775390625e-8;
}

}  // namespace pmo
