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

// The ten round keys (k0 + r*W0, k1 + r*W1), r = 0..9, of one key.  Kernels
// get them precomputed in their launch parameters, so each round's key is a
// constant-bank operand instead of two adds per round.
struct PhiloxKeys {
    uint32_t k[20];
};

__host__ __device__ inline PhiloxKeys philox_round_keys(uint32_t k0, uint32_t k1) {
    PhiloxKeys rk;
    for (int r = 0; r < 10; ++r) {
        rk.k[2 * r] = k0 + (uint32_t)r * 0x9E3779B9u;
        rk.k[2 * r + 1] = k1 + (uint32_t)r * 0xBB67AE85u;
    }
    return rk;
}

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, const PhiloxKeys &rk) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c.x;
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ rk.k[2 * r], lo1, hi0 ^ c.w ^ rk.k[2 * r + 1], lo0);
    }
    return c;
}

// Counters (n, y, z, w) whose y and z stay fixed while n runs (a photon's
// draws): in round 0 the product of z, and in round 1 the product of round
// 0's first output word (z's product xor y xor key), do not depend on n.
// PhiloxFixed holds what those two products leave behind, so a draw runs
// rounds 0 and 1 with one multiplier pair each.  The words are those of
// philox4x32_10(make_uint4(n, y, z, w), rk), bit for bit.
struct PhiloxFixed {
    uint32_t e;   // round-1 output x = hi(M1 * z1) ^ e
    uint32_t f;   // round-1 output z = w1 ^ f
    uint32_t d;   // round-1 output w
};

__device__ __forceinline__ PhiloxFixed philox_fixed(uint32_t y, uint32_t z,
                                                    const PhiloxKeys &rk) {
    const uint32_t a = __umulhi(0xCD9E8D57u, z) ^ y ^ rk.k[0];   // round-0 output x
    const uint32_t b = 0xCD9E8D57u * z;                           // round-0 output y
    PhiloxFixed p;
    p.e = b ^ rk.k[2];
    p.f = __umulhi(0xD2511F53u, a) ^ rk.k[3];
    p.d = 0xD2511F53u * a;
    return p;
}

__device__ __forceinline__ uint4 philox4x32_10_fixed(uint32_t n, uint32_t w,
                                                     const PhiloxFixed &p,
                                                     const PhiloxKeys &rk) {
    // round 0: only n's product varies
    const uint32_t z1 = __umulhi(0xD2511F53u, n) ^ w ^ rk.k[1];
    const uint32_t w1 = 0xD2511F53u * n;
    // round 1: only z1's product varies
    uint4 c = make_uint4(__umulhi(0xCD9E8D57u, z1) ^ p.e, 0xCD9E8D57u * z1, w1 ^ p.f, p.d);
#pragma unroll
    for (int r = 2; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c.x;
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ rk.k[2 * r], lo1, hi0 ^ c.w ^ rk.k[2 * r + 1], lo0);
    }
    return c;
}

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

// 32-bit word -> uniform in (0, 1]: 2 - f with f = 1 + (x >> 9) * 2^-23 the
// float whose mantissa is the word's top 23 bits, i.e. 1 - (x >> 9) * 2^-23.
// Every value is exact in float and in double, so the FP32 and FP64 builds
// consume identical draws; a bit merge and one subtraction replace an
// integer-to-float conversion and a multiply.
template <typename R>
__device__ __forceinline__ R u01(uint32_t x) {
    return (R)2 - (R)__uint_as_float((x >> 9) | 0x3f800000u);
}

}  // namespace pmo
