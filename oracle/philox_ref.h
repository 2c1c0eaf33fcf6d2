/*
 * philox_ref.h — Philox4x32-10 counter-based generator, host C.
 *
 * TEST INFRASTRUCTURE (oracle): used only by tests, smoke() and the CPU
 * baseline of bench.py, never by the product path.
 *
 * Written from the published algorithm (J. K. Salmon, M. A. Moraes,
 * R. O. Dror, D. E. Shaw, "Parallel random numbers: as easy as 1, 2, 3",
 * SC'11): ten rounds of two 32x32->64 multiplies with the multipliers
 * 0xD2511F53 / 0xCD9E8D57 and a Weyl key schedule 0x9E3779B9 / 0xBB67AE85.
 * The device kernels implement the same function; tests compare the two
 * word for word and compare the device one with cuRAND's Philox4_32_10.
 */
#ifndef PMO_PHILOX_REF_H
#define PMO_PHILOX_REF_H
#include <stdint.h>

static inline void pmo_philox4x32_10(const uint32_t ctr_in[4],
                                     const uint32_t key_in[2],
                                     uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * (uint64_t)c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * (uint64_t)c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* 32-bit word -> uniform in (0, 1]: 1 - (x >> 9) * 2^-23, the value the
   device forms as 2 - f from the float f = 1 + (x >> 9) * 2^-23.  Every value
   is exact in float and double, so FP32 and FP64 builds see identical draws. */
static inline double pmo_u01(uint32_t x) {
    return 1.0 - (double)(x >> 9) * (1.0 / 8388608.0);
}

#endif
