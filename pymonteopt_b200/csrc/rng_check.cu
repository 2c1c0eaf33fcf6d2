// rng_check.cu — device Philox words for known-answer tests of the random
// stream layout: the engine's own Philox4x32-10 and, beside it, cuRAND's
// Philox4_32_10 for the same (seed, subsequence, offset).
#include <curand_kernel.h>

#include "philox.cuh"
#include "pmo_internal.h"

namespace {

__global__ void philox_words_kernel(const uint32_t *ctr, uint32_t k0, uint32_t k1, uint32_t *out,
                                    int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4 c = make_uint4(ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3]);
    const uint4 r = pmo::philox4x32_10(c, make_uint2(k0, k1));
    out[4 * i] = r.x;
    out[4 * i + 1] = r.y;
    out[4 * i + 2] = r.z;
    out[4 * i + 3] = r.w;
}

// curand_init(seed, subsequence, 4 * block) then curand4(): the counter of
// that call is (block, 0, subsequence_lo, subsequence_hi) under key = seed.
__global__ void curand_philox_kernel(unsigned long long seed, const unsigned long long *subseq,
                                     const unsigned long long *block, uint32_t *out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    curandStatePhilox4_32_10_t st;
    curand_init(seed, subseq[i], 4ull * block[i], &st);
    const uint4 r = curand4(&st);
    out[4 * i] = r.x;
    out[4 * i + 1] = r.y;
    out[4 * i + 2] = r.z;
    out[4 * i + 3] = r.w;
}

}  // namespace

extern "C" {

int pmo_philox_words(const uint32_t *ctr, uint32_t key0, uint32_t key1, uint32_t *out, int n,
                     void *stream) {
    if (!ctr || !out || n < 0) return PMO_ERR_ARG;
    if (n == 0) return PMO_OK;
    philox_words_kernel<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        ctr, key0, key1, out, n);
    return cudaGetLastError() == cudaSuccess ? PMO_OK : PMO_ERR_CUDA;
}

int pmo_philox_words_curand(unsigned long long seed, const unsigned long long *subsequence,
                            const unsigned long long *block, uint32_t *out, int n, void *stream) {
    if (!subsequence || !block || !out || n < 0) return PMO_ERR_ARG;
    if (n == 0) return PMO_OK;
    curand_philox_kernel<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        seed, subsequence, block, out, n);
    return cudaGetLastError() == cudaSuccess ? PMO_OK : PMO_ERR_CUDA;
}

}  // extern "C"
