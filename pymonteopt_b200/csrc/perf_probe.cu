// perf_probe.cu — FP32 issue-rate probe: the measured denominator of the
// FP32-issue roofline of the transport kernel.  Each thread runs eight
// independent FFMA chains, so the FMA pipe, not latency, limits the rate.
#include "pmo_internal.h"

namespace {

__global__ void __launch_bounds__(256) ffma_probe_kernel(float *out, int iters, float a, float b) {
    float x0 = threadIdx.x * 1e-7f, x1 = x0 + 1e-6f, x2 = x0 + 2e-6f, x3 = x0 + 3e-6f;
    float x4 = x0 + 4e-6f, x5 = x0 + 5e-6f, x6 = x0 + 6e-6f, x7 = x0 + 7e-6f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
            x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
        }
    }
    const float s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == 12345.678f) out[blockIdx.x] = s;  // keeps the chains live
}

}  // namespace

extern "C" {

// Launch blocks x threads, each thread issuing iters * 128 FFMA instructions.
int pmo_fp32_probe(float *out, int blocks, int threads, int iters, void *stream) {
    if (!out || blocks < 1 || threads < 32 || threads > 256 || iters < 1) return PMO_ERR_ARG;
    ffma_probe_kernel<<<blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(
        out, iters, 0.999999f, 1e-7f);
    return cudaGetLastError() == cudaSuccess ? PMO_OK : PMO_ERR_CUDA;
}

}  // extern "C"
