// pmo_batched_api.cu — C ABI of the batched slab form: argument checks, the
// persistent launch, and the FP64 finalisation of per-problem results.
#include <cmath>

#include "pmo_internal.h"

namespace pmo {
struct BParams;
cudaError_t launch_batched_f32(const BParams &bp, int threads, int bps, cudaStream_t s);
cudaError_t launch_batched_f64(const BParams &bp, int threads, int bps, cudaStream_t s);
}  // namespace pmo

#include "vmc_batched.cuh"

using pmo::kWorkspaceBytes;

namespace {

// Rd, Tt, A, derivatives, energy residual; R(r) and its derivatives.
__global__ void batch_finalize_kernel(const pmo_slab *__restrict__ slabs, int n_problems,
                                      const double *__restrict__ sums,
                                      const float *__restrict__ bins, int nr,
                                      double *__restrict__ res, double *__restrict__ rr) {
    const int total = n_problems * (nr > 0 ? nr : 1);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int p = nr > 0 ? i / nr : i;
        const int b = nr > 0 ? i % nr : 0;
        const pmo_slab sl = slabs[p];
        const double N = (double)sl.photons;
        const double ims = sl.ms > 0.f ? 1.0 / (double)sl.ms : 0.0;
        const double *S = sums + (size_t)p * PMO_BS_N;
        if (b == 0 && res) {
            double *o = res + (size_t)p * PMO_BR_N;
            o[PMO_BR_RD] = S[PMO_BS_RD] / N;
            o[PMO_BR_TT] = S[PMO_BS_TT] / N;
            o[PMO_BR_A] = S[PMO_BS_ABS] / N;
            o[PMO_BR_DRD_DMA] = -S[PMO_BS_RD_L] / N;
            o[PMO_BR_DRD_DMS] = (S[PMO_BS_RD_N] * ims - S[PMO_BS_RD_L]) / N;
            o[PMO_BR_DTT_DMA] = -S[PMO_BS_TT_L] / N;
            o[PMO_BR_DTT_DMS] = (S[PMO_BS_TT_N] * ims - S[PMO_BS_TT_L]) / N;
            const double in = S[PMO_BS_WINIT] + S[PMO_BS_RGAIN];
            const double out = S[PMO_BS_RD] + S[PMO_BS_TT] + S[PMO_BS_ABS] + S[PMO_BS_RLOSS] +
                               S[PMO_BS_ERRW];
            o[PMO_BR_BALANCE] = in > 0.0 ? (in - out) / in : 0.0;
        }
        if (nr > 0 && rr) {
            const double dr = (double)sl.dr;
            const double area = 2.0 * 3.14159265358979323846 * (b + 0.5) * dr * dr;
            const float *B = bins + ((size_t)p * nr + b) * 3;
            double *o = rr + ((size_t)p * nr + b) * 3;
            o[0] = (double)B[0] / (area * N);
            o[1] = -(double)B[1] / (area * N);
            o[2] = ((double)B[2] * ims - (double)B[1]) / (area * N);
        }
    }
}

}  // namespace

extern "C" {

int pmo_run_batched(const pmo_batch *b, const pmo_launch *launch, void *workspace,
                    size_t workspace_bytes, void *stream) {
    if (!b || !b->slabs || b->n_problems < 1 || !b->items || b->n_items < 0 || !b->sums)
        return PMO_ERR_ARG;
    if (b->nr < 0 || (b->nr > 0 && !b->bins)) return PMO_ERR_ARG;
    if (b->precision != PMO_FP32 && b->precision != PMO_FP64) return PMO_ERR_ARG;
    if (b->tally_mode != PMO_BT_THREAD && b->tally_mode != PMO_BT_GLOBAL) return PMO_ERR_ARG;
    if (!workspace || workspace_bytes < kWorkspaceBytes) return PMO_ERR_WORKSPACE;
    const int threads = launch && launch->block_threads > 0 ? launch->block_threads : 128;
    if (threads % 32 != 0 || threads > 512) return PMO_ERR_ARG;
    const int bps = launch ? launch->blocks_per_sm : 0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned long long *work = static_cast<unsigned long long *>(workspace);
    // work[0]: next item (0); work[1]: launch start time (min over blocks)
    if (cudaMemsetAsync(work, 0, sizeof(unsigned long long), s) != cudaSuccess) return PMO_ERR_CUDA;
    if (cudaMemsetAsync(work + 1, 0xff, sizeof(unsigned long long), s) != cudaSuccess)
        return PMO_ERR_CUDA;
    if (b->n_items == 0) return PMO_OK;
    pmo::BParams bp;
    bp.slabs = b->slabs;
    bp.n_problems = b->n_problems;
    bp.items = b->items;
    bp.n_items = b->n_items;
    bp.key0 = (uint32_t)b->seed;
    bp.key1 = (uint32_t)(b->seed >> 32);
    bp.rk = pmo::philox_round_keys(bp.key0, bp.key1);
    bp.nr = b->nr;
    bp.sums = b->sums;
    bp.bins = b->bins;
    bp.remaining = b->remaining;
    bp.t_done = b->t_done;
    bp.max_events = b->max_events;
    bp.tally_mode = b->tally_mode;
    bp.work = work;
    const cudaError_t e = b->precision == PMO_FP64 ? pmo::launch_batched_f64(bp, threads, bps, s)
                                                   : pmo::launch_batched_f32(bp, threads, bps, s);
    return e == cudaSuccess ? PMO_OK : PMO_ERR_CUDA;
}

int pmo_batch_finalize(const pmo_batch *b, double *results, double *rr, void *stream) {
    if (!b || !b->slabs || b->n_problems < 1 || !b->sums) return PMO_ERR_ARG;
    if (!results && !rr) return PMO_ERR_ARG;
    if (rr && (b->nr <= 0 || !b->bins)) return PMO_ERR_ARG;
    const int total = b->n_problems * (b->nr > 0 ? b->nr : 1);
    int blocks = (total + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    batch_finalize_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        b->slabs, b->n_problems, b->sums, b->bins, b->nr, results, rr);
    return cudaGetLastError() == cudaSuccess ? PMO_OK : PMO_ERR_CUDA;
}

}  // extern "C"
