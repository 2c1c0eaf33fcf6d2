// pmo_stack_api.cu — C ABI of the batched layered-slab form: argument checks,
// the persistent launch, and the FP64 finalisation of per-problem results.
#include "pmo_internal.h"

namespace pmo {
struct SParams;
cudaError_t launch_stack_f32(const SParams &sp, int threads, int bps, cudaStream_t s);
cudaError_t launch_stack_f64(const SParams &sp, int threads, int bps, cudaStream_t s);
}  // namespace pmo

#include "vmc_stack.cuh"

using pmo::kWorkspaceBytes;

namespace {

// Rd, Tt, A, energy residual and per-layer derivatives; R(r) and its
// per-layer derivatives.  One thread per (problem, bin).
__global__ void stack_finalize_kernel(const pmo_stack *__restrict__ stacks, int n_problems,
                                      const pmo_layer *__restrict__ layers, int n_layer_rows,
                                      const double *__restrict__ sums,
                                      const float *__restrict__ bins, int nr,
                                      double *__restrict__ res, double *__restrict__ rr) {
    const int total = n_problems * (nr > 0 ? nr : 1);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int p = nr > 0 ? i / nr : i;
        const int b = nr > 0 ? i % nr : 0;
        const pmo_stack st = stacks[p];
        const int nl = (int)st.n_layers;
        const bool ok = nl >= 1 && nl <= PMO_MAX_LAYERS &&
                        (uint64_t)st.first_layer + (uint64_t)nl <= (uint64_t)n_layer_rows;
        const double N = (double)st.photons;
        const double *S = sums + (size_t)p * PMO_SS_N;
        if (b == 0 && res) {
            double *o = res + (size_t)p * PMO_SR_N;
            for (int q = 0; q < PMO_SR_N; ++q) o[q] = 0.0;
            o[PMO_SR_RD] = S[PMO_SS_RD] / N;
            o[PMO_SR_TT] = S[PMO_SS_TT] / N;
            o[PMO_SR_A] = S[PMO_SS_ABS] / N;
            const double in = S[PMO_SS_WINIT] + S[PMO_SS_RGAIN];
            const double out = S[PMO_SS_RD] + S[PMO_SS_TT] + S[PMO_SS_ABS] + S[PMO_SS_RLOSS] +
                               S[PMO_SS_ERRW];
            o[PMO_SR_BALANCE] = in > 0.0 ? (in - out) / in : 0.0;
            if (ok) {
                for (int l = 0; l < nl; ++l) {
                    const float ms = layers[st.first_layer + l].ms;
                    const double ims = ms > 0.f ? 1.0 / (double)ms : 0.0;
                    const double *Sl = S + PMO_SS_LAYER0 + 4 * l;
                    double *ol = o + PMO_SR_LAYER0 + 4 * l;
                    ol[0] = -Sl[0] / N;
                    ol[1] = (Sl[1] * ims - Sl[0]) / N;
                    ol[2] = -Sl[2] / N;
                    ol[3] = (Sl[3] * ims - Sl[2]) / N;
                }
            }
        }
        if (nr > 0 && rr) {
            const double dr = (double)st.dr;
            const double area = 2.0 * 3.14159265358979323846 * (b + 0.5) * dr * dr;
            const float *B = bins + ((size_t)p * nr + b) * PMO_SB_N;
            double *o = rr + ((size_t)p * nr + b) * PMO_SB_N;
            for (int q = 0; q < PMO_SB_N; ++q) o[q] = 0.0;
            o[0] = (double)B[0] / (area * N);
            if (ok) {
                for (int l = 0; l < nl; ++l) {
                    const float ms = layers[st.first_layer + l].ms;
                    const double ims = ms > 0.f ? 1.0 / (double)ms : 0.0;
                    const double wl = (double)B[1 + 2 * l], wn = (double)B[2 + 2 * l];
                    o[1 + 2 * l] = -wl / (area * N);
                    o[2 + 2 * l] = (wn * ims - wl) / (area * N);
                }
            }
        }
    }
}

}  // namespace

extern "C" {

int pmo_run_stack_batch(const pmo_stack_batch *b, const pmo_launch *launch, void *workspace,
                        size_t workspace_bytes, void *stream) {
    if (!b || !b->stacks || b->n_problems < 1 || !b->layers || b->n_layer_rows < 1 ||
        !b->items || b->n_items < 0 || !b->sums)
        return PMO_ERR_ARG;
    if (b->nr < 0 || (b->nr > 0 && !b->bins)) return PMO_ERR_ARG;
    if (b->precision != PMO_FP32 && b->precision != PMO_FP64) return PMO_ERR_ARG;
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
    pmo::SParams sp;
    sp.stacks = b->stacks;
    sp.n_problems = b->n_problems;
    sp.layers = b->layers;
    sp.n_layer_rows = b->n_layer_rows;
    sp.items = b->items;
    sp.n_items = b->n_items;
    sp.key0 = (uint32_t)b->seed;
    sp.key1 = (uint32_t)(b->seed >> 32);
    sp.rk = pmo::philox_round_keys(sp.key0, sp.key1);
    sp.nr = b->nr;
    sp.sums = b->sums;
    sp.bins = b->bins;
    sp.remaining = b->remaining;
    sp.t_done = b->t_done;
    sp.max_events = b->max_events;
    sp.work = work;
    const cudaError_t e = b->precision == PMO_FP64 ? pmo::launch_stack_f64(sp, threads, bps, s)
                                                   : pmo::launch_stack_f32(sp, threads, bps, s);
    return e == cudaSuccess ? PMO_OK : PMO_ERR_CUDA;
}

int pmo_stack_batch_finalize(const pmo_stack_batch *b, double *results, double *rr,
                             void *stream) {
    if (!b || !b->stacks || b->n_problems < 1 || !b->layers || b->n_layer_rows < 1 || !b->sums)
        return PMO_ERR_ARG;
    if (!results && !rr) return PMO_ERR_ARG;
    if (rr && (b->nr <= 0 || !b->bins)) return PMO_ERR_ARG;
    const int total = b->n_problems * (b->nr > 0 ? b->nr : 1);
    int blocks = (total + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    stack_finalize_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        b->stacks, b->n_problems, b->layers, b->n_layer_rows, b->sums, b->bins, b->nr, results,
        rr);
    return cudaGetLastError() == cudaSuccess ? PMO_OK : PMO_ERR_CUDA;
}

}  // extern "C"
