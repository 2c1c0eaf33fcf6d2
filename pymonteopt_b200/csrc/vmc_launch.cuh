// vmc_launch.cuh — persistent-grid launch of the transport kernel for one
// arithmetic type.  Included by vmc_plain_f32.cu and vmc_plain_f64.cu, which
// are compiled with different floating-point flags.
#pragma once
#include <atomic>

#include "vmc_batched.cuh"
#include "vmc_stack.cuh"
#include "vmc_transport.cuh"

namespace pmo {

// SM count of the current device, cached per device ordinal.  Launches may come
// from several host threads at once, so the cache entries are atomics (two
// threads that miss together both query the same value).
inline int device_sm_count() {
    static std::atomic<int> cached[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (dev < 0 || dev >= 64) return 0;
    int sms = cached[dev].load(std::memory_order_relaxed);
    if (!sms) {
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return 0;
        cached[dev].store(sms, std::memory_order_relaxed);
    }
    return sms;
}

template <typename R, int PROPS, int FLU, bool SKIP, bool GRAD = false>
cudaError_t launch_plain_t(const KParams &kp, int threads, int blocks_per_sm, cudaStream_t s,
                           LaunchShape *out) {
    auto kern = vmc_plain_kernel<R, PROPS, FLU, SKIP, GRAD>;
    size_t smem = SmemLayout<R>::total(kp.hist_n, FLU, kp.win_dim);
    if (GRAD && kp.fd_n > 0) smem += SmemLayout<R>::fd_bytes(threads);
    cudaError_t e;
    if (smem > 48 * 1024) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const int sms = device_sm_count();
    if (sms <= 0) return cudaErrorNoDevice;
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem);
    if (e != cudaSuccess) return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    const int per_sm = blocks_per_sm > 0 && blocks_per_sm < occ ? blocks_per_sm : occ;
    uint64_t blocks = (uint64_t)sms * per_sm;
    const uint64_t useful = (kp.count + threads - 1) / threads;
    if (blocks > useful) blocks = useful > 0 ? useful : 1;
    kern<<<(unsigned)blocks, threads, smem, s>>>(kp);
    if (out) {
        out->block_threads = threads;
        out->blocks = (int)blocks;
        out->smem = smem;
    }
    return cudaGetLastError();
}

template <typename R, bool SKIP>
cudaError_t launch_plain_label(const KParams &kp, int flu, int threads, int bps, cudaStream_t s,
                               LaunchShape *out) {
    if (flu == PMO_FLU_NONE)
        return launch_plain_t<R, PMO_PROPS_LABEL, PMO_FLU_NONE, SKIP>(kp, threads, bps, s, out);
    if (flu == PMO_FLU_GLOBAL)
        return launch_plain_t<R, PMO_PROPS_LABEL, PMO_FLU_GLOBAL, SKIP>(kp, threads, bps, s, out);
    return launch_plain_t<R, PMO_PROPS_LABEL, PMO_FLU_SHARED, SKIP>(kp, threads, bps, s, out);
}

// Uniform-box stepping whenever a voxel-word map is given and the optics are
// per label; per-voxel optics step voxel by voxel.
template <typename R>
cudaError_t launch_plain_r(const KParams &kp, int props, int flu, int threads, int bps,
                           cudaStream_t s, LaunchShape *out) {
    if (props == PMO_PROPS_LABEL) {
        if (kp.words) return launch_plain_label<R, true>(kp, flu, threads, bps, s, out);
        return launch_plain_label<R, false>(kp, flu, threads, bps, s, out);
    }
    if (flu == PMO_FLU_NONE)
        return launch_plain_t<R, PMO_PROPS_VOXEL, PMO_FLU_NONE, false>(kp, threads, bps, s, out);
    if (flu == PMO_FLU_GLOBAL)
        return launch_plain_t<R, PMO_PROPS_VOXEL, PMO_FLU_GLOBAL, false>(kp, threads, bps, s, out);
    return launch_plain_t<R, PMO_PROPS_VOXEL, PMO_FLU_SHARED, false>(kp, threads, bps, s, out);
}

// Gradient replay: no fluence; uniform boxes only when the problem carries a
// voxel-word map (per-label derivatives only).
template <typename R>
cudaError_t launch_grad_r(const KParams &kp, int props, int threads, int bps, cudaStream_t s) {
    if (props == PMO_PROPS_LABEL) {
        if (kp.words)
            return launch_plain_t<R, PMO_PROPS_LABEL, PMO_FLU_NONE, true, true>(kp, threads, bps, s,
                                                                                nullptr);
        return launch_plain_t<R, PMO_PROPS_LABEL, PMO_FLU_NONE, false, true>(kp, threads, bps, s,
                                                                             nullptr);
    }
    return launch_plain_t<R, PMO_PROPS_VOXEL, PMO_FLU_NONE, false, true>(kp, threads, bps, s,
                                                                         nullptr);
}

template <typename R>
cudaError_t launch_batched_r(const BParams &bp, int threads, int blocks_per_sm, cudaStream_t s) {
    auto kern = vmc_batched_kernel<R>;
    const size_t smem =
        bp.tally_mode == PMO_BT_THREAD ? (size_t)threads * kSlots * sizeof(double) : 0;
    cudaError_t e;
    if (smem > 48 * 1024) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const int sms = device_sm_count();
    if (sms <= 0) return cudaErrorNoDevice;
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem);
    if (e != cudaSuccess) return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    const int per_sm = blocks_per_sm > 0 && blocks_per_sm < occ ? blocks_per_sm : occ;
    kern<<<sms * per_sm, threads, smem, s>>>(bp);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_stack_r(const SParams &sp, int threads, int blocks_per_sm, cudaStream_t s) {
    auto kern = vmc_stack_kernel<R>;
    const size_t smem = (size_t)threads * 2 * PMO_MAX_LAYERS * sizeof(R);
    cudaError_t e;
    if (smem > 48 * 1024) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const int sms = device_sm_count();
    if (sms <= 0) return cudaErrorNoDevice;
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem);
    if (e != cudaSuccess) return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    const int per_sm = blocks_per_sm > 0 && blocks_per_sm < occ ? blocks_per_sm : occ;
    kern<<<sms * per_sm, threads, smem, s>>>(sp);
    return cudaGetLastError();
}

}  // namespace pmo
