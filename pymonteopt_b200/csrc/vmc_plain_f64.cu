// vmc_plain_f64.cu — FP64 instantiation of the transport kernel: the
// per-photon oracle build.  Compiled with -fmad=false so that every product
// and sum rounds separately, like the CPU oracle; the remaining differences
// come from the math library (log, sincospi).
#include "vmc_launch.cuh"

namespace pmo {
cudaError_t launch_plain_f64(const KParams &kp, int props, int flu, int threads, int bps,
                             cudaStream_t s, LaunchShape *out) {
    return launch_plain_r<double>(kp, props, flu, threads, bps, s, out);
}
cudaError_t launch_grad_f64(const KParams &kp, int props, int threads, int bps,
                            cudaStream_t s) {
    return launch_grad_r<double>(kp, props, threads, bps, s);
}
cudaError_t launch_batched_f64(const BParams &bp, int threads, int bps, cudaStream_t s) {
    return launch_batched_r<double>(bp, threads, bps, s);
}
cudaError_t launch_stack_f64(const SParams &sp, int threads, int bps, cudaStream_t s) {
    return launch_stack_r<double>(sp, threads, bps, s);
}
}  // namespace pmo
