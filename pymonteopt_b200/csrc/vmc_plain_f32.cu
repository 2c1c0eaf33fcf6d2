// vmc_plain_f32.cu — FP32 instantiation of the transport kernel (the product).
// Compiled with -ftz=true -prec-div=false -prec-sqrt=false: single-precision
// divides and square roots use the hardware approximations.
#include "vmc_launch.cuh"

namespace pmo {
cudaError_t launch_plain_f32(const KParams &kp, int props, int flu, int threads, int bps,
                             cudaStream_t s, LaunchShape *out) {
    return launch_plain_r<float>(kp, props, flu, threads, bps, s, out);
}
cudaError_t launch_grad_f32(const KParams &kp, int props, int threads, int bps,
                            cudaStream_t s) {
    return launch_grad_r<float>(kp, props, threads, bps, s);
}
cudaError_t launch_batched_f32(const BParams &bp, int threads, int bps, cudaStream_t s) {
    return launch_batched_r<float>(bp, threads, bps, s);
}
cudaError_t launch_stack_f32(const SParams &sp, int threads, int bps, cudaStream_t s) {
    return launch_stack_r<float>(sp, threads, bps, s);
}
}  // namespace pmo
