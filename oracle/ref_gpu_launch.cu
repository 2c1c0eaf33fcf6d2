// Launcher for the reference's own GPU kernel cuVMC (test and baseline
// infrastructure; never part of the product).
//
// cuvmc_reference.cu is the kernel source string of
// pymopt/voxel_gpu/_cukernel.py:10-229, written unchanged into oracle/_ref
// by oracle/ref_gpu_build.py.  This file only adds the launch that
// VoxelModel.start() performs through CuPy (pymopt/voxel_gpu/_classes.py:105-112):
// one thread per photon, ceil(nPh / threadnum) blocks of threadnum threads.
// The state arrays are updated in place, as in the reference.
#include "cuvmc_reference.cu"

#include <cuda_runtime.h>

extern "C" {

// 0 on success, else the CUDA error code of the launch.
int ref_cuvmc_launch(int *add, float *p, float *v, float *w, float *ma, float *ms, float *n,
                     float *g, char *voxel_model, float l, int M, int L, int nPh,
                     char end_point, int rand_seed, int threadnum, void *stream) {
    if (nPh <= 0 || threadnum <= 0 || threadnum > 1024) return (int)cudaErrorInvalidValue;
    const unsigned blocks = (unsigned)((nPh + threadnum - 1) / threadnum);
    cuVMC<<<blocks, threadnum, 0, static_cast<cudaStream_t>(stream)>>>(
        add, p, v, w, ma, ms, n, g, voxel_model, l, M, L, nPh, end_point, rand_seed);
    return (int)cudaGetLastError();
}

}  // extern "C"
