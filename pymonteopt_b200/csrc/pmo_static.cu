// pmo_static.cu — pmo_run_plain for callers that cannot allocate device memory.
//
// pmo_run_plain needs a small device workspace (the photon-chunk counter the
// warps draw photon ids from), which its caller allocates.  Some callers cannot
// allocate device memory themselves: a plugin inside a host application that
// owns every device allocation through its own memory pool, or a caller on a
// latency-critical path where cudaMalloc, which may synchronise the device, is
// not allowed.  pmo_run_plain_static runs the same transport with that scratch
// in a file-scope device array instead, so the caller passes only the problem,
// its tally buffers and a stream.
#include <mutex>

#include "pmo_internal.h"

namespace {

// Largest workspace pmo_run_plain_static can provide.  Every GPU that loads
// this library holds this array until the process exits.
constexpr size_t kStaticWorkspaceBytes = 512;

// Shared by every call on a device; it keeps the last call's contents.
// pmo_run_plain clears the photon counter in it (stream-ordered) before each
// launch, so calls in sequence on one stream are fine, but calls that overlap
// on the GPU (two streams, or two host threads) race on it.
static __device__ __align__(256) unsigned char g_static_workspace[kStaticWorkspaceBytes];

std::mutex g_mutex;
void *g_workspace_ptr[64] = {};

// Device address of g_static_workspace on the current device.  In host code
// the array's name is only a host-side stand-in, not a device address, so the
// address is looked up once per device, with that device current.
int static_workspace(void **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PMO_ERR_CUDA;
    if (dev < 0 || dev >= 64) return PMO_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_workspace_ptr[dev]) {
        void *ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, g_static_workspace) != cudaSuccess || !ptr)
            return PMO_ERR_CUDA;
        g_workspace_ptr[dev] = ptr;
    }
    *out = g_workspace_ptr[dev];
    return PMO_OK;
}

}  // namespace

extern "C" int pmo_run_plain_static(const pmo_problem *prob, const pmo_tallies *tal,
                                    const pmo_launch *launch, void *stream) {
    if (pmo_workspace_bytes() > kStaticWorkspaceBytes) return PMO_ERR_WORKSPACE;
    void *ws = nullptr;
    const int st = static_workspace(&ws);
    if (st != PMO_OK) return st;
    return pmo_run_plain(prob, tal, launch, ws, kStaticWorkspaceBytes, stream);
}
