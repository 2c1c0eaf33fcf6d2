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
#include <cuda.h>

#include <mutex>
#include <utility>
#include <vector>

#include "pmo_internal.h"

namespace {

// Shared by every call in one CUDA context; it keeps the last call's contents.
// pmo_run_plain clears the photon counter in it (stream-ordered) before each
// launch, so calls in sequence on one stream are fine, but calls that overlap
// on the GPU (two streams, or two host threads) race on it.  Every GPU that
// loads this library holds the array until the process exits.
static __device__ __align__(256) unsigned char g_static_workspace[PMO_STATIC_WORKSPACE_BYTES];

// In host code the array's name is only a host-side stand-in, not a device
// address.  Its device address belongs to the CUDA context the module was
// loaded into, so it is cached per context, keyed by the context's unique id
// (cuCtxGetId: ids are never reused within a process, so a context destroyed
// by cudaDeviceReset and its successor get different entries).
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

std::mutex g_mutex;
std::vector<std::pair<unsigned long long, void *>> g_cache;
bool g_entry_points_looked_up = false;
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

// Unique id of the context current on this thread, 0 when there is none or the
// driver does not offer the query.  Call with g_mutex held.
unsigned long long current_context_id() {
    if (!g_entry_points_looked_up) {
        g_entry_points_looked_up = true;
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &fn, 12000, cudaEnableDefault,
                                             &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
        fn = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &fn, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(fn);
    }
    if (!g_ctx_get_current || !g_ctx_get_id) return 0;
    CUcontext ctx = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    unsigned long long id = 0;
    if (g_ctx_get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of g_static_workspace in the current context.  The first call
// in a context looks it up with cudaGetSymbolAddress (which also loads the
// module into the context if it is not loaded yet); later calls in that context
// reuse it.  Without the context query the address is looked up on every call.
int static_workspace(void **out) {
    std::lock_guard<std::mutex> lock(g_mutex);
    unsigned long long id = current_context_id();
    if (id)
        for (const auto &e : g_cache)
            if (e.first == id) {
                *out = e.second;
                return PMO_OK;
            }
    void *ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_static_workspace) != cudaSuccess || !ptr)
        return PMO_ERR_CUDA;
    if (!id) id = current_context_id();   // the lookup made the primary context current
    if (id) g_cache.emplace_back(id, ptr);
    *out = ptr;
    return PMO_OK;
}

}  // namespace

extern "C" int pmo_run_plain_static(const pmo_problem *prob, const pmo_tallies *tal,
                                    const pmo_launch *launch, void *stream) {
    // kWorkspaceBytes <= PMO_STATIC_WORKSPACE_BYTES is also checked at compile
    // time (pmo_internal.h); the run-time check keeps the documented error
    if (!prob || !tal) return PMO_ERR_ARG;   // before any CUDA call
    if (pmo_workspace_bytes() > sizeof(g_static_workspace)) return PMO_ERR_WORKSPACE;
    void *ws = nullptr;
    const int st = static_workspace(&ws);
    if (st != PMO_OK) return st;
    return pmo_run_plain(prob, tal, launch, ws, sizeof(g_static_workspace), stream);
}
