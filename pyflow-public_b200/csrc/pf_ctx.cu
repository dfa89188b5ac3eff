// pf_ctx.cu -- per-CUDA-context bookkeeping of the library.
//
// Kernel function attributes (the dynamic shared-memory limits the larger
// kernels need) and addresses of __device__ symbols belong to a CUDA context,
// not to a device: a host application may make its own context current, and
// a context destroyed and created again (cudaDeviceReset) starts without
// them.  The library therefore keys such one-time set-up by the unique id of
// the context current on the calling thread (cuCtxGetId, reached through
// cudaGetDriverEntryPoint so the library links only the runtime).
#include <cuda.h>  // driver-API types only

#include <mutex>
#include <vector>

#include "pf_common.cuh"
#include "pf_kernels.cuh"

namespace pf {

namespace {

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

std::mutex g_ctx_mu;
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;

struct Done {
    const void* key;
    unsigned long long ctx;
};
std::vector<Done> g_done;  // (key, context) pairs whose set-up has run

int context_id_locked(unsigned long long* id) {
    *id = 0;
    if (!g_ctx_current || !g_ctx_id) {
        void* f1 = nullptr;
        void* f2 = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) !=
                cudaSuccess || q1 != cudaDriverEntryPointSuccess || !f1 ||
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) !=
                cudaSuccess || q2 != cudaDriverEntryPointSuccess || !f2)
            return PF_ERR_CUDA;
        g_ctx_current = (CtxGetCurrentFn)f1;
        g_ctx_id = (CtxGetIdFn)f2;
    }
    CUcontext c = nullptr;
    if (g_ctx_current(&c) != CUDA_SUCCESS) return PF_ERR_CUDA;
    if (c && g_ctx_id(c, id) != CUDA_SUCCESS) return PF_ERR_CUDA;
    return PF_OK;
}

}  // namespace

int context_id(unsigned long long* id) {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    return context_id_locked(id);
}

cudaError_t once_per_context(const void* key, cudaError_t (*setup)()) {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    unsigned long long id = 0;
    if (context_id_locked(&id) != PF_OK) return cudaErrorUnknown;
    if (id != 0)
        for (const Done& d : g_done)
            if (d.key == key && d.ctx == id) return cudaSuccess;
    // with no context current yet, the set-up's runtime calls make the
    // device's primary context current; look its id up afterwards
    const cudaError_t e = setup();
    if (e != cudaSuccess) return e;
    if (id == 0 && (context_id_locked(&id) != PF_OK || id == 0)) return cudaSuccess;
    g_done.push_back(Done{key, id});
    return cudaSuccess;
}

}  // namespace pf
