// pf_noalloc.cu -- BiCGStab pressure solve whose scratch memory belongs to the
// library, for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc or hand the library a workspace: code
// embedded in a host application whose device-memory budget is owned by
// another allocator, real-time loops that must not allocate after start-up,
// or plugins that receive only their input and output buffers.  For them,
// pf_bicgstab_solve_noalloc runs the same FP64 solve as pf_bicgstab_solve but
// takes its scratch from a fixed array compiled into this library:
//
//   * The array, g_noalloc_scratch, is a file-scope static __device__ array of
//     kNoallocBytes (16.25 MiB).  Every GPU that loads the library holds it
//     until the process exits.  It fits grids of at most kNoallocMaxCells
//     (64^3 = 262144) cells; larger grids are rejected with
//     PF_ERR_TOO_LARGE and nothing is launched.
//   * Host code cannot use the array's name as a device address (on the host
//     it names a host-side shadow).  A __device__ array has one address per
//     CUDA context (not per device), so the call looks the address up with
//     cudaGetSymbolAddress once per context -- the first call in a context,
//     with that context current -- and caches it under the context's unique
//     id (cuCtxGetId, pf::context_id).  A host application that makes its own context
//     current, or a context destroyed and created again (cudaDeviceReset),
//     therefore gets a fresh lookup, never a stale address.  The first call
//     in a context may load the library's device code, so make it before any
//     stream capture.
//   * Every call shares the one array, and the array keeps the previous
//     call's contents.  The solve clears what must start at zero (its scalar
//     block and reduction counter) and initialises every vector it reads, so
//     consecutive calls are independent.  Calls that overlap on the GPU (for
//     example on two streams) race on the array and must be serialised by the
//     caller.
//   * The call allocates nothing: no cudaMalloc, cudaFree or allocating
//     library routine.
#include <mutex>

#include "pf_common.cuh"
#include "pf_kernels.cuh"

namespace {

constexpr long long kNoallocMaxCells = 64LL * 64 * 64;
// the FP64 solve's 8 vectors of kNoallocMaxCells cells plus its scalar block
// and reduction partials (with alignment slack); the call also checks the
// exact size the solve needs against this bound at run time
constexpr size_t kNoallocBytes = 8 * (size_t)kNoallocMaxCells * sizeof(double) + 256 * 1024;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

// scratch address per context id (a small ring: the oldest entry is reused
// when a process has created more contexts than it holds)
constexpr int kMaxContexts = 64;
struct CtxScratch {
    unsigned long long id;
    void* ptr;
};
std::mutex g_noalloc_mu;
CtxScratch g_noalloc_tab[kMaxContexts];
int g_noalloc_used = 0, g_noalloc_next = 0;

// Device address of the scratch array in the context the runtime uses on
// this thread (looked up once per context).
int noalloc_scratch(void** out) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    unsigned long long id = 0;
    int rc = pf::context_id(&id);
    if (rc != PF_OK) return rc;
    if (id != 0)
        for (int e = 0; e < g_noalloc_used; ++e)
            if (g_noalloc_tab[e].id == id) {
                *out = g_noalloc_tab[e].ptr;
                return PF_OK;
            }
    // set-up in this context: with no context current yet, this call makes
    // the device's primary context current, as any runtime call would
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return PF_ERR_CUDA;
    if (id == 0 && ((rc = pf::context_id(&id)) != PF_OK || id == 0)) return PF_ERR_CUDA;
    g_noalloc_tab[g_noalloc_next] = CtxScratch{id, p};
    g_noalloc_next = (g_noalloc_next + 1) % kMaxContexts;
    if (g_noalloc_used < kMaxContexts) ++g_noalloc_used;
    *out = p;
    return PF_OK;
}

}  // namespace

extern "C" int pf_bicgstab_solve_noalloc(const pf_grid* g, double rho,
                                         double dt, double min_res,
                                         int max_it, const double* source,
                                         double* DP, double* p, void* stream,
                                         pf_solve_info* info) {
    if (!g || g->nx < 2 || g->ny < 2 || g->nz < 2 || !(g->dx > 0) || !(g->dy > 0) ||
        !(g->dz > 0) || !source || !DP || !p || !(dt != 0.0))
        return PF_ERR_BAD_ARG;
    const long long n = (long long)g->nx * g->ny * g->nz;
    if (n > kNoallocMaxCells || pf::poisson_ws_bytes(g, PF_FP64) > kNoallocBytes)
        return PF_ERR_TOO_LARGE;
    void* ws = nullptr;
    const int rc = noalloc_scratch(&ws);
    if (rc != PF_OK) return rc;
    return pf::bicgstab_solve(g, PF_FP64, rho, dt, min_res, max_it, source, DP, p, ws,
                              (cudaStream_t)stream, info);
}
