// pf_slab.cu -- x-slab decomposition of the periodic box over ranks: the
// distributed form of solver_bicgstab.solve (src/solver/pressure.py:196-297)
// and the slab helpers around it.  Replaces the reference's decomposition
// and ghost exchange (decomp, communicate_border,
// src/library/parallel.py:118-414) and its scalar reductions (comms.parallel_sum
// / parallel_max, src/library/parallel.py:60-94) for grids split along x.
//
// A rank holds planes [x0, x0 + nxl) of the global box as a LOCAL EXTENDED
// grid of nxl + 2h planes, [nx][ny][nz] with z fastest like every field of
// this library: h ghost planes, the interior, h ghost planes.  Planes are
// contiguous, so a halo exchange moves h * ny * nz doubles per side with no
// packing.  Kernels that do not reduce (the RK4 predictor, divergence,
// projection) run unchanged on the extended grid: an interior plane depends
// on planes at most one away per stencil, so after an exchange of h planes
// the whole four-stage predictor is exact on the interior (h >= 4); what they
// write on ghost planes is overwritten by the next exchange.
//
// The solve follows the reference's iteration literally -- three global
// reductions per iteration (rho1 = (res, res0); gamma = (vv, res0); (s,t) and
// (t,t)), then max|res| for the stop test -- with every per-element operation
// of the reference (torch's add_(alpha, x) as one fused multiply-add).  Each
// reduction point is: a kernel writes this rank's sums over its interior into
// `send`; the caller gathers every rank's `send` into `recv` (rank order);
// the next phase folds `recv` in rank order on one thread, so every rank
// computes bitwise the same scalars and takes the same branch.  Scalars never
// leave the device; the caller polls the stop flag (pf_slab_bicg_info).
//
// Phases (the caller's loop, one rank):
//   init -> gather -> START;
//   repeat: exchange(pp, 1) -> APPLY_P -> gather -> S -> exchange(s, 1) ->
//           APPLY_S -> gather -> FINAL -> gather -> P (folds the stop test)
// until the stop flag is set; then p += DP (pf_slab_add) and, after an
// exchange of DP, the projection.
#include <cmath>

#include "pf_common.cuh"
#include "pf_kernels.cuh"
#include "pf_profile.cuh"
#include "pf_sweep.cuh"

namespace pf {
namespace {

struct SlabScalars {
    double rho1, rho2, alpha, omega, max_res0, max_res, min_res;
    int iter, max_it, done, status;
    unsigned int counter;
};

constexpr int kSlabVals = 2;      // values per rank in `send`
constexpr int kSlabMaxRanks = 4096;

struct Slab {
    Dims d;          // the extended local grid
    int h;           // ghost planes per side
    long long off;   // first interior cell: h * ny * nz
    long long nint;  // interior cells: (nx - 2h) * ny * nz
};

struct SlabVecs {
    double *res, *res0, *pp, *vv, *s, *t;
};

struct SlabWs {
    SlabScalars* sc;
    double* part;  // kSlabVals x kMaxPartials block partials
    SlabVecs v;
};

Slab make_slab(const pf_grid* g, int h) {
    Slab s;
    s.d = Dims{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    s.h = h;
    s.off = (long long)h * g->ny * g->nz;
    s.nint = (long long)(g->nx - 2 * h) * g->ny * g->nz;
    return s;
}

size_t slab_ws_bytes(const pf_grid* g) {
    const size_t n = (size_t)g->nx * g->ny * g->nz;
    return align256(sizeof(SlabScalars)) + align256(kSlabVals * kMaxPartials * sizeof(double)) +
           6 * align256(n * sizeof(double));
}

SlabWs carve_slab(const pf_grid* g, void* ws) {
    const size_t n = (size_t)g->nx * g->ny * g->nz;
    char* p = (char*)ws;
    SlabWs w;
    w.sc = (SlabScalars*)p;
    p += align256(sizeof(SlabScalars));
    w.part = (double*)p;
    p += align256(kSlabVals * kMaxPartials * sizeof(double));
    double** vs[6] = {&w.v.res, &w.v.res0, &w.v.pp, &w.v.vv, &w.v.s, &w.v.t};
    for (double** q : vs) {
        *q = (double*)p;
        p += align256(n * sizeof(double));
    }
    return w;
}

int pointwise_blocks(long long n) {
    const long long b = (n + kBlock * 4 - 1) / (kBlock * 4);
    return (int)std::max<long long>(1, std::min<long long>(b, std::min(num_sms() * 8, kMaxPartials)));
}

__device__ __forceinline__ bool slab_last(SlabScalars* sc) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (tid0()) last = atomicAdd(&sc->counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (last) __threadfence();
    return last;
}

// the last block sums (or maxes) the partials in block order and writes send[slot]
template <bool MAX>
__device__ double finish_blocks(const double* part, int nblocks, double* sh) {
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    double v = 0.0;
    for (int b = tid; b < nblocks; b += kBlock) {
        const double x = ((volatile const double*)part)[b];
        v = MAX ? nanmax(v, x) : v + x;
    }
    return MAX ? block_max<kBlock>(v, sh) : block_sum<kBlock>(v, sh);
}

// ------------------------------------------------------------------ init
// res = res0 = (div * rho/dt) * (-vol) on the interior (the reference's
// source_P *= rho/dt; source_P *= -vol; src/solver/pressure.py:205-212);
// DP, pp, vv, s, t = 0 on every plane.  send = [(res, res0), max|res|].
__global__ void __launch_bounds__(kBlock)
slab_init(Slab sl, SlabWs w, const double* __restrict__ div, double c1, double c2,
          double* __restrict__ DP, double* __restrict__ send, double min_res, int max_it) {
    __shared__ double sh[32];
    double s = 0.0, m = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < sl.d.n; q += stride) {
        DP[q] = 0.0;
        w.v.pp[q] = 0.0;
        w.v.vv[q] = 0.0;
        w.v.s[q] = 0.0;
        w.v.t[q] = 0.0;
        double r = 0.0;
        if (q >= sl.off && q < sl.off + sl.nint) {
            r = (div[q] * c1) * c2;
            s += r * r;
            m = nanmax(m, fabs(r));
        }
        w.v.res[q] = r;
        w.v.res0[q] = r;
    }
    const double bs = block_sum<kBlock>(s, sh);
    const double bm = block_max<kBlock>(m, sh);
    if (tid0()) { w.part[blockIdx.x] = bs; w.part[kMaxPartials + blockIdx.x] = bm; }
    if (slab_last(w.sc)) {
        const double tot = finish_blocks<false>(w.part, gridDim.x, sh);
        const double mx = finish_blocks<true>(w.part + kMaxPartials, gridDim.x, sh);
        if (tid0()) {
            send[0] = tot;
            send[1] = mx;
            SlabScalars* sc = w.sc;
            sc->rho1 = 1.0; sc->rho2 = 1.0; sc->alpha = 0.0; sc->omega = 1.0;
            sc->max_res0 = 0.0; sc->max_res = 0.0; sc->min_res = min_res;
            sc->iter = 0; sc->max_it = max_it; sc->done = 0; sc->status = PF_OK;
            sc->counter = 0u;
        }
    }
}

// ------------------------------------------------------------------ folds
// One thread folds the gathered values of every rank in rank order.
enum { kFoldStart = 0, kFoldNext = 1, kFoldGamma = 2, kFoldOmega = 3 };

__global__ void slab_fold(SlabScalars* sc, const double* __restrict__ recv, int world, int mode) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (mode != kFoldStart && sc->done) return;
    double a = 0.0, b = 0.0;
    for (int r = 0; r < world; ++r) {
        a += recv[r * kSlabVals];
        b = (mode == kFoldOmega) ? b + recv[r * kSlabVals + 1] : nanmax(b, recv[r * kSlabVals + 1]);
    }
    if (mode == kFoldStart) {
        // max_res0 (src/solver/pressure.py:213) and rho1 of iteration 1
        sc->max_res0 = b;
        sc->rho1 = a;
    } else if (mode == kFoldNext) {
        // end of an iteration (src/solver/pressure.py:276-289): rho2 = rho1,
        // the stop test on max|res| / max_res0, then rho1 of the next one
        sc->rho2 = sc->rho1;
        sc->rho1 = a;
        const double mr = b / sc->max_res0;
        sc->max_res = mr;
        sc->iter += 1;
        if (!(mr == mr)) { sc->done = 1; sc->status = PF_NONFINITE; }
        else if (mr <= sc->min_res) { sc->done = 1; sc->status = PF_OK; }
        else if (sc->iter >= sc->max_it) { sc->done = 1; sc->status = PF_MAXIT; }
    } else if (mode == kFoldGamma) {
        // gamma = (vv, res0); gamma == 0 leaves the loop before DP changes
        if (a == 0.0) { sc->done = 1; sc->status = PF_BREAKDOWN; }
        else sc->alpha = sc->rho1 / a;
    } else {
        // omega = (s, t) / (t, t); (t, t) == 0 leaves after DP += alpha pp
        if (b == 0.0) { sc->done = 1; sc->status = PF_BREAKDOWN; }
        else sc->omega = a / b;
    }
}

// ------------------------------------------------------------------ pointwise
// pp = (pp - omega vv) beta + res, beta = alpha rho1 / (rho2 omega)
// (src/solver/pressure.py:229-234)
__global__ void __launch_bounds__(kBlock)
slab_pupdate(Slab sl, SlabWs w) {
    const SlabScalars* sc = w.sc;
    if (sc->done) return;
    const double omega = sc->omega;
    const double beta = sc->alpha * sc->rho1 / (sc->rho2 * omega);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long q = sl.off + blockIdx.x * (long long)blockDim.x + threadIdx.x;
         q < sl.off + sl.nint; q += stride) {
        double p = fma(-omega, w.v.vv[q], w.v.pp[q]);
        p = p * beta;
        w.v.pp[q] = p + w.v.res[q];
    }
}

// DP += alpha pp; s = res - alpha vv (src/solver/pressure.py:250-255)
__global__ void __launch_bounds__(kBlock)
slab_supdate(Slab sl, SlabWs w, double* __restrict__ DP) {
    const SlabScalars* sc = w.sc;
    if (sc->done) return;
    const double alpha = sc->alpha;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long q = sl.off + blockIdx.x * (long long)blockDim.x + threadIdx.x;
         q < sl.off + sl.nint; q += stride) {
        DP[q] = fma(alpha, w.v.pp[q], DP[q]);
        w.v.s[q] = fma(-alpha, w.v.vv[q], w.v.res[q]);
    }
}

// DP += omega s; res = s - omega t; send = [(res, res0), max|res|]
// (src/solver/pressure.py:269-283)
__global__ void __launch_bounds__(kBlock)
slab_final(Slab sl, SlabWs w, double* __restrict__ DP, double* __restrict__ send) {
    __shared__ double sh[32];
    SlabScalars* sc = w.sc;
    if (sc->done) return;
    const double omega = sc->omega;
    double s = 0.0, m = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long q = sl.off + blockIdx.x * (long long)blockDim.x + threadIdx.x;
         q < sl.off + sl.nint; q += stride) {
        const double sv = w.v.s[q];
        DP[q] = fma(omega, sv, DP[q]);
        const double r = fma(-omega, w.v.t[q], sv);
        w.v.res[q] = r;
        s += r * w.v.res0[q];
        m = nanmax(m, fabs(r));
    }
    const double bs = block_sum<kBlock>(s, sh);
    const double bm = block_max<kBlock>(m, sh);
    if (tid0()) { w.part[blockIdx.x] = bs; w.part[kMaxPartials + blockIdx.x] = bm; }
    if (slab_last(sc)) {
        const double tot = finish_blocks<false>(w.part, gridDim.x, sh);
        const double mx = finish_blocks<true>(w.part + kMaxPartials, gridDim.x, sh);
        if (tid0()) { send[0] = tot; send[1] = mx; sc->counter = 0u; }
    }
}

// ------------------------------------------------------------------ operator
// out = A in on the interior (Pressure_Base.applyOperator,
// src/solver/pressure.py:54-84, the terms in the order of laplace_kernel):
// x neighbours from the planes beside the interior (ghost planes at its
// ends), y and z wrap.  APPLY_P: vv = A pp, send = [(vv, res0), 0];
// APPLY_S: t = A s, send = [(s, t), (t, t)].  A block of 32 x 8 threads walks
// 32 (z) x 8 (y) tiles of the interior planes, tile index += grid size.
template <bool S_PHASE>
__global__ void __launch_bounds__(kBlock)
slab_apply(Slab sl, SlabWs w, LapCoef<double> cf, double* __restrict__ send) {
    __shared__ double sh[32];
    SlabScalars* sc = w.sc;
    if (sc->done) return;
    const Dims d = sl.d;
    const double* A = S_PHASE ? w.v.s : w.v.pp;
    double* B = S_PHASE ? w.v.t : w.v.vv;
    const int tz = (d.nz + 31) / 32, ty = (d.ny + 7) / 8;
    const long long ntiles = (long long)tz * ty * (d.nx - 2 * sl.h);
    double s1 = 0.0, s2 = 0.0;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int k = (int)(t % tz) * 32 + threadIdx.x;
        const int j = (int)((t / tz) % ty) * 8 + threadIdx.y;
        const int i = sl.h + (int)(t / ((long long)tz * ty));
        if (k >= d.nz || j >= d.ny) continue;
        const long long q = idx(d, i, j, k);
        const double c = A[q];
        double b = 0.0;
        b += A[idx(d, i - 1, j, k)] * cf.c[0][0];
        b += c * cf.c[0][1];
        b += A[idx(d, i + 1, j, k)] * cf.c[0][2];
        b += A[idx(d, i, wrap(j - 1, d.ny), k)] * cf.c[1][0];
        b += c * cf.c[1][1];
        b += A[idx(d, i, wrap(j + 1, d.ny), k)] * cf.c[1][2];
        b += A[idx(d, i, j, wrap(k - 1, d.nz))] * cf.c[2][0];
        b += c * cf.c[2][1];
        b += A[idx(d, i, j, wrap(k + 1, d.nz))] * cf.c[2][2];
        B[q] = b;
        if (S_PHASE) { s1 += c * b; s2 += b * b; }
        else s1 += b * w.v.res0[q];
    }
    const double b1 = block_sum<kBlock>(s1, sh);
    const double b2 = S_PHASE ? block_sum<kBlock>(s2, sh) : 0.0;
    if (tid0()) { w.part[blockIdx.x] = b1; w.part[kMaxPartials + blockIdx.x] = b2; }
    if (slab_last(sc)) {
        const double t1 = finish_blocks<false>(w.part, gridDim.x, sh);
        const double t2 = S_PHASE ? finish_blocks<false>(w.part + kMaxPartials, gridDim.x, sh) : 0.0;
        if (tid0()) { send[0] = t1; send[1] = t2; sc->counter = 0u; }
    }
}

// p += DP on the interior (src/solver/pressure.py:293-294)
__global__ void __launch_bounds__(kBlock)
slab_add(Slab sl, const double* __restrict__ DP, double* __restrict__ p) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long q = sl.off + blockIdx.x * (long long)blockDim.x + threadIdx.x;
         q < sl.off + sl.nint; q += stride)
        p[q] = p[q] + DP[q];
}

__global__ void slab_info(const SlabScalars* sc, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    out[0] = sc->max_res;
    out[1] = (double)sc->iter;
    out[2] = (double)sc->status;
    out[3] = (double)sc->done;
}

// blocks of the apply kernel: every SM busy, at most kMaxPartials
int apply_blocks(const Slab& sl) {
    const long long nt = (long long)((sl.d.nz + 31) / 32) * ((sl.d.ny + 7) / 8) * (sl.d.nx - 2 * sl.h);
    return (int)std::max<long long>(1, std::min<long long>(nt, std::min(num_sms() * 8, kMaxPartials)));
}

}  // namespace
}  // namespace pf

using namespace pf;

static bool slab_ok(const pf_grid* g, int halo) {
    return g && g->ny >= 2 && g->nz >= 2 && halo >= 1 && g->nx - 2 * halo >= 1 &&
           g->dx > 0 && g->dy > 0 && g->dz > 0;
}

static int rc_of(cudaError_t e) { return e == cudaSuccess ? PF_OK : PF_ERR_CUDA; }

extern "C" {

size_t pf_slab_workspace_bytes(const pf_grid* g) {
    if (!g || g->nx < 1 || g->ny < 1 || g->nz < 1) return 0;
    return slab_ws_bytes(g);
}

int pf_slab_bicg_vectors(const pf_grid* g, void* ws, double** pp, double** s) {
    if (!g || !ws || !pp || !s) return PF_ERR_BAD_ARG;
    const SlabWs w = carve_slab(g, ws);
    *pp = w.v.pp;
    *s = w.v.s;
    return PF_OK;
}

int pf_slab_bicg_init(const pf_grid* g, int halo, double rho, double dt, double min_res,
                      int max_it, const double* div, double* DP, void* ws, size_t ws_bytes,
                      double* send, void* stream) {
    if (!slab_ok(g, halo) || !div || !DP || !send || !ws || ((uintptr_t)ws & 255) ||
        ws_bytes < slab_ws_bytes(g) || !(rho != 0.0) || !(dt != 0.0) || max_it < 1)
        return PF_ERR_BAD_ARG;
    const Slab sl = make_slab(g, halo);
    const SlabWs w = carve_slab(g, ws);
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemsetAsync(&w.sc->counter, 0, sizeof(unsigned int), s) != cudaSuccess)
        return PF_ERR_CUDA;
    const double vol = (g->dx * g->dy) * g->dz;
    PF_LAUNCH("slab_init", s, slab_init<<<pointwise_blocks(sl.d.n), kBlock, 0, s>>>(
        sl, w, div, rho / dt, -1.0 * vol, DP, send, min_res, max_it));
    return rc_of(cudaGetLastError());
}

int pf_slab_bicg_phase(const pf_grid* g, int halo, int phase, const double* recv, int world,
                       double* DP, void* ws, double* send, void* stream) {
    if (!slab_ok(g, halo) || !ws || ((uintptr_t)ws & 255) || phase < PF_SLAB_START ||
        phase > PF_SLAB_FINAL)
        return PF_ERR_BAD_ARG;
    const bool folds = phase == PF_SLAB_START || phase == PF_SLAB_NEXT || phase == PF_SLAB_S ||
                       phase == PF_SLAB_FINAL;
    if (folds && (!recv || world < 1 || world > kSlabMaxRanks)) return PF_ERR_BAD_ARG;
    if ((phase == PF_SLAB_S || phase == PF_SLAB_FINAL) && !DP) return PF_ERR_BAD_ARG;
    if ((phase == PF_SLAB_APPLY_P || phase == PF_SLAB_APPLY_S || phase == PF_SLAB_FINAL) && !send)
        return PF_ERR_BAD_ARG;
    const Slab sl = make_slab(g, halo);
    const SlabWs w = carve_slab(g, ws);
    cudaStream_t s = (cudaStream_t)stream;
    const int nb = pointwise_blocks(sl.nint);
    switch (phase) {
        case PF_SLAB_START:
        case PF_SLAB_NEXT:
            PF_LAUNCH("slab_fold", s, slab_fold<<<1, 32, 0, s>>>(
                w.sc, recv, world, phase == PF_SLAB_START ? kFoldStart : kFoldNext));
            PF_LAUNCH("slab_pupdate", s, slab_pupdate<<<nb, kBlock, 0, s>>>(sl, w));
            break;
        case PF_SLAB_APPLY_P:
        case PF_SLAB_APPLY_S: {
            const int ab = apply_blocks(sl);
            if (phase == PF_SLAB_APPLY_P)
                PF_LAUNCH("slab_apply_p", s, slab_apply<false><<<ab, dim3(32, 8), 0, s>>>(
                    sl, w, lap_coef<double>(g), send));
            else
                PF_LAUNCH("slab_apply_s", s, slab_apply<true><<<ab, dim3(32, 8), 0, s>>>(
                    sl, w, lap_coef<double>(g), send));
            break;
        }
        case PF_SLAB_S:
            PF_LAUNCH("slab_fold", s, slab_fold<<<1, 32, 0, s>>>(w.sc, recv, world, kFoldGamma));
            PF_LAUNCH("slab_supdate", s, slab_supdate<<<nb, kBlock, 0, s>>>(sl, w, DP));
            break;
        case PF_SLAB_FINAL:
            PF_LAUNCH("slab_fold", s, slab_fold<<<1, 32, 0, s>>>(w.sc, recv, world, kFoldOmega));
            PF_LAUNCH("slab_final", s, slab_final<<<nb, kBlock, 0, s>>>(sl, w, DP, send));
            break;
    }
    return rc_of(cudaGetLastError());
}

int pf_slab_bicg_info(const pf_grid* g, void* ws, double* out_dev, void* stream) {
    if (!g || !ws || !out_dev) return PF_ERR_BAD_ARG;
    const SlabWs w = carve_slab(g, ws);
    cudaStream_t s = (cudaStream_t)stream;
    slab_info<<<1, 32, 0, s>>>(w.sc, out_dev);
    return rc_of(cudaGetLastError());
}

int pf_slab_add(const pf_grid* g, int halo, const double* DP, double* p, void* stream) {
    if (!slab_ok(g, halo) || !DP || !p) return PF_ERR_BAD_ARG;
    const Slab sl = make_slab(g, halo);
    cudaStream_t s = (cudaStream_t)stream;
    PF_LAUNCH("slab_add", s, slab_add<<<pointwise_blocks(sl.nint), kBlock, 0, s>>>(sl, DP, p));
    return rc_of(cudaGetLastError());
}

}  // extern "C"
