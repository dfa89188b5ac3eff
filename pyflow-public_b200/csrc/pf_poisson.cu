// pf_poisson.cu -- pressure Poisson solvers, divergence, projection, stats.
//
// BiCGStab (solver_bicgstab.solve, src/solver/pressure.py:196-297) runs as
// three fused kernels per iteration around its three global reductions:
//   phase A: pp' = (pp - omega vv) beta + res, vv' = A pp', gamma = (vv', res0)
//   phase B: s = res - alpha vv',             t = A s,     (s,t), (t,t)
//   phase C: DP += alpha pp' + omega s, res = s - omega t, (res,res0), max|res|
// A is the 7-point operator of Pressure_Base.applyOperator
// (src/solver/pressure.py:54-84, coefficients metric_staggered.py:84-102).
// Phases A and B evaluate their stencil operand on the fly: a block stages
// one x-plane of the operand (with its y/z halo) in shared memory, computing
// each value from res/pp/vv as it is loaded, and marches along x keeping the
// i-1, i, i+1 planes of its own cells in registers.  Old/new pp and vv live in
// ping-pong buffers chosen by the iteration parity read from device memory.
//
// All scalars (rho1, rho2, alpha, omega, ...) stay in device memory; each
// reduction is finished by the last block to arrive (fixed summation order,
// so results are bitwise reproducible run to run), which also evaluates the
// reference's stop tests and sets a `done` flag that makes every later
// kernel of the solve return immediately.  The host only polls that flag.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "pf_common.cuh"
#include "pf_kernels.cuh"
#include "pf_profile.cuh"

namespace pf {

struct BicgScalars {
    double rho1, rho2, alpha, omega, gamma, buf1, buf2;
    double max_res0, max_res, min_res;
    double scale;      // mixed: max|r| of the current refinement pass
    double max_b;      // mixed: max|b|
    int iter, done, status, max_it;
    unsigned int counter;
    int pad[3];
};

template <typename T>
struct LapCoef {
    T c[3][3];
};

template <typename T>
static LapCoef<T> lap_coef(const pf_grid* g) {
    // metric_uniform.__init__ (metric_staggered.py:84-102) in FP64, then cast
    const double dxi = 1.0 / g->dx, dyi = 1.0 / g->dy, dzi = 1.0 / g->dz;
    const double vol = (g->dx * g->dy) * g->dz;
    const double di[3] = {dxi, dyi, dzi};
    LapCoef<T> c;
    for (int q = 0; q < 3; ++q) {
        c.c[q][0] = T((di[q] * di[q]) * (-1.0 * vol));
        c.c[q][1] = T(((-2.0 * di[q]) * di[q]) * (-1.0 * vol));
        c.c[q][2] = T((di[q] * di[q]) * (-1.0 * vol));
    }
    return c;
}

struct Tiling {
    int ntz, nty, ntx, xc;
    long long ntiles;
};

static int num_sms() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

static Tiling make_tiling(const Dims& d) {
    Tiling t;
    t.ntz = (d.nz + kTileZ - 1) / kTileZ;
    t.nty = (d.ny + kTileY - 1) / kTileY;
    const long long yz = (long long)t.ntz * t.nty;
    const long long want = (long long)num_sms() * 4;  // tiles to fill the GPU
    long long xc = (yz * d.nx) / want;
    xc = std::max<long long>(4, std::min<long long>(32, xc));
    t.xc = (int)std::min<long long>(xc, d.nx);
    t.ntx = (d.nx + t.xc - 1) / t.xc;
    t.ntiles = yz * t.ntx;
    return t;
}

static int tiled_grid(const Tiling& t) {
    return (int)std::min<long long>(t.ntiles, std::min(num_sms() * 6, kMaxPartials));
}

static int pointwise_grid(long long n) {
    long long b = (n + kBlock * 4 - 1) / (kBlock * 4);
    return (int)std::max<long long>(1, std::min<long long>(b, std::min(num_sms() * 8, kMaxPartials)));
}

// --------------------------------------------------------------------------
// Tiled 7-point sweep.  load(i,j,k) returns the operand at a cell; epi(i,j,k,
// centre, Ax) consumes the operator value at each owned cell.  Block: 32 x 8
// threads, tile 32 (z) x 16 (y) x xc (x); each thread owns rows ty, ty+8.
// --------------------------------------------------------------------------
template <typename T, typename Load, typename Epi>
__device__ __forceinline__ void sweep_tiles(const Dims& d, const Tiling& tl,
                                            const LapCoef<T>& cf, Load& load,
                                            Epi& epi) {
    __shared__ T sm[kTileY + 2][kTileZ + 2];
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (long long t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int tz = (int)(t % tl.ntz);
        const long long r = t / tl.ntz;
        const int tyy = (int)(r % tl.nty);
        const int txx = (int)(r / tl.nty);
        const int k0 = tz * kTileZ, j0 = tyy * kTileY, i0 = txx * tl.xc;
        const int i1 = min(i0 + tl.xc, d.nx);
        const int ez = min(kTileZ, d.nz - k0), ey = min(kTileY, d.ny - j0);
        const int k = k0 + tx;
        const int jr0 = j0 + ty, jr1 = j0 + ty + 8;
        const bool v0 = (tx < ez) && (ty < ey), v1 = (tx < ez) && (ty + 8 < ey);
        T p0 = T(0), p1 = T(0), c0 = T(0), c1 = T(0), n0 = T(0), n1 = T(0);
        const int im = wrap(i0 - 1, d.nx);
        if (v0) { p0 = load(im, jr0, k); c0 = load(i0, jr0, k); }
        if (v1) { p1 = load(im, jr1, k); c1 = load(i0, jr1, k); }
        for (int i = i0; i < i1; ++i) {
            const int ip = wrap(i + 1, d.nx);
            if (v0) { n0 = load(ip, jr0, k); sm[ty + 1][tx + 1] = c0; }
            if (v1) { n1 = load(ip, jr1, k); sm[ty + 9][tx + 1] = c1; }
            if (ty == 0) {
                if (tx < ez) sm[0][tx + 1] = load(i, wrap(j0 - 1, d.ny), k0 + tx);
            } else if (ty == 1) {
                if (tx < ez) sm[ey + 1][tx + 1] = load(i, wrap(j0 + ey, d.ny), k0 + tx);
            } else if (ty == 2) {
                if (tx < ey) sm[tx + 1][0] = load(i, j0 + tx, wrap(k0 - 1, d.nz));
            } else if (ty == 3) {
                if (tx < ey) sm[tx + 1][ez + 1] = load(i, j0 + tx, wrap(k0 + ez, d.nz));
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const bool vq = q ? v1 : v0;
                if (!vq) continue;
                const int yy = ty + 8 * q + 1, zz = tx + 1;
                const T pc = q ? p1 : p0, cc = q ? c1 : c0, nc = q ? n1 : n0;
                T b = T(0);
                b += pc * cf.c[0][0];
                b += cc * cf.c[0][1];
                b += nc * cf.c[0][2];
                b += sm[yy - 1][zz] * cf.c[1][0];
                b += cc * cf.c[1][1];
                b += sm[yy + 1][zz] * cf.c[1][2];
                b += sm[yy][zz - 1] * cf.c[2][0];
                b += cc * cf.c[2][1];
                b += sm[yy][zz + 1] * cf.c[2][2];
                epi(i, q ? jr1 : jr0, k, cc, b);
            }
            __syncthreads();
            p0 = c0; c0 = n0; p1 = c1; c1 = n1;
        }
    }
}

// Last-block completion: returns true in every thread of the last block.
__device__ __forceinline__ bool arrive_last(BicgScalars* sc) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        const unsigned prev = atomicAdd(&sc->counter, 1u);
        last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

// Sum (or max) of gridDim.x partials in a fixed order, by the calling block.
template <bool MAX>
__device__ double finish(const double* part, double* sh) {
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int nt = blockDim.x * blockDim.y;
    double v = 0.0;
    for (int b = tid; b < (int)gridDim.x; b += nt) {
        const double x = ((volatile const double*)part)[b];
        v = MAX ? nanmax(v, x) : v + x;
    }
    return MAX ? block_max<kBlock>(v, sh) : block_sum<kBlock>(v, sh);
}

// ---------------------------------------------------------------- init
// FP64 path: res = res0 = (source * rho/dt) * (-vol); DP = pp = vv = 0.
// Mixed inner pass: res = res0 = T(r / scale) where r is the FP64 residual.
template <typename T, bool FROM_RESIDUAL>
__global__ void __launch_bounds__(kBlock)
bicg_init(Dims d, BicgScalars* sc, double* part, const double* src, double c1,
          double c2, T* res, T* res0, T* xs, T* pp0, T* pp1, T* vv0, T* vv1,
          int max_it, double min_res) {
    __shared__ double sh[32];
    double s = 0.0, m = 0.0;
    const double inv = FROM_RESIDUAL ? 1.0 / sc->scale : 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < d.n;
         q += (long long)gridDim.x * blockDim.x) {
        T r;
        if (FROM_RESIDUAL) r = T(src[q] * inv);
        else r = T((src[q] * c1) * c2);
        res[q] = r; res0[q] = r;
        xs[q] = T(0); pp0[q] = T(0); pp1[q] = T(0); vv0[q] = T(0); vv1[q] = T(0);
        s += double(r) * double(r);
        m = nanmax(m, fabs(double(r)));
    }
    const double bs = block_sum<kBlock>(s, sh);
    const double bm = block_max<kBlock>(m, sh);
    if (threadIdx.x == 0) { part[blockIdx.x] = bs; part[kMaxPartials + blockIdx.x] = bm; }
    if (arrive_last(sc)) {
        const double tot = finish<false>(part, sh);
        const double mx = finish<true>(part + kMaxPartials, sh);
        if (threadIdx.x == 0) {
            sc->rho1 = tot; sc->rho2 = 1.0; sc->alpha = 0.0; sc->omega = 1.0;
            sc->max_res0 = mx; sc->max_res = 0.0; sc->iter = 0; sc->done = 0;
            sc->status = PF_OK; sc->max_it = max_it; sc->min_res = min_res;
            sc->counter = 0u;
        }
    }
}

// ---------------------------------------------------------------- phase A
template <typename T>
__global__ void __launch_bounds__(kBlock)
bicg_phase_a(Dims d, Tiling tl, LapCoef<T> cf, BicgScalars* sc, double* part,
             const T* __restrict__ res, const T* __restrict__ res0, T* pp0,
             T* pp1, T* vv0, T* vv1) {
    __shared__ double sh[32];
    if (sc->done) return;
    const int par = sc->iter & 1;
    const T* ppo = par ? pp1 : pp0;
    const T* vvo = par ? vv1 : vv0;
    T* ppn = par ? pp0 : pp1;
    T* vvn = par ? vv0 : vv1;
    const double beta_d = (sc->alpha * sc->rho1) / (sc->rho2 * sc->omega);
    const T beta = T(beta_d), omega = T(sc->omega);
    double acc = 0.0;
    auto load = [&](int i, int j, int k) -> T {
        const long long q = idx(d, i, j, k);
        T x = fma(-omega, vvo[q], ppo[q]);  // pp.sub_(omega, vv)
        x = x * beta;                       // pp.mul_(beta)
        return x + res[q];                  // pp.add_(res)
    };
    auto epi = [&](int i, int j, int k, T c, T b) {
        const long long q = idx(d, i, j, k);
        ppn[q] = c;
        vvn[q] = b;
        acc += double(b) * double(res0[q]);
    };
    sweep_tiles<T>(d, tl, cf, load, epi);
    const double bs = block_sum<kBlock>(acc, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) part[blockIdx.x] = bs;
    if (arrive_last(sc)) {
        const double gamma = finish<false>(part, sh);
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            sc->gamma = gamma;
            if (gamma == 0.0) {
                sc->done = 1;
                sc->status = PF_BREAKDOWN;
            } else {
                sc->alpha = sc->rho1 / gamma;
            }
            sc->counter = 0u;
        }
    }
}

// ---------------------------------------------------------------- phase B
template <typename T>
__global__ void __launch_bounds__(kBlock)
bicg_phase_b(Dims d, Tiling tl, LapCoef<T> cf, BicgScalars* sc, double* part,
             const T* __restrict__ res, const T* vv0, const T* vv1,
             T* __restrict__ t) {
    __shared__ double sh[32];
    if (sc->done) return;
    const int par = sc->iter & 1;
    const T* vv = par ? vv0 : vv1;  // written by phase A of this iteration
    const T alpha = T(sc->alpha);
    double a1 = 0.0, a2 = 0.0;
    auto load = [&](int i, int j, int k) -> T {
        const long long q = idx(d, i, j, k);
        return fma(-alpha, vv[q], res[q]);  // s = res; s.sub_(alpha, vv)
    };
    auto epi = [&](int i, int j, int k, T c, T b) {
        t[idx(d, i, j, k)] = b;
        a1 += double(c) * double(b);
        a2 += double(b) * double(b);
    };
    sweep_tiles<T>(d, tl, cf, load, epi);
    const double b1 = block_sum<kBlock>(a1, sh);
    const double b2 = block_sum<kBlock>(a2, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        part[blockIdx.x] = b1;
        part[kMaxPartials + blockIdx.x] = b2;
    }
    if (arrive_last(sc)) {
        const double buf1 = finish<false>(part, sh);
        const double buf2 = finish<false>(part + kMaxPartials, sh);
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            sc->buf1 = buf1; sc->buf2 = buf2;
            if (buf2 == 0.0) {
                sc->done = 2;  // phase C applies DP += alpha pp, then stops
                sc->status = PF_BREAKDOWN;
            } else {
                sc->omega = buf1 / buf2;
            }
            sc->counter = 0u;
        }
    }
}

// ---------------------------------------------------------------- phase C
template <typename T>
__global__ void __launch_bounds__(kBlock)
bicg_phase_c(Dims d, BicgScalars* sc, double* part, T* __restrict__ res,
             const T* __restrict__ res0, const T* pp0, const T* pp1,
             const T* vv0, const T* vv1, const T* __restrict__ t,
             T* __restrict__ x) {
    __shared__ double sh[32];
    const int done = sc->done;
    if (done == 1) return;
    const int par = sc->iter & 1;
    const T* pp = par ? pp0 : pp1;
    const T* vv = par ? vv0 : vv1;
    const T alpha = T(sc->alpha), omega = T(sc->omega);
    double s1 = 0.0, m = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < d.n;
         q += (long long)gridDim.x * blockDim.x) {
        T dp = fma(alpha, pp[q], x[q]);  // DP.add_(alpha, pp)
        if (done == 0) {
            const T s = fma(-alpha, vv[q], res[q]);
            dp = fma(omega, s, dp);             // DP.add_(omega, s)
            const T r = fma(-omega, t[q], s);   // res = s; res.sub_(omega, t)
            res[q] = r;
            s1 += double(r) * double(res0[q]);
            m = nanmax(m, fabs(double(r)));
        }
        x[q] = dp;
    }
    const double bs = block_sum<kBlock>(s1, sh);
    const double bm = block_max<kBlock>(m, sh);
    if (threadIdx.x == 0) { part[blockIdx.x] = bs; part[kMaxPartials + blockIdx.x] = bm; }
    if (arrive_last(sc)) {
        const double rho1 = finish<false>(part, sh);
        const double mx = finish<true>(part + kMaxPartials, sh);
        if (threadIdx.x == 0) {
            if (done == 2) {
                sc->done = 1;
            } else {
                sc->rho2 = sc->rho1;
                sc->rho1 = rho1;
                const double mr = mx / sc->max_res0;
                sc->max_res = mr;
                sc->iter += 1;
                if (!(mr == mr) || isinf(mr)) {
                    sc->done = 1; sc->status = PF_NONFINITE;
                } else if (mr <= sc->min_res) {
                    sc->done = 1; sc->status = PF_OK;
                } else if (sc->iter >= sc->max_it) {
                    sc->done = 1; sc->status = PF_MAXIT;
                }
            }
            sc->counter = 0u;
        }
    }
}

// ------------------------------------------------ mixed-precision refinement
// b = (source*rho/dt)*(-vol) in FP64, DP = 0, max|b|.
__global__ void __launch_bounds__(kBlock)
mixed_b_init(Dims d, BicgScalars* sc, double* part, const double* src,
             double c1, double c2, double* b, double* x) {
    __shared__ double sh[32];
    double m = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < d.n;
         q += (long long)gridDim.x * blockDim.x) {
        const double r = (src[q] * c1) * c2;
        b[q] = r;
        x[q] = 0.0;
        m = nanmax(m, fabs(r));
    }
    const double bm = block_max<kBlock>(m, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = bm;
    if (arrive_last(sc)) {
        const double mx = finish<true>(part, sh);
        if (threadIdx.x == 0) { sc->max_b = mx; sc->scale = mx; sc->counter = 0u; }
    }
}

// x += scale * e  (FP64 accumulate of the FP32 correction)
__global__ void __launch_bounds__(kBlock)
mixed_update(Dims d, const BicgScalars* sc, const float* e, double* x) {
    const double s = sc->scale;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < d.n;
         q += (long long)gridDim.x * blockDim.x)
        x[q] = x[q] + s * double(e[q]);
}

// r = b - A x in FP64 and max|r| (the refinement's true residual)
__global__ void __launch_bounds__(kBlock)
mixed_residual(Dims d, Tiling tl, LapCoef<double> cf, BicgScalars* sc,
               double* part, const double* __restrict__ b,
               const double* __restrict__ x, double* __restrict__ r) {
    __shared__ double sh[32];
    double m = 0.0;
    auto load = [&](int i, int j, int k) -> double { return x[idx(d, i, j, k)]; };
    auto epi = [&](int i, int j, int k, double c, double ax) {
        const long long q = idx(d, i, j, k);
        const double v = b[q] - ax;
        r[q] = v;
        m = nanmax(m, fabs(v));
    };
    sweep_tiles<double>(d, tl, cf, load, epi);
    const double bm = block_max<kBlock>(m, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) part[blockIdx.x] = bm;
    if (arrive_last(sc)) {
        const double mx = finish<true>(part, sh);
        if (threadIdx.x == 0 && threadIdx.y == 0) { sc->scale = mx; sc->counter = 0u; }
    }
}

// p += DP (src/solver/pressure.py:294)
__global__ void __launch_bounds__(kBlock)
add_inplace(long long n, const double* a, double* p) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x)
        p[q] = p[q] + a[q];
}

// ------------------------------------------------------------ workspace
struct PoissonWs {
    BicgScalars* sc;
    double* part;      // 2 x kMaxPartials
    void* vec;         // solver vectors
};

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

size_t poisson_ws_bytes(const pf_grid* g, int prec) {
    const size_t n = (size_t)g->nx * g->ny * g->nz;
    size_t b = align256(sizeof(BicgScalars)) + align256(2 * kMaxPartials * sizeof(double));
    if (prec == PF_FP64) {
        b += 7 * align256(n * sizeof(double));  // res res0 pp0 pp1 vv0 vv1 t
    } else {
        b += 8 * align256(n * sizeof(float));   // + e
        b += 2 * align256(n * sizeof(double));  // b, r
    }
    return b;
}

template <typename T>
struct BicgVecs {
    T *res, *res0, *pp0, *pp1, *vv0, *vv1, *t;
};

template <typename T>
static BicgVecs<T> carve(char*& p, size_t n) {
    BicgVecs<T> v;
    T** f[7] = {&v.res, &v.res0, &v.pp0, &v.pp1, &v.vv0, &v.vv1, &v.t};
    for (auto ptr : f) { *ptr = (T*)p; p += align256(n * sizeof(T)); }
    return v;
}

static int read_scalars(BicgScalars* dev, BicgScalars* host, cudaStream_t s) {
    if (cudaMemcpyAsync(host, dev, sizeof(BicgScalars), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return PF_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PF_ERR_CUDA;
    return PF_OK;
}

// Enqueue BiCGStab iterations in chunks, polling the device `done` flag
// between chunks.  Kernels of a finished solve return at once, so the
// iterations enqueued past convergence cost only their launch.
template <typename T>
static int run_iterations(const Dims& d, const Tiling& tl, const LapCoef<T>& cf,
                          BicgScalars* sc, double* part, const BicgVecs<T>& v,
                          T* x, cudaStream_t s, BicgScalars* hs) {
    const int gt = tiled_grid(tl), gp = pointwise_grid(d.n);
    dim3 blk2(32, 8);
    int chunk = 4;
    for (int guard = 0; guard < 1 << 20; ++guard) {
        for (int c = 0; c < chunk; ++c) {
            PF_LAUNCH(sizeof(T) == 8 ? "bicg_phase_a_f64" : "bicg_phase_a_f32", s, bicg_phase_a<T><<<gt, blk2, 0, s>>>(d, tl, cf, sc, part, v.res, v.res0, v.pp0, v.pp1, v.vv0, v.vv1));
            PF_LAUNCH(sizeof(T) == 8 ? "bicg_phase_b_f64" : "bicg_phase_b_f32", s, bicg_phase_b<T><<<gt, blk2, 0, s>>>(d, tl, cf, sc, part, v.res, v.vv0, v.vv1, v.t));
            PF_LAUNCH(sizeof(T) == 8 ? "bicg_phase_c_f64" : "bicg_phase_c_f32", s, bicg_phase_c<T><<<gp, kBlock, 0, s>>>(d, sc, part, v.res, v.res0, v.pp0, v.pp1, v.vv0, v.vv1, v.t, x));
        }
        if (cudaGetLastError() != cudaSuccess) return PF_ERR_CUDA;
        const int rc = read_scalars(sc, hs, s);
        if (rc) return rc;
        if (hs->done) return PF_OK;
        chunk = std::min(chunk * 2, 32);
    }
    return PF_ERR_CUDA;
}

int bicgstab_solve(const pf_grid* g, int prec, double rho, double dt,
                   double min_res, int max_it, const double* source,
                   double* DP, double* p, void* ws, cudaStream_t s,
                   pf_solve_info* info) {
    Dims d{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    const size_t n = (size_t)d.n;
    char* ptr = (char*)ws;
    BicgScalars* sc = (BicgScalars*)ptr; ptr += align256(sizeof(BicgScalars));
    double* part = (double*)ptr; ptr += align256(2 * kMaxPartials * sizeof(double));
    const Tiling tl = make_tiling(d);
    const int gp = pointwise_grid(d.n);
    const double vol = (g->dx * g->dy) * g->dz;
    const double c1 = rho / dt, c2 = -1.0 * vol;
    BicgScalars hs;
    std::memset(&hs, 0, sizeof(hs));
    if (cudaMemsetAsync(sc, 0, sizeof(BicgScalars), s) != cudaSuccess) return PF_ERR_CUDA;
    pf_solve_info out{0.0, 0, 1, PF_OK};
    if (prec == PF_FP64) {
        BicgVecs<double> v = carve<double>(ptr, n);
        const LapCoef<double> cf = lap_coef<double>(g);
        PF_LAUNCH("bicg_init_f64", s, bicg_init<double, false><<<gp, kBlock, 0, s>>>(d, sc, part, source, c1, c2, v.res, v.res0, DP,
                                                       v.pp0, v.pp1, v.vv0, v.vv1, max_it, min_res));
        // the reference loop always runs at least one iteration
        int rc = run_iterations<double>(d, tl, cf, sc, part, v, DP, s, &hs);
        if (rc) return rc;
        out.max_res = hs.max_res; out.iterations = hs.iter; out.status = hs.status;
    } else {
        BicgVecs<float> v = carve<float>(ptr, n);
        float* e = (float*)ptr; ptr += align256(n * sizeof(float));
        double* b = (double*)ptr; ptr += align256(n * sizeof(double));
        double* r = (double*)ptr; ptr += align256(n * sizeof(double));
        const LapCoef<float> cf = lap_coef<float>(g);
        const LapCoef<double> cfd = lap_coef<double>(g);
        dim3 blk2(32, 8);
        const int gt = tiled_grid(tl);
        PF_LAUNCH("mixed_b_init", s, mixed_b_init<<<gp, kBlock, 0, s>>>(d, sc, part, source, c1, c2, b, DP));
        if (read_scalars(sc, &hs, s)) return PF_ERR_CUDA;
        const double max_b = hs.max_b;
        // inner tolerance relative to the pass's initial residual; FP32
        // BiCGStab reliably contracts by this much before it stagnates
        const double inner_tol = 1e-4;
        const int max_outer = 30;
        int total = 0, status = PF_OK, outer = 0;
        double ratio = max_b > 0 ? 1.0 : 0.0, prev_ratio = 2.0;
        for (;; ++outer) {
            if (outer > 0) {
                PF_LAUNCH("mixed_update", s, mixed_update<<<gp, kBlock, 0, s>>>(d, sc, e, DP));
                PF_LAUNCH("mixed_residual", s, mixed_residual<<<gt, blk2, 0, s>>>(d, tl, cfd, sc, part, b, DP, r));
                if (read_scalars(sc, &hs, s)) return PF_ERR_CUDA;
                ratio = max_b > 0 ? hs.scale / max_b : 0.0;
            }
            if (!(ratio == ratio)) { status = PF_NONFINITE; break; }
            if (ratio <= min_res || max_b == 0.0) { status = PF_OK; break; }
            if (outer >= max_outer || total >= max_it) { status = PF_MAXIT; break; }
            if (outer > 1 && ratio > 0.5 * prev_ratio) { status = PF_STAGNATION; break; }
            prev_ratio = ratio;
            PF_LAUNCH("bicg_init_f32", s, bicg_init<float, true><<<gp, kBlock, 0, s>>>(d, sc, part, outer == 0 ? b : r, 0.0, 0.0,
                                                         v.res, v.res0, e, v.pp0, v.pp1, v.vv0, v.vv1,
                                                         max_it - total, inner_tol));
            const int rc = run_iterations<float>(d, tl, cf, sc, part, v, e, s, &hs);
            if (rc) return rc;
            total += hs.iter;
            if (hs.status == PF_NONFINITE) { status = PF_NONFINITE; break; }
        }
        out.max_res = ratio; out.iterations = total; out.outer = outer; out.status = status;
    }
    PF_LAUNCH("add_inplace", s, add_inplace<<<gp, kBlock, 0, s>>>(d.n, DP, p));
    if (cudaGetLastError() != cudaSuccess) return PF_ERR_CUDA;
    if (info) *info = out;
    return PF_OK;
}

// ------------------------------------------------------------------ Jacobi
// One sweep of solver_jacobi.solve (src/solver/pressure.py:141-147).
__global__ void __launch_bounds__(kBlock)
jacobi_sweep(Dims d, const double* __restrict__ pold, const double* __restrict__ src,
             double* __restrict__ pnew) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    const double DInv = -1.0 / 6.0;
    double x = -pold[idx(d, wrap(i + 1, d.nx), j, k)];
    x = x - pold[idx(d, wrap(i - 1, d.nx), j, k)];
    x = x - pold[idx(d, i, wrap(j + 1, d.ny), k)];
    x = x - pold[idx(d, i, wrap(j - 1, d.ny), k)];
    x = x - pold[idx(d, i, j, wrap(k + 1, d.nz))];
    x = x - pold[idx(d, i, j, wrap(k - 1, d.nz))];
    x = x + src[idx(d, i, j, k)];
    pnew[idx(d, i, j, k)] = x * DInv;
}

// scaled source, max|.| for the initial residual, then * dx^2
__global__ void __launch_bounds__(kBlock)
jacobi_prep(Dims d, BicgScalars* sc, double* part, const double* src, double c1,
            double dx2, double* s_out, double* p, double* pold) {
    __shared__ double sh[32];
    double m = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < d.n;
         q += (long long)gridDim.x * blockDim.x) {
        const double a = src[q] * c1;
        m = nanmax(m, fabs(a));
        s_out[q] = a * dx2;
        p[q] = 0.0;
        if (pold) pold[q] = 0.0;
    }
    const double bm = block_max<kBlock>(m, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = bm;
    if (arrive_last(sc)) {
        const double mx = finish<true>(part, sh);
        if (threadIdx.x == 0) { sc->max_res0 = mx; sc->counter = 0u; }
    }
}

// res = (A p) * -1 + source/dx^2, max|res| / max_res0
__global__ void __launch_bounds__(kBlock)
jacobi_residual(Dims d, Tiling tl, LapCoef<double> cf, BicgScalars* sc,
                double* part, const double* __restrict__ sdx, double dx2,
                const double* __restrict__ p) {
    __shared__ double sh[32];
    double m = 0.0;
    auto load = [&](int i, int j, int k) -> double { return p[idx(d, i, j, k)]; };
    auto epi = [&](int i, int j, int k, double c, double ax) {
        const double v = ax * -1.0 + sdx[idx(d, i, j, k)] / dx2;
        m = nanmax(m, fabs(v));
    };
    sweep_tiles<double>(d, tl, cf, load, epi);
    const double bm = block_max<kBlock>(m, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) part[blockIdx.x] = bm;
    if (arrive_last(sc)) {
        const double mx = finish<true>(part, sh);
        if (threadIdx.x == 0 && threadIdx.y == 0) { sc->max_res = mx / sc->max_res0; sc->counter = 0u; }
    }
}

int jacobi_solve(const pf_grid* g, double rho, double dt, int n_it,
                 const double* source, double* pold, double* p, void* ws,
                 cudaStream_t s, double* max_res) {
    Dims d{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    const size_t n = (size_t)d.n;
    char* ptr = (char*)ws;
    BicgScalars* sc = (BicgScalars*)ptr; ptr += align256(sizeof(BicgScalars));
    double* part = (double*)ptr; ptr += align256(2 * kMaxPartials * sizeof(double));
    double* sdx = (double*)ptr; ptr += align256(n * sizeof(double));
    double* tmp = (double*)ptr;
    const int gp = pointwise_grid(d.n);
    const double dx2 = std::pow(g->dx, 2.0);
    if (cudaMemsetAsync(sc, 0, sizeof(BicgScalars), s) != cudaSuccess) return PF_ERR_CUDA;
    PF_LAUNCH("jacobi_prep", s, jacobi_prep<<<gp, kBlock, 0, s>>>(d, sc, part, source, rho / dt, dx2, sdx, p, nullptr));
    dim3 blk(32, 8), grd((d.nz + 31) / 32, (d.ny + 7) / 8, d.nx);
    // iterate: pold <- p; p <- sweep(pold).  Ping-pong between p and tmp so
    // that the last two iterates land in p (last) and pold (previous).
    for (int it = 0; it < n_it; ++it) {
        const bool last = (it == n_it - 1);
        double* src_buf = (it == 0) ? p : ((it & 1) ? tmp : p);
        double* dst_buf = (it & 1) ? p : tmp;
        if (last) {
            cudaMemcpyAsync(pold, src_buf, n * sizeof(double), cudaMemcpyDeviceToDevice, s);
            PF_LAUNCH("jacobi_sweep", s, jacobi_sweep<<<grd, blk, 0, s>>>(d, pold, sdx, p));
        } else {
            PF_LAUNCH("jacobi_sweep", s, jacobi_sweep<<<grd, blk, 0, s>>>(d, src_buf, sdx, dst_buf));
        }
    }
    const Tiling tl = make_tiling(d);
    PF_LAUNCH("jacobi_residual", 0, jacobi_residual<<<tiled_grid(tl), dim3(32, 8), 0, s>>>(d, tl, lap_coef<double>(g), sc, part, sdx, dx2, p));
    if (cudaGetLastError() != cudaSuccess) return PF_ERR_CUDA;
    BicgScalars hs;
    if (read_scalars(sc, &hs, s)) return PF_ERR_CUDA;
    if (max_res) *max_res = hs.max_res;
    return PF_OK;
}

// ------------------------------------------------------- small operators
__global__ void __launch_bounds__(256)
div_kernel(Dims d, const double* __restrict__ u, const double* __restrict__ v,
           const double* __restrict__ w, double dxi, double dyi, double dzi,
           double* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    const long long q = idx(d, i, j, k);
    double a = (u[idx(d, wrap(i + 1, d.nx), j, k)] - u[q]) * dxi;
    a += (v[idx(d, i, wrap(j + 1, d.ny), k)] - v[q]) * dyi;
    a += (w[idx(d, i, j, wrap(k + 1, d.nz))] - w[q]) * dzi;
    out[q] = a;
}

__global__ void __launch_bounds__(256)
laplace_kernel(Dims d, LapCoef<double> cf, const double* __restrict__ A,
               double* __restrict__ B) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    const double c = A[idx(d, i, j, k)];
    double b = 0.0;
    b += A[idx(d, wrap(i - 1, d.nx), j, k)] * cf.c[0][0];
    b += c * cf.c[0][1];
    b += A[idx(d, wrap(i + 1, d.nx), j, k)] * cf.c[0][2];
    b += A[idx(d, i, wrap(j - 1, d.ny), k)] * cf.c[1][0];
    b += c * cf.c[1][1];
    b += A[idx(d, i, wrap(j + 1, d.ny), k)] * cf.c[1][2];
    b += A[idx(d, i, j, wrap(k - 1, d.nz))] * cf.c[2][0];
    b += c * cf.c[2][1];
    b += A[idx(d, i, j, wrap(k + 1, d.nz))] * cf.c[2][2];
    B[idx(d, i, j, k)] = b;
}

__global__ void __launch_bounds__(256)
vel_corr_kernel(Dims d, const double* __restrict__ DP, double scale, double dxi,
                double dyi, double dzi, double* __restrict__ u,
                double* __restrict__ v, double* __restrict__ w) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    const long long q = idx(d, i, j, k);
    const double c = DP[q];
    const double gx = (c - DP[idx(d, wrap(i - 1, d.nx), j, k)]) * dxi;
    const double gy = (c - DP[idx(d, i, wrap(j - 1, d.ny), k)]) * dyi;
    const double gz = (c - DP[idx(d, i, j, wrap(k - 1, d.nz))]) * dzi;
    u[q] = fma(-scale, gx, u[q]);  // var.sub_(scale, grad)
    v[q] = fma(-scale, gy, v[q]);
    w[q] = fma(-scale, gz, w[q]);
}

// max|u|, max|v|, max|w|, sum(u^2+v^2+w^2), max|div u|
__global__ void __launch_bounds__(256)
stats_kernel(Dims d, BicgScalars* sc, double* part, const double* __restrict__ u,
             const double* __restrict__ v, const double* __restrict__ w,
             double dxi, double dyi, double dzi, double* out) {
    __shared__ double sh[32];
    double mu_ = 0, mv = 0, mw = 0, s = 0, md = 0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < d.n;
         q += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(q % d.nz);
        const long long r = q / d.nz;
        const int j = (int)(r % d.ny), i = (int)(r / d.ny);
        const double a = u[q], b = v[q], c = w[q];
        mu_ = nanmax(mu_, fabs(a)); mv = nanmax(mv, fabs(b)); mw = nanmax(mw, fabs(c));
        s += (a * a + b * b) + c * c;
        double dv = (u[idx(d, wrap(i + 1, d.nx), j, k)] - a) * dxi;
        dv += (v[idx(d, i, wrap(j + 1, d.ny), k)] - b) * dyi;
        dv += (w[idx(d, i, j, wrap(k + 1, d.nz))] - c) * dzi;
        md = nanmax(md, fabs(dv));
    }
    double r[5] = {block_max<kBlock>(mu_, sh), block_max<kBlock>(mv, sh),
                   block_max<kBlock>(mw, sh), block_sum<kBlock>(s, sh),
                   block_max<kBlock>(md, sh)};
    if (threadIdx.x == 0)
        for (int c = 0; c < 5; ++c) part[c * kMaxPartials + blockIdx.x] = r[c];
    if (arrive_last(sc)) {
        double f[5];
        for (int c = 0; c < 5; ++c)
            f[c] = (c == 3) ? finish<false>(part + c * kMaxPartials, sh)
                            : finish<true>(part + c * kMaxPartials, sh);
        if (threadIdx.x == 0) {
            out[0] = f[0]; out[1] = f[1]; out[2] = f[2];
            out[3] = f[3] / double(d.n) * 0.5;
            out[4] = f[4];
            sc->counter = 0u;
        }
    }
}

size_t stats_ws_bytes(const pf_grid*) {
    return align256(sizeof(BicgScalars)) + align256(5 * kMaxPartials * sizeof(double));
}

cudaError_t launch_stats(const pf_grid* g, const double* u, const double* v,
                         const double* w, double* out, void* ws, cudaStream_t s) {
    Dims d{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    char* ptr = (char*)ws;
    BicgScalars* sc = (BicgScalars*)ptr; ptr += align256(sizeof(BicgScalars));
    double* part = (double*)ptr;
    cudaMemsetAsync(sc, 0, sizeof(BicgScalars), s);
    PF_LAUNCH("stats", s, stats_kernel<<<pointwise_grid(d.n), kBlock, 0, s>>>(d, sc, part, u, v, w, 1.0 / g->dx,
                                                       1.0 / g->dy, 1.0 / g->dz, out));
    return cudaGetLastError();
}

static dim3 cgrid(const Dims& d) { return dim3((d.nz + 31) / 32, (d.ny + 7) / 8, d.nx); }

cudaError_t launch_div(const pf_grid* g, const double* u, const double* v,
                       const double* w, double* div, cudaStream_t s) {
    Dims d{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    PF_LAUNCH("div_vel", 0, div_kernel<<<cgrid(d), dim3(32, 8), 0, s>>>(d, u, v, w, 1.0 / g->dx, 1.0 / g->dy, 1.0 / g->dz, div));
    return cudaGetLastError();
}

cudaError_t launch_laplace(const pf_grid* g, const double* A, double* B, cudaStream_t s) {
    Dims d{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    PF_LAUNCH("laplace_apply", 0, laplace_kernel<<<cgrid(d), dim3(32, 8), 0, s>>>(d, lap_coef<double>(g), A, B));
    return cudaGetLastError();
}

cudaError_t launch_vel_corr(const pf_grid* g, const double* DP, double scale,
                            double* u, double* v, double* w, cudaStream_t s) {
    Dims d{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    PF_LAUNCH("vel_corr", 0, vel_corr_kernel<<<cgrid(d), dim3(32, 8), 0, s>>>(d, DP, scale, 1.0 / g->dx, 1.0 / g->dy,
                                                     1.0 / g->dz, u, v, w));
    return cudaGetLastError();
}

}  // namespace pf
