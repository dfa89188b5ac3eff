// pf_mg.cu -- multigrid-preconditioned FP32 BiCGStab, the inner solver of the
// PF_MIXED_MG pressure refinement (no counterpart in the reference, whose
// solver_bicgstab, src/solver/pressure.py:196-297, is unpreconditioned).
//
// Right-preconditioned BiCGStab on A e = r (A = -vol L, the operator of
// Pressure_Base.applyOperator, src/solver/pressure.py:54-84):
//   p  = res + beta (p - omega v)      ph = M p     v = A ph    alpha = rho/(v,res0)
//   s  = res - alpha v                 sh = M s     t = A sh    omega = (t,s)/(t,t)
//   e += alpha ph + omega sh           res = s - omega t        rho' = (res,res0)
// M is one V(2,2) cycle of cell-centred geometric multigrid:
//   * levels halve every dimension while all are even, down to <= 512 cells;
//     level l uses the same 7-point operator with spacing 2^l h (the coarse
//     right-hand side is the SUM of the 8 fine residuals, because A carries
//     the cell volume);
//   * smoother: weighted Jacobi, omega = 6/7 (the optimal damping of the 3-D
//     7-point Laplacian); the two pre-smoothing sweeps start from zero and are
//     evaluated in one pass as x = w (2 b - w A b), w = omega / diag(A);
//   * restriction: sum of the 8 children's residuals b - A x, computed from x
//     in the same kernel; prolongation: trilinear (weights 27, 9, 3, 1 / 64);
//   * coarsest level: mean removed (the periodic operator is singular), then
//     48 Jacobi sweeps by one CTA in shared memory.
// M is a fixed linear operator (fixed sweep counts), as BiCGStab requires.
// At the finest level the p update and s = res - alpha v are fused into the
// first smoothing pass, which computes them for every cell it loads.
//
// All vectors are FP32; every dot product and max accumulates in FP64 and is
// finished by the last block (fixed order).  Scalars stay on the device.
#include <cmath>

#include "pf_common.cuh"
#include "pf_kernels.cuh"
#include "pf_mg.cuh"
#include "pf_profile.cuh"

namespace pf {

constexpr float kMgOmega = 6.0f / 7.0f;
constexpr int kMgCoarseSweeps = 48;

// ------------------------------------------------------------ sweep phases
// Sources of the first (from-zero) smoothing pass.
struct SrcPlain {  // b of a coarse level
    const float* b;
    struct Raw { float b; };
    __device__ void setup(const BicgScalars*) {}
    __device__ Raw raw(long long q) const { return Raw{b[q]}; }
    __device__ float op(const Raw& a) const { return a.b; }
    __device__ void store(long long, float) const {}
};

struct SrcP {  // p' = res + beta (p - omega v), stored to p_new
    const float *res, *p_old, *v;
    float* p_new;
    float beta, omega;
    struct Raw { float r, p, v; };
    __device__ void setup(const BicgScalars* sc) {
        beta = float((sc->rho1 / sc->rho2) * (sc->alpha / sc->omega));
        omega = float(sc->omega);
    }
    __device__ Raw raw(long long q) const { return Raw{res[q], p_old[q], v[q]}; }
    __device__ float op(const Raw& a) const {
        return fmaf(beta, fmaf(-omega, a.v, a.p), a.r);
    }
    __device__ void store(long long q, float c) const { p_new[q] = c; }
};

struct SrcS {  // s = res - alpha v, stored to s
    const float *res, *v;
    float* s;
    float alpha;
    struct Raw { float r, v; };
    __device__ void setup(const BicgScalars* sc) { alpha = float(sc->alpha); }
    __device__ Raw raw(long long q) const { return Raw{res[q], v[q]}; }
    __device__ float op(const Raw& a) const { return fmaf(-alpha, a.v, a.r); }
    __device__ void store(long long q, float c) const { s[q] = c; }
};

// x = w (2 b - w A b): two weighted-Jacobi sweeps from x = 0
template <class Src>
struct PhaseSmooth0 {
    static constexpr int R = 4;
    Src src;
    float* x;
    float wd;
    using Raw = typename Src::Raw;
    struct Ext {};
    __device__ Raw raw(long long q) const { return src.raw(q); }
    __device__ Ext ext(long long) const { return Ext{}; }
    __device__ float op(const Raw& a) const { return src.op(a); }
    __device__ void epi(long long q, float c, float ab, const Raw&, const Ext&) {
        src.store(q, c);
        x[q] = wd * (2.0f * c - wd * ab);
    }
};

// out = x + w (b - A x): one weighted-Jacobi sweep
struct PhaseSmooth {
    static constexpr int R = 4;
    const float *x, *b;
    float* out;
    float wd;
    struct Raw { float x; };
    struct Ext { float b; };
    __device__ Raw raw(long long q) const { return Raw{x[q]}; }
    __device__ Ext ext(long long q) const { return Ext{b[q]}; }
    __device__ float op(const Raw& a) const { return a.x; }
    __device__ void epi(long long q, float c, float ax, const Raw&, const Ext& e) {
        out[q] = fmaf(wd, e.b - ax, c);
    }
};

// v = A ph and (v, res0)
struct PhaseAv {
    static constexpr int R = 4;
    const float *ph, *res0;
    float* v;
    double dot;
    struct Raw { float x; };
    struct Ext { float r0; };
    __device__ Raw raw(long long q) const { return Raw{ph[q]}; }
    __device__ Ext ext(long long q) const { return Ext{res0[q]}; }
    __device__ float op(const Raw& a) const { return a.x; }
    __device__ void epi(long long q, float, float ax, const Raw&, const Ext& e) {
        v[q] = ax;
        dot += double(ax) * double(e.r0);
    }
};

// t = A sh, (t, s) and (t, t)
struct PhaseAt {
    static constexpr int R = 4;
    const float *sh, *s;
    float* t;
    double ts, tt;
    struct Raw { float x; };
    struct Ext { float s; };
    __device__ Raw raw(long long q) const { return Raw{sh[q]}; }
    __device__ Ext ext(long long q) const { return Ext{s[q]}; }
    __device__ float op(const Raw& a) const { return a.x; }
    __device__ void epi(long long q, float, float ax, const Raw&, const Ext& e) {
        t[q] = ax;
        ts += double(ax) * double(e.s);
        tt += double(ax) * double(ax);
    }
};

// ------------------------------------------------------------------ kernels
template <class Src>
__global__ void __launch_bounds__(kBlock, 2)
mg_smooth0(Dims d, Tiling tl, LapCoef<float> cf, const BicgScalars* sc,
           PhaseSmooth0<Src> ph) {
    if (sc->done) return;
    ph.src.setup(sc);
    sweep<float>(d, tl, cf, ph);
}

__global__ void __launch_bounds__(kBlock, 2)
mg_smooth(Dims d, Tiling tl, LapCoef<float> cf, const BicgScalars* sc, PhaseSmooth ph) {
    if (sc->done) return;
    sweep<float>(d, tl, cf, ph);
}

// bc[I,J,K] = sum over the 8 children of (b - A x) on the fine level
__global__ void __launch_bounds__(256)
mg_restrict(Dims f, LapCoef<float> cf, const float* __restrict__ b,
            const float* __restrict__ x, Dims c, float* __restrict__ bc,
            const BicgScalars* sc) {
    if (sc->done) return;
    const int K = blockIdx.x * 32 + threadIdx.x, J = blockIdx.y * 8 + threadIdx.y;
    const int I = blockIdx.z;
    if (K >= c.nz || J >= c.ny) return;
    long long ia[4], jb[4];
    int kc[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        ia[a] = (long long)wrap(2 * I - 1 + a, f.nx) * f.ny * f.nz;
        jb[a] = (long long)wrap(2 * J - 1 + a, f.ny) * f.nz;
        kc[a] = wrap(2 * K - 1 + a, f.nz);
    }
    // x on the 2x2x2 block and its 24 face neighbours
    float xv[4][4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int bb = 0; bb < 4; ++bb)
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) {
                const int core = (a == 1 || a == 2) + (bb == 1 || bb == 2) + (cc == 1 || cc == 2);
                xv[a][bb][cc] = core >= 2 ? __ldg(x + ia[a] + jb[bb] + kc[cc]) : 0.0f;
            }
    float sum = 0.0f;
#pragma unroll
    for (int a = 1; a < 3; ++a)
#pragma unroll
        for (int bb = 1; bb < 3; ++bb)
#pragma unroll
            for (int cc = 1; cc < 3; ++cc) {
                const float xc = xv[a][bb][cc];
                float ax = 0.0f;
                ax += xv[a - 1][bb][cc] * cf.c[0][0];
                ax += xc * cf.c[0][1];
                ax += xv[a + 1][bb][cc] * cf.c[0][2];
                ax += xv[a][bb - 1][cc] * cf.c[1][0];
                ax += xc * cf.c[1][1];
                ax += xv[a][bb + 1][cc] * cf.c[1][2];
                ax += xv[a][bb][cc - 1] * cf.c[2][0];
                ax += xc * cf.c[2][1];
                ax += xv[a][bb][cc + 1] * cf.c[2][2];
                sum += __ldg(b + ia[a] + jb[bb] + kc[cc]) - ax;
            }
    bc[idx(c, I, J, K)] = sum;
}

// x += P xc (trilinear, cell-centred)
__global__ void __launch_bounds__(256)
mg_prolong(Dims f, Dims c, const float* __restrict__ xc, float* __restrict__ x,
           const BicgScalars* sc) {
    if (sc->done) return;
    const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= f.nz || j >= f.ny) return;
    const int I = i >> 1, J = j >> 1, K = k >> 1;
    const int I2 = wrap(I + ((i & 1) ? 1 : -1), c.nx);
    const int J2 = wrap(J + ((j & 1) ? 1 : -1), c.ny);
    const int K2 = wrap(K + ((k & 1) ? 1 : -1), c.nz);
    const long long a0 = (long long)I * c.ny * c.nz, a1 = (long long)I2 * c.ny * c.nz;
    const long long b0 = (long long)J * c.nz, b1 = (long long)J2 * c.nz;
    const float v000 = __ldg(xc + a0 + b0 + K), v100 = __ldg(xc + a1 + b0 + K);
    const float v010 = __ldg(xc + a0 + b1 + K), v001 = __ldg(xc + a0 + b0 + K2);
    const float v110 = __ldg(xc + a1 + b1 + K), v101 = __ldg(xc + a1 + b0 + K2);
    const float v011 = __ldg(xc + a0 + b1 + K2), v111 = __ldg(xc + a1 + b1 + K2);
    const float e = (27.0f * v000 + 9.0f * (v100 + v010 + v001) +
                     3.0f * (v110 + v101 + v011) + v111) * (1.0f / 64.0f);
    const long long q = idx(f, i, j, k);
    x[q] = x[q] + e;
}

// Coarsest level: remove the mean of b, then Jacobi sweeps in shared memory.
constexpr int kCoarseThreads = 1024;
__global__ void __launch_bounds__(kCoarseThreads)
mg_coarse(Dims d, LapCoef<float> cf, float wd, const float* __restrict__ b,
          float* __restrict__ x, const BicgScalars* sc) {
    if (sc->done) return;
    extern __shared__ float smem[];
    __shared__ double shd[32];
    __shared__ float mean_s;
    const int n = (int)d.n;
    float* sb = smem;
    float* s0 = smem + n;
    float* s1 = s0 + n;
    const int tid = threadIdx.x;
    double acc = 0.0;
    for (int q = tid; q < n; q += blockDim.x) {
        const float v = b[q];
        sb[q] = v;
        acc += double(v);
    }
    const double tot = block_sum<kCoarseThreads>(acc, shd);
    if (tid == 0) mean_s = float(tot / double(n));
    __syncthreads();
    const float mean = mean_s;
    for (int q = tid; q < n; q += blockDim.x) {
        const float v = sb[q] - mean;
        sb[q] = v;
        s0[q] = wd * v;
    }
    __syncthreads();
    const int nyz = d.ny * d.nz;
    for (int it = 1; it < kMgCoarseSweeps; ++it) {
        for (int q = tid; q < n; q += blockDim.x) {
            const int i = q / nyz, r = q - i * nyz, j = r / d.nz, k = r - j * d.nz;
            const int im = wrap(i - 1, d.nx) * nyz, ip = wrap(i + 1, d.nx) * nyz;
            const int jm = wrap(j - 1, d.ny) * d.nz, jp = wrap(j + 1, d.ny) * d.nz;
            const int km = wrap(k - 1, d.nz), kp = wrap(k + 1, d.nz);
            const int ic = i * nyz, jc = j * d.nz;
            const float xc = s0[q];
            float ax = 0.0f;
            ax += s0[im + jc + k] * cf.c[0][0];
            ax += xc * cf.c[0][1];
            ax += s0[ip + jc + k] * cf.c[0][2];
            ax += s0[ic + jm + k] * cf.c[1][0];
            ax += xc * cf.c[1][1];
            ax += s0[ic + jp + k] * cf.c[1][2];
            ax += s0[ic + jc + km] * cf.c[2][0];
            ax += xc * cf.c[2][1];
            ax += s0[ic + jc + kp] * cf.c[2][2];
            s1[q] = fmaf(wd, sb[q] - ax, xc);
        }
        __syncthreads();
        float* tmp = s0; s0 = s1; s1 = tmp;
    }
    for (int q = tid; q < n; q += blockDim.x) x[q] = s0[q];
}

// v = A ph, gamma = (v, res0), alpha = rho / gamma
__global__ void __launch_bounds__(kBlock, 2)
mg_av(Dims d, Tiling tl, LapCoef<float> cf, BicgScalars* sc, double* part,
      const float* ph, const float* res0, float* v, int use_cond,
      cudaGraphConditionalHandle cond) {
    __shared__ double sh[32];
    if (sc->done) return;
    PhaseAv p{ph, res0, v, 0.0};
    sweep<float>(d, tl, cf, p);
    const double bs = block_sum<kBlock>(p.dot, sh);
    if (tid0()) part[blockIdx.x] = bs;
    if (arrive_last(sc)) {
        const double gamma = finish<false>(part, sh);
        if (tid0()) {
            sc->gamma = gamma;
            if (!(gamma == gamma) || isinf(gamma)) {
                sc->status = PF_NONFINITE; sc->done = 1;
            } else if (gamma == 0.0) {
                sc->status = PF_BREAKDOWN; sc->done = 1;
            } else {
                sc->alpha = sc->rho1 / gamma;
            }
            if (sc->done && use_cond) cudaGraphSetConditional(cond, 0);
            sc->counter = 0u;
        }
    }
}

// t = A sh, omega = (t, s) / (t, t)
__global__ void __launch_bounds__(kBlock, 2)
mg_at(Dims d, Tiling tl, LapCoef<float> cf, BicgScalars* sc, double* part,
      const float* shv, const float* s, float* t) {
    __shared__ double sh[32];
    if (sc->done) return;
    PhaseAt p{shv, s, t, 0.0, 0.0};
    sweep<float>(d, tl, cf, p);
    const double b0 = block_sum<kBlock>(p.ts, sh);
    const double b1 = block_sum<kBlock>(p.tt, sh);
    if (tid0()) { part[blockIdx.x] = b0; part[kMaxPartials + blockIdx.x] = b1; }
    if (arrive_last(sc)) {
        const double ts = finish<false>(part, sh);
        const double tt = finish<false>(part + kMaxPartials, sh);
        if (tid0()) {
            sc->buf1 = ts; sc->buf2 = tt;
            // (t,t) = 0 means s = 0: e += alpha ph finishes the solve
            sc->omega = tt > 0.0 ? ts / tt : 0.0;
            sc->counter = 0u;
        }
    }
}

// e += alpha ph + omega sh; res = s - omega t; rho' = (res, res0); stop test
__global__ void __launch_bounds__(kBlock)
mg_update(Dims d, BicgScalars* sc, double* part, float* e, const float* ph,
          const float* shv, const float* s, const float* t, float* res,
          const float* res0, int use_cond, cudaGraphConditionalHandle cond) {
    __shared__ double sh[32];
    if (sc->done) {
        if (use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(cond, 0);
        return;
    }
    const float alpha = float(sc->alpha), omega = float(sc->omega);
    double dot = 0.0, mx = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < d.n;
         q += (long long)gridDim.x * blockDim.x) {
        float x = fmaf(alpha, ph[q], e[q]);
        e[q] = fmaf(omega, shv[q], x);
        const float r = fmaf(-omega, t[q], s[q]);
        res[q] = r;
        dot += double(r) * double(res0[q]);
        mx = nanmax(mx, fabs(double(r)));
    }
    const double bs = block_sum<kBlock>(dot, sh);
    const double bm = block_max<kBlock>(mx, sh);
    if (threadIdx.x == 0) { part[blockIdx.x] = bs; part[kMaxPartials + blockIdx.x] = bm; }
    if (arrive_last(sc)) {
        const double rho = finish<false>(part, sh);
        const double mr = finish<true>(part + kMaxPartials, sh) / sc->max_res0;
        if (threadIdx.x == 0) {
            const int it = sc->iter + 1;
            sc->iter = it;
            sc->max_res = mr;
            sc->rho2 = sc->rho1;
            sc->rho1 = rho;
            bool stop = true;
            if (!(mr == mr) || isinf(mr)) sc->status = PF_NONFINITE;
            else if (mr <= sc->min_res || sc->buf2 == 0.0) sc->status = PF_OK;
            else if (it >= sc->max_it) sc->status = PF_MAXIT;
            else if (rho == 0.0 || sc->omega == 0.0) sc->status = PF_BREAKDOWN;
            else stop = false;
            if (stop) {
                sc->done = 1;
                if (use_cond) cudaGraphSetConditional(cond, 0);
            }
            sc->counter = 0u;
        }
    }
}

// res = res0 = float(r / scale); e = p = v = 0; rho = (res, res0)
__global__ void __launch_bounds__(kBlock)
mg_init(Dims d, BicgScalars* sc, double* part, const double* __restrict__ r,
        float* res, float* res0, float* e, float* p0, float* p1, float* v,
        int max_it, double tol) {
    __shared__ double sh[32];
    const double inv = sc->scale > 0.0 ? 1.0 / sc->scale : 0.0;
    double s = 0.0, m = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < d.n;
         q += (long long)gridDim.x * blockDim.x) {
        const float x = float(r[q] * inv);
        res[q] = x; res0[q] = x;
        e[q] = 0.0f; p0[q] = 0.0f; p1[q] = 0.0f; v[q] = 0.0f;
        s += double(x) * double(x);
        m = nanmax(m, fabs(double(x)));
    }
    const double bs = block_sum<kBlock>(s, sh);
    const double bm = block_max<kBlock>(m, sh);
    if (threadIdx.x == 0) { part[blockIdx.x] = bs; part[kMaxPartials + blockIdx.x] = bm; }
    if (arrive_last(sc)) {
        const double tot = finish<false>(part, sh);
        const double mx = finish<true>(part + kMaxPartials, sh);
        if (threadIdx.x == 0) {
            sc->rho1 = tot; sc->rho2 = 1.0; sc->alpha = 0.0; sc->omega = 1.0;
            sc->buf1 = 0.0; sc->buf2 = 1.0;
            sc->max_res0 = mx; sc->max_res = 1.0; sc->iter = 0; sc->k = 0;
            sc->max_it = max_it; sc->min_res = tol; sc->status = PF_OK;
            sc->done = (mx > 0.0 && mx == mx && !isinf(mx)) ? 0 : 1;
            if (!(mx == mx) || isinf(mx)) sc->status = PF_NONFINITE;
            sc->counter = 0u;
        }
    }
}

// ------------------------------------------------------------------- host
int mg_levels(const pf_grid* g, MgLevel* lv) {
    pf_grid cur = *g;
    int L = 0;
    for (;;) {
        MgLevel& l = lv[L];
        l.d = Dims{cur.nx, cur.ny, cur.nz, (long long)cur.nx * cur.ny * cur.nz};
        l.cf = lap_coef<float>(&cur);
        const LapCoef<double> c64 = lap_coef<double>(&cur);
        const double diag = c64.c[0][1] + c64.c[1][1] + c64.c[2][1];
        l.wd = float(double(kMgOmega) / diag);
        l.b = l.x = l.t = nullptr;
        l.tl = make_tiling(l.d, 32);
        ++L;
        if (l.d.n <= kMgCoarseTarget || L == kMgMaxLevels) break;
        if ((cur.nx | cur.ny | cur.nz) & 1) break;
        if (cur.nx < 4 || cur.ny < 4 || cur.nz < 4) break;
        cur.nx /= 2; cur.ny /= 2; cur.nz /= 2;
        cur.dx *= 2.0; cur.dy *= 2.0; cur.dz *= 2.0;
    }
    if (L < 2 || lv[L - 1].d.n > kMgCoarseMax) return 0;
    return L;
}

static constexpr int kMgFineVecs = 11;  // res res0 p0 p1 v s t ph sh e tmp

size_t mg_region_bytes(const pf_grid* g) {
    MgLevel lv[kMgMaxLevels];
    const int L = mg_levels(g, lv);
    if (!L) return 0;
    size_t b = kMgFineVecs * align256(lv[0].d.n * sizeof(float));
    for (int l = 1; l < L; ++l) b += 3 * align256(lv[l].d.n * sizeof(float));
    return b;
}

int mg_setup(const pf_grid* g, void* region, MgPlan* P) {
    P->L = mg_levels(g, P->lv);
    if (!P->L) return PF_ERR_BAD_ARG;
    static int dev_done[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !dev_done[dev]) {
        // the coarsest level may need up to 48 KiB of dynamic shared memory
        if (cudaFuncSetAttribute(mg_coarse, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(3 * kMgCoarseMax * sizeof(float))) != cudaSuccess)
            return PF_ERR_CUDA;
        dev_done[dev] = 1;
    }
    char* ptr = (char*)region;
    const size_t fb = align256(P->lv[0].d.n * sizeof(float));
    float** f[kMgFineVecs] = {&P->res, &P->res0, &P->p[0], &P->p[1], &P->v, &P->s,
                              &P->t, &P->ph, &P->sh, &P->e, &P->lv[0].t};
    for (auto q : f) { *q = (float*)ptr; ptr += fb; }
    for (int l = 1; l < P->L; ++l) {
        const size_t lb = align256(P->lv[l].d.n * sizeof(float));
        P->lv[l].b = (float*)ptr; ptr += lb;
        P->lv[l].x = (float*)ptr; ptr += lb;
        P->lv[l].t = (float*)ptr; ptr += lb;
    }
    return PF_OK;
}

static dim3 cgrid3(const Dims& d) { return dim3((d.nz + 31) / 32, (d.ny + 7) / 8, d.nx); }

// Restriction from level 0 (whose x and b are set), the coarse levels, and
// the up-sweep back to level 0's x.
static void vcycle_tail(const MgPlan& P, const float* b0, float* x0, BicgScalars* sc,
                        cudaStream_t s) {
    const dim3 blk(32, 8);
    const int L = P.L;
    for (int l = 0; l + 1 < L; ++l) {
        const MgLevel& f = P.lv[l];
        const MgLevel& c = P.lv[l + 1];
        const float* bl = l == 0 ? b0 : f.b;
        float* xl = l == 0 ? x0 : f.x;
        if (l > 0) {
            PhaseSmooth0<SrcPlain> ph{};
            ph.src.b = f.b; ph.x = f.x; ph.wd = f.wd;
            PF_LAUNCH("mg_smooth0", s, mg_smooth0<SrcPlain><<<tiled_grid(f.tl), blk, 0, s>>>(
                f.d, f.tl, f.cf, sc, ph));
        }
        PF_LAUNCH(l == 0 ? "mg_restrict_l0" : "mg_restrict", s, mg_restrict<<<cgrid3(c.d), blk, 0, s>>>(
            f.d, f.cf, bl, xl, c.d, c.b, sc));
    }
    {
        const MgLevel& c = P.lv[L - 1];
        const size_t smem = 3 * (size_t)c.d.n * sizeof(float);
        PF_LAUNCH("mg_coarse", s, mg_coarse<<<1, kCoarseThreads, smem, s>>>(
            c.d, c.cf, c.wd, c.b, c.x, sc));
    }
    for (int l = L - 2; l >= 0; --l) {
        const MgLevel& f = P.lv[l];
        const MgLevel& c = P.lv[l + 1];
        const float* bl = l == 0 ? b0 : f.b;
        float* xl = l == 0 ? x0 : f.x;
        const char* np = l == 0 ? "mg_prolong_l0" : "mg_prolong";
        const char* ns = l == 0 ? "mg_smooth_l0" : "mg_smooth";
        PF_LAUNCH(np, s, mg_prolong<<<cgrid3(f.d), blk, 0, s>>>(f.d, c.d, c.x, xl, sc));
        PhaseSmooth a{xl, bl, f.t, f.wd};
        PF_LAUNCH(ns, s, mg_smooth<<<tiled_grid(f.tl), blk, 0, s>>>(f.d, f.tl, f.cf, sc, a));
        PhaseSmooth b{f.t, bl, xl, f.wd};
        PF_LAUNCH(ns, s, mg_smooth<<<tiled_grid(f.tl), blk, 0, s>>>(f.d, f.tl, f.cf, sc, b));
    }
}

int mg_enqueue_init(const MgPlan& P, BicgScalars* sc, double* part, const double* rhs,
                    double tol, int max_it, cudaStream_t s) {
    const Dims& d = P.lv[0].d;
    PF_LAUNCH("mg_init", s, mg_init<<<pointwise_grid(d.n), kBlock, 0, s>>>(
        d, sc, part, rhs, P.res, P.res0, P.e, P.p[0], P.p[1], P.v, max_it, tol));
    return cudaGetLastError() == cudaSuccess ? PF_OK : PF_ERR_CUDA;
}

int mg_enqueue_iteration(const MgPlan& P, BicgScalars* sc, double* part, int k,
                         cudaStream_t s, int use_cond, cudaGraphConditionalHandle cond) {
    const MgLevel& f = P.lv[0];
    const dim3 blk(32, 8);
    const int gt = tiled_grid(f.tl);
    float* p_new = P.p[k & 1];
    const float* p_old = P.p[(k & 1) ^ 1];
    {   // p update fused into the first smoothing pass of M p
        PhaseSmooth0<SrcP> ph{};
        ph.src.res = P.res; ph.src.p_old = p_old; ph.src.v = P.v; ph.src.p_new = p_new;
        ph.x = P.ph; ph.wd = f.wd;
        PF_LAUNCH("mg_smooth0_p", s, mg_smooth0<SrcP><<<gt, blk, 0, s>>>(f.d, f.tl, f.cf, sc, ph));
    }
    vcycle_tail(P, p_new, P.ph, sc, s);
    PF_LAUNCH("mg_av", s, mg_av<<<gt, blk, 0, s>>>(f.d, f.tl, f.cf, sc, part, P.ph, P.res0,
                                                   P.v, use_cond, cond));
    {   // s = res - alpha v fused into the first smoothing pass of M s
        PhaseSmooth0<SrcS> ph{};
        ph.src.res = P.res; ph.src.v = P.v; ph.src.s = P.s;
        ph.x = P.sh; ph.wd = f.wd;
        PF_LAUNCH("mg_smooth0_s", s, mg_smooth0<SrcS><<<gt, blk, 0, s>>>(f.d, f.tl, f.cf, sc, ph));
    }
    vcycle_tail(P, P.s, P.sh, sc, s);
    PF_LAUNCH("mg_at", s, mg_at<<<gt, blk, 0, s>>>(f.d, f.tl, f.cf, sc, part, P.sh, P.s, P.t));
    PF_LAUNCH("mg_update", s, mg_update<<<pointwise_grid(f.d.n), kBlock, 0, s>>>(
        f.d, sc, part, P.e, P.ph, P.sh, P.s, P.t, P.res, P.res0, use_cond, cond));
    return cudaGetLastError() == cudaSuccess ? PF_OK : PF_ERR_CUDA;
}

int mg_inner_solve(const MgPlan& P, BicgScalars* sc, double* part, const double* rhs,
                   double tol, int max_it, cudaStream_t s, BicgScalars* hs) {
    int rc = mg_enqueue_init(P, sc, part, rhs, tol, std::max(1, max_it), s);
    if (rc) return rc;
    int k = 0, chunk = 2;
    for (int guard = 0; guard < (1 << 20); ++guard) {
        for (int c = 0; c < chunk; ++c, ++k) {
            rc = mg_enqueue_iteration(P, sc, part, k, s);
            if (rc) return rc;
        }
        if (cudaMemcpyAsync(hs, sc, sizeof(BicgScalars), cudaMemcpyDeviceToHost, s) != cudaSuccess)
            return PF_ERR_CUDA;
        if (cudaStreamSynchronize(s) != cudaSuccess) return PF_ERR_CUDA;
        if (hs->done) return PF_OK;
        chunk = std::min(chunk * 2, 8);
    }
    return PF_ERR_CUDA;
}

}  // namespace pf
