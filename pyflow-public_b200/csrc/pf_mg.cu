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
//   * levels halve every dimension while all are even, down to <= 64 cells;
//     level l uses the same 7-point operator with spacing 2^l h (the coarse
//     right-hand side is the SUM of the 8 fine residuals, because A carries
//     the cell volume);
//   * smoother: weighted Jacobi, omega = 6/7 (the optimal damping of the 3-D
//     7-point Laplacian); the two pre-smoothing sweeps start from zero and are
//     evaluated in one pass as x = w (2 b - w A b), w = omega / diag(A);
//   * restriction: sum of the 8 children's residuals b - A x, computed from x
//     in the same kernel; prolongation: trilinear (weights 27, 9, 3, 1 / 64);
//   * coarsest level (<= 64 cells when the grid halves that far): solved
//     exactly with the pseudo-inverse of its periodic operator (from the
//     Fourier eigenvalues; the operator is singular), else mean removal and
//     Jacobi sweeps.
// M is a fixed linear operator (fixed sweep counts), as BiCGStab requires.
// At the finest level the p update and s = res - alpha v are fused into the
// first smoothing pass, which computes them for every cell it loads.
//
// Execution by level size: large levels (the finest always) use the tiled
// sweep of pf_sweep.cuh (prolongation: one thread per coarse cell updating its
// 8 children); mid-size levels one thread per cell (a sweep's plane-by-plane
// march is latency-bound on small grids) with the prolongation fused into the
// first post-smoothing pass; every level of at most 512 cells (and the
// coarsest level, at most 4096 cells) runs inside ONE CTA in shared memory
// (mg_bottom), so the bottom of the V-cycle is a single launch.
//
// All vectors are FP32; every dot product and max accumulates in FP64 and is
// finished by the last block (fixed order).  Scalars stay on the device.
#include <cmath>
#include <cstdlib>

#include <cooperative_groups.h>

#include "pf_common.cuh"
#include "pf_kernels.cuh"
#include "pf_mg.cuh"
#include "pf_profile.cuh"

namespace pf {

constexpr float kMgOmega = 6.0f / 7.0f;
constexpr int kMgCoarseSweeps = 32;

// ------------------------------------------------------------ sweep phases
// Sources of the first (from-zero) smoothing pass.
struct SrcPlain {  // b of a coarse level
    static constexpr int kRows = 8;
    const float* b;
    struct Raw { float b; };
    __device__ void setup(const BicgScalars*) {}
    __device__ Raw raw(long long q, int = 0, int = 0, int = 0) const { return Raw{b[q]}; }
    __device__ float op(const Raw& a) const { return a.b; }
    __device__ void store(long long, float) const {}
};

struct SrcP {  // p' = res + beta (p - omega v), stored to p_new
    static constexpr int kRows = 4;
    const float *res, *p_old, *v;
    float* p_new;
    float beta, omega;
    struct Raw { float r, p, v; };
    __device__ void setup(const BicgScalars* sc) {
        beta = float((sc->rho1 / sc->rho2) * (sc->alpha / sc->omega));
        omega = float(sc->omega);
    }
    __device__ Raw raw(long long q, int = 0, int = 0, int = 0) const { return Raw{res[q], p_old[q], v[q]}; }
    __device__ float op(const Raw& a) const {
        return fmaf(beta, fmaf(-omega, a.v, a.p), a.r);
    }
    __device__ void store(long long q, float c) const { p_new[q] = c; }
};

// The p update of the first iteration of a pass (beta == 0): the same
// expression with p = v = 0, which are not read (they hold nothing yet).
struct SrcP0 {
    static constexpr int kRows = 4;
    const float* res;
    float* p_new;
    float beta, omega;
    struct Raw { float r; };
    __device__ Raw raw(long long q, int = 0, int = 0, int = 0) const { return Raw{res[q]}; }
    __device__ float op(const Raw& a) const { return fmaf(beta, fmaf(-omega, 0.0f, 0.0f), a.r); }
    __device__ void store(long long q, float c) const { p_new[q] = c; }
};

struct SrcS {  // s = res - alpha v, stored to s
    static constexpr int kRows = 4;
    const float *res, *v;
    float* s;
    float alpha;
    struct Raw { float r, v; };
    __device__ void setup(const BicgScalars* sc) { alpha = float(sc->alpha); }
    __device__ Raw raw(long long q, int = 0, int = 0, int = 0) const { return Raw{res[q], v[q]}; }
    __device__ float op(const Raw& a) const { return fmaf(-alpha, a.v, a.r); }
    __device__ void store(long long q, float c) const { s[q] = c; }
};

// x = w (2 b - w A b): two weighted-Jacobi sweeps from x = 0
template <class Src>
struct PhaseSmooth0 {
    static constexpr int R = Src::kRows;
    Src src;
    float* x;
    float wd;
    using Raw = typename Src::Raw;
    struct Ext {};
    __device__ Raw raw(long long q, int = 0, int = 0, int = 0) const { return src.raw(q); }
    __device__ Ext ext(long long) const { return Ext{}; }
    __device__ float op(const Raw& a) const { return src.op(a); }
    __device__ void epi(long long q, float c, float ab, const Raw&, const Ext&) {
        src.store(q, c);
        x[q] = wd * (2.0f * c - wd * ab);
    }
};

// out = x + w (b - A x): one weighted-Jacobi sweep
struct PhaseSmooth {
    static constexpr int R = 8;  // one field in: 8 rows per thread keep more loads in flight
    const float *x, *b;
    float* out;
    float wd;
    struct Raw { float x; };
    struct Ext { float b; };
    __device__ Raw raw(long long q, int = 0, int = 0, int = 0) const { return Raw{x[q]}; }
    __device__ Ext ext(long long q) const { return Ext{b[q]}; }
    __device__ float op(const Raw& a) const { return a.x; }
    __device__ void epi(long long q, float c, float ax, const Raw&, const Ext& e) {
        out[q] = fmaf(wd, e.b - ax, c);
    }
};

// v = A ph and (v, res0)
struct PhaseAv {
    static constexpr int R = 8;  // one field in: 8 rows per thread keep more loads in flight
    const float *ph, *res0;
    float* v;
    double dot;
    struct Raw { float x; };
    struct Ext { float r0; };
    __device__ Raw raw(long long q, int = 0, int = 0, int = 0) const { return Raw{ph[q]}; }
    __device__ Ext ext(long long q) const { return Ext{res0[q]}; }
    __device__ float op(const Raw& a) const { return a.x; }
    __device__ void epi(long long q, float, float ax, const Raw&, const Ext& e) {
        v[q] = ax;
        dot += double(ax) * double(e.r0);
    }
};

// t = A sh, (t, s) and (t, t)
struct PhaseAt {
    static constexpr int R = 8;  // one field in: 8 rows per thread keep more loads in flight
    const float *sh, *s;
    float* t;
    double ts, tt;
    struct Raw { float x; };
    struct Ext { float s; };
    __device__ Raw raw(long long q, int = 0, int = 0, int = 0) const { return Raw{sh[q]}; }
    __device__ Ext ext(long long q) const { return Ext{s[q]}; }
    __device__ float op(const Raw& a) const { return a.x; }
    __device__ void epi(long long q, float, float ax, const Raw&, const Ext& e) {
        t[q] = ax;
        ts += double(ax) * double(e.s);
        tt += double(ax) * double(ax);
    }
};

// The same phases for sweep_async (FP32 grids with nz a multiple of 32).
// Sources of the first smoothing pass, from their raw input fields:
struct AsyncPlain {  // b of a coarse level
    static constexpr int NR = 1;
    __device__ void setup(const BicgScalars*) {}
    __device__ float op(const float* r) const { return r[0]; }
    __device__ void store(long long, float) const {}
};

struct AsyncS {  // s = res - alpha v from (res, v), stored to s
    static constexpr int NR = 2;
    float* s;
    float alpha;
    __device__ void setup(const BicgScalars* sc) { alpha = float(sc->alpha); }
    __device__ float op(const float* r) const { return fmaf(-alpha, r[1], r[0]); }
    __device__ void store(long long q, float c) const { s[q] = c; }
};

template <class S>
struct AsyncSmooth0 {  // x = w (2 b - w A b), b = the source's operand
    static constexpr int NR = S::NR, NE = 0;
    S src;
    const float* rf[NR];
    const float* ef[1];
    float* x;
    float wd;
    __device__ float op(const float* r) const { return src.op(r); }
    __device__ void epi(long long q, float c, float ab, const float*) {
        src.store(q, c);
        x[q] = wd * (2.0f * c - wd * ab);
    }
};

struct AsyncSmooth {  // out = x + w (b - A x)
    static constexpr int NR = 1, NE = 1;
    const float* rf[1];
    const float* ef[1];
    float* out;
    float wd;
    __device__ float op(const float* r) const { return r[0]; }
    __device__ void epi(long long q, float c, float ax, const float* e) {
        out[q] = fmaf(wd, e[0] - ax, c);
    }
};

struct AsyncAv {  // v = A ph, (v, res0)
    static constexpr int NR = 1, NE = 1;
    const float* rf[1];
    const float* ef[1];
    float* v;
    double dot;
    __device__ float op(const float* r) const { return r[0]; }
    __device__ void epi(long long q, float, float ax, const float* e) {
        v[q] = ax;
        dot += double(ax) * double(e[0]);
    }
};

struct AsyncAt {  // t = A sh, (t, s), (t, t)
    static constexpr int NR = 1, NE = 1;
    const float* rf[1];
    const float* ef[1];
    float* t;
    double ts, tt;
    __device__ float op(const float* r) const { return r[0]; }
    __device__ void epi(long long q, float, float ax, const float* e) {
        t[q] = ax;
        ts += double(ax) * double(e[0]);
        tt += double(ax) * double(ax);
    }
};

// Tile heights of the cp.async sweeps: 32 rows for one input field, 16 for
// the two-field first pass of M s (its plane ring stays small enough for two
// blocks per SM).
constexpr int kAsTY1 = 32, kAsTYn = 16;

// ------------------------------------------------------------------ kernels
template <class Src>
__global__ void __launch_bounds__(kBlock, 2)
mg_smooth0(Dims d, Tiling tl, LapCoef<float> cf, const BicgScalars* sc,
           PhaseSmooth0<Src> ph) {
    pdl_wait();
    if (sc->done) return;
    ph.src.setup(sc);
    sweep<float>(d, tl, cf, ph);
}

// The p update and first smoothing pass of M p; the first iteration of a
// pass (beta == 0) reads neither p nor v.
__global__ void __launch_bounds__(kBlock, 2)
mg_smooth0_p(Dims d, Tiling tl, LapCoef<float> cf, const BicgScalars* sc,
             PhaseSmooth0<SrcP> ph) {
    pdl_wait();
    if (sc->done) return;
    ph.src.setup(sc);
    if (ph.src.beta == 0.0f) {
        PhaseSmooth0<SrcP0> p0{};
        p0.src = SrcP0{ph.src.res, ph.src.p_new, ph.src.beta, ph.src.omega};
        p0.x = ph.x;
        p0.wd = ph.wd;
        sweep<float>(d, tl, cf, p0);
    } else {
        sweep<float>(d, tl, cf, ph);
    }
}

__global__ void __launch_bounds__(kBlock, 2)
mg_smooth(Dims d, Tiling tl, LapCoef<float> cf, const BicgScalars* sc, PhaseSmooth ph) {
    pdl_wait();
    if (sc->done) return;
    sweep<float>(d, tl, cf, ph);
}

template <int TY, int TZ, class S>
__global__ void __launch_bounds__(kBlock, 2)
mg_smooth0_as(Dims d, Tiling tl, LapCoef<float> cf, const BicgScalars* sc, AsyncSmooth0<S> ph) {
    pdl_wait();
    if (sc->done) return;
    ph.src.setup(sc);
    sweep_async<TY, TZ>(d, tl, cf, ph);
}

template <int TZ>
__global__ void __launch_bounds__(kBlock, 2)
mg_smooth_as(Dims d, Tiling tl, LapCoef<float> cf, const BicgScalars* sc, AsyncSmooth ph) {
    pdl_wait();
    if (sc->done) return;
    sweep_async<kAsTY1, TZ>(d, tl, cf, ph);
}

// bc[I,J,K] = sum over the 8 children of (b - A x) on the fine level.  One
// thread per coarse (J, K) and TWO coarse planes I0, I0 + 1 (fine x planes
// 2 I0 - 1 .. 2 I0 + 4 loaded once); each fine row pair 2K, 2K + 1 is one
// 8-byte load, and the z halos 2K - 1, 2K + 2 come from the neighbouring
// lanes (loaded only at the warp's edges and the grid's periodic wrap).
// Lanes past c.nz compute on a clamped K (so every lane takes part in the
// shuffles) and store nothing.  A x in fused multiply-adds with one centre
// coefficient, as the cp.async sweeps.  Needs fine dims = 2 x coarse dims.
__global__ void __launch_bounds__(256)
mg_restrict(Dims f, LapCoef<float> cf, const float* __restrict__ b,
            const float* __restrict__ x, Dims c, float* __restrict__ bc,
            const BicgScalars* sc) {
    pdl_wait();
    if (sc->done) return;
    const int K = blockIdx.x * 32 + threadIdx.x, J = blockIdx.y * 8 + threadIdx.y;
    const int I0 = blockIdx.z * 2;
    if (J >= c.ny) return;  // uniform across the warp (threadIdx.y is)
    const bool ok = K < c.nz;
    const int Kc = ok ? K : c.nz - 1;
    const bool ledge = threadIdx.x == 0, redge = threadIdx.x == 31 || Kc + 1 >= c.nz;
    long long ia[6], jb[4];
#pragma unroll
    for (int a = 0; a < 6; ++a) ia[a] = (long long)pmod(2 * I0 - 1 + a, f.nx) * f.ny * f.nz;
#pragma unroll
    for (int a = 0; a < 4; ++a) jb[a] = (long long)wrap(2 * J - 1 + a, f.ny) * f.nz;
    const int kl = wrap(2 * Kc - 1, f.nz), kr = wrap(2 * Kc + 2, f.nz);
    const float cen = (cf.c[0][1] + cf.c[1][1]) + cf.c[2][1];
    // x pairs (2K, 2K+1) of fine rows (a, bb); the four corner rows are unused
    float2 xp[6][4];
#pragma unroll
    for (int a = 0; a < 6; ++a)
#pragma unroll
        for (int bb = 0; bb < 4; ++bb) {
            const bool need = (a >= 1 && a <= 4) || bb == 1 || bb == 2;
            xp[a][bb] = need ? __ldg(reinterpret_cast<const float2*>(x + ia[a] + jb[bb] + 2 * Kc))
                             : make_float2(0.0f, 0.0f);
        }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        float sum = 0.0f;
#pragma unroll
        for (int a = 1 + 2 * h; a < 3 + 2 * h; ++a)
#pragma unroll
            for (int bb = 1; bb < 3; ++bb) {
                float zl = __shfl_up_sync(0xffffffffu, xp[a][bb].y, 1);
                float zr = __shfl_down_sync(0xffffffffu, xp[a][bb].x, 1);
                if (ledge) zl = __ldg(x + ia[a] + jb[bb] + kl);
                if (redge) zr = __ldg(x + ia[a] + jb[bb] + kr);
                const float2 bv = __ldg(reinterpret_cast<const float2*>(b + ia[a] + jb[bb] + 2 * Kc));
                const float z[4] = {zl, xp[a][bb].x, xp[a][bb].y, zr};
#pragma unroll
                for (int cc = 1; cc < 3; ++cc) {
                    auto at = [&](int aa, int b2) { return cc == 1 ? xp[aa][b2].x : xp[aa][b2].y; };
                    float ax = z[cc] * cen;
                    ax = fmaf(at(a - 1, bb), cf.c[0][0], ax);
                    ax = fmaf(at(a + 1, bb), cf.c[0][2], ax);
                    ax = fmaf(at(a, bb - 1), cf.c[1][0], ax);
                    ax = fmaf(at(a, bb + 1), cf.c[1][2], ax);
                    ax = fmaf(z[cc - 1], cf.c[2][0], ax);
                    ax = fmaf(z[cc + 1], cf.c[2][2], ax);
                    sum += (cc == 1 ? bv.x : bv.y) - ax;
                }
            }
        if (ok && I0 + h < c.nx) bc[idx(c, I0 + h, J, K)] = sum;
    }
}

// ------------------------------------------------- one thread per cell
__device__ __forceinline__ float lap7(const float* __restrict__ x, const Dims& d,
                                      const LapCoef<float>& cf, int i, int j, int k,
                                      float xc) {
    const long long P = (long long)d.ny * d.nz;
    const long long ci = (long long)i * P, cj = (long long)j * d.nz;
    float ax = 0.0f;
    ax += __ldg(x + (long long)wrap(i - 1, d.nx) * P + cj + k) * cf.c[0][0];
    ax += xc * cf.c[0][1];
    ax += __ldg(x + (long long)wrap(i + 1, d.nx) * P + cj + k) * cf.c[0][2];
    ax += __ldg(x + ci + (long long)wrap(j - 1, d.ny) * d.nz + k) * cf.c[1][0];
    ax += xc * cf.c[1][1];
    ax += __ldg(x + ci + (long long)wrap(j + 1, d.ny) * d.nz + k) * cf.c[1][2];
    ax += __ldg(x + ci + cj + wrap(k - 1, d.nz)) * cf.c[2][0];
    ax += xc * cf.c[2][1];
    ax += __ldg(x + ci + cj + wrap(k + 1, d.nz)) * cf.c[2][2];
    return ax;
}

// trilinear prolongation of the coarse level to fine cell (i, j, k)
__device__ __forceinline__ float prolong_at(const float* __restrict__ xc, const Dims& c,
                                            int i, int j, int k) {
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
    return (27.0f * v000 + 9.0f * (v100 + v010 + v001) + 3.0f * (v110 + v101 + v011) + v111) *
           (1.0f / 64.0f);
}

#define PF_CELL_IDX(d)                                                       \
    const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y; \
    const int i = blockIdx.z;                                                \
    if (k >= (d).nz || j >= (d).ny) return;                                  \
    const long long q = idx((d), i, j, k)

// x = w (2 b - w A b)
__global__ void __launch_bounds__(256)
mg_smooth0_pw(Dims d, LapCoef<float> cf, float wd, const float* __restrict__ b,
              float* __restrict__ x, const BicgScalars* sc) {
    pdl_wait();
    if (sc->done) return;
    PF_CELL_IDX(d);
    const float bc = b[q];
    x[q] = wd * (2.0f * bc - wd * lap7(b, d, cf, i, j, k, bc));
}

// out = x + w (b - A x)
__global__ void __launch_bounds__(256)
mg_smooth_pw(Dims d, LapCoef<float> cf, float wd, const float* __restrict__ x,
             const float* __restrict__ b, float* __restrict__ out, const BicgScalars* sc) {
    pdl_wait();
    if (sc->done) return;
    PF_CELL_IDX(d);
    const float xc = x[q];
    out[q] = fmaf(wd, b[q] - lap7(x, d, cf, i, j, k, xc), xc);
}

// y = x + P xc at the cell and its six neighbours; out = y + w (b - A y)
__global__ void __launch_bounds__(256)
mg_prolong_smooth_pw(Dims d, Dims c, LapCoef<float> cf, float wd,
                     const float* __restrict__ xc, const float* __restrict__ x,
                     const float* __restrict__ b, float* __restrict__ out,
                     const BicgScalars* sc) {
    pdl_wait();
    if (sc->done) return;
    PF_CELL_IDX(d);
    auto y = [&](int a, int bb, int cc) {
        return __ldg(x + idx(d, a, bb, cc)) + prolong_at(xc, c, a, bb, cc);
    };
    const int im = wrap(i - 1, d.nx), ip = wrap(i + 1, d.nx);
    const int jm = wrap(j - 1, d.ny), jp = wrap(j + 1, d.ny);
    const int km = wrap(k - 1, d.nz), kp = wrap(k + 1, d.nz);
    const float yc = y(i, j, k);
    float ax = 0.0f;
    ax += y(im, j, k) * cf.c[0][0];
    ax += yc * cf.c[0][1];
    ax += y(ip, j, k) * cf.c[0][2];
    ax += y(i, jm, k) * cf.c[1][0];
    ax += yc * cf.c[1][1];
    ax += y(i, jp, k) * cf.c[1][2];
    ax += y(i, j, km) * cf.c[2][0];
    ax += yc * cf.c[2][1];
    ax += y(i, j, kp) * cf.c[2][2];
    out[q] = fmaf(wd, b[q] - ax, yc);
}

// Swept levels: x += P xc with one thread per coarse cell, which loads its
// 3x3x3 coarse neighbourhood once and updates its 8 children (z pairs as one
// 8-byte access).  Needs even fine dimensions (always true below the top).
__global__ void __launch_bounds__(256)
mg_prolong_add(Dims f, Dims c, const float* __restrict__ xc, float* __restrict__ x,
               const BicgScalars* sc) {
    pdl_wait();
    if (sc->done) return;
    const int K = blockIdx.x * 32 + threadIdx.x, J = blockIdx.y * 8 + threadIdx.y;
    const int I = blockIdx.z;
    if (K >= c.nz || J >= c.ny) return;
    float v[3][3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const long long pa = (long long)wrap(I + a - 1, c.nx) * c.ny * c.nz;
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const long long pb = pa + (long long)wrap(J + b - 1, c.ny) * c.nz;
#pragma unroll
            for (int e = 0; e < 3; ++e) v[a][b][e] = __ldg(xc + pb + wrap(K + e - 1, c.nz));
        }
    }
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            // child (2I+a, 2J+b, 2K+cc): far neighbours at offset -1 (child 0) or +1 (child 1)
            const int A2 = a ? 2 : 0, B2 = b ? 2 : 0;
            float e2[2];
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const int C2 = cc ? 2 : 0;
                e2[cc] = (27.0f * v[1][1][1] + 9.0f * (v[A2][1][1] + v[1][B2][1] + v[1][1][C2]) +
                          3.0f * (v[A2][B2][1] + v[A2][1][C2] + v[1][B2][C2]) + v[A2][B2][C2]) *
                         (1.0f / 64.0f);
            }
            const long long q = idx(f, 2 * I + a, 2 * J + b, 2 * K);
            float2 xv = *reinterpret_cast<const float2*>(x + q);
            xv.x = xv.x + e2[0];
            xv.y = xv.y + e2[1];
            *reinterpret_cast<float2*>(x + q) = xv;
        }
}

// The same with two coarse z cells per thread when the fine z extent is a
// multiple of 4: its four fine z cells are one 16-byte access per fine row,
// the coarse z pair one 8-byte load per coarse row (z neighbours from the
// adjacent lanes), so each thread moves 4 x 16 bytes of x in 8 accesses.
__global__ void __launch_bounds__(256)
mg_prolong_add4(Dims f, Dims c, const float* __restrict__ xc, float* __restrict__ x,
                const BicgScalars* sc) {
    pdl_wait();
    if (sc->done) return;
    const int Kp = blockIdx.x * 32 + threadIdx.x, J = blockIdx.y * 8 + threadIdx.y;
    const int I = blockIdx.z;
    if (J >= c.ny) return;  // uniform across the warp
    const int np = c.nz >> 1;
    const bool ok = Kp < np;
    const int Kc = ok ? Kp : np - 1;  // lanes past the row compute on a clamped pair
    const bool ledge = threadIdx.x == 0, redge = threadIdx.x == 31 || Kc + 1 >= np;
    const int km = wrap(2 * Kc - 1, c.nz), kp = wrap(2 * Kc + 2, c.nz);
    float v[3][3][4];  // coarse planes I-1..I+1, rows J-1..J+1, z 2Kc-1 .. 2Kc+2
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const long long pa = (long long)wrap(I + a - 1, c.nx) * c.ny * c.nz;
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const long long pb = pa + (long long)wrap(J + b - 1, c.ny) * c.nz;
            const float2 m = __ldg(reinterpret_cast<const float2*>(xc + pb + 2 * Kc));
            float l = __shfl_up_sync(0xffffffffu, m.y, 1);
            float r = __shfl_down_sync(0xffffffffu, m.x, 1);
            if (ledge) l = __ldg(xc + pb + km);
            if (redge) r = __ldg(xc + pb + kp);
            v[a][b][0] = l;
            v[a][b][1] = m.x;
            v[a][b][2] = m.y;
            v[a][b][3] = r;
        }
    }
    if (!ok) return;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            // fine z 4Kc + m: K at index 1 + (m >> 1), far neighbour K -+ 1
            const int A2 = a ? 2 : 0, B2 = b ? 2 : 0;
            auto e = [&](int kk, int k2) {
                return (27.0f * v[1][1][kk] + 9.0f * (v[A2][1][kk] + v[1][B2][kk] + v[1][1][k2]) +
                        3.0f * (v[A2][B2][kk] + v[A2][1][k2] + v[1][B2][k2]) + v[A2][B2][k2]) *
                       (1.0f / 64.0f);
            };
            const long long q = idx(f, 2 * I + a, 2 * J + b, 4 * Kc);
            float4 xv = *reinterpret_cast<const float4*>(x + q);
            xv.x = xv.x + e(1, 0);
            xv.y = xv.y + e(1, 2);
            xv.z = xv.z + e(2, 1);
            xv.w = xv.w + e(2, 3);
            *reinterpret_cast<float4*>(x + q) = xv;
        }
}

// ------------------------------------------------- grid-wide mid levels
// The one-thread-per-cell levels G .. C-1 together with the restriction from
// and the prolongation into the swept level G - 1 above them, as two
// cooperative launches per V-cycle (down: restriction into G, then for each
// level smoothing from zero and restriction; up: for each level the
// prolongation and the two post-smoothing sweeps, then the prolongation into
// level G - 1), the phases separated by grid barriers.  Every phase is the
// arithmetic of the per-level kernel it replaces (mg_restrict, mg_smooth0_pw,
// mg_prolong_smooth_pw + mg_smooth_pw, mg_prolong_add), so the V-cycle is
// bit-identical to the per-level launches.  Data written within the launch
// is read through L2 (ld.cg), not the incoherent L1.
struct MgMid {
    int g0, g1;                   // levels g0 .. g1 - 1 run here; g0 - 1 is swept
    Dims d[kMgMaxLevels];
    LapCoef<float> cf[kMgMaxLevels];
    float wd[kMgMaxLevels];
    float* b[kMgMaxLevels];
    float* x[kMgMaxLevels];
    float* t[kMgMaxLevels];
    const float* bs;              // level g0 - 1: right-hand side and working iterate
    float* xs;
};

__device__ __forceinline__ float ldcg(const float* p) { return __ldcg(p); }

// the grid's blocks meet; false (and gbar[2] set) if the wait gave up
__device__ bool grid_barrier(unsigned* gbar) {
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile unsigned* gen = gbar + 1;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(gbar, 1u) == gridDim.x - 1) {
            atomicExch(gbar, 0u);
            __threadfence();
            atomicAdd(gbar + 1, 1u);
        } else {
            long long it = 0;
            while (*gen == g) {
                if (++it > (1LL << 22) || ((volatile unsigned*)gbar)[2]) { ok = 0; break; }
                __nanosleep(32);
            }
        }
        __threadfence();
        if (!ok) atomicExch(gbar + 2, 1u);
        ok_s = ok;
    }
    __syncthreads();
    return ok_s != 0;
}

// A x at (i, j, k) in the order of lap7, loads through L2
__device__ __forceinline__ float lap7_cg(const float* x, const Dims& d, const LapCoef<float>& cf,
                                         int i, int j, int k, float xc) {
    const long long P = (long long)d.ny * d.nz;
    const long long ci = (long long)i * P, cj = (long long)j * d.nz;
    float ax = 0.0f;
    ax += ldcg(x + (long long)wrap(i - 1, d.nx) * P + cj + k) * cf.c[0][0];
    ax += xc * cf.c[0][1];
    ax += ldcg(x + (long long)wrap(i + 1, d.nx) * P + cj + k) * cf.c[0][2];
    ax += ldcg(x + ci + (long long)wrap(j - 1, d.ny) * d.nz + k) * cf.c[1][0];
    ax += xc * cf.c[1][1];
    ax += ldcg(x + ci + (long long)wrap(j + 1, d.ny) * d.nz + k) * cf.c[1][2];
    ax += ldcg(x + ci + cj + wrap(k - 1, d.nz)) * cf.c[2][0];
    ax += xc * cf.c[2][1];
    ax += ldcg(x + ci + cj + wrap(k + 1, d.nz)) * cf.c[2][2];
    return ax;
}

// the correction prolong_at adds at fine cell (i, j, k), loads through L2
__device__ __forceinline__ float prolong_cg(const float* xc, const Dims& c, int i, int j, int k) {
    const int I = i >> 1, J = j >> 1, K = k >> 1;
    const int I2 = wrap(I + ((i & 1) ? 1 : -1), c.nx);
    const int J2 = wrap(J + ((j & 1) ? 1 : -1), c.ny);
    const int K2 = wrap(K + ((k & 1) ? 1 : -1), c.nz);
    const long long a0 = (long long)I * c.ny * c.nz, a1 = (long long)I2 * c.ny * c.nz;
    const long long b0 = (long long)J * c.nz, b1 = (long long)J2 * c.nz;
    const float v000 = ldcg(xc + a0 + b0 + K), v100 = ldcg(xc + a1 + b0 + K);
    const float v010 = ldcg(xc + a0 + b1 + K), v001 = ldcg(xc + a0 + b0 + K2);
    const float v110 = ldcg(xc + a1 + b1 + K), v101 = ldcg(xc + a1 + b0 + K2);
    const float v011 = ldcg(xc + a0 + b1 + K2), v111 = ldcg(xc + a1 + b1 + K2);
    return (27.0f * v000 + 9.0f * (v100 + v010 + v001) + 3.0f * (v110 + v101 + v011) + v111) *
           (1.0f / 64.0f);
}

// bc[I, J, K] = sum over the 8 children of (b - A x), in mg_restrict's order
__device__ __forceinline__ float restrict_cg(const float* b, const float* x, const Dims& f,
                                             const LapCoef<float>& cf, int I, int J, int K) {
    const float cen = (cf.c[0][1] + cf.c[1][1]) + cf.c[2][1];
    const long long P = (long long)f.ny * f.nz;
    float sum = 0.0f;
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        const int i = 2 * I + a;
        const long long pi = (long long)i * P, pm = (long long)pmod(i - 1, f.nx) * P,
                        pp = (long long)pmod(i + 1, f.nx) * P;
#pragma unroll
        for (int bb = 0; bb < 2; ++bb) {
            const int j = 2 * J + bb;
            const long long rj = (long long)j * f.nz, rm = (long long)wrap(j - 1, f.ny) * f.nz,
                            rp = (long long)wrap(j + 1, f.ny) * f.nz;
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const int k = 2 * K + cc;
                float ax = ldcg(x + pi + rj + k) * cen;
                ax = fmaf(ldcg(x + pm + rj + k), cf.c[0][0], ax);
                ax = fmaf(ldcg(x + pp + rj + k), cf.c[0][2], ax);
                ax = fmaf(ldcg(x + pi + rm + k), cf.c[1][0], ax);
                ax = fmaf(ldcg(x + pi + rp + k), cf.c[1][2], ax);
                ax = fmaf(ldcg(x + pi + rj + wrap(k - 1, f.nz)), cf.c[2][0], ax);
                ax = fmaf(ldcg(x + pi + rj + wrap(k + 1, f.nz)), cf.c[2][2], ax);
                sum += ldcg(b + pi + rj + k) - ax;
            }
        }
    }
    return sum;
}

__device__ __forceinline__ void cell_of(long long q, const Dims& d, int& i, int& j, int& k) {
    k = (int)(q % d.nz);
    const long long r = q / d.nz;
    j = (int)(r % d.ny);
    i = (int)(r / d.ny);
}

#define PF_GRID_LOOP(q, n) \
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < (n); \
         q += (long long)gridDim.x * blockDim.x)

__global__ void __launch_bounds__(256)
mg_mid_down(MgMid M, const BicgScalars* sc, unsigned* gbar) {
    if (sc->done || gbar[2]) return;
    const int g0 = M.g0;
    {   // restriction from the swept level g0 - 1 into level g0's b
        const Dims f = M.d[g0 - 1], c = M.d[g0];
        PF_GRID_LOOP(Q, c.n) {
            int I, J, K;
            cell_of(Q, c, I, J, K);
            M.b[g0][Q] = restrict_cg(M.bs, M.xs, f, M.cf[g0 - 1], I, J, K);
        }
    }
    for (int l = g0; l < M.g1; ++l) {
        if (!grid_barrier(gbar)) return;
        const Dims d = M.d[l];
        const float wd = M.wd[l];
        PF_GRID_LOOP(q, d.n) {  // x = w (2 b - w A b)
            int i, j, k;
            cell_of(q, d, i, j, k);
            const float bc = ldcg(M.b[l] + q);
            M.x[l][q] = wd * (2.0f * bc - wd * lap7_cg(M.b[l], d, M.cf[l], i, j, k, bc));
        }
        if (!grid_barrier(gbar)) return;
        const Dims c = M.d[l + 1];
        PF_GRID_LOOP(Q, c.n) {
            int I, J, K;
            cell_of(Q, c, I, J, K);
            M.b[l + 1][Q] = restrict_cg(M.b[l], M.x[l], d, M.cf[l], I, J, K);
        }
    }
}

__global__ void __launch_bounds__(256)
mg_mid_up(MgMid M, const BicgScalars* sc, unsigned* gbar) {
    if (sc->done || gbar[2]) return;
    for (int l = M.g1 - 1; l >= M.g0; --l) {
        const Dims d = M.d[l], c = M.d[l + 1];
        const float wd = M.wd[l];
        float* x = M.x[l];
        float* t = M.t[l];
        const float* b = M.b[l];
        PF_GRID_LOOP(q, d.n) {  // x += P xc
            int i, j, k;
            cell_of(q, d, i, j, k);
            x[q] = ldcg(x + q) + prolong_cg(M.x[l + 1], c, i, j, k);
        }
        if (!grid_barrier(gbar)) return;
        PF_GRID_LOOP(q, d.n) {  // t = x + w (b - A x)
            int i, j, k;
            cell_of(q, d, i, j, k);
            const float xc = ldcg(x + q);
            t[q] = fmaf(wd, ldcg(b + q) - lap7_cg(x, d, M.cf[l], i, j, k, xc), xc);
        }
        if (!grid_barrier(gbar)) return;
        PF_GRID_LOOP(q, d.n) {  // x = t + w (b - A t)
            int i, j, k;
            cell_of(q, d, i, j, k);
            const float tc = ldcg(t + q);
            x[q] = fmaf(wd, ldcg(b + q) - lap7_cg(t, d, M.cf[l], i, j, k, tc), tc);
        }
        if (!grid_barrier(gbar)) return;
    }
    {   // prolongation into the swept level g0 - 1
        const Dims f = M.d[M.g0 - 1], c = M.d[M.g0];
        PF_GRID_LOOP(q, f.n) {
            int i, j, k;
            cell_of(q, f, i, j, k);
            M.xs[q] = M.xs[q] + prolong_cg(M.x[M.g0], c, i, j, k);
        }
    }
}

// ------------------------------------------------- bottom of the V-cycle
// All levels of at most kMgBottomMax cells in one CTA: b, x, t of each level
// live in shared memory.  Same operations as the global kernels.
constexpr int kBottomThreads = 1024;

struct MgBottom {
    int nlev;
    Dims d[kMgMaxLevels];
    LapCoef<float> cf[kMgMaxLevels];
    float wd[kMgMaxLevels];
    float inv_p[kMgMaxLevels];  // 1 / (ny nz) and 1 / nz, for index decoding
    float inv_z[kMgMaxLevels];
    int off[kMgMaxLevels];      // float offset of the level's b; x and t follow
    const float* pinv;          // coarsest level's pseudo-inverse, or null
};


// Pseudo-inverse of the periodic coarsest-level operator (singular: constant
// null space), from its Fourier eigen-decomposition:
//   A^+[p][r] = (1/N) sum_{k != 0} cos(sum_q 2 pi k_q (p_q - r_q) / n_q) / lambda(k),
//   lambda(k) = sum_q c_q (2 - 2 cos(2 pi k_q / n_q)),  c_q = vol / h_q^2.
// Symmetric; applying it also removes the mean of the right-hand side.
__global__ void __launch_bounds__(256)
mg_coarse_pinv(Dims d, double cx, double cy, double cz, float* __restrict__ out) {
    pdl_wait();
    // A^+ is circulant: A^+[p][r] depends on (p - r) mod n only.  The block
    // tabulates 1/lambda(k), then 4 threads per difference vector sum its
    // Fourier series over interleaved k (fixed order), and the matrix is
    // filled from the N values.
    __shared__ double ilam[kMgPinvMax];
    __shared__ double part[kMgPinvMax][4];
    __shared__ double tab[kMgPinvMax];
    const int N = (int)d.n;
    const double tp = 6.283185307179586;
    const int nyz = d.ny * d.nz;
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
        const int kz = k % d.nz, ky = (k / d.nz) % d.ny, kx = k / nyz;
        const double lam = cx * (2.0 - 2.0 * cos(tp * kx / d.nx)) +
                           cy * (2.0 - 2.0 * cos(tp * ky / d.ny)) +
                           cz * (2.0 - 2.0 * cos(tp * kz / d.nz));
        ilam[k] = k == 0 ? 0.0 : 1.0 / lam;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 4 * N; t += blockDim.x) {
        const int q = t >> 2, lane = t & 3;
        const int dz = q % d.nz, dy = (q / d.nz) % d.ny, dx = q / nyz;
        double acc = 0.0;
        for (int k = 1 + lane; k < N; k += 4) {
            const int kz = k % d.nz, ky = (k / d.nz) % d.ny, kx = k / nyz;
            const double ph = tp * (double(kx * dx) / d.nx + double(ky * dy) / d.ny +
                                    double(kz * dz) / d.nz);
            acc += cos(ph) * ilam[k];
        }
        part[q][lane] = acc;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < N; q += blockDim.x)
        tab[q] = (((part[q][0] + part[q][1]) + part[q][2]) + part[q][3]) / double(N);
    __syncthreads();
    for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
        const int p = e / N, r = e - p * N;
        const int pz = p % d.nz, py = (p / d.nz) % d.ny, px = p / nyz;
        const int rz = r % d.nz, ry = (r / d.nz) % d.ny, rx = r / nyz;
        const int q = ((px - rx + d.nx) % d.nx * d.ny + (py - ry + d.ny) % d.ny) * d.nz +
                      (pz - rz + d.nz) % d.nz;
        out[e] = float(tab[q]);
    }
}

__device__ __forceinline__ float lap7_s(const float* x, const Dims& d,
                                        const LapCoef<float>& cf, int i, int j, int k,
                                        float xc) {
    const int P = d.ny * d.nz, ci = i * P, cj = j * d.nz;
    float ax = 0.0f;
    ax += x[wrap(i - 1, d.nx) * P + cj + k] * cf.c[0][0];
    ax += xc * cf.c[0][1];
    ax += x[wrap(i + 1, d.nx) * P + cj + k] * cf.c[0][2];
    ax += x[ci + wrap(j - 1, d.ny) * d.nz + k] * cf.c[1][0];
    ax += xc * cf.c[1][1];
    ax += x[ci + wrap(j + 1, d.ny) * d.nz + k] * cf.c[1][2];
    ax += x[ci + cj + wrap(k - 1, d.nz)] * cf.c[2][0];
    ax += xc * cf.c[2][1];
    ax += x[ci + cj + wrap(k + 1, d.nz)] * cf.c[2][2];
    return ax;
}

// q -> (i, j, k) by float reciprocals: exact for q < 2^16 (the quotients are
// at least 0.5 / 4096 away from an integer, far above the rounding error)
__device__ __forceinline__ void decode(int q, const Dims& d, float inv_p, float inv_z,
                                       int& i, int& j, int& k) {
    const int P = d.ny * d.nz;
    i = int((float(q) + 0.5f) * inv_p);
    const int r = q - i * P;
    j = int((float(r) + 0.5f) * inv_z);
    k = r - j * d.nz;
}

// The coarsest pseudo-inverse (<= 64 x 64) into shared memory.
__device__ __forceinline__ void bottom_load_pinv(const MgBottom& P, float* sm) {
    if (!P.pinv) return;
    const int last = P.nlev - 1;
    const int nc = (int)P.d[last].n;
    float* pv = sm + P.off[last] + 3 * nc;
    for (int q = threadIdx.x; q < nc * nc; q += blockDim.x) pv[q] = __ldg(P.pinv + q);
}

// One V-cycle over the levels of P, all in this CTA's shared memory `sm`:
// the first level's b is in place on entry (and the pseudo-inverse, if any);
// its x is in place on exit.  Block-wide barriers only.
__device__ void bottom_cycle(const MgBottom& P, float* sm) {
    __shared__ double shd[32];
    __shared__ float mean_s;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int last = P.nlev - 1;
    // down: pre-smooth from zero, restrict
    for (int l = 0; l < last; ++l) {
        const Dims d = P.d[l], c = P.d[l + 1];
        const int n = (int)d.n;
        float* b = sm + P.off[l];
        float* x = b + n;
        const float wd = P.wd[l];
        for (int q = tid; q < n; q += nt) {
            int i, j, k;
            decode(q, d, P.inv_p[l], P.inv_z[l], i, j, k);
            x[q] = wd * (2.0f * b[q] - wd * lap7_s(b, d, P.cf[l], i, j, k, b[q]));
        }
        __syncthreads();
        float* bc = sm + P.off[l + 1];
        for (int Q = tid; Q < (int)c.n; Q += nt) {
            int I, J, K;
            decode(Q, c, P.inv_p[l + 1], P.inv_z[l + 1], I, J, K);
            float sum = 0.0f;
            for (int a = 0; a < 2; ++a)
                for (int bb = 0; bb < 2; ++bb)
                    for (int cc = 0; cc < 2; ++cc) {
                        const int i = 2 * I + a, j = 2 * J + bb, k = 2 * K + cc;
                        const int qq = (i * d.ny + j) * d.nz + k;
                        sum += b[qq] - lap7_s(x, d, P.cf[l], i, j, k, x[qq]);
                    }
            bc[Q] = sum;
        }
        __syncthreads();
    }
    // coarsest: x = A^+ b, or mean removal then Jacobi sweeps (x <-> t)
    if (P.pinv) {
        // x = A^+ b: 16 threads per row, 16-lane shuffle reduction
        const int n = (int)P.d[last].n;
        const float* b = sm + P.off[last];
        float* x = sm + P.off[last] + n;
        const float* pv = sm + P.off[last] + 3 * n;
        // whole warps take part in every pass of the loop (the bound is a
        // multiple of 32, like the block), so the shuffles see all lanes
        const int tot = ((16 * n + 31) / 32) * 32;
        for (int t = tid; t < tot; t += nt) {
            const int p = t >> 4, part = t & 15;
            float acc = 0.0f;
            if (p < n)
                for (int r = part; r < n; r += 16) acc = fmaf(pv[r * n + p], b[r], acc);
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o, 16);
            if (part == 0 && p < n) x[p] = acc;
        }
        __syncthreads();
    } else {
        const Dims d = P.d[last];
        const int n = (int)d.n;
        float* b = sm + P.off[last];
        float* x = b + n;
        float* t = x + n;
        const float wd = P.wd[last];
        double acc = 0.0;
        for (int q = tid; q < n; q += nt) acc += double(b[q]);
        const double tot = block_sum<kBottomThreads>(acc, shd);
        if (tid == 0) mean_s = float(tot / double(n));
        __syncthreads();
        const float mean = mean_s;
        for (int q = tid; q < n; q += nt) {
            const float v = b[q] - mean;
            b[q] = v;
            x[q] = wd * v;
        }
        __syncthreads();
        for (int it = 1; it < kMgCoarseSweeps; ++it) {
            for (int q = tid; q < n; q += nt) {
                int i, j, k;
                decode(q, d, P.inv_p[last], P.inv_z[last], i, j, k);
                const float xc = x[q];
                t[q] = fmaf(wd, b[q] - lap7_s(x, d, P.cf[last], i, j, k, xc), xc);
            }
            __syncthreads();
            float* tmp = x; x = t; t = tmp;
        }
        // the result must sit in the level's x slot
        if (x != b + n) {
            for (int q = tid; q < n; q += nt) b[n + q] = x[q];
            __syncthreads();
        }
    }
    // up: prolong, two post-smoothing sweeps
    for (int l = last - 1; l >= 0; --l) {
        const Dims d = P.d[l], c = P.d[l + 1];
        const int n = (int)d.n;
        float* b = sm + P.off[l];
        float* x = b + n;
        float* t = x + n;
        const float* xc = sm + P.off[l + 1] + c.n;
        const float wd = P.wd[l];
        for (int q = tid; q < n; q += nt) {
            int i, j, k;
            decode(q, d, P.inv_p[l], P.inv_z[l], i, j, k);
            const int I = i >> 1, J = j >> 1, K = k >> 1;
            const int I2 = wrap(I + ((i & 1) ? 1 : -1), c.nx);
            const int J2 = wrap(J + ((j & 1) ? 1 : -1), c.ny);
            const int K2 = wrap(K + ((k & 1) ? 1 : -1), c.nz);
            auto C = [&](int a, int bb, int cc) { return xc[(a * c.ny + bb) * c.nz + cc]; };
            const float e = (27.0f * C(I, J, K) + 9.0f * (C(I2, J, K) + C(I, J2, K) + C(I, J, K2)) +
                             3.0f * (C(I2, J2, K) + C(I2, J, K2) + C(I, J2, K2)) + C(I2, J2, K2)) *
                            (1.0f / 64.0f);
            x[q] = x[q] + e;
        }
        __syncthreads();
        for (int q = tid; q < n; q += nt) {
            int i, j, k;
            decode(q, d, P.inv_p[l], P.inv_z[l], i, j, k);
            const float v = x[q];
            t[q] = fmaf(wd, b[q] - lap7_s(x, d, P.cf[l], i, j, k, v), v);
        }
        __syncthreads();
        for (int q = tid; q < n; q += nt) {
            int i, j, k;
            decode(q, d, P.inv_p[l], P.inv_z[l], i, j, k);
            const float v = t[q];
            x[q] = fmaf(wd, b[q] - lap7_s(t, d, P.cf[l], i, j, k, v), v);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kBottomThreads)
mg_bottom(MgBottom P, const float* __restrict__ gb, float* __restrict__ gx,
          const BicgScalars* sc) {
    pdl_wait();
    if (sc->done) return;
    extern __shared__ float sm[];
    const int n = (int)P.d[0].n;
    float* b = sm + P.off[0];
    for (int q = threadIdx.x; q < n; q += blockDim.x) b[q] = gb[q];
    bottom_load_pinv(P, sm);
    __syncthreads();
    bottom_cycle(P, sm);
    const float* x = sm + P.off[0] + n;
    for (int q = threadIdx.x; q < n; q += blockDim.x) gx[q] = x[q];
}

// ------------------------------------------------- cluster bottom
// Levels of at most kMgClusterMax cells whose x extent divides among the
// kClusterCtas CTAs of one thread-block cluster, together with the bottom
// levels below them, run as ONE launch: each CTA keeps its x planes of b, x
// and t of every split level in its shared memory and reads the neighbouring
// CTAs' boundary planes through distributed shared memory (a per-CTA table
// maps every plane of every split level to the owner's shared memory); the
// hardware cluster barrier separates the phases.  The levels below the split
// ones live in CTA 0, which runs bottom_cycle on them while the other CTAs
// wait at the barrier.  Every operation is the one the per-level global
// kernels perform (same arithmetic, same order): smoothing as mg_smooth0_pw
// and mg_smooth_pw, restriction as mg_restrict, prolongation as prolong_at.
struct MgCluster {
    int ns;                               // split levels
    Dims d[kMgMaxLevels];
    LapCoef<float> cf[kMgMaxLevels];
    float wd[kMgMaxLevels];
    int pp[kMgMaxLevels];                 // x planes per CTA
    float inv_p[kMgMaxLevels];            // 1 / (ny nz), 1 / nz: decode of plane-blocked indices
    float inv_z[kMgMaxLevels];
    int off[kMgMaxLevels];                // float offset of the level's b (pp ny nz); x, t follow
    int toff[kMgMaxLevels];               // plane-table entry offset of the level: [3][nx]
    int whole;                            // float offset of the whole levels (w.off relative to it)
    int tab;                              // float offset of the plane table (8-byte entries)
    MgBottom w;                           // the levels below, in CTA 0
};

// A x at (j, k) of the plane pc from the planes pm (i - 1) and pp (i + 1),
// in the order of lap7.
__device__ __forceinline__ float lap_planes(const float* pm, const float* pc, const float* pp,
                                            const Dims& d, const LapCoef<float>& cf, int j, int k,
                                            float xc) {
    const int cj = j * d.nz;
    float ax = 0.0f;
    ax += pm[cj + k] * cf.c[0][0];
    ax += xc * cf.c[0][1];
    ax += pp[cj + k] * cf.c[0][2];
    ax += pc[wrap(j - 1, d.ny) * d.nz + k] * cf.c[1][0];
    ax += xc * cf.c[1][1];
    ax += pc[wrap(j + 1, d.ny) * d.nz + k] * cf.c[1][2];
    ax += pc[cj + wrap(k - 1, d.nz)] * cf.c[2][0];
    ax += xc * cf.c[2][1];
    ax += pc[cj + wrap(k + 1, d.nz)] * cf.c[2][2];
    return ax;
}

__global__ void __launch_bounds__(kBottomThreads, 1)
mg_cluster(MgCluster P, const float* __restrict__ gb, float* __restrict__ gx,
           const BicgScalars* sc) {
    pdl_wait();
    // uniform over the cluster: no CTA has touched another's memory yet
    if (sc->done) return;
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) float sm[];
    const int rank = (int)cl.block_rank();
    const int tid = threadIdx.x, nt = blockDim.x;
    float** tab = reinterpret_cast<float**>(sm + P.tab);
    float* whole0 = cl.map_shared_rank(sm + P.whole, 0);
    const Dims dw = P.w.d[0];
    const int plw = dw.ny * dw.nz;
    // plane i of array a (0 b, 1 x, 2 t) of level r: a split level's plane
    // in its owner's shared memory, or the first whole level's in CTA 0's
    auto plane = [&](int r, int a, int i) -> float* {
        if (r < P.ns) return tab[P.toff[r] + a * P.d[r].nx + i];
        return whole0 + P.w.off[0] + a * (int)dw.n + i * plw;
    };
    for (int r = 0; r < P.ns; ++r) {
        const int nx = P.d[r].nx, pl = P.d[r].ny * P.d[r].nz, cells = P.pp[r] * pl;
        for (int e = tid; e < 3 * nx; e += nt) {
            const int a = e / nx, i = e - a * nx;
            const int owner = i / P.pp[r], li = i - owner * P.pp[r];
            tab[P.toff[r] + e] = cl.map_shared_rank(sm + P.off[r] + a * cells + li * pl, owner);
        }
    }
    {   // this CTA's planes of the first level's b
        const int cells = P.pp[0] * P.d[0].ny * P.d[0].nz;
        const float* src = gb + (long long)rank * cells;
        float* b = sm + P.off[0];
        for (int q = tid; q < cells; q += nt) b[q] = src[q];
    }
    if (rank == 0) bottom_load_pinv(P.w, sm + P.whole);
    cl.sync();
    // down: pre-smooth from zero, restrict
    for (int r = 0; r < P.ns; ++r) {
        const Dims d = P.d[r];
        const LapCoef<float> cf = P.cf[r];
        const int pl = d.ny * d.nz, cells = P.pp[r] * pl, i0 = rank * P.pp[r];
        const Dims loc{P.pp[r], d.ny, d.nz, (long long)cells};
        float* b = sm + P.off[r];
        float* x = b + cells;
        const float wd = P.wd[r];
        for (int q = tid; q < cells; q += nt) {
            int il, j, k;
            decode(q, loc, P.inv_p[r], P.inv_z[r], il, j, k);
            const int i = i0 + il;
            const float* pc = b + il * pl;
            const float bc = pc[j * d.nz + k];
            const float ab = lap_planes(plane(r, 0, wrap(i - 1, d.nx)), pc,
                                        plane(r, 0, wrap(i + 1, d.nx)), d, cf, j, k, bc);
            x[q] = wd * (2.0f * bc - wd * ab);
        }
        cl.sync();
        // coarse planes I whose first child plane 2I is this CTA's
        const bool cs = r + 1 < P.ns;
        const Dims c = cs ? P.d[r + 1] : dw;
        const float cip = cs ? P.inv_p[r + 1] : P.w.inv_p[0];
        const float ciz = cs ? P.inv_z[r + 1] : P.w.inv_z[0];
        const int I0 = (i0 + 1) >> 1, I1 = (i0 + P.pp[r] + 1) >> 1;
        const int ccells = (I1 - I0) * c.ny * c.nz;
        const Dims cloc{I1 - I0, c.ny, c.nz, (long long)ccells};
        const float cen = (cf.c[0][1] + cf.c[1][1]) + cf.c[2][1];
        for (int q = tid; q < ccells; q += nt) {
            int Il, J, K;
            decode(q, cloc, cip, ciz, Il, J, K);
            const int I = I0 + Il;
            float sum = 0.0f;
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                const int i = 2 * I + a;
                const float* xm = plane(r, 1, wrap(i - 1, d.nx));
                const float* xc = plane(r, 1, i);
                const float* xp = plane(r, 1, wrap(i + 1, d.nx));
                const float* bi = plane(r, 0, i);
#pragma unroll
                for (int bb = 0; bb < 2; ++bb) {
                    const int j = 2 * J + bb;
                    const int jm = wrap(j - 1, d.ny) * d.nz, jp = wrap(j + 1, d.ny) * d.nz;
#pragma unroll
                    for (int cc = 0; cc < 2; ++cc) {
                        const int k = 2 * K + cc, q0 = j * d.nz + k;
                        float ax = xc[q0] * cen;
                        ax = fmaf(xm[q0], cf.c[0][0], ax);
                        ax = fmaf(xp[q0], cf.c[0][2], ax);
                        ax = fmaf(xc[jm + k], cf.c[1][0], ax);
                        ax = fmaf(xc[jp + k], cf.c[1][2], ax);
                        ax = fmaf(xc[j * d.nz + wrap(k - 1, d.nz)], cf.c[2][0], ax);
                        ax = fmaf(xc[j * d.nz + wrap(k + 1, d.nz)], cf.c[2][2], ax);
                        sum += bi[q0] - ax;
                    }
                }
            }
            plane(r + 1, 0, I)[J * c.nz + K] = sum;
        }
        cl.sync();
    }
    // the levels below, in CTA 0
    if (rank == 0) bottom_cycle(P.w, sm + P.whole);
    cl.sync();
    // up: x += P xc, two post-smoothing sweeps
    for (int r = P.ns - 1; r >= 0; --r) {
        const Dims d = P.d[r];
        const LapCoef<float> cf = P.cf[r];
        const int pl = d.ny * d.nz, cells = P.pp[r] * pl, i0 = rank * P.pp[r];
        const Dims loc{P.pp[r], d.ny, d.nz, (long long)cells};
        const Dims c = r + 1 < P.ns ? P.d[r + 1] : dw;
        float* b = sm + P.off[r];
        float* x = b + cells;
        float* t = x + cells;
        const float wd = P.wd[r];
        for (int q = tid; q < cells; q += nt) {
            int il, j, k;
            decode(q, loc, P.inv_p[r], P.inv_z[r], il, j, k);
            const int i = i0 + il;
            const int I = i >> 1, J = j >> 1, K = k >> 1;
            const int I2 = wrap(I + ((i & 1) ? 1 : -1), c.nx);
            const int J2 = wrap(J + ((j & 1) ? 1 : -1), c.ny);
            const int K2 = wrap(K + ((k & 1) ? 1 : -1), c.nz);
            const float* c0 = plane(r + 1, 1, I);
            const float* c1 = plane(r + 1, 1, I2);
            const int b0 = J * c.nz, b1 = J2 * c.nz;
            const float v000 = c0[b0 + K], v100 = c1[b0 + K];
            const float v010 = c0[b1 + K], v001 = c0[b0 + K2];
            const float v110 = c1[b1 + K], v101 = c1[b0 + K2];
            const float v011 = c0[b1 + K2], v111 = c1[b1 + K2];
            const float e = (27.0f * v000 + 9.0f * (v100 + v010 + v001) +
                             3.0f * (v110 + v101 + v011) + v111) * (1.0f / 64.0f);
            x[q] = x[q] + e;
        }
        cl.sync();
        for (int pass = 0; pass < 2; ++pass) {
            const int ai = pass == 0 ? 1 : 2;   // smooth x -> t, then t -> x
            float* in = pass == 0 ? x : t;
            float* out = pass == 0 ? t : x;
            for (int q = tid; q < cells; q += nt) {
                int il, j, k;
                decode(q, loc, P.inv_p[r], P.inv_z[r], il, j, k);
                const int i = i0 + il;
                const float* pc = in + il * pl;
                const float v = pc[j * d.nz + k];
                const float ax = lap_planes(plane(r, ai, wrap(i - 1, d.nx)), pc,
                                            plane(r, ai, wrap(i + 1, d.nx)), d, cf, j, k, v);
                out[q] = fmaf(wd, b[q] - ax, v);
            }
            cl.sync();
        }
    }
    {   // this CTA's planes of the first level's x
        const int cells = P.pp[0] * P.d[0].ny * P.d[0].nz;
        const float* x = sm + P.off[0] + cells;
        float* dst = gx + (long long)rank * cells;
        for (int q = tid; q < cells; q += nt) dst[q] = x[q];
    }
}

static size_t bottom_smem_floats(const MgPlan& P) {
    size_t f = 0;
    for (int l = P.B; l < P.L; ++l) f += 3 * (size_t)P.lv[l].d.n;
    if (P.pinv) f += (size_t)P.lv[P.L - 1].d.n * P.lv[P.L - 1].d.n;  // the pseudo-inverse
    return f;
}

static MgBottom bottom_params(const MgPlan& P) {
    MgBottom m{};
    m.nlev = P.L - P.B;
    int off = 0;
    for (int l = P.B; l < P.L; ++l) {
        const int r = l - P.B;
        m.d[r] = P.lv[l].d;
        m.cf[r] = P.lv[l].cf;
        m.wd[r] = P.lv[l].wd;
        m.inv_p[r] = 1.0f / float(P.lv[l].d.ny * P.lv[l].d.nz);
        m.inv_z[r] = 1.0f / float(P.lv[l].d.nz);
        m.off[r] = off;
        off += 3 * (int)P.lv[l].d.n;
    }
    m.pinv = P.pinv;
    return m;
}

// Shared-memory layout of the cluster kernel (floats): split levels' planes,
// the bottom levels (CTA 0), the plane table (8-byte entries).
static MgCluster cluster_params(const MgPlan& P, size_t* floats) {
    MgCluster m{};
    m.ns = P.B - P.C;
    int off = 0, toff = 0;
    for (int l = P.C; l < P.B; ++l) {
        const int r = l - P.C;
        const MgLevel& v = P.lv[l];
        m.d[r] = v.d;
        m.cf[r] = v.cf;
        m.wd[r] = v.wd;
        m.pp[r] = v.d.nx / kClusterCtas;
        m.inv_p[r] = 1.0f / float(v.d.ny * v.d.nz);
        m.inv_z[r] = 1.0f / float(v.d.nz);
        m.off[r] = off;
        off += 3 * m.pp[r] * v.d.ny * v.d.nz;
        m.toff[r] = toff;
        toff += 3 * v.d.nx;
    }
    m.whole = off;
    m.w = bottom_params(P);
    off += (int)bottom_smem_floats(P);
    off = (off + 1) & ~1;
    m.tab = off;
    off += 2 * toff;
    *floats = (size_t)off;
    return m;
}

static constexpr size_t kClusterSmemMax = 200 * 1024;

// Launch configuration of the cluster kernel: one cluster of kClusterCtas
// CTAs, optionally with programmatic dependent launch (`at` holds two entries).
static cudaLaunchConfig_t cluster_config(size_t smem, cudaStream_t s, cudaLaunchAttribute* at,
                                         bool pdl) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(kClusterCtas);
    cfg.blockDim = dim3(kBottomThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = kClusterCtas;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if (pdl) {  // as the per-level kernels (pdl_wait() at entry)
        at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[1].val.programmaticStreamSerializationAllowed = 1;
        cfg.numAttrs = 2;
    }
    return cfg;
}

static cudaError_t launch_cluster(const MgCluster& m, size_t smem, const float* gb, float* gx,
                                  const BicgScalars* sc, cudaStream_t s) {
    cudaLaunchAttribute at[2];
    const cudaLaunchConfig_t cfg = cluster_config(smem, s, at, true);
    return cudaLaunchKernelEx(&cfg, mg_cluster, m, gb, gx, sc);
}

// Whether this device runs the plan's cluster kernel (shared memory within
// kClusterSmemMax and at least one cluster resident); otherwise the split
// levels fall back to the per-level kernels.
static cudaError_t cluster_attrs() {
    return cudaFuncSetAttribute(mg_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kClusterSmemMax);
}

static bool cluster_usable(const MgPlan& P) {
    size_t fl = 0;
    cluster_params(P, &fl);
    const size_t bytes = fl * sizeof(float);
    if (bytes > kClusterSmemMax) return false;
    // once per CUDA context (function attributes belong to the context)
    if (once_per_context((const void*)&cluster_attrs, &cluster_attrs) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    cudaLaunchAttribute at[2];
    const cudaLaunchConfig_t cfg = cluster_config(bytes, nullptr, at, false);
    int nc = 0;
    if (cudaOccupancyMaxActiveClusters(&nc, mg_cluster, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return nc >= 1;
}

// v = A ph, gamma = (v, res0), alpha = rho / gamma (TZ: cp.async tile width,
// 0 for the register-prefetch sweep)
template <int TZ>
__global__ void __launch_bounds__(kBlock, 2)
mg_av(Dims d, Tiling tl, LapCoef<float> cf, BicgScalars* sc, double* part,
      const float* ph, const float* res0, float* v, int use_cond,
      cudaGraphConditionalHandle cond) {
    pdl_wait();
    __shared__ double sh[32];
    if (sc->done) return;
    double dot;
    if constexpr (TZ > 0) {
        AsyncAv p{{ph}, {res0}, v, 0.0};
        sweep_async<kAsTY1, TZ>(d, tl, cf, p);
        dot = p.dot;
    } else {
        PhaseAv p{ph, res0, v, 0.0};
        sweep<float>(d, tl, cf, p);
        dot = p.dot;
    }
    const double bs = block_sum<kBlock>(dot, sh);
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
template <int TZ>
__global__ void __launch_bounds__(kBlock, 2)
mg_at(Dims d, Tiling tl, LapCoef<float> cf, BicgScalars* sc, double* part,
      const float* shv, const float* s, float* t) {
    pdl_wait();
    __shared__ double sh[32];
    if (sc->done) return;
    double ts, tt;
    if constexpr (TZ > 0) {
        AsyncAt p{{shv}, {s}, t, 0.0, 0.0};
        sweep_async<kAsTY1, TZ>(d, tl, cf, p);
        ts = p.ts; tt = p.tt;
    } else {
        PhaseAt p{shv, s, t, 0.0, 0.0};
        sweep<float>(d, tl, cf, p);
        ts = p.ts; tt = p.tt;
    }
    const double b0 = block_sum<kBlock>(ts, sh);
    const double b1 = block_sum<kBlock>(tt, sh);
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
    pdl_wait();
    __shared__ double sh[32];
    if (sc->done) {
        if (use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(cond, 0);
        return;
    }
    const float alpha = float(sc->alpha), omega = float(sc->omega);
    // the first iteration of a pass starts from e = 0 (e is not read)
    const bool first = sc->iter == 0;
    double dot = 0.0, mx = 0.0;
    auto cell = [&](float& ev, float phv, float shq, float sv, float tv, float r0, float& rv) {
        const float x = fmaf(alpha, phv, ev);
        ev = fmaf(omega, shq, x);
        rv = fmaf(-omega, tv, sv);
        dot += double(rv) * double(r0);
        mx = nanmax(mx, fabs(double(rv)));
    };
    // four cells per thread with 16-byte accesses (all vectors are 256-byte
    // aligned), then the tail
    const long long n4 = d.n >> 2;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += stride) {
        float4 ev = first ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : reinterpret_cast<const float4*>(e)[i];
        const float4 pv = reinterpret_cast<const float4*>(ph)[i];
        const float4 hv = reinterpret_cast<const float4*>(shv)[i];
        const float4 sv = reinterpret_cast<const float4*>(s)[i];
        const float4 tv = reinterpret_cast<const float4*>(t)[i];
        const float4 zv = reinterpret_cast<const float4*>(res0)[i];
        float4 rv;
        cell(ev.x, pv.x, hv.x, sv.x, tv.x, zv.x, rv.x);
        cell(ev.y, pv.y, hv.y, sv.y, tv.y, zv.y, rv.y);
        cell(ev.z, pv.z, hv.z, sv.z, tv.z, zv.z, rv.z);
        cell(ev.w, pv.w, hv.w, sv.w, tv.w, zv.w, rv.w);
        reinterpret_cast<float4*>(e)[i] = ev;
        reinterpret_cast<float4*>(res)[i] = rv;
    }
    for (long long q = 4 * n4 + blockIdx.x * (long long)blockDim.x + threadIdx.x; q < d.n;
         q += stride) {
        float ev = first ? 0.0f : e[q], rv;
        cell(ev, ph[q], shv[q], s[q], t[q], res0[q], rv);
        e[q] = ev;
        res[q] = rv;
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

// res = res0 = float(r / scale); rho = (res, res0).  e, p and v are not
// cleared: the first iteration reads none of them (beta == 0 in the p
// update, e = 0 in mg_update), and a pass that ends before its first
// iteration folds nothing (fold_* skip iter == 0).
__global__ void __launch_bounds__(kBlock)
mg_init(Dims d, BicgScalars* sc, double* part, const double* __restrict__ r,
        float* res, float* res0, float* e, float* p0, float* p1, float* v,
        int max_it, double tol, double outer_tol) {
    pdl_wait();
    __shared__ double sh[32];
    const double inv = sc->scale > 0.0 ? 1.0 / sc->scale : 0.0;
    double s = 0.0, m = 0.0;
    auto cell = [&](double rq) {
        const float x = float(rq * inv);
        s += double(x) * double(x);
        m = nanmax(m, fabs(double(x)));
        return x;
    };
    // four cells per thread with 16-byte accesses (all vectors are 256-byte
    // aligned), then the tail
    const long long n4 = d.n >> 2;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += stride) {
        const double2 a = reinterpret_cast<const double2*>(r)[2 * i];
        const double2 b = reinterpret_cast<const double2*>(r)[2 * i + 1];
        float4 x;
        x.x = cell(a.x);
        x.y = cell(a.y);
        x.z = cell(b.x);
        x.w = cell(b.y);
        reinterpret_cast<float4*>(res)[i] = x;
        reinterpret_cast<float4*>(res0)[i] = x;
    }
    for (long long q = 4 * n4 + blockIdx.x * (long long)blockDim.x + threadIdx.x; q < d.n;
         q += stride) {
        const float x = cell(r[q]);
        res[q] = x; res0[q] = x;
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
            // a pass only has to close the remaining gap to the refinement's
            // tolerance (with a 3x margin): the last pass stops early
            double t = tol;
            if (outer_tol > 0.0 && sc->true_res > 0.0 && sc->max_b > 0.0)
                t = fmin(0.5, fmax(tol, 0.3 * outer_tol * sc->max_b / sc->true_res));
            sc->max_it = max_it; sc->min_res = t; sc->status = PF_OK;
            sc->done = (mx > 0.0 && mx == mx && !isinf(mx)) ? 0 : 1;
            if (!(mx == mx) || isinf(mx)) sc->status = PF_NONFINITE;
            sc->counter = 0u;
        }
    }
}

// ------------------------------------------------------------------- host
int mg_levels(const pf_grid* g, MgLevel* lv, int* bottom) {
    pf_grid cur = *g;
    int L = 0;
    for (;;) {
        MgLevel& l = lv[L];
        l.d = Dims{cur.nx, cur.ny, cur.nz, (long long)cur.nx * cur.ny * cur.nz};
        l.cf = lap_coef<float>(&cur);
        const LapCoef<double> c64 = lap_coef<double>(&cur);
        const double diag = c64.c[0][1] + c64.c[1][1] + c64.c[2][1];
        l.wd = float(double(kMgOmega) / diag);
        for (int q = 0; q < 3; ++q) l.cq[q] = -c64.c[q][2];
        l.b = l.x = l.t = nullptr;
        l.tl = make_tiling(l.d, 32);
        l.tl8 = make_tiling(l.d, 64);
        l.az = l.d.nz % 64 == 0 ? 64 : (l.d.nz % 32 == 0 ? 32 : 0);
        l.ta1 = make_tiling(l.d, kAsTY1, l.az ? l.az : 32);
        l.tan = make_tiling(l.d, kAsTYn, l.az ? l.az : 32);
        l.kind = (L == 0 || l.d.n >= kMgSweepMin) ? kMgSwept
                 : (l.d.n > kMgBottomLevel ? kMgPointwise : kMgBottom);
        ++L;
        if (l.d.n <= kMgCoarseTarget || L == kMgMaxLevels) break;
        if ((cur.nx | cur.ny | cur.nz) & 1) break;
        if (cur.nx < 4 || cur.ny < 4 || cur.nz < 4) break;
        cur.nx /= 2; cur.ny /= 2; cur.nz /= 2;
        cur.dx *= 2.0; cur.dy *= 2.0; cur.dz *= 2.0;
    }
    // the coarsest level always runs in the bottom kernel
    if (L >= 2 && lv[L - 1].kind == kMgPointwise && lv[L - 1].d.n <= kMgBottomMax)
        lv[L - 1].kind = kMgBottom;
    int B = 0;
    while (B < L && lv[B].kind != kMgBottom) ++B;
    if (L < 2 || B == 0 || B == L) return 0;
    // the cluster kernel takes the levels just above the bottom ones that
    // split evenly into x planes per CTA
    for (int l = B - 1; l >= 1; --l) {
        const MgLevel& v = lv[l];
        if (v.kind != kMgPointwise || v.d.n > kMgClusterMax || v.d.nx % kClusterCtas) break;
        lv[l].kind = kMgCluster;
    }
    *bottom = B;
    return L;
}

static constexpr int kMgFineVecs = 11;  // res res0 p0 p1 v s t ph sh e tmp

size_t mg_region_bytes(const pf_grid* g) {
    MgLevel lv[kMgMaxLevels];
    int B = 0;
    const int L = mg_levels(g, lv, &B);
    if (!L) return 0;
    size_t b = kMgFineVecs * align256(lv[0].d.n * sizeof(float));
    for (int l = 1; l < L; ++l) b += 3 * align256(lv[l].d.n * sizeof(float));
    const long long nc = lv[L - 1].d.n;
    if (nc <= kMgPinvMax) b += align256((size_t)(nc * nc) * sizeof(float));
    return b + kMgBarrierBytes;
}

template <class K>
static bool smem_attr(K kernel, size_t bytes) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)bytes) != cudaSuccess;
}

// dynamic shared memory limits of the cp.async sweeps of tile width TZ
template <int TZ>
static bool async_attrs() {
    return smem_attr(mg_smooth0_as<kAsTY1, TZ, AsyncPlain>,
                     async_sweep_smem<kAsTY1, TZ, AsyncSmooth0<AsyncPlain>>()) ||
           smem_attr(mg_smooth0_as<kAsTYn, TZ, AsyncS>,
                     async_sweep_smem<kAsTYn, TZ, AsyncSmooth0<AsyncS>>()) ||
           smem_attr(mg_smooth_as<TZ>, async_sweep_smem<kAsTY1, TZ, AsyncSmooth>()) ||
           smem_attr(mg_av<TZ>, async_sweep_smem<kAsTY1, TZ, AsyncAv>()) ||
           smem_attr(mg_at<TZ>, async_sweep_smem<kAsTY1, TZ, AsyncAt>());
}

// Dynamic shared-memory limits of the multigrid kernels.
static cudaError_t mg_attrs() {
    // the bottom levels (at most 4096 + 512 + 64 + ... cells, 3 arrays each)
    // need more than the default 48 KiB of shared memory
    const int bytes = int(sizeof(float) * (3 * (kMgBottomMax + kMgBottomMax / 7 + 64) +
                                            kMgPinvMax * kMgPinvMax));
    const cudaError_t e = cudaFuncSetAttribute(mg_bottom, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               bytes);
    if (e != cudaSuccess) return e;
    // the cp.async sweeps' plane rings (up to ~93 KiB)
    if (async_attrs<32>() || async_attrs<64>()) return cudaErrorInvalidValue;
    return cudaSuccess;
}

int mg_setup(const pf_grid* g, void* region, MgPlan* P) {
    P->L = mg_levels(g, P->lv, &P->B);
    if (!P->L) return PF_ERR_BAD_ARG;
    P->C = P->B;
    while (P->C > 1 && P->lv[P->C - 1].kind == kMgCluster) --P->C;
    if (P->C < P->B && !cluster_usable(*P)) {
        for (int l = P->C; l < P->B; ++l) P->lv[l].kind = kMgPointwise;
        P->C = P->B;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    // once per CUDA context (function attributes belong to the context)
    if (once_per_context((const void*)&mg_attrs, &mg_attrs) != cudaSuccess) return PF_ERR_CUDA;
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
    const long long nc = P->lv[P->L - 1].d.n;
    P->pinv = nc <= kMgPinvMax ? (float*)ptr : nullptr;
    if (nc <= kMgPinvMax) ptr += align256((size_t)(nc * nc) * sizeof(float));
    P->gbar = (unsigned*)ptr;
    // the one-thread-per-cell levels below the swept ones: cooperative launches
    P->G = P->C;
    while (P->G > 1 && P->lv[P->G - 1].kind == kMgPointwise) --P->G;
    P->coop = 0;
    // Opt-in (PF_MG_COOP=1 in the environment): the two forms give
    // bit-identical results; the cooperative one launches 100 instead of 188
    // kernels per 128^3 step but replays 28 % slower in a captured step
    // (1.88 against 1.47 ms: its grid barriers cost more than the per-level
    // launches, whose launch latency programmatic dependent launch hides)
    const char* env = std::getenv("PF_MG_COOP");
    const bool allow = env && env[0] == '1';
    if (allow && P->G < P->C && P->lv[P->G - 1].kind == kMgSwept) {
        int coop = 0, per_down = 0, per_up = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
        if (coop &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_down, mg_mid_down, 256, 0) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_up, mg_mid_up, 256, 0) == cudaSuccess &&
            std::min(per_down, per_up) >= 1) {
            // at most two blocks per SM, so concurrent solves' launches fit together
            P->coop_grid = num_sms() * std::min(2, std::min(per_down, per_up));
            P->coop = 1;
        }
        cudaGetLastError();
    }
    return PF_OK;
}

static dim3 cgrid3(const Dims& d) { return dim3((d.nz + 31) / 32, (d.ny + 7) / 8, d.nx); }
// restriction / prolongation: two coarse planes per thread
static dim3 cgrid3h(const Dims& c) { return dim3((c.nz + 31) / 32, (c.ny + 7) / 8, (c.nx + 1) / 2); }

// Launchers of the cp.async sweeps for the level's tile width.
template <int TY, class S>
static void smooth0_as(const MgLevel& f, const BicgScalars* sc, const AsyncSmooth0<S>& ph,
                       const char* name, cudaStream_t s) {
    const dim3 blk(32, 8);
    const Tiling& tl = TY == kAsTY1 ? f.ta1 : f.tan;
    if (f.az == 64)
        PF_LAUNCH(name, s, launch_pdl(mg_smooth0_as<TY, 64, S>, dim3(tiled_grid(tl)), dim3(blk),
            async_sweep_smem<TY, 64, AsyncSmooth0<S>>(), s, f.d, tl, f.cf, sc, ph));
    else
        PF_LAUNCH(name, s, launch_pdl(mg_smooth0_as<TY, 32, S>, dim3(tiled_grid(tl)), dim3(blk),
            async_sweep_smem<TY, 32, AsyncSmooth0<S>>(), s, f.d, tl, f.cf, sc, ph));
}

static void smooth_as(const MgLevel& f, const BicgScalars* sc, const AsyncSmooth& ph,
                      const char* name, cudaStream_t s) {
    const dim3 blk(32, 8);
    if (f.az == 64)
        PF_LAUNCH(name, s, launch_pdl(mg_smooth_as<64>, dim3(tiled_grid(f.ta1)), dim3(blk),
            async_sweep_smem<kAsTY1, 64, AsyncSmooth>(), s, f.d, f.ta1, f.cf, sc, ph));
    else
        PF_LAUNCH(name, s, launch_pdl(mg_smooth_as<32>, dim3(tiled_grid(f.ta1)), dim3(blk),
            async_sweep_smem<kAsTY1, 32, AsyncSmooth>(), s, f.d, f.ta1, f.cf, sc, ph));
}

// The cooperative mid-level launches (see mg_mid_down / mg_mid_up): levels
// G .. C-1 with the swept level G - 1 (right-hand side bs, iterate xs).
static MgMid mid_params(const MgPlan& P, const float* bs, float* xs) {
    MgMid m{};
    m.g0 = P.G;
    m.g1 = P.C;
    for (int l = P.G - 1; l <= P.C; ++l) {
        m.d[l] = P.lv[l].d;
        m.cf[l] = P.lv[l].cf;
        m.wd[l] = P.lv[l].wd;
        m.b[l] = P.lv[l].b;
        m.x[l] = P.lv[l].x;
        m.t[l] = P.lv[l].t;
    }
    m.bs = bs;
    m.xs = xs;
    return m;
}

static cudaError_t launch_mid(bool up, const MgPlan& P, const float* bs, float* xs,
                              const BicgScalars* sc, cudaStream_t s) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(P.coop_grid);
    cfg.blockDim = dim3(256);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const MgMid m = mid_params(P, bs, xs);
    return up ? cudaLaunchKernelEx(&cfg, mg_mid_up, m, sc, P.gbar)
              : cudaLaunchKernelEx(&cfg, mg_mid_down, m, sc, P.gbar);
}

// Restriction from level 0 (whose x and b are set), the levels down to the
// bottom kernel, and the up-sweep back to level 0's x.
static void vcycle_tail(const MgPlan& P, const float* b0, float* x0, BicgScalars* sc,
                        cudaStream_t s) {
    const dim3 blk(32, 8);
    const bool coop = P.coop && P.G < P.C;  // levels G .. C-1 in the cooperative launches
    const int down_end = coop ? P.G : P.C;
    for (int l = 0; l < down_end; ++l) {
        const MgLevel& f = P.lv[l];
        const MgLevel& c = P.lv[l + 1];
        const float* bl = l == 0 ? b0 : f.b;
        float* xl = l == 0 ? x0 : f.x;
        if (l > 0) {
            if (f.kind == kMgSwept && f.az) {
                AsyncSmooth0<AsyncPlain> ph{{}, {f.b}, {nullptr}, f.x, f.wd};
                smooth0_as<kAsTY1>(f, sc, ph, "mg_smooth0", s);
            } else if (f.kind == kMgSwept) {
                PhaseSmooth0<SrcPlain> ph{};
                ph.src.b = f.b; ph.x = f.x; ph.wd = f.wd;
                PF_LAUNCH("mg_smooth0", s, launch_pdl(mg_smooth0<SrcPlain>, dim3(tiled_grid(f.tl8)), dim3(blk), 0, s,
                    f.d, f.tl8, f.cf, sc, ph));
            } else {
                PF_LAUNCH("mg_smooth0_pw", s, launch_pdl(mg_smooth0_pw, dim3(cgrid3(f.d)), dim3(blk), 0, s,
                    f.d, f.cf, f.wd, f.b, f.x, sc));
            }
        }
        if (coop && l == P.G - 1)
            PF_LAUNCH("mg_mid_down", s, launch_mid(false, P, bl, xl, sc, s));
        else
            PF_LAUNCH(l == 0 ? "mg_restrict_l0" : "mg_restrict", s, launch_pdl(mg_restrict, dim3(cgrid3h(c.d)), dim3(blk), 0, s,
                f.d, f.cf, bl, xl, c.d, c.b, sc));
    }
    if (P.C < P.B) {
        size_t fl = 0;
        const MgCluster m = cluster_params(P, &fl);
        PF_LAUNCH("mg_cluster", s, launch_cluster(m, fl * sizeof(float), P.lv[P.C].b, P.lv[P.C].x, sc, s));
    } else {
        const MgBottom m = bottom_params(P);
        const size_t smem = bottom_smem_floats(P) * sizeof(float);
        PF_LAUNCH("mg_bottom", s, launch_pdl(mg_bottom, dim3(1), dim3(kBottomThreads), smem, s,
            m, P.lv[P.B].b, P.lv[P.B].x, sc));
    }
    if (coop) {
        const int l = P.G - 1;
        PF_LAUNCH("mg_mid_up", s, launch_mid(true, P, l == 0 ? b0 : P.lv[l].b,
                                             l == 0 ? x0 : P.lv[l].x, sc, s));
    }
    for (int l = (coop ? P.G : P.C) - 1; l >= 0; --l) {
        const MgLevel& f = P.lv[l];
        const MgLevel& c = P.lv[l + 1];
        const float* bl = l == 0 ? b0 : f.b;
        float* xl = l == 0 ? x0 : f.x;
        if (f.kind == kMgSwept) {
            const char* np = l == 0 ? "mg_prolong_l0" : "mg_prolong";
            const char* ns = l == 0 ? "mg_smooth_l0" : "mg_smooth";
            if (coop && l == P.G - 1) {
                // the prolongation from level G ran in mg_mid_up
            } else if (f.d.nz % 4 == 0)
                PF_LAUNCH(np, s, launch_pdl(mg_prolong_add4, dim3((c.d.nz / 2 + 31) / 32, (c.d.ny + 7) / 8, c.d.nx),
                    dim3(blk), 0, s, f.d, c.d, c.x, xl, sc));
            else
                PF_LAUNCH(np, s, launch_pdl(mg_prolong_add, dim3(cgrid3(c.d)), dim3(blk), 0, s, f.d, c.d, c.x, xl, sc));
            if (f.az) {
                smooth_as(f, sc, AsyncSmooth{{xl}, {bl}, f.t, f.wd}, ns, s);
                smooth_as(f, sc, AsyncSmooth{{f.t}, {bl}, xl, f.wd}, ns, s);
            } else {
                PhaseSmooth a{xl, bl, f.t, f.wd};
                PF_LAUNCH(ns, s, launch_pdl(mg_smooth, dim3(tiled_grid(f.tl8)), dim3(blk), 0, s, f.d, f.tl8, f.cf, sc, a));
                PhaseSmooth b{f.t, bl, xl, f.wd};
                PF_LAUNCH(ns, s, launch_pdl(mg_smooth, dim3(tiled_grid(f.tl8)), dim3(blk), 0, s, f.d, f.tl8, f.cf, sc, b));
            }
        } else {
            PF_LAUNCH("mg_prolong_smooth_pw", s, launch_pdl(mg_prolong_smooth_pw, dim3(cgrid3(f.d)), dim3(blk), 0, s,
                f.d, c.d, f.cf, f.wd, c.x, xl, bl, f.t, sc));
            PF_LAUNCH("mg_smooth_pw", s, launch_pdl(mg_smooth_pw, dim3(cgrid3(f.d)), dim3(blk), 0, s,
                f.d, f.cf, f.wd, f.t, bl, xl, sc));
        }
    }
}

int mg_enqueue_setup(const MgPlan& P, cudaStream_t s) {
    if (P.coop && cudaMemsetAsync(P.gbar, 0, 4 * sizeof(unsigned), s) != cudaSuccess)
        return PF_ERR_CUDA;
    if (P.pinv) {
        const MgLevel& c = P.lv[P.L - 1];
        PF_LAUNCH("mg_coarse_pinv", s, launch_pdl(mg_coarse_pinv, dim3(1), dim3(256), 0, s,
            c.d, c.cq[0], c.cq[1], c.cq[2], P.pinv));
    }
    return cudaGetLastError() == cudaSuccess ? PF_OK : PF_ERR_CUDA;
}

int mg_enqueue_init(const MgPlan& P, BicgScalars* sc, double* part, const double* rhs,
                    double tol, int max_it, cudaStream_t s, double outer_tol) {
    const Dims& d = P.lv[0].d;
    PF_LAUNCH("mg_init", s, launch_pdl(mg_init, dim3(pointwise_grid(d.n)), dim3(kBlock), 0, s,
        d, sc, part, rhs, P.res, P.res0, P.e, P.p[0], P.p[1], P.v, max_it, tol, outer_tol));
    return cudaGetLastError() == cudaSuccess ? PF_OK : PF_ERR_CUDA;
}

int mg_enqueue_iteration(const MgPlan& P, BicgScalars* sc, double* part, int k,
                         cudaStream_t s, int use_cond, cudaGraphConditionalHandle cond) {
    const MgLevel& f = P.lv[0];
    const dim3 blk(32, 8);
    const int gt = tiled_grid(f.tl), gt8 = tiled_grid(f.tl8);
    float* p_new = P.p[k & 1];
    const float* p_old = P.p[(k & 1) ^ 1];
    {   // p update fused into the first smoothing pass of M p (three input
        // fields: the register sweep beats the cp.async ring here)
        PhaseSmooth0<SrcP> ph{};
        ph.src.res = P.res; ph.src.p_old = p_old; ph.src.v = P.v; ph.src.p_new = p_new;
        ph.x = P.ph; ph.wd = f.wd;
        PF_LAUNCH("mg_smooth0_p", s, launch_pdl(mg_smooth0_p, dim3(gt), dim3(blk), 0, s, f.d, f.tl, f.cf, sc, ph));
    }
    vcycle_tail(P, p_new, P.ph, sc, s);
    const int ga = tiled_grid(f.ta1);
    if (f.az == 64)
        PF_LAUNCH("mg_av", s, launch_pdl(mg_av<64>, dim3(ga), dim3(blk), async_sweep_smem<kAsTY1, 64, AsyncAv>(),
                                         s, f.d, f.ta1, f.cf, sc, part, P.ph, P.res0, P.v, use_cond, cond));
    else if (f.az == 32)
        PF_LAUNCH("mg_av", s, launch_pdl(mg_av<32>, dim3(ga), dim3(blk), async_sweep_smem<kAsTY1, 32, AsyncAv>(),
                                         s, f.d, f.ta1, f.cf, sc, part, P.ph, P.res0, P.v, use_cond, cond));
    else
        PF_LAUNCH("mg_av", s, launch_pdl(mg_av<0>, dim3(gt8), dim3(blk), 0, s, f.d, f.tl8, f.cf, sc,
                                         part, P.ph, P.res0, P.v, use_cond, cond));
    if (f.az) {  // s = res - alpha v fused into the first smoothing pass of M s
        AsyncSmooth0<AsyncS> ph{{P.s, 0.0f}, {P.res, P.v}, {nullptr}, P.sh, f.wd};
        smooth0_as<kAsTYn>(f, sc, ph, "mg_smooth0_s", s);
    } else {
        PhaseSmooth0<SrcS> ph{};
        ph.src.res = P.res; ph.src.v = P.v; ph.src.s = P.s;
        ph.x = P.sh; ph.wd = f.wd;
        PF_LAUNCH("mg_smooth0_s", s, launch_pdl(mg_smooth0<SrcS>, dim3(gt), dim3(blk), 0, s, f.d, f.tl, f.cf, sc, ph));
    }
    vcycle_tail(P, P.s, P.sh, sc, s);
    if (f.az == 64)
        PF_LAUNCH("mg_at", s, launch_pdl(mg_at<64>, dim3(ga), dim3(blk), async_sweep_smem<kAsTY1, 64, AsyncAt>(),
                                         s, f.d, f.ta1, f.cf, sc, part, P.sh, P.s, P.t));
    else if (f.az == 32)
        PF_LAUNCH("mg_at", s, launch_pdl(mg_at<32>, dim3(ga), dim3(blk), async_sweep_smem<kAsTY1, 32, AsyncAt>(),
                                         s, f.d, f.ta1, f.cf, sc, part, P.sh, P.s, P.t));
    else
        PF_LAUNCH("mg_at", s, launch_pdl(mg_at<0>, dim3(gt8), dim3(blk), 0, s, f.d, f.tl8, f.cf, sc,
                                         part, P.sh, P.s, P.t));
    PF_LAUNCH("mg_update", s, launch_pdl(mg_update, dim3(pointwise_grid(f.d.n)), dim3(kBlock), 0, s,
        f.d, sc, part, P.e, P.ph, P.sh, P.s, P.t, P.res, P.res0, use_cond, cond));
    return cudaGetLastError() == cudaSuccess ? PF_OK : PF_ERR_CUDA;
}

int mg_inner_solve(const MgPlan& P, BicgScalars* sc, double* part, const double* rhs,
                   double tol, int max_it, cudaStream_t s, BicgScalars* hs, double outer_tol) {
    int rc = mg_enqueue_init(P, sc, part, rhs, tol, std::max(1, max_it), s, outer_tol);
    if (rc) return rc;
    // with per-kernel timing on, poll after every iteration so no launch of
    // a finished solve (which returns at once) enters the kernel averages
    const bool exact = prof_on();
    int k = 0, chunk = exact ? 1 : 2;
    for (int guard = 0; guard < (1 << 20); ++guard) {
        for (int c = 0; c < chunk; ++c, ++k) {
            rc = mg_enqueue_iteration(P, sc, part, k, s);
            if (rc) return rc;
        }
        if (cudaMemcpyAsync(hs, sc, sizeof(BicgScalars), cudaMemcpyDeviceToHost, s) != cudaSuccess)
            return PF_ERR_CUDA;
        if (cudaStreamSynchronize(s) != cudaSuccess) return PF_ERR_CUDA;
        if (hs->done) return PF_OK;
        chunk = exact ? 1 : std::min(chunk * 2, 8);
    }
    return PF_ERR_CUDA;
}

}  // namespace pf
