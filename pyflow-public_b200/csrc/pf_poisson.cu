// pf_poisson.cu -- pressure Poisson solvers, divergence, projection, stats.
//
// BiCGStab (solver_bicgstab.solve, src/solver/pressure.py:196-297) with the
// operator of Pressure_Base.applyOperator (src/solver/pressure.py:54-84,
// coefficients metric_staggered.py:84-102) runs as TWO fused kernels per
// iteration, one per remaining global reduction:
//
//   kernel CA (iteration k): finish iteration k-1 and start iteration k
//     s   = res - alpha vv            (alpha, omega of iteration k-1)
//     res = s - omega t               (the reference's residual update)
//     DP += alpha pp + omega s        (two fused multiply-adds, same order)
//     pp  = (pp - omega vv) beta + res,  beta = alpha rho1 / (rho2 omega)
//     vv  = A pp,   gamma = (vv, res0),   max|res| -> stop test of k-1
//   kernel B (iteration k):
//     s = res - alpha vv,  t = A s,  (s,t), (t,t), (s,res0), (t,res0)
//     omega = (s,t)/(t,t);  rho1 of iteration k+1 = (s,res0) - omega (t,res0)
//
// Every per-element operation is the reference's (same operands, same fused
// multiply-adds: torch's add_(alpha, x) is one fma); only the scalar rho1 is
// formed from two dot products instead of (res, res0), which changes its
// rounding, not its value.  The reference needs three reductions and 17 field
// passes per iteration; this needs two and 14.
//
// Both kernels evaluate their stencil operand on the fly: a block owns a
// 32 (z) x 8R (y) tile, stages one x-plane of the operand plus its y/z halo in
// shared memory, and marches along x keeping the i-1, i, i+1 operand values of
// its own cells in registers.  The raw inputs of plane i+2 (and the halo of
// plane i+1) are loaded one iteration ahead so each thread keeps 15-30 loads
// in flight.  pp, vv and res, read at neighbours and rewritten by kernel CA,
// live in two buffer sets chosen by the parity of a device-side counter.
//
// All scalars stay in device memory; each reduction is finished by the last
// block to arrive (fixed summation order: bitwise reproducible), which also
// applies the reference's stop tests and sets a `done` flag that makes every
// later kernel of the solve return immediately.  The host only polls it.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "pf_common.cuh"
#include "pf_kernels.cuh"
#include "pf_sweep.cuh"
#include "pf_grad.cuh"
#include "pf_mg.cuh"
#include "pf_profile.cuh"

namespace pf {


// Solver vectors.  set 0/1: res, pp, vv written by kernel CA of even/odd k.
template <typename T>
struct BicgVecs {
    T* res[2];
    T* pp[2];
    T* vv[2];
    T *t, *res0;
};

// ---------------------------------------------------------------- init
// FP64 path: res = res0 = (source * rho/dt) * (-vol); DP = pp = vv = 0.
// Mixed inner pass: res = res0 = T(r / scale) where r is the FP64 residual.
// Writes buffer set 1 (read by the first kernel CA).
template <typename T, bool FROM_RESIDUAL>
__global__ void __launch_bounds__(kBlock)
bicg_init(Dims d, BicgScalars* sc, double* part, const double* src, double c1,
          double c2, BicgVecs<T> v, T* x, int max_it, double min_res) {
    __shared__ double sh[32];
    double s = 0.0, m = 0.0;
    const double inv = (FROM_RESIDUAL && sc->scale > 0.0) ? 1.0 / sc->scale : 0.0;
    T* res = v.res[1];
    T* pp = v.pp[1];
    T* vv = v.vv[1];
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < d.n;
         q += (long long)gridDim.x * blockDim.x) {
        T r;
        if (FROM_RESIDUAL) r = T(src[q] * inv);
        else r = T((src[q] * c1) * c2);
        res[q] = r;
        v.res0[q] = r;
        x[q] = T(0); pp[q] = T(0); vv[q] = T(0); v.t[q] = T(0);
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
            sc->max_res0 = mx; sc->max_res = 0.0; sc->k = 0; sc->iter = 0;
            sc->done = 0; sc->status = PF_OK; sc->max_it = max_it;
            sc->min_res = min_res; sc->counter = 0u;
        }
    }
}

// ---------------------------------------------------------------- kernel CA
template <typename T>
struct PhaseCA {
    static constexpr int R = 2;
    const T *res_o, *pp_o, *vv_o, *t, *res0;
    T *x, *res_n, *pp_n, *vv_n;
    T alpha, omega, beta;
    bool fin;  // finish the previous iteration (k > 0)
    double gam, mx;
    struct Raw { T r, p, v, t; };
    struct Ext { T x, r0; };
    __device__ Raw raw(long long q, int = 0, int = 0, int = 0) const { return Raw{res_o[q], pp_o[q], vv_o[q], t[q]}; }
    __device__ Ext ext(long long q) const { return Ext{fin ? x[q] : T(0), res0[q]}; }
    __device__ T resid(const Raw& a) const {
        if (!fin) return a.r;
        const T s = fma(-alpha, a.v, a.r);  // s = res; s.sub_(alpha, vv)
        return fma(-omega, a.t, s);         // res = s; res.sub_(omega, t)
    }
    __device__ T op(const Raw& a) const {
        const T rn = resid(a);
        T q = fma(-omega, a.v, a.p);        // pp.sub_(omega, vv)
        q = q * beta;                       // pp.mul_(beta)
        return q + rn;                      // pp.add_(res)
    }
    __device__ void epi(long long q, T c, T b, const Raw& a, const Ext& e) {
        T rn = a.r;
        if (fin) {
            const T s = fma(-alpha, a.v, a.r);
            rn = fma(-omega, a.t, s);
            T xv = fma(alpha, a.p, e.x);    // DP.add_(alpha, pp)
            x[q] = fma(omega, s, xv);       // DP.add_(omega, s)
        }
        res_n[q] = rn;
        pp_n[q] = c;
        vv_n[q] = b;
        gam += double(b) * double(e.r0);
        mx = nanmax(mx, fabs(double(rn)));
    }
};

template <typename T>
__global__ void __launch_bounds__(kBlock, 2)
bicg_ca(Dims d, Tiling tl, LapCoef<T> cf, BicgScalars* sc, double* part,
        BicgVecs<T> v, T* __restrict__ x, int use_cond = 0,
        cudaGraphConditionalHandle cond = 0) {
    __shared__ double sh[32];
    const int done = sc->done;
    if (done == 1) {
        if (use_cond && blockIdx.x == 0 && tid0()) cudaGraphSetConditional(cond, 0);
        return;
    }
    const int k = sc->k;
    const bool odd = k & 1;  // CA(k) writes set k&1 and reads the other
    if (done == 2) {
        // (t,t) == 0 breakdown: the reference has applied DP += alpha pp and
        // stops (src/solver/pressure.py:251,266-267)
        const T alpha = T(sc->alpha);
        const T* pp = odd ? v.pp[0] : v.pp[1];
        const long long nt = (long long)gridDim.x * blockDim.x * blockDim.y;
        for (long long q = blockIdx.x * (long long)blockDim.x * blockDim.y +
                           threadIdx.y * blockDim.x + threadIdx.x;
             q < d.n; q += nt)
            x[q] = fma(alpha, pp[q], x[q]);
        if (arrive_last(sc) && tid0()) {
            sc->done = 1;
            sc->counter = 0u;
            if (use_cond) cudaGraphSetConditional(cond, 0);
        }
        return;
    }
    PhaseCA<T> ph;
    ph.res_o = odd ? v.res[0] : v.res[1];
    ph.pp_o = odd ? v.pp[0] : v.pp[1];
    ph.vv_o = odd ? v.vv[0] : v.vv[1];
    ph.t = v.t; ph.res0 = v.res0; ph.x = x;
    ph.res_n = odd ? v.res[1] : v.res[0];
    ph.pp_n = odd ? v.pp[1] : v.pp[0];
    ph.vv_n = odd ? v.vv[1] : v.vv[0];
    ph.alpha = T(sc->alpha);
    ph.omega = T(sc->omega);
    ph.beta = T((sc->alpha * sc->rho1) / (sc->rho2 * sc->omega));
    ph.fin = k > 0;
    ph.gam = 0.0; ph.mx = 0.0;
    sweep<T>(d, tl, cf, ph);
    const double bs = block_sum<kBlock>(ph.gam, sh);
    const double bm = block_max<kBlock>(ph.mx, sh);
    if (tid0()) { part[blockIdx.x] = bs; part[kMaxPartials + blockIdx.x] = bm; }
    if (arrive_last(sc)) {
        const double gamma = finish<false>(part, sh);
        const double mxr = finish<true>(part + kMaxPartials, sh);
        if (tid0()) {
            bool stop = false;
            if (k > 0) {
                // stop tests of iteration k (src/solver/pressure.py:279-287)
                sc->iter = k;
                const double mr = mxr / sc->max_res0;
                sc->max_res = mr;
                if (!(mr == mr) || isinf(mr)) { stop = true; sc->status = PF_NONFINITE; }
                else if (mr <= sc->min_res) { stop = true; sc->status = PF_OK; }
                else if (k >= sc->max_it) { stop = true; sc->status = PF_MAXIT; }
            }
            if (!stop) {
                sc->gamma = gamma;
                if (gamma == 0.0) { stop = true; sc->status = PF_BREAKDOWN; }
                else sc->alpha = sc->rho1 / gamma;
            }
            if (stop) {
                sc->done = 1;
                if (use_cond) cudaGraphSetConditional(cond, 0);
            }
            sc->k = k + 1;
            sc->counter = 0u;
        }
    }
}

// ---------------------------------------------------------------- kernel B
template <typename T>
struct PhaseB {
    static constexpr int R = Rows<T>::R;
    const T *res, *vv, *res0;
    T* t;
    T alpha;
    double st, tt, sr, tr;
    struct Raw { T r, v; };
    struct Ext { T r0; };
    __device__ Raw raw(long long q, int = 0, int = 0, int = 0) const { return Raw{res[q], vv[q]}; }
    __device__ Ext ext(long long q) const { return Ext{res0[q]}; }
    __device__ T op(const Raw& a) const { return fma(-alpha, a.v, a.r); }
    __device__ void epi(long long q, T c, T b, const Raw&, const Ext& e) {
        t[q] = b;
        st += double(c) * double(b);
        tt += double(b) * double(b);
        sr += double(c) * double(e.r0);
        tr += double(b) * double(e.r0);
    }
};

template <typename T>
__global__ void __launch_bounds__(kBlock, 2)
bicg_b(Dims d, Tiling tl, LapCoef<T> cf, BicgScalars* sc, double* part,
       BicgVecs<T> v, int use_cond = 0, cudaGraphConditionalHandle cond = 0) {
    __shared__ double sh[32];
    if (sc->done) {
        if (sc->done == 1 && use_cond && blockIdx.x == 0 && tid0())
            cudaGraphSetConditional(cond, 0);
        return;
    }
    const bool odd = (sc->k - 1) & 1;  // set written by the CA kernel just run
    PhaseB<T> ph;
    ph.res = odd ? v.res[1] : v.res[0];
    ph.vv = odd ? v.vv[1] : v.vv[0];
    ph.res0 = v.res0; ph.t = v.t;
    ph.alpha = T(sc->alpha);
    ph.st = ph.tt = ph.sr = ph.tr = 0.0;
    sweep<T>(d, tl, cf, ph);
    const double b0 = block_sum<kBlock>(ph.st, sh);
    const double b1 = block_sum<kBlock>(ph.tt, sh);
    const double b2 = block_sum<kBlock>(ph.sr, sh);
    const double b3 = block_sum<kBlock>(ph.tr, sh);
    if (tid0()) {
        part[blockIdx.x] = b0;
        part[kMaxPartials + blockIdx.x] = b1;
        part[2 * kMaxPartials + blockIdx.x] = b2;
        part[3 * kMaxPartials + blockIdx.x] = b3;
    }
    if (arrive_last(sc)) {
        const double buf1 = finish<false>(part, sh);
        const double buf2 = finish<false>(part + kMaxPartials, sh);
        const double sr = finish<false>(part + 2 * kMaxPartials, sh);
        const double tr = finish<false>(part + 3 * kMaxPartials, sh);
        if (tid0()) {
            sc->buf1 = buf1; sc->buf2 = buf2;
            if (buf2 == 0.0) {
                sc->done = 2;
                sc->status = PF_BREAKDOWN;
            } else {
                const double omega = buf1 / buf2;
                sc->omega = omega;
                sc->rho2 = sc->rho1;
                sc->rho1 = sr - omega * tr;  // (s - omega t, res0)
            }
            sc->counter = 0u;
        }
    }
}

// ------------------------------------------------ mixed-precision refinement
// b = (source*rho/dt)*(-vol) in FP64, max|b|; DP = 0 unless x is null (a
// solve that starts from the DP it is given).
__global__ void __launch_bounds__(kBlock)
mixed_b_init(Dims d, BicgScalars* sc, double* part, const double* src,
             double c1, double c2, double* b, double* x, double* r_copy) {
    __shared__ double sh[32];
    double m = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < d.n;
         q += (long long)gridDim.x * blockDim.x) {
        const double r = (src[q] * c1) * c2;
        b[q] = r;
        if (x) x[q] = 0.0;
        if (r_copy) r_copy[q] = r;
        m = nanmax(m, fabs(r));
    }
    const double bm = block_max<kBlock>(m, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = bm;
    if (arrive_last(sc)) {
        const double mx = finish<true>(part, sh);
        if (threadIdx.x == 0) {
            sc->max_b = mx; sc->scale = mx; sc->true_res = mx;
            sc->outer = 0; sc->total = 0; sc->counter = 0u;
            sc->use64 = 0; sc->prev_ratio = 2.0;
        }
    }
}

// Refinement update: x += scale * e (FP64 accumulate of a pass's correction,
// scale = max|r| of the residual the pass solved for).
template <typename T>
__global__ void __launch_bounds__(kBlock)
fold_correction(Dims d, const BicgScalars* sc, const T* e, double* x, int guard = 0) {
    // graph mode: a pass that ended non-finite or in breakdown is discarded
    if (guard && (sc->status == PF_NONFINITE || sc->status == PF_BREAKDOWN)) return;
    // a pass that stopped before its first iteration has e = 0 (and may not
    // have written it)
    if (sc->iter == 0) return;
    const double s = sc->scale;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < d.n;
         q += (long long)gridDim.x * blockDim.x)
        x[q] = x[q] + s * double(e[q]);
}

// r = b - A x in FP64 and max|r| (the refinement's true residual)
struct PhaseResidual {
    static constexpr int R = 4;
    const double *x, *b;
    double* r;
    double mx;
    struct Raw { double x; };
    struct Ext { double b; };
    __device__ Raw raw(long long q, int = 0, int = 0, int = 0) const { return Raw{x[q]}; }
    __device__ Ext ext(long long q) const { return Ext{b[q]}; }
    __device__ double op(const Raw& a) const { return a.x; }
    __device__ void epi(long long q, double, double ax, const Raw&, const Ext& e) {
        const double v = e.b - ax;
        r[q] = v;
        mx = nanmax(mx, fabs(v));
    }
};

__global__ void __launch_bounds__(kBlock, 2)
mixed_residual(Dims d, Tiling tl, LapCoef<double> cf, BicgScalars* sc,
               double* part, const double* __restrict__ b,
               const double* __restrict__ x, double* __restrict__ r) {
    __shared__ double sh[32];
    PhaseResidual ph{x, b, r, 0.0};
    sweep<double>(d, tl, cf, ph);
    const double bm = block_max<kBlock>(ph.mx, sh);
    if (tid0()) part[blockIdx.x] = bm;
    if (arrive_last(sc)) {
        const double mx = finish<true>(part, sh);
        if (tid0()) { sc->true_res = mx; sc->scale = mx; sc->counter = 0u; }
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

static constexpr int kNumPartials = 4;

size_t poisson_ws_bytes(const pf_grid* g, int prec) {
    const size_t n = (size_t)g->nx * g->ny * g->nz;
    size_t b = align256(sizeof(BicgScalars)) +
               align256(kNumPartials * kMaxPartials * sizeof(double));
    if (prec == PF_FP64) {
        b += 8 * align256(n * sizeof(double));  // res[2] pp[2] vv[2] t res0
    } else {
        // inner vectors + correction: FP32 passes, or FP64 passes after an
        // FP32 pass fails (the two sets share one region), then b and r
        b += 9 * align256(n * sizeof(double));
        b += 2 * align256(n * sizeof(double));
    }
    return b;
}

template <typename T>
static BicgVecs<T> carve(char*& p, size_t n) {
    BicgVecs<T> v;
    T** f[8] = {&v.res[0], &v.res[1], &v.pp[0], &v.pp[1], &v.vv[0], &v.vv[1], &v.t, &v.res0};
    for (auto ptr : f) { *ptr = (T*)p; p += align256(n * sizeof(T)); }
    return v;
}

static LapCoef<double> cf64(const pf_grid* g) { return lap_coef<double>(g); }

static int read_scalars(BicgScalars* dev, BicgScalars* host, cudaStream_t s) {
    if (cudaMemcpyAsync(host, dev, sizeof(BicgScalars), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return PF_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PF_ERR_CUDA;
    return PF_OK;
}

// Enqueue BiCGStab iterations in chunks, polling the device `done` flag
// between chunks; kernels of a finished solve return at once.  Launch order:
// CA(0), then pairs (B(k), CA(k+1)), so every chunk ends with a CA and the
// last iteration of a chunk is finished before polling.
template <typename T>
static int run_iterations(const Dims& d, const LapCoef<T>& cf,
                          BicgScalars* sc, double* part, const BicgVecs<T>& v,
                          T* x, cudaStream_t s, BicgScalars* hs) {
    const Tiling ta = make_tiling(d, 8 * PhaseCA<T>::R);
    const Tiling tb = make_tiling(d, 8 * PhaseB<T>::R);
    const int ga = tiled_grid(ta), gb = tiled_grid(tb);
    dim3 blk2(32, 8);
    const char* nca = sizeof(T) == 8 ? "bicg_ca_f64" : "bicg_ca_f32";
    const char* nb = sizeof(T) == 8 ? "bicg_b_f64" : "bicg_b_f32";
    PF_LAUNCH(nca, s, bicg_ca<T><<<ga, blk2, 0, s>>>(d, ta, cf, sc, part, v, x));
    // with per-kernel timing on, poll after every iteration so no launch of
    // a finished solve (which returns at once) enters the kernel averages
    const bool exact = prof_on();
    int chunk = exact ? 1 : 4;
    for (int guard = 0; guard < (1 << 20); ++guard) {
        for (int c = 0; c < chunk; ++c) {
            PF_LAUNCH(nb, s, bicg_b<T><<<gb, blk2, 0, s>>>(d, tb, cf, sc, part, v));
            PF_LAUNCH(nca, s, bicg_ca<T><<<ga, blk2, 0, s>>>(d, ta, cf, sc, part, v, x));
        }
        if (cudaGetLastError() != cudaSuccess) return PF_ERR_CUDA;
        const int rc = read_scalars(sc, hs, s);
        if (rc) return rc;
        if (hs->done == 1) return PF_OK;
        chunk = exact ? 1 : std::min(chunk * 2, 32);
    }
    return PF_ERR_CUDA;
}

int bicgstab_solve(const pf_grid* g, int prec, double rho, double dt,
                   double min_res, int max_it, const double* source,
                   double* DP, double* p, void* ws, cudaStream_t s,
                   pf_solve_info* info) {
    // PF_WARM_START (mixed forms): the refinement starts from the DP given
    const bool warm = (prec & PF_WARM_START) != 0 && (prec & 0xFF) != PF_FP64;
    prec &= 0xFF;
    Dims d{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    const size_t n = (size_t)d.n;
    char* ptr = (char*)ws;
    BicgScalars* sc = (BicgScalars*)ptr; ptr += align256(sizeof(BicgScalars));
    double* part = (double*)ptr; ptr += align256(kNumPartials * kMaxPartials * sizeof(double));
    const int gp = pointwise_grid(d.n);
    const double vol = (g->dx * g->dy) * g->dz;
    const double c1 = rho / dt, c2 = -1.0 * vol;
    BicgScalars hs;
    std::memset(&hs, 0, sizeof(hs));
    if (cudaMemsetAsync(sc, 0, sizeof(BicgScalars), s) != cudaSuccess) return PF_ERR_CUDA;
    pf_solve_info out{0.0, 0, 1, PF_OK};
    // the reference loop always runs at least one iteration
    max_it = std::max(max_it, 1);
    if (prec == PF_FP64) {
        BicgVecs<double> v = carve<double>(ptr, n);
        const LapCoef<double> cf = lap_coef<double>(g);
        PF_LAUNCH("bicg_init_f64", s, bicg_init<double, false><<<gp, kBlock, 0, s>>>(
            d, sc, part, source, c1, c2, v, DP, max_it, min_res));
        int rc = run_iterations<double>(d, cf, sc, part, v, DP, s, &hs);
        if (rc) return rc;
        out.max_res = hs.max_res; out.iterations = hs.iter; out.status = hs.status;
    } else {
        // Iterative refinement: each pass solves A e = r / max|r| with BiCGStab
        // on FP32 vectors (FP64 dot products) to kInnerTol, then
        // x += max|r| e and r = b - A x in FP64, until max|r| / max|b| reaches
        // the reference's tolerance.  A pass that ends non-finite or in
        // breakdown is discarded, and a pass that gains less than 2x switches
        // the solve to FP64 inner passes, so the refinement always converges
        // like the FP64 solver.
        char* region = ptr;
        BicgVecs<float> v32 = carve<float>(ptr, n);
        float* e32 = (float*)ptr;
        ptr = region + 9 * align256(n * sizeof(double));
        char* r64 = region;
        BicgVecs<double> v64 = carve<double>(r64, n);
        double* e64 = (double*)r64;
        double* b = (double*)ptr; ptr += align256(n * sizeof(double));
        double* r = (double*)ptr; ptr += align256(n * sizeof(double));
        const Tiling tld = make_tiling(d, 8 * PhaseResidual::R);
        const LapCoef<float> cf = lap_coef<float>(g);
        const LapCoef<double> cfd = lap_coef<double>(g);
        const double kInnerTol = 1e-4;
        const int kMaxOuter = 40;
        // PF_MIXED_MG: the FP32 passes run the multigrid-preconditioned solver
        // (its vectors share the same region) when the grid coarsens
        MgPlan mg;
        if (prec == PF_MIXED_MG && mg_region_bytes(g) <= 9 * align256(n * sizeof(double))) {
            const int rc = mg_setup(g, region, &mg);
            if (rc != PF_OK && rc != PF_ERR_BAD_ARG) return rc;
            if (mg.L && mg_enqueue_setup(mg, s) != PF_OK) return PF_ERR_CUDA;
        }
        PF_LAUNCH("mixed_b_init", s, mixed_b_init<<<gp, kBlock, 0, s>>>(d, sc, part, source, c1, c2, b,
                                                                       warm ? nullptr : DP, nullptr));
        if (read_scalars(sc, &hs, s)) return PF_ERR_CUDA;
        const double max_b = hs.max_b;
        int status = PF_OK, outer = 0, total = 0;
        bool use64 = false;
        double ratio = max_b > 0 ? 1.0 : 0.0, prev_ratio = 2.0;
        if (!(max_b == max_b)) status = PF_NONFINITE;
        while (status == PF_OK && max_b > 0.0) {
            if (outer > 0 || warm) {
                PF_LAUNCH("mixed_residual", s, mixed_residual<<<tiled_grid(tld), dim3(32, 8), 0, s>>>(
                    d, tld, cfd, sc, part, b, DP, r));
                if (read_scalars(sc, &hs, s)) return PF_ERR_CUDA;
                ratio = hs.true_res / max_b;
            }
            if (!(ratio == ratio) || std::isinf(ratio)) { status = PF_NONFINITE; break; }
            if (ratio <= min_res) break;
            if (outer >= kMaxOuter || total >= max_it) { status = PF_MAXIT; break; }
            if (!use64 && outer > 1 && ratio > 0.5 * prev_ratio) use64 = true;
            prev_ratio = ratio;
            const double* rhs = (outer == 0 && !warm) ? b : r;
            ++outer;
            if (!use64) {
                float* e = e32;
                if (mg.L) {
                    const int rc = mg_inner_solve(mg, sc, part, rhs, kInnerTol, max_it - total, s,
                                                  &hs, min_res);
                    if (rc) return rc;
                    e = mg.e;
                } else {
                    PF_LAUNCH("bicg_init_f32", s, bicg_init<float, true><<<gp, kBlock, 0, s>>>(
                        d, sc, part, rhs, 0.0, 0.0, v32, e32, max_it - total, kInnerTol));
                    const int rc = run_iterations<float>(d, cf, sc, part, v32, e32, s, &hs);
                    if (rc) return rc;
                }
                total += hs.iter;
                if (hs.status == PF_NONFINITE || hs.status == PF_BREAKDOWN) {
                    use64 = true;  // discard this pass: x is unchanged
                    continue;
                }
                PF_LAUNCH("fold_correction", s, fold_correction<float><<<gp, kBlock, 0, s>>>(d, sc, e, DP));
            } else {
                // an FP64 pass finishes the solve: its tolerance is the
                // remaining reduction
                const double tol64 = std::min(0.5, 0.5 * min_res / ratio);
                PF_LAUNCH("bicg_init_f64", s, bicg_init<double, true><<<gp, kBlock, 0, s>>>(
                    d, sc, part, rhs, 0.0, 0.0, v64, e64, max_it - total, tol64));
                const int rc = run_iterations<double>(d, cf64(g), sc, part, v64, e64, s, &hs);
                if (rc) return rc;
                total += hs.iter;
                if (hs.status == PF_NONFINITE) { status = PF_NONFINITE; break; }
                PF_LAUNCH("fold_correction", s, fold_correction<double><<<gp, kBlock, 0, s>>>(d, sc, e64, DP));
            }
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
struct PhaseJacobiRes {
    static constexpr int R = 2;
    const double *p, *sdx;
    double dx2, mx;
    struct Raw { double p; };
    struct Ext { double s; };
    __device__ Raw raw(long long q, int = 0, int = 0, int = 0) const { return Raw{p[q]}; }
    __device__ Ext ext(long long q) const { return Ext{sdx[q]}; }
    __device__ double op(const Raw& a) const { return a.p; }
    __device__ void epi(long long, double, double ax, const Raw&, const Ext& e) {
        const double v = ax * -1.0 + e.s / dx2;
        mx = nanmax(mx, fabs(v));
    }
};

__global__ void __launch_bounds__(kBlock, 2)
jacobi_residual(Dims d, Tiling tl, LapCoef<double> cf, BicgScalars* sc,
                double* part, const double* __restrict__ sdx, double dx2,
                const double* __restrict__ p) {
    __shared__ double sh[32];
    PhaseJacobiRes ph{p, sdx, dx2, 0.0};
    sweep<double>(d, tl, cf, ph);
    const double bm = block_max<kBlock>(ph.mx, sh);
    if (tid0()) part[blockIdx.x] = bm;
    if (arrive_last(sc)) {
        const double mx = finish<true>(part, sh);
        if (tid0()) { sc->max_res = mx / sc->max_res0; sc->counter = 0u; }
    }
}

int jacobi_solve(const pf_grid* g, double rho, double dt, int n_it,
                 const double* source, double* pold, double* p, void* ws,
                 cudaStream_t s, double* max_res) {
    Dims d{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    const size_t n = (size_t)d.n;
    char* ptr = (char*)ws;
    BicgScalars* sc = (BicgScalars*)ptr; ptr += align256(sizeof(BicgScalars));
    double* part = (double*)ptr; ptr += align256(kNumPartials * kMaxPartials * sizeof(double));
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
    const Tiling tl = make_tiling(d, 8 * PhaseJacobiRes::R);
    PF_LAUNCH("jacobi_residual", s, jacobi_residual<<<tiled_grid(tl), dim3(32, 8), 0, s>>>(d, tl, lap_coef<double>(g), sc, part, sdx, dx2, p));
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

// max|u|, max|v|, max|w|, sum(u^2+v^2+w^2), max|div u| (and, with DISS, the
// sum of S_ij S_ij of the cell-centred strain rate): one warp per (i, j) row
// of cells, its lanes along z (row and neighbour-row offsets computed once per
// row).  out[3] = TKE = 0.5 <u^2 + v^2 + w^2>, out[5] = 2 nu <S_ij S_ij>.
template <bool DISS>
__global__ void __launch_bounds__(256)
stats_kernel(Dims d, BicgScalars* sc, double* part, const double* __restrict__ u,
             const double* __restrict__ v, const double* __restrict__ w,
             double dxi, double dyi, double dzi, double nu, double* out) {
    constexpr int NC = DISS ? 6 : 5;
    __shared__ double sh[32];
    double mu_ = 0, mv = 0, mw = 0, s = 0, md = 0, ss = 0;
    const int lane = threadIdx.x & 31;
    const int nrows = d.nx * d.ny, wpb = blockDim.x >> 5;
    for (int row = blockIdx.x * wpb + (threadIdx.x >> 5); row < nrows; row += gridDim.x * wpb) {
        const int i = row / d.ny, j = row - i * d.ny;
        const long long base = (long long)row * d.nz;
        const long long bx = ((long long)wrap(i + 1, d.nx) * d.ny + j) * d.nz;
        const long long by = ((long long)i * d.ny + wrap(j + 1, d.ny)) * d.nz;
        for (int k = lane; k < d.nz; k += 32) {
            const long long q = base + k;
            const double a = u[q], b = v[q], c = w[q];
            mu_ = nanmax(mu_, fabs(a)); mv = nanmax(mv, fabs(b)); mw = nanmax(mw, fabs(c));
            s += (a * a + b * b) + c * c;
            double dv = (u[bx + k] - a) * dxi;
            dv += (v[by + k] - b) * dyi;
            dv += (w[base + wrap(k + 1, d.nz)] - c) * dzi;
            md = nanmax(md, fabs(dv));
            if (DISS) {
                const Grad9 g = grad_center(d, u, v, w, i, j, k, dxi, dyi, dzi);
                const double s12 = 0.5 * (g.uy + g.vx);
                const double s13 = 0.5 * (g.uz + g.wx);
                const double s23 = 0.5 * (g.vz + g.wy);
                ss += ((g.ux * g.ux + g.vy * g.vy) + g.wz * g.wz) +
                      2.0 * ((s12 * s12 + s13 * s13) + s23 * s23);
            }
        }
    }
    double r[6] = {block_max<kBlock>(mu_, sh), block_max<kBlock>(mv, sh),
                   block_max<kBlock>(mw, sh), block_sum<kBlock>(s, sh),
                   block_max<kBlock>(md, sh), DISS ? block_sum<kBlock>(ss, sh) : 0.0};
    if (threadIdx.x == 0)
        for (int c = 0; c < NC; ++c) part[c * kMaxPartials + blockIdx.x] = r[c];
    if (arrive_last(sc)) {
        double f[6];
        for (int c = 0; c < NC; ++c)
            f[c] = (c == 3 || c == 5) ? finish<false>(part + c * kMaxPartials, sh)
                                      : finish<true>(part + c * kMaxPartials, sh);
        if (threadIdx.x == 0) {
            out[0] = f[0]; out[1] = f[1]; out[2] = f[2];
            out[3] = f[3] / double(d.n) * 0.5;
            out[4] = f[4];
            if (DISS) out[5] = 2.0 * nu * (f[5] / double(d.n));
            sc->counter = 0u;
        }
    }
}

size_t stats_ws_bytes(const pf_grid*) {
    return align256(sizeof(BicgScalars)) + align256(6 * kMaxPartials * sizeof(double));
}

static cudaError_t launch_stats_impl(const pf_grid* g, const double* u, const double* v,
                                     const double* w, bool diss, double nu, double* out,
                                     void* ws, cudaStream_t s) {
    Dims d{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    char* ptr = (char*)ws;
    BicgScalars* sc = (BicgScalars*)ptr; ptr += align256(sizeof(BicgScalars));
    double* part = (double*)ptr;
    cudaMemsetAsync(sc, 0, sizeof(BicgScalars), s);
    const double dxi = 1.0 / g->dx, dyi = 1.0 / g->dy, dzi = 1.0 / g->dz;
    if (diss)
        PF_LAUNCH("flow_stats", s, stats_kernel<true><<<pointwise_grid(d.n), kBlock, 0, s>>>(
            d, sc, part, u, v, w, dxi, dyi, dzi, nu, out));
    else
        PF_LAUNCH("stats", s, stats_kernel<false><<<pointwise_grid(d.n), kBlock, 0, s>>>(
            d, sc, part, u, v, w, dxi, dyi, dzi, 0.0, out));
    return cudaGetLastError();
}

cudaError_t launch_stats(const pf_grid* g, const double* u, const double* v,
                         const double* w, double* out, void* ws, cudaStream_t s) {
    return launch_stats_impl(g, u, v, w, false, 0.0, out, ws, s);
}

cudaError_t launch_flow_stats(const pf_grid* g, const double* u, const double* v,
                              const double* w, double nu, double* out, void* ws,
                              cudaStream_t s) {
    return launch_stats_impl(g, u, v, w, true, nu, out, ws, s);
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


// ============================================================================
// Whole time step as one CUDA graph.
//
// The step (predictor, divergence, Poisson solve, p += DP, projection,
// statistics) is captured once per plan; the BiCGStab iteration loop is a
// conditional WHILE node whose body is (kernel B, kernel CA): kernel CA clears
// the condition when the solve stops (converged, iteration limit, breakdown,
// non-finite), so a whole step runs without any host synchronisation.  The
// mixed-precision refinement is an outer WHILE node (inner pass, fold,
// FP64 residual, control) cleared by the control kernel.  A pass that ends
// non-finite or in breakdown is discarded and ends the solve with that status
// (the host-driven solve switches to FP64 passes instead).  Every kernel that
// can find the solve already stopped clears the condition as well, so each
// loop ends after at most max_it iterations.
// ============================================================================

// Refinement control (one thread): after the FP64 residual of a pass, count the
// pass and its inner iterations and decide whether another pass runs, with
// the host-driven solve's rules: an FP32 pass that ended non-finite or in
// breakdown was discarded (its fold skipped) and the solve continues with
// FP64 passes, as it does once two FP32 passes in a row gain less than 2x.
__global__ void mixed_control(BicgScalars* sc, double min_res, int max_outer,
                              int max_it, cudaGraphConditionalHandle cond) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    sc->outer += 1;
    sc->total += sc->iter;
    // max|b| == 0: nothing to solve; a NaN max|b| gives a NaN ratio
    const double ratio = sc->max_b == 0.0 ? 0.0 : sc->true_res / sc->max_b;
    const int pass = sc->status;  // status of the inner pass just run
    const bool failed32 = !sc->use64 && (pass == PF_NONFINITE || pass == PF_BREAKDOWN);
    bool stop = true;
    if (sc->use64 && pass == PF_NONFINITE) sc->status = PF_NONFINITE;
    else if (!(ratio == ratio) || isinf(ratio)) sc->status = PF_NONFINITE;
    else if (ratio <= min_res) sc->status = PF_OK;
    else if (sc->outer >= max_outer || sc->total >= max_it) sc->status = PF_MAXIT;
    else stop = false;
    if (!stop) {
        if (failed32 || (!sc->use64 && sc->outer > 1 && ratio > 0.5 * sc->prev_ratio))
            sc->use64 = 1;
        sc->prev_ratio = ratio;
    }
    sc->max_res = ratio;
    if (stop) cudaGraphSetConditional(cond, 0);
}

// Start of a refinement pass: choose the FP64 or the FP32 pass.
__global__ void pass_branch(const BicgScalars* sc, cudaGraphConditionalHandle if64) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    cudaGraphSetConditional(if64, sc->use64 ? 1u : 0u);
}

// An FP64 pass finishes the solve: its inner tolerance is the remaining
// reduction (set after bicg_init, before the first kernel CA reads it).
__global__ void pass_tol64(BicgScalars* sc, double min_res) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double ratio = sc->max_b == 0.0 ? 0.0 : sc->true_res / sc->max_b;
    sc->min_res = ratio > 0.0 ? fmin(0.5, 0.5 * min_res / ratio) : 0.5;
}

// x += scale * e of the pass just run (its precision is sc->use64); an FP32
// pass that ended non-finite or in breakdown is discarded.
__global__ void __launch_bounds__(kBlock)
fold_mixed(Dims d, const BicgScalars* sc, const float* e32, const double* e64, double* x) {
    const bool f64 = sc->use64 != 0;
    if (!f64 && (sc->status == PF_NONFINITE || sc->status == PF_BREAKDOWN)) return;
    if (f64 && sc->status == PF_NONFINITE) return;
    if (sc->iter == 0) return;  // no iteration ran: e = 0, possibly unwritten
    const double s = sc->scale;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < d.n;
         q += (long long)gridDim.x * blockDim.x)
        x[q] = x[q] + s * (f64 ? e64[q] : double(e32[q]));
}

// copy the solve's result next to the monitor statistics:
// info[0] = max_res, info[1] = iterations, info[2] = status,
// info[3] += iterations and info[4] += 1 (running totals over launches)
__global__ void step_info(const BicgScalars* sc, int mixed, double* info) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double it = double(mixed ? sc->total : sc->iter);
    info[0] = sc->max_res;
    info[1] = it;
    info[2] = double(sc->status);
    info[3] += it;
    info[4] += 1.0;
}

struct StepPlan {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

static int capture_begin(cudaStream_t cs, cudaGraph_t target) {
    cudaError_t e = target ? cudaStreamBeginCaptureToGraph(cs, target, nullptr, nullptr, 0,
                                                          cudaStreamCaptureModeThreadLocal)
                           : cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    return e == cudaSuccess ? PF_OK : PF_ERR_CUDA;
}

static int capture_end(cudaStream_t cs, cudaGraph_t* g) {
    return cudaStreamEndCapture(cs, g) == cudaSuccess ? PF_OK : PF_ERR_CUDA;
}

// Re-arms a WHILE condition (the default value is applied only when the
// whole graph is launched, not each time a nested loop is entered).
__global__ void arm_condition(cudaGraphConditionalHandle h) {
    if (threadIdx.x == 0 && blockIdx.x == 0) cudaGraphSetConditional(h, 1);
}

// Adds a WHILE node after `dep` whose body is returned in *body.  With
// `make_handle` the handle (default 1 at every graph launch) is created here
// and written to *handle; otherwise *handle is used as given.
static int add_while(cudaGraph_t g, cudaGraphNode_t dep, cudaGraphNode_t* node,
                     cudaGraph_t* body, cudaGraphConditionalHandle* handle,
                     bool make_handle = true) {
    if (make_handle &&
        cudaGraphConditionalHandleCreate(handle, g, 1, cudaGraphCondAssignDefault) != cudaSuccess)
        return PF_ERR_CUDA;
    cudaGraphNodeParams prm = {cudaGraphNodeTypeConditional};
    prm.conditional.handle = *handle;
    prm.conditional.type = cudaGraphCondTypeWhile;
    prm.conditional.size = 1;
    if (cudaGraphAddNode(node, g, dep ? &dep : nullptr, dep ? 1 : 0, &prm) != cudaSuccess)
        return PF_ERR_CUDA;
    *body = prm.conditional.phGraph_out[0];
    return PF_OK;
}

static int add_child(cudaGraph_t g, cudaGraphNode_t dep, cudaGraph_t child,
                     cudaGraphNode_t* node) {
    return cudaGraphAddChildGraphNode(node, g, dep ? &dep : nullptr, dep ? 1 : 0, child) ==
                   cudaSuccess ? PF_OK : PF_ERR_CUDA;
}

// Plan workspace: [div: n doubles][scalar block][reduction partials][region R]
// R holds, at different times of the step, the predictor's stage buffers, the
// solver vectors and the statistics scratch.  The scalar block is written only
// by the solver kernels.
static constexpr size_t kPlanPinvBytes = (size_t)kMgPinvMax * kMgPinvMax * sizeof(float);

size_t step_plan_ws_bytes(const pf_grid* g, int prec) {
    const size_t n = (size_t)g->nx * g->ny * g->nz;
    size_t vecs = prec == PF_FP64 ? 8 * align256(n * sizeof(double))
                                  : 11 * align256(n * sizeof(double));
    size_t r = std::max(std::max(predictor_ws_bytes(g, prec), vecs), stats_ws_bytes(g));
    // PF_MIXED_MG: the coarsest level's pseudo-inverse in a slot of its own
    // (the region r is reused by the predictor every step), computed once
    const size_t pinv = prec == PF_MIXED_MG ? kPlanPinvBytes + kMgBarrierBytes : 0;
    return align256(n * sizeof(double)) + align256(sizeof(BicgScalars)) +
           align256(kNumPartials * kMaxPartials * sizeof(double)) + align256(r) + pinv;
}

// Pointers of one request's plan workspace (see step_plan_ws_bytes).
struct PlanLayout {
    Dims d;
    double* div;
    BicgScalars* sc;
    double* part;
    char* R;
    BicgVecs<double> v64;
    BicgVecs<float> v32;
    float* e32;
    double *bb, *rr;
    MgPlan mg;
};

static int plan_layout(const pf_grid* g, int prec, void* ws, PlanLayout* L) {
    L->d = Dims{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    const size_t n = (size_t)L->d.n;
    char* ptr = (char*)ws;
    L->div = (double*)ptr; ptr += align256(n * sizeof(double));
    L->sc = (BicgScalars*)ptr; ptr += align256(sizeof(BicgScalars));
    L->part = (double*)ptr; ptr += align256(kNumPartials * kMaxPartials * sizeof(double));
    L->R = ptr;
    // FP64 vectors, or FP32 vectors + correction followed by b and r (FP64)
    char* vp = L->R;
    L->v64 = carve<double>(vp, n);
    vp = L->R;
    L->v32 = carve<float>(vp, n);
    L->e32 = (float*)vp;
    L->bb = (double*)(L->R + 9 * align256(n * sizeof(double)));
    L->rr = (double*)(L->R + 10 * align256(n * sizeof(double)));
    // PF_MIXED_MG: multigrid-preconditioned inner passes when the grid
    // coarsens (vectors in the region of the FP32 solver vectors)
    L->mg = MgPlan();
    if (prec == PF_MIXED_MG && mg_region_bytes(g) <= 9 * align256(n * sizeof(double))) {
        const int e = mg_setup(g, L->R, &L->mg);
        if (e != PF_OK && e != PF_ERR_BAD_ARG) return e;
        // the pseudo-inverse lives in the last slot of the workspace, outside
        // the region the predictor overwrites, and is computed once here
        if (L->mg.L && L->mg.pinv)
            L->mg.pinv = (float*)((char*)ws + step_plan_ws_bytes(g, prec) - kPlanPinvBytes -
                                  kMgBarrierBytes);
        // the grid-barrier words too: the region is rewritten every step
        if (L->mg.L)
            L->mg.gbar = (unsigned*)((char*)ws + step_plan_ws_bytes(g, prec) - kMgBarrierBytes);
    }
    return PF_OK;
}

// Adds one request's step after the predictor (node `dep`) to graph G:
// divergence and solver set-up, the solver's WHILE loop(s), then p += DP,
// the projection and the monitor statistics.  *end gets the last node.
static int add_solve_chain(cudaGraph_t G, cudaGraphNode_t dep, const pf_grid* g, int prec,
                           PlanLayout& P, double* u, double* v, double* w, double* p,
                           double* DP, double rho, double dt, double min_res, int max_it,
                           double* stats, cudaStream_t cs, cudaGraphNode_t* end) {
    const Dims d = P.d;
    BicgScalars* sc = P.sc;
    double* part = P.part;
    const int gp = pointwise_grid(d.n);
    const double vol = (g->dx * g->dy) * g->dz;
    const double c1 = rho / dt, c2 = -1.0 * vol;
    max_it = std::max(max_it, 1);
    dim3 blk2(32, 8);
    int rc = PF_OK;
    // ---- divergence, solver set-up
    cudaGraph_t seg1 = nullptr;
    if ((rc = capture_begin(cs, nullptr))) return rc;
    launch_div(g, u, v, w, P.div, cs);
    if (prec == PF_FP64) {
        const LapCoef<double> cf = lap_coef<double>(g);
        const Tiling ta = make_tiling(d, 8 * PhaseCA<double>::R);
        bicg_init<double, false><<<gp, kBlock, 0, cs>>>(d, sc, part, P.div, c1, c2, P.v64, DP,
                                                       max_it, min_res);
        bicg_ca<double><<<tiled_grid(ta), blk2, 0, cs>>>(d, ta, cf, sc, part, P.v64, DP);
    } else {
        // the refinement starts from the previous step's DP (zero before the
        // first step): its first residual is r = b - A DP, and the stop test
        // stays the reference's, max|b - A DP| <= min_res max|b|
        const Tiling tld = make_tiling(d, 8 * PhaseResidual::R);
        mixed_b_init<<<gp, kBlock, 0, cs>>>(d, sc, part, P.div, c1, c2, P.bb, nullptr, nullptr);
        mixed_residual<<<tiled_grid(tld), blk2, 0, cs>>>(d, tld, lap_coef<double>(g), sc, part,
                                                        P.bb, DP, P.rr);
    }
    if ((rc = capture_end(cs, &seg1))) return rc;
    cudaGraphNode_t n1, nw;
    rc = add_child(G, dep, seg1, &n1);
    cudaGraphDestroy(seg1);
    if (rc) return rc;
    cudaGraph_t body;
    cudaGraphConditionalHandle h;
    if ((rc = add_while(G, n1, &nw, &body, &h))) return rc;
    if (prec == PF_FP64) {
        const LapCoef<double> cf = lap_coef<double>(g);
        const Tiling ta = make_tiling(d, 8 * PhaseCA<double>::R);
        const Tiling tb = make_tiling(d, 8 * PhaseB<double>::R);
        if ((rc = capture_begin(cs, body))) return rc;
        bicg_b<double><<<tiled_grid(tb), blk2, 0, cs>>>(d, tb, cf, sc, part, P.v64, 1, h);
        bicg_ca<double><<<tiled_grid(ta), blk2, 0, cs>>>(d, ta, cf, sc, part, P.v64, DP, 1, h);
        if ((rc = capture_end(cs, &body))) return rc;
    } else {
        const LapCoef<float> cf = lap_coef<float>(g);
        const LapCoef<double> cfd = lap_coef<double>(g);
        const Tiling ta = make_tiling(d, 8 * PhaseCA<float>::R);
        const Tiling tb = make_tiling(d, 8 * PhaseB<float>::R);
        const Tiling tld = make_tiling(d, 8 * PhaseResidual::R);
        const double kInnerTol = 1e-4;
        const MgPlan& mg = P.mg;
        float* ecorr = mg.L ? mg.e : P.e32;
        // FP64 inner vectors (the same region: a pass uses one set)
        char* r64 = P.R;
        BicgVecs<double> v64 = carve<double>(r64, (size_t)d.n);
        double* e64 = (double*)r64;
        const LapCoef<double> cf64 = lap_coef<double>(g);
        const Tiling ta64 = make_tiling(d, 8 * PhaseCA<double>::R);
        const Tiling tb64 = make_tiling(d, 8 * PhaseB<double>::R);
        // outer body: branch kernel, IF(use64) {FP64 pass} ELSE {FP32 pass},
        // then fold + residual + control
        cudaGraphConditionalHandle h32, h64, hif;
        if (cudaGraphConditionalHandleCreate(&hif, body, 0, cudaGraphCondAssignDefault) !=
                cudaSuccess)
            return PF_ERR_CUDA;
        // a one-thread kernel node: func(args...) with the given argument list
        auto add_tiny = [](cudaGraph_t gr, void* func, void** args, cudaGraphNode_t* node) {
            cudaKernelNodeParams kp;
            std::memset(&kp, 0, sizeof(kp));
            kp.func = func;
            kp.gridDim = dim3(1);
            kp.blockDim = dim3(32);
            kp.kernelParams = args;
            return cudaGraphAddKernelNode(node, gr, nullptr, 0, &kp) == cudaSuccess ? PF_OK
                                                                                     : PF_ERR_CUDA;
        };
        cudaGraphNode_t b0, bif, b3;
        {
            BicgScalars* scp = sc;
            void* args[] = {&scp, &hif};
            if ((rc = add_tiny(body, (void*)pass_branch, args, &b0))) return rc;
        }
        cudaGraph_t br64, br32;
        {
            cudaGraphNodeParams prm = {cudaGraphNodeTypeConditional};
            prm.conditional.handle = hif;
            prm.conditional.type = cudaGraphCondTypeIf;
            prm.conditional.size = 2;
            if (cudaGraphAddNode(&bif, body, &b0, 1, &prm) != cudaSuccess) return PF_ERR_CUDA;
            br64 = prm.conditional.phGraph_out[0];
            br32 = prm.conditional.phGraph_out[1];
        }
        // FP32 branch: re-arm its loop, set-up, then the inner WHILE (the
        // handle belongs to the branch graph that holds the loop)
        {
            cudaGraph_t pre = nullptr, inner_body = nullptr;
            cudaGraphNode_t a0, c1n, cw;
            if (cudaGraphConditionalHandleCreate(&h32, br32, 1, cudaGraphCondAssignDefault) !=
                cudaSuccess)
                return PF_ERR_CUDA;
            void* args[] = {&h32};
            if ((rc = add_tiny(br32, (void*)arm_condition, args, &a0))) return rc;
            if ((rc = capture_begin(cs, nullptr))) return rc;
            if (mg.L) {
                mg_enqueue_init(mg, sc, part, P.rr, kInnerTol, max_it, cs, min_res);
            } else {
                bicg_init<float, true><<<gp, kBlock, 0, cs>>>(d, sc, part, P.rr, 0.0, 0.0, P.v32,
                                                             P.e32, max_it, kInnerTol);
                bicg_ca<float><<<tiled_grid(ta), blk2, 0, cs>>>(d, ta, cf, sc, part, P.v32,
                                                               P.e32);
            }
            if ((rc = capture_end(cs, &pre))) return rc;
            rc = add_child(br32, a0, pre, &c1n);
            cudaGraphDestroy(pre);
            if (rc) return rc;
            if ((rc = add_while(br32, c1n, &cw, &inner_body, &h32, false))) return rc;
            if ((rc = capture_begin(cs, inner_body))) return rc;
            if (mg.L) {
                // two iterations per pass of the body: the p buffers alternate
                mg_enqueue_iteration(mg, sc, part, 0, cs, 1, h32);
                mg_enqueue_iteration(mg, sc, part, 1, cs, 1, h32);
            } else {
                bicg_b<float><<<tiled_grid(tb), blk2, 0, cs>>>(d, tb, cf, sc, part, P.v32, 1,
                                                              h32);
                bicg_ca<float><<<tiled_grid(ta), blk2, 0, cs>>>(d, ta, cf, sc, part, P.v32,
                                                               P.e32, 1, h32);
            }
            if ((rc = capture_end(cs, &inner_body))) return rc;
        }
        // FP64 branch: re-arm, set-up with the remaining tolerance, its WHILE
        {
            cudaGraph_t pre = nullptr, inner_body = nullptr;
            cudaGraphNode_t a0, c1n, cw;
            if (cudaGraphConditionalHandleCreate(&h64, br64, 1, cudaGraphCondAssignDefault) !=
                cudaSuccess)
                return PF_ERR_CUDA;
            void* args[] = {&h64};
            if ((rc = add_tiny(br64, (void*)arm_condition, args, &a0))) return rc;
            if ((rc = capture_begin(cs, nullptr))) return rc;
            bicg_init<double, true><<<gp, kBlock, 0, cs>>>(d, sc, part, P.rr, 0.0, 0.0, v64, e64,
                                                          max_it, 0.5);
            pass_tol64<<<1, 32, 0, cs>>>(sc, min_res);
            bicg_ca<double><<<tiled_grid(ta64), blk2, 0, cs>>>(d, ta64, cf64, sc, part, v64, e64);
            if ((rc = capture_end(cs, &pre))) return rc;
            rc = add_child(br64, a0, pre, &c1n);
            cudaGraphDestroy(pre);
            if (rc) return rc;
            if ((rc = add_while(br64, c1n, &cw, &inner_body, &h64, false))) return rc;
            if ((rc = capture_begin(cs, inner_body))) return rc;
            bicg_b<double><<<tiled_grid(tb64), blk2, 0, cs>>>(d, tb64, cf64, sc, part, v64, 1, h64);
            bicg_ca<double><<<tiled_grid(ta64), blk2, 0, cs>>>(d, ta64, cf64, sc, part, v64, e64,
                                                              1, h64);
            if ((rc = capture_end(cs, &inner_body))) return rc;
        }
        cudaGraph_t post = nullptr;
        if ((rc = capture_begin(cs, nullptr))) return rc;
        fold_mixed<<<gp, kBlock, 0, cs>>>(d, sc, ecorr, e64, DP);
        mixed_residual<<<tiled_grid(tld), blk2, 0, cs>>>(d, tld, cfd, sc, part, P.bb, DP, P.rr);
        mixed_control<<<1, 32, 0, cs>>>(sc, min_res, 40, max_it, h);
        if ((rc = capture_end(cs, &post))) return rc;
        rc = add_child(body, bif, post, &b3);
        cudaGraphDestroy(post);
        if (rc) return rc;
    }
    // ---- p += DP, projection, statistics
    cudaGraph_t seg3 = nullptr;
    if ((rc = capture_begin(cs, nullptr))) return rc;
    step_info<<<1, 32, 0, cs>>>(sc, prec != PF_FP64 ? 1 : 0, stats + 5);
    add_inplace<<<gp, kBlock, 0, cs>>>(d.n, DP, p);
    launch_vel_corr(g, DP, dt / rho, u, v, w, cs);
    launch_stats(g, u, v, w, stats, P.R, cs);
    if ((rc = capture_end(cs, &seg3))) return rc;
    rc = add_child(G, nw, seg3, end);
    cudaGraphDestroy(seg3);
    return rc;
}

// Captures the body of `enqueue(cs)` as a child node of G (no dependency).
template <class F>
static int add_captured(cudaGraph_t G, cudaStream_t cs, F enqueue, cudaGraphNode_t* node) {
    cudaGraph_t seg = nullptr;
    int rc = capture_begin(cs, nullptr);
    if (rc) return rc;
    const cudaError_t e = enqueue(cs);
    rc = capture_end(cs, &seg);
    if (rc) return rc;
    if (e != cudaSuccess) { cudaGraphDestroy(seg); return PF_ERR_CUDA; }
    rc = add_child(G, nullptr, seg, node);
    cudaGraphDestroy(seg);
    return rc;
}

static void plan_free(StepPlan* plan) {
    if (plan->exec) cudaGraphExecDestroy(plan->exec);
    if (plan->graph) cudaGraphDestroy(plan->graph);
    delete plan;
}

ClosureLayout closure_layout(const pf_grid* g, int prec, int kind) {
    const size_t n = (size_t)g->nx * g->ny * g->nz;
    const size_t tsz = prec == PF_FP64 ? sizeof(double) : sizeof(float);
    ClosureLayout L{0, 0, 0, 0};
    if (kind == PF_CLOSURE_SMAGORINSKY || kind == PF_CLOSURE_GRADIENT) {
        L.bytes = (kind == PF_CLOSURE_SMAGORINSKY ? 1 : 6) * n * tsz;
        return L;
    }
    // MLP: scales + reduction scratch, the FP64 stresses, their float copy
    L.f64 = align256(256 + mlp_scales_ws_bytes());
    L.stage = L.f64;
    L.bytes = L.f64 + align256(6 * n * sizeof(double));
    if (prec != PF_FP64) {
        L.stage = L.bytes;
        L.bytes += align256(6 * n * sizeof(float));
    }
    return L;
}

// the SFS pre-step of a plan (src/data/domain.py:347-355): the closure's
// field from the fields the previous step left, in the stages' type
static cudaError_t enqueue_closure(const pf_grid* g, int prec, const pf_step_closure* c,
                                   double mu, const double* u, const double* v, const double* w,
                                   cudaStream_t st) {
    char* f = (char*)c->field;
    const bool f32 = prec != PF_FP64;
    if (c->kind != PF_CLOSURE_MLP)
        return launch_sgs(g, c->kind - 1, u, v, w, c->coef,
                          c->kind == PF_CLOSURE_SMAGORINSKY ? mu : 0.0, f, f32, st);
    const ClosureLayout L = closure_layout(g, prec, c->kind);
    float* scales = (float*)f;
    cudaError_t e = launch_mlp_scales(g, u, v, w, c->coef, scales, f + 256, st);
    if (e != cudaSuccess) return e;
    e = launch_mlp(g, u, v, w, c->wpack, scales, (double*)(f + L.f64), c->err, st);
    if (e != cudaSuccess || !f32) return e;
    const long long n6 = 6LL * g->nx * g->ny * g->nz;
    return launch_to_float((const double*)(f + L.f64), (float*)(f + L.stage), n6, st);
}

int step_plan_create(const pf_grid* g, int prec, int rk4, double* u, double* v,
                     double* w, double* p, double* DP, double mu, double rho,
                     double dt, double min_res, int max_it, const pf_step_closure* c,
                     void* ws, double* stats, void** out) {
    PlanLayout P;
    int rc = plan_layout(g, prec, ws, &P);
    if (rc != PF_OK) return rc;
    if (predictor_prepare(prec) != cudaSuccess) return PF_ERR_CUDA;
    if (c && c->kind == PF_CLOSURE_MLP && mlp_prepare() != cudaSuccess) return PF_ERR_CUDA;
    cudaStream_t cs;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return PF_ERR_CUDA;
    if (P.mg.L) {
        if (mg_enqueue_setup(P.mg, cs) != PF_OK || cudaStreamSynchronize(cs) != cudaSuccess) {
            cudaStreamDestroy(cs);
            return PF_ERR_CUDA;
        }
    }
    prof_suspend(true);
    StepPlan* plan = new StepPlan();
    do {
        if (cudaGraphCreate(&plan->graph, 0) != cudaSuccess) { rc = PF_ERR_CUDA; break; }
        cudaGraph_t G = plan->graph;
        cudaGraphNode_t n0, nend;
        // the SFS pre-step reads the fields the previous step left; the
        // stages read its field in their own type
        const void* cf = c ? (const char*)c->field + closure_layout(g, prec, c->kind).stage : nullptr;
        const void* visc = c && c->kind == PF_CLOSURE_SMAGORINSKY ? cf : nullptr;
        const void* sfs = c && c->kind != PF_CLOSURE_SMAGORINSKY ? cf : nullptr;
        if ((rc = add_captured(G, cs, [&](cudaStream_t st) {
                 if (c) {
                     const cudaError_t e = enqueue_closure(g, prec, c, mu, u, v, w, st);
                     if (e != cudaSuccess) return e;
                 }
                 return launch_predictor(g, prec, rk4, u, v, w, visc, mu, rho, sfs, dt, P.R, st);
             }, &n0)))
            break;
        if ((rc = add_solve_chain(G, n0, g, prec, P, u, v, w, p, DP, rho, dt, min_res, max_it,
                                  stats, cs, &nend)))
            break;
        if (cudaGraphInstantiate(&plan->exec, G, 0) != cudaSuccess) { rc = PF_ERR_CUDA; break; }
    } while (0);
    prof_suspend(false);
    if (rc == PF_OK &&
        (cudaMemsetAsync(P.sc, 0, sizeof(BicgScalars), cs) != cudaSuccess ||
         cudaStreamSynchronize(cs) != cudaSuccess))
        rc = PF_ERR_CUDA;
    cudaStreamDestroy(cs);
    if (rc != PF_OK) {
        plan_free(plan);
        cudaGetLastError();
        return rc;
    }
    *out = plan;
    return PF_OK;
}

int batch_plan_create(int prec, int rk4, const pf_batch_member* m, int count, void* table,
                      void** out) {
    if (count < 1 || count > kMaxBatch) return PF_ERR_BAD_ARG;
    PlanLayout* P = new PlanLayout[count];
    int rc = PF_OK;
    for (int r = 0; r < count && rc == PF_OK; ++r) rc = plan_layout(&m[r].grid, prec, m[r].ws, &P[r]);
    if (rc != PF_OK) { delete[] P; return rc; }
    // the requests' solves run as parallel branches: their mid levels stay on
    // the per-level kernels (no grid-barrier launches that could wait on one
    // another for room on the SMs)
    for (int r = 0; r < count; ++r) P[r].mg.coop = 0;
    if (predictor_prepare(prec) != cudaSuccess) { delete[] P; return PF_ERR_CUDA; }
    cudaStream_t cs;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) {
        delete[] P;
        return PF_ERR_CUDA;
    }
    // the grouped predictor's members, and each request's one-time set-up
    GroupMember gm[kMaxBatch];
    for (int r = 0; r < count; ++r)
        gm[r] = GroupMember{m[r].grid, m[r].u, m[r].v, m[r].w, m[r].mu, m[r].rho, m[r].dt,
                            P[r].R};
    rc = grouped_predictor_tables(prec, rk4, gm, count, table, cs);
    // one-time set-up of members that join a plan for the first time; a
    // member carried over from an earlier plan may still be computing there
    // and is not touched
    for (int r = 0; r < count && rc == PF_OK; ++r)
        if (m[r].fresh && P[r].mg.L && mg_enqueue_setup(P[r].mg, cs) != PF_OK) rc = PF_ERR_CUDA;
    if (rc == PF_OK && cudaStreamSynchronize(cs) != cudaSuccess) rc = PF_ERR_CUDA;
    StepPlan* plan = new StepPlan();
    prof_suspend(true);
    do {
        if (rc != PF_OK) break;
        if (cudaGraphCreate(&plan->graph, 0) != cudaSuccess) { rc = PF_ERR_CUDA; break; }
        cudaGraph_t G = plan->graph;
        cudaGraphNode_t n0;
        if ((rc = add_captured(G, cs, [&](cudaStream_t st) {
                 return launch_grouped_predictor(prec, rk4, gm, count, table, st);
             }, &n0)))
            break;
        // the requests' solves run as independent branches of the graph
        for (int r = 0; r < count && rc == PF_OK; ++r) {
            cudaGraphNode_t nend;
            rc = add_solve_chain(G, n0, &m[r].grid, prec, P[r], m[r].u, m[r].v, m[r].w, m[r].p,
                                 m[r].DP, m[r].rho, m[r].dt, m[r].min_res, m[r].max_it,
                                 m[r].stats, cs, &nend);
        }
        if (rc != PF_OK) break;
        if (cudaGraphInstantiate(&plan->exec, G, 0) != cudaSuccess) { rc = PF_ERR_CUDA; break; }
    } while (0);
    prof_suspend(false);
    for (int r = 0; r < count && rc == PF_OK; ++r)
        if (m[r].fresh && cudaMemsetAsync(P[r].sc, 0, sizeof(BicgScalars), cs) != cudaSuccess)
            rc = PF_ERR_CUDA;
    if (rc == PF_OK && cudaStreamSynchronize(cs) != cudaSuccess) rc = PF_ERR_CUDA;
    cudaStreamDestroy(cs);
    delete[] P;
    if (rc != PF_OK) {
        plan_free(plan);
        cudaGetLastError();
        return rc;
    }
    *out = plan;
    return PF_OK;
}

int step_plan_launch(void* plan, int nsteps, cudaStream_t s) {
    StepPlan* pl = (StepPlan*)plan;
    for (int i = 0; i < nsteps; ++i)
        if (cudaGraphLaunch(pl->exec, s) != cudaSuccess) return PF_ERR_CUDA;
    return PF_OK;
}

int step_plan_destroy(void* plan) {
    if (plan) plan_free((StepPlan*)plan);
    return PF_OK;
}

}  // namespace pf
