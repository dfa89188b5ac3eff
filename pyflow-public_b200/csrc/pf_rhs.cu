// pf_rhs.cu -- staggered Navier-Stokes right-hand side and RK4/Euler stages.
//
// rhs_NavierStokes.evaluate (src/solver/velocity.py:221-355) computed per cell
// from a 3x3x3 neighbourhood, with the stage arithmetic of RK4.step
// (src/solver/advancer.py:75-113) fused into the epilogue, so one launch per
// stage reads the stage state once and writes the next stage state and the
// running k-sum:
//   stage 1  : acc  = k1,            uT  = h*k1 + u      (h = dt/2)
//   stage 2,3: acc += 2*k,           uT' = h*k  + u
//   stage 4  : u    = u + dt/6*(acc + k4)   (reference stage-4 state u + h*k3)
// Euler.step (src/solver/advancer.py:49-57): u = u + k*dt.
// The flux expressions keep the reference's operation order (see
// pf_common.cuh), including the edge-averaged viscosity one cell below the
// off-diagonal flux (metric_staggered.py:127-144 vs :378-384).
#include <algorithm>
#include <cstring>
#include <vector>

#include "pf_common.cuh"
#include "pf_kernels.cuh"
#include "pf_profile.cuh"
#include "pf_sweep.cuh"
#include "pf_flux.cuh"

namespace pf {

template <typename T, typename TI>
struct RhsArgs {
    const TI* u;
    const TI* v;
    const TI* w;
    const T* visc;  // nullptr: constant mu
    const T* sfs;   // nullptr or FXX,FYY,FZZ,FXY,FXZ,FYZ
    T mu, rho, dxi, dyi, dzi;
};


// Neighbourhood of cell (i, j, k) read from global memory (any viscosity /
// SFS configuration): wrapped plane / row / column offsets of the neighbours
// i-2 .. i+1 are computed once, every load is then two adds.
template <typename T, typename TI>
struct GatherSrc {
    const RhsArgs<T, TI>* a;
    long long xo[4];
    int yo[4], zo[4];
    long long n;
    __device__ GatherSrc(const Dims& d, const RhsArgs<T, TI>& args, int i, int j, int k) : a(&args) {
        const long long P = (long long)d.ny * d.nz;
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            xo[o] = (long long)wrap(i + o - 2, d.nx) * P;
            yo[o] = wrap(j + o - 2, d.ny) * d.nz;
            zo[o] = wrap(k + o - 2, d.nz);
        }
        n = d.n;
    }
    __device__ long long off(int di, int dj, int dk) const {
        return xo[di + 2] + (long long)(yo[dj + 2] + zo[dk + 2]);
    }
    __device__ T u(int di, int dj, int dk) const { return T(__ldg(a->u + off(di, dj, dk))); }
    __device__ T v(int di, int dj, int dk) const { return T(__ldg(a->v + off(di, dj, dk))); }
    __device__ T w(int di, int dj, int dk) const { return T(__ldg(a->w + off(di, dj, dk))); }
    __device__ T visc(int di, int dj, int dk) const { return __ldg(a->visc + off(di, dj, dk)); }
    __device__ T sfs(int c, int di, int dj, int dk) const {
        return __ldg(a->sfs + (long long)c * n + off(di, dj, dk));
    }
};

template <typename T, typename TI>
__device__ inline void rhs_cell(const Dims& d, const RhsArgs<T, TI>& a, int i, int j, int k,
                                T& ru, T& rv, T& rw) {
    GatherSrc<T, TI> S(d, a, i, j, k);
    rhs_core<T>(S, a.mu, a.rho, a.dxi, a.dyi, a.dzi, a.visc != nullptr, a.sfs != nullptr,
                ru, rv, rw);
}

enum StageMode { kModeRhs = 0, kModeFirst = 1, kModeMid = 2, kModeLast = 3, kModeK = 4 };

// Stage arithmetic of one cell (the epilogue of every stage kernel).
template <typename T, typename TS, typename TA, int MODE>
__device__ __forceinline__ void stage_store(long long q, T ku, T kv, T kw, double* u,
                                            double* v, double* w, TS* su, TS* sv, TS* sw,
                                            TA* au, TA* av, TA* aw, T* ru, T* rv, T* rw,
                                            double hdt, double c6) {
    if (MODE == kModeRhs) {
        ru[q] = ku; rv[q] = kv; rw[q] = kw;
    } else if (MODE == kModeFirst || MODE == kModeMid) {
        // ZAXPY(h, k, u) = h*k + u (src/data/state.py:157-165)
        su[q] = TS(hdt * double(ku) + u[q]);
        sv[q] = TS(hdt * double(kv) + v[q]);
        sw[q] = TS(hdt * double(kw) + w[q]);
        if (MODE == kModeFirst) {
            au[q] = TA(ku); av[q] = TA(kv); aw[q] = TA(kw);
        } else {
            au[q] = TA(T(au[q]) + T(2.0) * ku);
            av[q] = TA(T(av[q]) + T(2.0) * kv);
            aw[q] = TA(T(aw[q]) + T(2.0) * kw);
        }
    } else if (MODE == kModeLast) {
        u[q] = u[q] + c6 * (double(T(au[q]) + ku));
        v[q] = v[q] + c6 * (double(T(av[q]) + kv));
        w[q] = w[q] + c6 * (double(T(aw[q]) + kw));
    } else {  // kModeK: k alone (Euler applies it in a second pass)
        au[q] = TA(ku); av[q] = TA(kv); aw[q] = TA(kw);
    }
}

// TS: stage-state storage type; TA: k-sum storage type.  Gather form: any
// viscosity / SFS configuration.
template <typename T, typename TI, typename TS, typename TA, int MODE>
__global__ void __launch_bounds__(256)
rhs_stage_kernel(Dims d, RhsArgs<T, TI> a, double* __restrict__ u,
                 double* __restrict__ v, double* __restrict__ w,
                 TS* __restrict__ su, TS* __restrict__ sv, TS* __restrict__ sw,
                 TA* __restrict__ au, TA* __restrict__ av, TA* __restrict__ aw,
                 T* __restrict__ ru, T* __restrict__ rv, T* __restrict__ rw,
                 double hdt, double c6) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    T ku, kv, kw;
    rhs_cell<T, TI>(d, a, i, j, k, ku, kv, kw);
    stage_store<T, TS, TA, MODE>(idx(d, i, j, k), ku, kv, kw, u, v, w, su, sv, sw, au, av,
                                 aw, ru, rv, rw, hdt, c6);
}

// ---------------------------------------------------------------------------
// Tiled form (constant viscosity, no SFS stresses: the DNS hot path).  A block
// of 32 x 8 threads owns a 32 (z) x 16 (y) tile and marches along x.  The
// velocity of planes i-1, i, i+1 (with a one-cell y/z halo, corners included)
// sits in a four-slot ring in shared memory; while plane i is computed,
// cp.async copies plane i+2 into the free slot and the per-cell stage inputs
// of plane i+1 (u, v, w and the k-sum) into a second buffer, so no thread
// waits on global memory inside the march and no registers hold the
// prefetch.  Every global value is read once per tile; the flux arithmetic
// is rhs_core, unchanged.
// ---------------------------------------------------------------------------
constexpr int kRhsTY = 16;
constexpr int kRhsSY = kRhsTY + 2, kRhsSZ = 34;
constexpr int kRhsPos = kRhsSY * kRhsSZ;        // halo-extended plane tile
constexpr int kRhsPPT = (kRhsPos + 255) / 256;  // positions per thread
constexpr int kRhsCells = 32 * kRhsTY;          // owned cells per plane

template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if (BYTES == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" :: "r"(s), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" :: "r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// dynamic shared memory of the tiled stage kernel
template <typename T, typename TI, typename TA, int MODE>
struct RhsSmem {
    // FP64 input planes of an FP32 stage (the state u of the first stage or
    // of Euler's k) are staged as FP64 and converted to T once per position
    static constexpr bool kConv = sizeof(TI) > sizeof(T);
    static constexpr bool kU = MODE == kModeFirst || MODE == kModeMid || MODE == kModeLast;
    static constexpr bool kA = MODE == kModeMid || MODE == kModeLast;
    static constexpr size_t kEu = (kU && !kConv) ? 2 * 3 * kRhsCells * sizeof(double) : 0;  // [2][3][cells]
    static constexpr size_t kStg = kConv ? 4 * 3 * kRhsPos * sizeof(TI) : 0;             // [4][3][pos]
    static constexpr size_t kRing = 4 * 3 * kRhsPos * (kConv ? sizeof(T) : sizeof(TI)); // [4][3][pos]
    static constexpr size_t kEa = kA ? 2 * 3 * kRhsCells * sizeof(TA) : 0;               // [2][3][cells]
    // y-plus terms of the rows 2 ty - 1 (8 x 32) and z-plus terms of the
    // halo column z = -1 (16 rows) of the face form
    static constexpr size_t kFaces = ((8 * 32 * sizeof(YFace<T>) + kRhsTY * sizeof(ZFace<T>)) + 15) &
                                     ~size_t(15);
    static constexpr size_t bytes = kEu + kStg + kRing + kEa + kFaces;
};

template <typename T>
__device__ __forceinline__ ZFace<T> shfl_up_z(const ZFace<T>& z) {
    constexpr unsigned m = 0xffffffffu;
    return ZFace<T>{__shfl_up_sync(m, z.fxz, 1), __shfl_up_sync(m, z.fyz, 1),
                    __shfl_up_sync(m, z.fzz, 1), __shfl_up_sync(m, z.cuw, 1),
                    __shfl_up_sync(m, z.cvw, 1), __shfl_up_sync(m, z.cww, 1)};
}

template <typename T, typename TI>
struct SmemSrc {
    const TI* ring;  // [4][3][kRhsPos]
    int s0, s1, s2;  // slots of planes i-1, i, i+1
    int y, z;        // the cell in the halo-extended tile
    __device__ const TI* f(int fld, int di) const {
        const int sl = di < 0 ? s0 : (di == 0 ? s1 : s2);
        return ring + (sl * 3 + fld) * kRhsPos;
    }
    __device__ T u(int di, int dj, int dk) const { return T(f(0, di)[(y + dj) * kRhsSZ + z + dk]); }
    __device__ T v(int di, int dj, int dk) const { return T(f(1, di)[(y + dj) * kRhsSZ + z + dk]); }
    __device__ T w(int di, int dj, int dk) const { return T(f(2, di)[(y + dj) * kRhsSZ + z + dk]); }
    __device__ T visc(int, int, int) const { return T(0); }
    __device__ T sfs(int, int, int, int) const { return T(0); }
};

// The right-hand side of this thread's two cells of plane i (rows 2 ty and
// 2 ty + 1, column tx of the tile) in the face form of pf_flux.cuh: every cell
// computes its plus-face terms once; its x-minus terms are the x-plus terms
// of the same cell on the previous plane (xf; on the tile's first plane they
// are computed from plane i - 1), its y-minus terms those of the row below
// (the thread's own first row, or through shared memory from thread ty - 1;
// row -1 of the tile is computed by the first warp), its z-minus terms those
// of the lane below (a shuffle; lane 0 reads the halo column z = -1, computed
// by the second warp).  Bit-identical to rhs_core (checked on the host).
// Every thread of the block must call it (it holds a block barrier); cells
// outside the grid compute on wrapped data and are not stored.
template <typename T, typename TI>
__device__ __forceinline__ void
rhs_plane_faces(const TI* ring, int s0, int s1, int s2, const FluxCoef<T>& fc, bool first,
                XFace<T> (&xf)[2], YFace<T>* sY, ZFace<T>* sZh, T (&k3)[2][3]) {
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    PlusFaces<T> pf[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const SmemSrc<T, TI> src{ring, s0, s1, s2, 2 * ty + r + 1, tx + 1};
        pf[r] = plus_faces<T>(src, fc);
    }
    if (ty < 7) sY[(ty + 1) * 32 + tx] = pf[1].y;
    if (tid < 32) {            // row -1: its y-plus terms are the y-minus terms of row 0
        const SmemSrc<T, TI> src{ring, s0, s1, s2, 0, tid + 1};
        sY[tid] = plus_faces<T, false, true, false>(src, fc).y;
    } else if (tid < 32 + kRhsTY) {  // column z = -1: z-plus terms for lane 0
        const int row = tid - 32;
        const SmemSrc<T, TI> src{ring, s0, s1, s2, row + 1, 0};
        sZh[row] = plus_faces<T, false, false, true>(src, fc).z;
    }
    XFace<T> xm[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        if (first) {
            const SmemSrc<T, TI> src{ring, s0, s1, s2, 2 * ty + r + 1, tx + 1};
            const Shifted<SmemSrc<T, TI>> prev{src, -1, 0, 0};
            xm[r] = plus_faces<T, true, false, false>(prev, fc).x;
        } else {
            xm[r] = xf[r];
        }
    }
    ZFace<T> zm[2] = {shfl_up_z(pf[0].z), shfl_up_z(pf[1].z)};
    __syncthreads();
    if (tx == 0) {
        zm[0] = sZh[2 * ty];
        zm[1] = sZh[2 * ty + 1];
    }
    assemble_faces(pf[0], xm[0], sY[ty * 32 + tx], zm[0], fc, k3[0][0], k3[0][1], k3[0][2]);
    assemble_faces(pf[1], xm[1], pf[0].y, zm[1], fc, k3[1][0], k3[1][1], k3[1][2]);
    xf[0] = pf[0].x;
    xf[1] = pf[1].x;
}

// The tiled stage for an FP64 input of an FP32 stage (first RK4 stage,
// Euler's k): plane x's FP64 values arrive by cp.async in stg slot
// (x - i0 + 1) & 3, and the thread that copied a position converts it into
// the FP32 ring slot of the same number once the copy has landed (a thread's
// own copies need no barrier).  Plane i + 2 is converted after plane i is
// computed, so one barrier per plane orders conversion and use; the first
// stage's FP64 u of the owned cells comes from plane i's stg slot.
template <typename T, typename TI, typename TS, typename TA, int MODE>
__device__ __forceinline__ void
rhs_tile_conv(const Dims& d, const Tiling& tl, const RhsArgs<T, TI>& a,
              double* __restrict__ u, double* __restrict__ v, double* __restrict__ w,
              TS* __restrict__ su, TS* __restrict__ sv, TS* __restrict__ sw,
              TA* __restrict__ au, TA* __restrict__ av, TA* __restrict__ aw,
              double hdt, long long t) {
    static_assert(MODE == kModeFirst || MODE == kModeK, "FP64 input planes: first stage or k");
    using SM = RhsSmem<T, TI, TA, MODE>;
    extern __shared__ __align__(16) unsigned char smraw[];
    TI* stg = reinterpret_cast<TI*>(smraw);
    T* ring = reinterpret_cast<T*>(smraw + SM::kStg);
    YFace<T>* sY = reinterpret_cast<YFace<T>*>(smraw + SM::kEu + SM::kStg + SM::kRing + SM::kEa);
    ZFace<T>* sZh = reinterpret_cast<ZFace<T>*>(sY + 8 * 32);
    const FluxCoef<T> fc = flux_coef<T>(a.mu, a.rho, a.dxi, a.dyi, a.dzi);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const long long plane = (long long)d.ny * d.nz;
    const TI* fld[3] = {a.u, a.v, a.w};
    TA* A[3] = {au, av, aw};
    TS* S[3] = {su, sv, sw};
    {
        const int tz = (int)(t % tl.ntz);
        const long long rr = t / tl.ntz;
        const int tyy = (int)(rr % tl.nty), txx = (int)(rr / tl.nty);
        const int k0 = tz * 32, j0 = tyy * kRhsTY, i0 = txx * tl.xc;
        const int i1 = min(i0 + tl.xc, d.nx);
        const int ez = min(32, d.nz - k0), ey = min(kRhsTY, d.ny - j0);
        long long goff[kRhsPPT];
        int soff[kRhsPPT];
        bool pv[kRhsPPT];
#pragma unroll
        for (int p = 0; p < kRhsPPT; ++p) {
            const int pos = tid + 256 * p;
            pv[p] = pos < kRhsPos;
            const int yy = pv[p] ? pos / kRhsSZ : 0, zz = pv[p] ? pos - yy * kRhsSZ : 0;
            goff[p] = (long long)pmod(j0 + yy - 1, d.ny) * d.nz + pmod(k0 + zz - 1, d.nz);
            soff[p] = yy * kRhsSZ + zz;
        }
        // this thread's owned cells: rows 2 ty and 2 ty + 1 of column tx
        bool cv[2];
        long long coff[2];
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int jl = 2 * ty + r;
            cv[r] = tx < ez && jl < ey;
            coff[r] = (long long)(j0 + jl) * d.nz + k0 + tx;
        }
        auto slot = [&](int x) { return (x - i0 + 1) & 3; };
        auto load_stg = [&](int x) {
            const long long base = (long long)pmod(x, d.nx) * plane;
            TI* dst = stg + slot(x) * 3 * kRhsPos;
#pragma unroll
            for (int f = 0; f < 3; ++f)
#pragma unroll
                for (int p = 0; p < kRhsPPT; ++p)
                    if (pv[p]) cp_async<sizeof(TI)>(dst + f * kRhsPos + soff[p], fld[f] + base + goff[p]);
        };
        auto convert = [&](int x) {
            const TI* src = stg + slot(x) * 3 * kRhsPos;
            T* dst = ring + slot(x) * 3 * kRhsPos;
#pragma unroll
            for (int f = 0; f < 3; ++f)
#pragma unroll
                for (int p = 0; p < kRhsPPT; ++p)
                    if (pv[p]) dst[f * kRhsPos + soff[p]] = T(src[f * kRhsPos + soff[p]]);
        };
        load_stg(i0 - 1);
        load_stg(i0);
        load_stg(i0 + 1);
        cp_async_commit();
        if (i0 + 1 < i1) load_stg(i0 + 2);
        cp_async_commit();
        cp_async_wait_groups<1>();
        convert(i0 - 1);
        convert(i0);
        convert(i0 + 1);
        __syncthreads();
        XFace<T> xf[2];  // x-plus terms of this thread's two cells on the previous plane
        for (int i = i0; i < i1; ++i) {
            const int c = i - i0;
            const int s0 = c & 3, s1 = (c + 1) & 3, s2 = (c + 2) & 3;
            if (i + 2 < i1) load_stg(i + 3);
            cp_async_commit();
            T k3[2][3];
            rhs_plane_faces<T, T>(ring, s0, s1, s2, fc, i == i0, xf, sY, sZh, k3);
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                if (!cv[r]) continue;
                const int jl = 2 * ty + r;
                const long long q = (long long)i * plane + coff[r];
                const int pc = (jl + 1) * kRhsSZ + tx + 1;
#pragma unroll
                for (int f = 0; f < 3; ++f) {
                    const T kf = k3[r][f];
                    if (MODE == kModeFirst) {
                        // ZAXPY(h, k, u) = h*k + u (src/data/state.py:157-165)
                        S[f][q] = TS(hdt * double(kf) + double(stg[(s1 * 3 + f) * kRhsPos + pc]));
                        A[f][q] = TA(kf);
                    } else {  // kModeK
                        A[f][q] = TA(kf);
                    }
                }
            }
            cp_async_wait_groups<1>();
            if (i + 1 < i1) convert(i + 2);
            __syncthreads();
        }
        cp_async_wait_all();
        __syncthreads();
    }
}

template <typename T, typename TI, typename TS, typename TA, int MODE>
__device__ __forceinline__ void
rhs_tile(const Dims& d, const Tiling& tl, const RhsArgs<T, TI>& a, double* __restrict__ u,
         double* __restrict__ v, double* __restrict__ w,
         TS* __restrict__ su, TS* __restrict__ sv, TS* __restrict__ sw,
         TA* __restrict__ au, TA* __restrict__ av, TA* __restrict__ aw,
         double hdt, double c6, long long t) {
    using SM = RhsSmem<T, TI, TA, MODE>;
    extern __shared__ __align__(16) unsigned char smraw[];
    double* eu = reinterpret_cast<double*>(smraw);
    TI* ring = reinterpret_cast<TI*>(smraw + SM::kEu);
    TA* ea = reinterpret_cast<TA*>(smraw + SM::kEu + SM::kRing);
    YFace<T>* sY = reinterpret_cast<YFace<T>*>(smraw + SM::kEu + SM::kStg + SM::kRing + SM::kEa);
    ZFace<T>* sZh = reinterpret_cast<ZFace<T>*>(sY + 8 * 32);
    const FluxCoef<T> fc = flux_coef<T>(a.mu, a.rho, a.dxi, a.dyi, a.dzi);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const long long plane = (long long)d.ny * d.nz;
    const TI* fld[3] = {a.u, a.v, a.w};
    double* U[3] = {u, v, w};
    TA* A[3] = {au, av, aw};
    TS* S[3] = {su, sv, sw};
    {
        const int tz = (int)(t % tl.ntz);
        const long long rr = t / tl.ntz;
        const int tyy = (int)(rr % tl.nty), txx = (int)(rr / tl.nty);
        const int k0 = tz * 32, j0 = tyy * kRhsTY, i0 = txx * tl.xc;
        const int i1 = min(i0 + tl.xc, d.nx);
        const int ez = min(32, d.nz - k0), ey = min(kRhsTY, d.ny - j0);
        long long goff[kRhsPPT];
        int soff[kRhsPPT];
        bool pv[kRhsPPT];
#pragma unroll
        for (int p = 0; p < kRhsPPT; ++p) {
            const int pos = tid + 256 * p;
            pv[p] = pos < kRhsPos;
            const int yy = pv[p] ? pos / kRhsSZ : 0, zz = pv[p] ? pos - yy * kRhsSZ : 0;
            goff[p] = (long long)pmod(j0 + yy - 1, d.ny) * d.nz + pmod(k0 + zz - 1, d.nz);
            soff[p] = yy * kRhsSZ + zz;
        }
        // this thread's owned cells: rows 2 ty and 2 ty + 1 of column tx
        bool cv[2];
        long long coff[2];
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int jl = 2 * ty + r;
            cv[r] = tx < ez && jl < ey;
            coff[r] = (long long)(j0 + jl) * d.nz + k0 + tx;
        }
        auto load_plane = [&](int x, int slot) {
            const long long base = (long long)pmod(x, d.nx) * plane;
#pragma unroll
            for (int f = 0; f < 3; ++f)
#pragma unroll
                for (int p = 0; p < kRhsPPT; ++p)
                    if (pv[p])
                        cp_async<sizeof(TI)>(ring + (slot * 3 + f) * kRhsPos + soff[p],
                                             fld[f] + base + goff[p]);
        };
        auto load_epi = [&](int x, int buf) {
            const long long base = (long long)x * plane;
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                if (!cv[r]) continue;
                const int c = (2 * ty + r) * 32 + tx;
#pragma unroll
                for (int f = 0; f < 3; ++f) {
                    if (SM::kU) cp_async<8>(eu + (buf * 3 + f) * kRhsCells + c, U[f] + base + coff[r]);
                    if (SM::kA)
                        cp_async<sizeof(TA)>(ea + (buf * 3 + f) * kRhsCells + c, A[f] + base + coff[r]);
                }
            }
        };
        // prologue: planes i0-1, i0, i0+1 into slots 0, 1, 2; stage inputs of i0
        load_plane(i0 - 1, 0);
        load_plane(i0, 1);
        load_plane(i0 + 1, 2);
        load_epi(i0, 0);
        cp_async_commit();
        cp_async_wait_all();
        __syncthreads();
        XFace<T> xf[2];  // x-plus terms of this thread's two cells on the previous plane
        for (int i = i0; i < i1; ++i) {
            const int c = i - i0;
            const int s0 = c & 3, s1 = (c + 1) & 3, s2 = (c + 2) & 3;
            const int buf = c & 1;
            if (i + 1 < i1) {
                load_plane(i + 2, (c + 3) & 3);
                load_epi(i + 1, buf ^ 1);
                cp_async_commit();
            }
            T k3[2][3];
            rhs_plane_faces<T, TI>(ring, s0, s1, s2, fc, i == i0, xf, sY, sZh, k3);
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                if (!cv[r]) continue;
                const int jl = 2 * ty + r;
                const long long q = (long long)i * plane + coff[r];
                const int cc = jl * 32 + tx;
#pragma unroll
                for (int f = 0; f < 3; ++f) {
                    const T kf = k3[r][f];
                    if (MODE == kModeFirst || MODE == kModeMid) {
                        // ZAXPY(h, k, u) = h*k + u (src/data/state.py:157-165)
                        S[f][q] = TS(hdt * double(kf) + eu[(buf * 3 + f) * kRhsCells + cc]);
                        if (MODE == kModeFirst) A[f][q] = TA(kf);
                        else A[f][q] = TA(T(ea[(buf * 3 + f) * kRhsCells + cc]) + T(2.0) * kf);
                    } else if (MODE == kModeLast) {
                        U[f][q] = eu[(buf * 3 + f) * kRhsCells + cc] +
                                  c6 * (double(T(ea[(buf * 3 + f) * kRhsCells + cc]) + kf));
                    } else {  // kModeK
                        A[f][q] = TA(kf);
                    }
                }
            }
            cp_async_wait_all();
            __syncthreads();
        }
    }
}

// One tile of a stage: the FP64-input form for an FP32 stage reading the
// FP64 state, the direct form otherwise.
template <typename T, typename TI, typename TS, typename TA, int MODE>
__device__ __forceinline__ void
stage_tile(const Dims& d, const Tiling& tl, const RhsArgs<T, TI>& a, double* u, double* v,
           double* w, TS* su, TS* sv, TS* sw, TA* au, TA* av, TA* aw, double hdt, double c6,
           long long t) {
    if constexpr (RhsSmem<T, TI, TA, MODE>::kConv)
        rhs_tile_conv<T, TI, TS, TA, MODE>(d, tl, a, u, v, w, su, sv, sw, au, av, aw, hdt, t);
    else
        rhs_tile<T, TI, TS, TA, MODE>(d, tl, a, u, v, w, su, sv, sw, au, av, aw, hdt, c6, t);
}

template <typename T, typename TI, typename TS, typename TA, int MODE>
__global__ void __launch_bounds__(256, 2)
rhs_stage_tiled(Dims d, Tiling tl, RhsArgs<T, TI> a, double* __restrict__ u,
                double* __restrict__ v, double* __restrict__ w,
                TS* __restrict__ su, TS* __restrict__ sv, TS* __restrict__ sw,
                TA* __restrict__ au, TA* __restrict__ av, TA* __restrict__ aw,
                double hdt, double c6) {
    for (long long t = blockIdx.x; t < tl.ntiles; t += gridDim.x)
        stage_tile<T, TI, TS, TA, MODE>(d, tl, a, u, v, w, su, sv, sw, au, av, aw, hdt, c6, t);
}

// Grouped stage: one launch advances the same RK4 stage of several
// independent solves (a batch of requests, any grid sizes).  jobs[r] (device
// memory) holds request r's grid, tiling, stage arguments and the index of
// its first tile in the batch's tile space; a block walks the batch's tiles
// (persistent loop), stages the tile's job in shared memory and runs the
// tile with it, so every tile computes exactly what the single-request
// launch computes.  A tile index outside every job's range (a table that does
// not match the launch) is skipped and recorded in *err.
template <typename T, typename TI>
struct StageJob {
    Dims d;
    Tiling tl;
    RhsArgs<T, TI> a;
    double *u, *v, *w;
    T *su, *sv, *sw, *au, *av, *aw;
    double hdt, c6;
    long long tile0;
};

constexpr int kMaxGroupJobs = kMaxBatch;

template <typename T, typename TI, int MODE>
__global__ void __launch_bounds__(256, 2)
rhs_stage_grouped(const StageJob<T, TI>* __restrict__ jobs, int njobs, long long ntiles,
                  int* __restrict__ err) {
    __shared__ long long first[kMaxGroupJobs];
    __shared__ StageJob<T, TI> J;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    njobs = min(njobs, kMaxGroupJobs);
    for (int r = tid; r < njobs; r += 256) first[r] = jobs[r].tile0;
    __syncthreads();
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        int lo = 0, hi = njobs - 1;  // last job whose first tile is <= t
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (first[mid] <= t) lo = mid; else hi = mid - 1;
        }
        // the previous tile is done with J (each tile ends at a barrier)
        __syncthreads();
        {
            static_assert(sizeof(StageJob<T, TI>) % 8 == 0, "job copied in 8-byte words");
            const unsigned long long* src = reinterpret_cast<const unsigned long long*>(jobs + lo);
            unsigned long long* dst = reinterpret_cast<unsigned long long*>(&J);
            for (int q = tid; q < (int)(sizeof(StageJob<T, TI>) / 8); q += 256) dst[q] = src[q];
        }
        __syncthreads();
        const long long local = t - J.tile0;
        if (local < 0 || local >= J.tl.ntiles) {
            if (tid == 0) atomicExch(err, 1);
            continue;
        }
        stage_tile<T, TI, T, T, MODE>(J.d, J.tl, J.a, J.u, J.v, J.w, J.su, J.sv, J.sw, J.au,
                                      J.av, J.aw, J.hdt, J.c6, local);
    }
}

// Sets the dynamic shared-memory limit of one tiled instance, once per CUDA
// context (function attributes belong to the context).
template <typename T, typename TI, int MODE>
static cudaError_t tiled_prepare_ctx() {
    cudaError_t e = cudaFuncSetAttribute(
        rhs_stage_tiled<T, TI, T, T, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int)RhsSmem<T, TI, T, MODE>::bytes);
    // a shared-memory carveout just large enough for two blocks per SM (the
    // rest stays L1): percent of the SM's 228 KiB
    if (e == cudaSuccess) {
        const size_t two = 2 * (RhsSmem<T, TI, T, MODE>::bytes + 1024);
        const int pct = (int)std::min<size_t>(100, (two * 100 + 228 * 1024 - 1) / (228 * 1024));
        e = cudaFuncSetAttribute(rhs_stage_tiled<T, TI, T, T, MODE>,
                                 cudaFuncAttributePreferredSharedMemoryCarveout, pct);
    }
    return e;
}

template <typename T, typename TI, int MODE>
static cudaError_t tiled_prepare() {
    return once_per_context((const void*)&tiled_prepare_ctx<T, TI, MODE>,
                            &tiled_prepare_ctx<T, TI, MODE>);
}

// Euler.step's update u += k dt (src/solver/advancer.py:49-57), applied after
// k is complete so no kernel reads a velocity another block has updated.
template <typename T>
__global__ void __launch_bounds__(256)
euler_apply(long long n, const T* __restrict__ ku, const T* __restrict__ kv,
            const T* __restrict__ kw, double dt, double* __restrict__ u,
            double* __restrict__ v, double* __restrict__ w) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        u[q] = u[q] + double(ku[q]) * dt;
        v[q] = v[q] + double(kv[q]) * dt;
        w[q] = w[q] + double(kw[q]) * dt;
    }
}

static dim3 cell_grid(const Dims& d) {
    return dim3((d.nz + 31) / 32, (d.ny + 7) / 8, d.nx);
}

template <typename T, typename TI>
static RhsArgs<T, TI> make_args(const pf_grid* g, const TI* u, const TI* v,
                                const TI* w, const T* visc, const T* sfs,
                                double mu, double rho) {
    RhsArgs<T, TI> a;
    a.u = u; a.v = v; a.w = w; a.visc = visc; a.sfs = sfs;
    a.mu = T(mu); a.rho = T(rho);
    a.dxi = T(1.0 / g->dx); a.dyi = T(1.0 / g->dy); a.dzi = T(1.0 / g->dz);
    return a;
}

cudaError_t launch_rhs(const pf_grid* g, int prec, const void* u,
                       const void* v, const void* w, const void* visc,
                       double mu, double rho, const void* sfs, void* ru,
                       void* rv, void* rw, cudaStream_t s) {
    Dims d{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    dim3 blk(32, 8);
    if (prec == PF_FP64) {
        auto a = make_args<double, double>(g, (const double*)u, (const double*)v, (const double*)w,
                                           (const double*)visc, (const double*)sfs, mu, rho);
        PF_LAUNCH("rhs_rhs_f64", s, rhs_stage_kernel<double, double, double, double, kModeRhs><<<cell_grid(d), blk, 0, s>>>(
            d, a, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
            (double*)ru, (double*)rv, (double*)rw, 0.0, 0.0));
    } else {
        auto a = make_args<float, float>(g, (const float*)u, (const float*)v, (const float*)w,
                                         (const float*)visc, (const float*)sfs, mu, rho);
        PF_LAUNCH("rhs_rhs_f32", s, rhs_stage_kernel<float, float, float, float, kModeRhs><<<cell_grid(d), blk, 0, s>>>(
            d, a, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
            (float*)ru, (float*)rv, (float*)rw, 0.0, 0.0));
    }
    return cudaGetLastError();
}

// One stage: the tiled kernel for constant viscosity without SFS stresses,
// the gather kernel otherwise.
template <typename T, typename TI, int MODE>
static cudaError_t stage(const char* name, const Dims& d, const RhsArgs<T, TI>& a, double* u,
                  double* v, double* w, T* st, T* acc, double hdt, double c6,
                  cudaStream_t s) {
    const long long n = d.n;
    T* su = st ? st : nullptr;
    T* sv = st ? st + n : nullptr;
    T* sw = st ? st + 2 * n : nullptr;
    dim3 blk(32, 8);
    if (!a.visc && !a.sfs) {
        const Tiling tl = make_tiling(d, kRhsTY);
        const cudaError_t e = tiled_prepare<T, TI, MODE>();
        if (e != cudaSuccess) return e;
        PF_LAUNCH(name, s, rhs_stage_tiled<T, TI, T, T, MODE><<<tiled_grid(tl), blk,
                                                              RhsSmem<T, TI, T, MODE>::bytes, s>>>(
            d, tl, a, u, v, w, su, sv, sw, acc, acc + n, acc + 2 * n, hdt, c6));
    } else {
        PF_LAUNCH(name, s, rhs_stage_kernel<T, TI, T, T, MODE><<<cell_grid(d), blk, 0, s>>>(
            d, a, u, v, w, su, sv, sw, acc, acc + n, acc + 2 * n, nullptr, nullptr, nullptr,
            hdt, c6));
    }
    return cudaGetLastError();
}

// Predictor step.  Workspace: stage states (2 ping-pong sets) and the k-sum,
// each 3 fields of the stage type (double for PF_FP64, float for the mixed
// forms).
template <typename T>
static cudaError_t predictor_impl(const pf_grid* g, int rk4, double* u,
                                  double* v, double* w, const T* visc,
                                  double mu, double rho, const T* sfs,
                                  double dt, T* ws, cudaStream_t s) {
    Dims d{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    const long long n = d.n;
    T *sa = ws, *sb = ws + 3 * n, *acc = ws + 6 * n;
    const double hdt = 0.5 * dt, c6 = dt / 6.0;
    const bool f64 = sizeof(T) == 8;
    auto a0 = make_args<T, double>(g, u, v, w, visc, sfs, mu, rho);
    if (!rk4) {
        cudaError_t e = stage<T, double, kModeK>(f64 ? "rhs_euler_f64" : "rhs_euler_f32", d,
                                                 a0, u, v, w, nullptr, acc, hdt, c6, s);
        if (e != cudaSuccess) return e;
        const int gp = (int)std::min<long long>((n + 1023) / 1024, 4096);
        PF_LAUNCH("euler_apply", s, euler_apply<T><<<gp, 256, 0, s>>>(
            n, acc, acc + n, acc + 2 * n, dt, u, v, w));
        return cudaGetLastError();
    }
    cudaError_t e = stage<T, double, kModeFirst>(f64 ? "rhs_first_f64" : "rhs_first_f32", d,
                                                 a0, u, v, w, sa, acc, hdt, c6, s);
    if (e != cudaSuccess) return e;
    auto a1 = make_args<T, T>(g, sa, sa + n, sa + 2 * n, visc, sfs, mu, rho);
    e = stage<T, T, kModeMid>(f64 ? "rhs_mid_f64" : "rhs_mid_f32", d, a1, u, v, w, sb, acc,
                              hdt, c6, s);
    if (e != cudaSuccess) return e;
    auto a2 = make_args<T, T>(g, sb, sb + n, sb + 2 * n, visc, sfs, mu, rho);
    e = stage<T, T, kModeMid>(f64 ? "rhs_mid_f64" : "rhs_mid_f32", d, a2, u, v, w, sa, acc,
                              hdt, c6, s);
    if (e != cudaSuccess) return e;
    // the reference's stage-4 state is u + dt/2 k3 = sa (Q1)
    e = stage<T, T, kModeLast>(f64 ? "rhs_last_f64" : "rhs_last_f32", d, a1, u, v, w, nullptr,
                               acc, hdt, c6, s);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Grouped predictor: the RK4 stages of a batch of requests, one launch per
// stage (rhs_stage_grouped over per-stage job tables in device memory).
// ---------------------------------------------------------------------------
template <typename T, typename TI, int MODE>
static cudaError_t grouped_prepare_ctx() {
    const size_t sm = RhsSmem<T, TI, T, MODE>::bytes;
    cudaError_t e = cudaFuncSetAttribute(rhs_stage_grouped<T, TI, MODE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e == cudaSuccess) {
        const size_t two = 2 * (sm + 1024);
        const int pct = (int)std::min<size_t>(100, (two * 100 + 228 * 1024 - 1) / (228 * 1024));
        e = cudaFuncSetAttribute(rhs_stage_grouped<T, TI, MODE>,
                                 cudaFuncAttributePreferredSharedMemoryCarveout, pct);
    }
    return e;
}

// once per CUDA context (function attributes belong to the context)
template <typename T, typename TI, int MODE>
static cudaError_t grouped_prepare() {
    return once_per_context((const void*)&grouped_prepare_ctx<T, TI, MODE>,
                            &grouped_prepare_ctx<T, TI, MODE>);
}

// Job of one request for one stage (the arguments the single-request
// predictor_impl passes to that stage).
template <typename T, typename TI>
static StageJob<T, TI> make_job(const GroupMember& m, const TI* in_u, const TI* in_v,
                                const TI* in_w, T* st, T* acc, long long tile0) {
    StageJob<T, TI> J;
    const pf_grid* g = &m.grid;
    J.d = Dims{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    J.tl = make_tiling(J.d, kRhsTY);
    const long long n = J.d.n;
    J.a = make_args<T, TI>(g, in_u, in_v, in_w, nullptr, nullptr, m.mu, m.rho);
    J.u = m.u; J.v = m.v; J.w = m.w;
    J.su = st; J.sv = st ? st + n : nullptr; J.sw = st ? st + 2 * n : nullptr;
    J.au = acc; J.av = acc + n; J.aw = acc + 2 * n;
    J.hdt = 0.5 * m.dt;
    J.c6 = m.dt / 6.0;
    J.tile0 = tile0;
    return J;
}

int grouped_predictor_prepare(int prec) {
    if (prec == PF_FP64) {
        if (grouped_prepare<double, double, kModeK>() ||
            grouped_prepare<double, double, kModeFirst>() ||
            grouped_prepare<double, double, kModeMid>() ||
            grouped_prepare<double, double, kModeLast>())
            return PF_ERR_CUDA;
        return PF_OK;
    }
    if (grouped_prepare<float, double, kModeK>() ||
        grouped_prepare<float, double, kModeFirst>() ||
        grouped_prepare<float, float, kModeMid>() ||
        grouped_prepare<float, float, kModeLast>())
        return PF_ERR_CUDA;
    return PF_OK;
}

// Table layout: [error flag, 256 B][stage 0 jobs][stage 1][stage 2][stage 3],
// each stage's slot of `count` jobs 256-byte aligned.
static size_t job_slot_bytes(int count) {
    const size_t j = std::max(std::max(sizeof(StageJob<double, double>),
                                       sizeof(StageJob<float, double>)),
                              sizeof(StageJob<float, float>));
    return ((size_t)std::max(count, 1) * j + 255) & ~size_t(255);
}

size_t grouped_predictor_table_bytes(int count) { return 256 + 4 * job_slot_bytes(count); }

template <typename T>
static long long group_tiles(const GroupMember* m, int count) {
    long long tiles = 0;
    for (int r = 0; r < count; ++r) {
        Dims d{m[r].grid.nx, m[r].grid.ny, m[r].grid.nz,
               (long long)m[r].grid.nx * m[r].grid.ny * m[r].grid.nz};
        tiles += make_tiling(d, kRhsTY).ntiles;
    }
    return tiles;
}

template <typename T>
static int tables_impl(int rk4, const GroupMember* m, int count, void* table, cudaStream_t s) {
    const size_t slot = job_slot_bytes(count);
    std::vector<unsigned char> host(grouped_predictor_table_bytes(count), 0);
    unsigned char* st0 = host.data() + 256;
    long long tiles = 0;
    for (int r = 0; r < count; ++r) {
        const long long n = (long long)m[r].grid.nx * m[r].grid.ny * m[r].grid.nz;
        T* ws = (T*)m[r].R;
        T *sa = ws, *sb = ws + 3 * n, *acc = ws + 6 * n;
        // the first stage (and Euler's k) reads the FP64 state u, v, w -- three
        // separate fields; later stages read a stage state, 3 consecutive fields
        if (!rk4) {
            auto J = make_job<T, double>(m[r], m[r].u, m[r].v, m[r].w, nullptr, acc, tiles);
            std::memcpy(st0 + r * sizeof(J), &J, sizeof(J));
            tiles += J.tl.ntiles;
        } else {
            auto J0 = make_job<T, double>(m[r], m[r].u, m[r].v, m[r].w, sa, acc, tiles);
            auto J1 = make_job<T, T>(m[r], sa, sa + n, sa + 2 * n, sb, acc, tiles);
            auto J2 = make_job<T, T>(m[r], sb, sb + n, sb + 2 * n, sa, acc, tiles);
            auto J3 = make_job<T, T>(m[r], sa, sa + n, sa + 2 * n, nullptr, acc, tiles);
            std::memcpy(st0 + 0 * slot + r * sizeof(J0), &J0, sizeof(J0));
            std::memcpy(st0 + 1 * slot + r * sizeof(J1), &J1, sizeof(J1));
            std::memcpy(st0 + 2 * slot + r * sizeof(J2), &J2, sizeof(J2));
            std::memcpy(st0 + 3 * slot + r * sizeof(J3), &J3, sizeof(J3));
            tiles += J0.tl.ntiles;
        }
    }
    if (tiles != group_tiles<T>(m, count)) return PF_ERR_BAD_ARG;
    if (cudaMemcpyAsync(table, host.data(), host.size(), cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return PF_ERR_CUDA;
    return PF_OK;
}

int grouped_predictor_tables(int prec, int rk4, const GroupMember* m, int count, void* table,
                             cudaStream_t s) {
    if (count < 1 || count > kMaxGroupJobs || !table) return PF_ERR_BAD_ARG;
    int rc = grouped_predictor_prepare(prec);
    if (rc != PF_OK) return rc;
    return prec == PF_FP64 ? tables_impl<double>(rk4, m, count, table, s)
                           : tables_impl<float>(rk4, m, count, table, s);
}

template <typename T>
static cudaError_t grouped_impl(int rk4, const GroupMember* m, int count, void* table,
                                cudaStream_t s) {
    if (count < 1 || count > kMaxGroupJobs) return cudaErrorInvalidValue;
    const size_t slot = job_slot_bytes(count);
    char* tb = (char*)table;
    int* err = (int*)tb;
    char* st0 = tb + 256;
    const long long tiles = group_tiles<T>(m, count);
    const int grid = (int)std::min<long long>(tiles, num_sms() * 2);
    const dim3 blk(32, 8);
    const bool f64 = sizeof(T) == 8;
    if (!rk4) {
        PF_LAUNCH(f64 ? "grouped_euler_f64" : "grouped_euler_f32", s,
                  (rhs_stage_grouped<T, double, kModeK><<<grid, blk,
                      RhsSmem<T, double, T, kModeK>::bytes, s>>>(
                      (const StageJob<T, double>*)st0, count, tiles, err)));
        for (int r = 0; r < count; ++r) {
            const long long n = (long long)m[r].grid.nx * m[r].grid.ny * m[r].grid.nz;
            const T* acc = (const T*)m[r].R + 6 * n;
            const int gp = (int)std::min<long long>((n + 1023) / 1024, 4096);
            PF_LAUNCH("euler_apply", s, euler_apply<T><<<gp, 256, 0, s>>>(
                n, acc, acc + n, acc + 2 * n, m[r].dt, m[r].u, m[r].v, m[r].w));
        }
        return cudaGetLastError();
    }
    PF_LAUNCH(f64 ? "grouped_first_f64" : "grouped_first_f32", s,
              (rhs_stage_grouped<T, double, kModeFirst><<<grid, blk,
                  RhsSmem<T, double, T, kModeFirst>::bytes, s>>>(
                  (const StageJob<T, double>*)st0, count, tiles, err)));
    PF_LAUNCH(f64 ? "grouped_mid_f64" : "grouped_mid_f32", s,
              (rhs_stage_grouped<T, T, kModeMid><<<grid, blk, RhsSmem<T, T, T, kModeMid>::bytes,
                  s>>>((const StageJob<T, T>*)(st0 + slot), count, tiles, err)));
    PF_LAUNCH(f64 ? "grouped_mid_f64" : "grouped_mid_f32", s,
              (rhs_stage_grouped<T, T, kModeMid><<<grid, blk, RhsSmem<T, T, T, kModeMid>::bytes,
                  s>>>((const StageJob<T, T>*)(st0 + 2 * slot), count, tiles, err)));
    PF_LAUNCH(f64 ? "grouped_last_f64" : "grouped_last_f32", s,
              (rhs_stage_grouped<T, T, kModeLast><<<grid, blk,
                  RhsSmem<T, T, T, kModeLast>::bytes, s>>>(
                  (const StageJob<T, T>*)(st0 + 3 * slot), count, tiles, err)));
    return cudaGetLastError();
}

cudaError_t launch_grouped_predictor(int prec, int rk4, const GroupMember* m, int count,
                                     void* table, cudaStream_t s) {
    return prec == PF_FP64 ? grouped_impl<double>(rk4, m, count, table, s)
                           : grouped_impl<float>(rk4, m, count, table, s);
}

cudaError_t predictor_prepare(int prec) {
    cudaError_t e = cudaSuccess;
    if (prec == PF_FP64) {
        if ((e = tiled_prepare<double, double, kModeK>())) return e;
        if ((e = tiled_prepare<double, double, kModeFirst>())) return e;
        if ((e = tiled_prepare<double, double, kModeMid>())) return e;
        return tiled_prepare<double, double, kModeLast>();
    }
    if ((e = tiled_prepare<float, double, kModeK>())) return e;
    if ((e = tiled_prepare<float, double, kModeFirst>())) return e;
    if ((e = tiled_prepare<float, float, kModeMid>())) return e;
    return tiled_prepare<float, float, kModeLast>();
}

size_t predictor_ws_bytes(const pf_grid* g, int prec) {
    const size_t n = (size_t)g->nx * g->ny * g->nz;
    return 9 * n * (prec == PF_FP64 ? sizeof(double) : sizeof(float));
}

cudaError_t launch_predictor(const pf_grid* g, int prec, int rk4, double* u,
                             double* v, double* w, const void* visc,
                             double mu, double rho, const void* sfs,
                             double dt, void* ws, cudaStream_t s) {
    if (prec == PF_FP64)
        return predictor_impl<double>(g, rk4, u, v, w, (const double*)visc, mu,
                                      rho, (const double*)sfs, dt, (double*)ws, s);
    return predictor_impl<float>(g, rk4, u, v, w, (const float*)visc, mu, rho,
                                 (const float*)sfs, dt, (float*)ws, s);
}

}  // namespace pf
