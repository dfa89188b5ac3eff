// pf_sweep.cuh -- solver building blocks shared by the Krylov and multigrid
// kernels: the device scalar block, Laplacian coefficients, the tiled 7-point
// sweep with one-plane-ahead prefetch, and last-block reductions.
#pragma once
#include <algorithm>

#include "pf_common.cuh"

namespace pf {

struct BicgScalars {
    double rho1, rho2, alpha, omega, gamma, buf1, buf2;
    double max_res0, max_res, min_res;
    double scale;      // mixed: max|r| of the current refinement pass
    double max_b;      // mixed: max|b|
    double true_res;   // mixed: max|b - A x| of the last refinement pass
    int outer, total;  // mixed graph mode: refinement passes, inner iterations
    int k;             // index of the next CA kernel
    int iter;          // completed iterations
    int done;          // 0 running, 1 stopped, 2 stop after DP += alpha pp
    int status, max_it;
    unsigned int counter;
    int use64;          // mixed graph mode: the next refinement pass runs in FP64
    double prev_ratio;  // mixed graph mode: true residual ratio after the previous pass
};

template <typename T>
struct LapCoef {
    T c[3][3];
};

template <typename T>
static inline LapCoef<T> lap_coef(const pf_grid* g) {
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

// rows of the tile owned by each thread: 4 for FP32, 2 for FP64
template <typename T>
struct Rows {
    static constexpr int R = sizeof(T) == 4 ? 4 : 2;
    static constexpr int TY = 8 * R;
};

struct Tiling {
    int ntz, nty, ntx, xc;
    long long ntiles;
};

static inline int num_sms() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

static inline Tiling make_tiling(const Dims& d, int ty, int tz = 32) {
    Tiling t;
    t.ntz = (d.nz + tz - 1) / tz;
    t.nty = (d.ny + ty - 1) / ty;
    const long long yz = (long long)t.ntz * t.nty;
    // split x so the tiles fill the resident blocks (2 per SM) in whole
    // waves: one tile per block when the grid is small, 64-plane tiles when
    // it is large
    const long long slots = (long long)num_sms() * 2;
    const long long chunks = std::max<long long>(1, slots / yz);
    long long xc = (d.nx + chunks - 1) / chunks;
    xc = std::max<long long>(4, std::min<long long>(64, xc));
    t.xc = (int)std::min<long long>(xc, d.nx);
    t.ntx = (d.nx + t.xc - 1) / t.xc;
    t.ntiles = yz * t.ntx;
    return t;
}

static inline int tiled_grid(const Tiling& t) {
    return (int)std::min<long long>(t.ntiles, std::min(num_sms() * 2, kMaxPartials));
}

static inline int pointwise_grid(long long n) {
    long long b = (n + kBlock * 4 - 1) / (kBlock * 4);
    return (int)std::max<long long>(1, std::min<long long>(b, std::min(num_sms() * 8, kMaxPartials)));
}

// --------------------------------------------------------------------------
// Tiled 7-point sweep with one-plane-ahead prefetch.  The phase object Ph
// provides
//   Raw raw(q, i, j, k) -- loads the operand inputs of cell q = (i, j, k),
//   T   op(raw) -- the stencil operand,
//   Ext ext(q)  -- loads the epilogue inputs of an owned cell,
//   epi(q, centre operand, A operand, raw, ext) -- consumes an owned cell.
// Block: 32 x 8 threads; tile 32 (z) x 8R (y) x xc (x).
// --------------------------------------------------------------------------
template <typename T, class Ph>
__device__ __forceinline__ void sweep(const Dims& d, const Tiling& tl,
                                      const LapCoef<T>& cf, Ph& ph) {
    constexpr int R = Ph::R, TY = 8 * Ph::R;
    using Raw = typename Ph::Raw;
    using Ext = typename Ph::Ext;
    __shared__ T sm[TY + 2][34];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const long long plane = (long long)d.ny * d.nz;
    for (long long t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int tz = (int)(t % tl.ntz);
        const long long rr = t / tl.ntz;
        const int tyy = (int)(rr % tl.nty), txx = (int)(rr / tl.nty);
        const int k0 = tz * 32, j0 = tyy * TY, i0 = txx * tl.xc;
        const int i1 = min(i0 + tl.xc, d.nx);
        const int ez = min(32, d.nz - k0), ey = min(TY, d.ny - j0);
        bool vr[R];
        long long off[R];
        const int kk = k0 + tx;  // z index of this thread's cells
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int jl = ty + 8 * r;
            vr[r] = (tx < ez) && (jl < ey);
            off[r] = (long long)(j0 + jl) * d.nz + kk;
        }
        // this thread's halo cell of each plane (at most 2*32 + 2*TY cells)
        bool hv = false;
        int hy = 0, hz = 0, hj = 0, hk = 0;
        if (tid < 64) {
            const int h = tid & 31;
            hv = h < ez;
            hz = h + 1;
            hk = k0 + h;
            if (tid < 32) { hy = 0; hj = wrap(j0 - 1, d.ny); }
            else { hy = ey + 1; hj = wrap(j0 + ey, d.ny); }
        } else if (tid < 64 + 2 * TY) {
            const int u = tid - 64, h = u % TY;
            hv = h < ey;
            hy = h + 1;
            hj = j0 + h;
            if (u < TY) { hz = 0; hk = wrap(k0 - 1, d.nz); }
            else { hz = ez + 1; hk = wrap(k0 + ez, d.nz); }
        }
        const long long hoff = (long long)hj * d.nz + hk;
        T opP[R], opC[R], opN[R];
        Raw rawC[R], rawN[R];
        Ext extC[R];
        Raw hraw{};
        {
            const int im = wrap(i0 - 1, d.nx), ip = wrap(i0 + 1, d.nx);
            const long long bm = (long long)im * plane;
            const long long b0 = (long long)i0 * plane;
            const long long b1 = (long long)ip * plane;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (vr[r]) {
                    const int jj = j0 + ty + 8 * r;
                    opP[r] = ph.op(ph.raw(bm + off[r], im, jj, kk));
                    rawC[r] = ph.raw(b0 + off[r], i0, jj, kk);
                    rawN[r] = ph.raw(b1 + off[r], ip, jj, kk);
                    extC[r] = ph.ext(b0 + off[r]);
                    opC[r] = ph.op(rawC[r]);
                }
            }
            if (hv) hraw = ph.raw(b0 + hoff, i0, hj, hk);
        }
        for (int i = i0; i < i1; ++i) {
            const bool more = i + 1 < i1;
            const int ih = wrap(i + 1, d.nx), in2 = wrap(i + 2, d.nx);
            const long long bi = (long long)i * plane;
            const long long bh = (long long)ih * plane;
            const long long bn = (long long)in2 * plane;
            Raw rawNN[R];
            Ext extN[R];
            Raw hrawN{};
            if (more) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (vr[r]) {
                        rawNN[r] = ph.raw(bn + off[r], in2, j0 + ty + 8 * r, kk);
                        extN[r] = ph.ext(bh + off[r]);
                    }
                }
                if (hv) hrawN = ph.raw(bh + hoff, ih, hj, hk);
            }
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (vr[r]) sm[ty + 8 * r + 1][tx + 1] = opC[r];
            if (hv) sm[hy][hz] = ph.op(hraw);
            __syncthreads();
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (!vr[r]) continue;
                opN[r] = ph.op(rawN[r]);
                const int yy = ty + 8 * r + 1, zz = tx + 1;
                T b = T(0);
                b += opP[r] * cf.c[0][0];
                b += opC[r] * cf.c[0][1];
                b += opN[r] * cf.c[0][2];
                b += sm[yy - 1][zz] * cf.c[1][0];
                b += opC[r] * cf.c[1][1];
                b += sm[yy + 1][zz] * cf.c[1][2];
                b += sm[yy][zz - 1] * cf.c[2][0];
                b += opC[r] * cf.c[2][1];
                b += sm[yy][zz + 1] * cf.c[2][2];
                ph.epi(bi + off[r], opC[r], b, rawC[r], extC[r]);
            }
            __syncthreads();
#pragma unroll
            for (int r = 0; r < R; ++r) {
                opP[r] = opC[r];
                opC[r] = opN[r];
                rawC[r] = rawN[r];
                if (more) { rawN[r] = rawNN[r]; extC[r] = extN[r]; }
            }
            if (more) hraw = hrawN;
        }
    }
}

// --------------------------------------------------------------------------
// FP32 sweep with a cp.async pipeline (grids whose z extent is a multiple of
// TZ).  Block 32 x 8 threads, tile TZ (z, 32 or 64) x TY (y) x xc (x); the
// input planes (with a one-cell y/z halo) arrive in shared memory kAsyncDep
// planes ahead of use through 16-byte cp.async copies (the z halos as the
// 16-byte chunks that end and start next to the tile), so no thread holds
// prefetched data in registers.  Wider z tiles make every row copy a longer
// contiguous run of the plane.  Each thread's copy offsets are fixed per tile
// and computed once.  The stencil is evaluated with fused multiply-adds and
// one combined centre coefficient (these sweeps serve only the FP32
// multigrid preconditioner, whose rounding is its own).  The phase object
// provides
//   NR input fields rf[] and NE (0 or 1) epilogue fields ef[],
//   float op(const float* raw)  -- the stencil operand of a cell from its NR
//                                  raw values,
//   epi(q, op_c, A op, e)       -- consumes an owned cell (e: NE values).
// Dynamic shared memory: async_sweep_smem<TY, TZ, Ph>() bytes.
// --------------------------------------------------------------------------
constexpr int kAsyncDep = 2;  // planes in flight ahead of use

template <int TY, int TZ, class Ph>
struct AsyncGeom {
    static_assert(TZ == 32 || TZ == 64, "tile width");
    static_assert(TY % 8 == 0, "tile height");
    static constexpr int SZ = TZ + 8;          // row stride: halo chunks at 0..3 and TZ+4..TZ+7
    static constexpr int RS = kAsyncDep + 4;   // raw plane slots (3 in use, DEP + 1 in flight)
    static constexpr int ES = kAsyncDep + 2;   // epilogue plane slots
    static constexpr int RPos = (TY + 2) * SZ;
    static constexpr int EPos = TY * TZ;
    static constexpr int NCH = TZ / 4 + 2;     // 16-byte chunks per raw row
    static constexpr size_t bytes =
        (size_t)(RS * Ph::NR * RPos + ES * Ph::NE * EPos) * sizeof(float);
};

template <int TY, int TZ, class Ph>
constexpr size_t async_sweep_smem() {
    return AsyncGeom<TY, TZ, Ph>::bytes;
}

template <int BYTES>
__device__ __forceinline__ void cp_async_sm(void* smem, const void* gmem) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
    if (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" :: "r"(a), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" :: "r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit_group() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait_groups() {
    asm volatile("cp.async.wait_group %0;\n" :: "n"(N) : "memory");
}

template <int TY, int TZ, class Ph>
__device__ __forceinline__ void sweep_async(const Dims& d, const Tiling& tl,
                                            const LapCoef<float>& cf, Ph& ph) {
    using G = AsyncGeom<TY, TZ, Ph>;
    constexpr int SZ = G::SZ, RS = G::RS, ES = G::ES, RPos = G::RPos, EPos = G::EPos;
    constexpr int NR = Ph::NR, NE = Ph::NE, NCH = G::NCH;
    constexpr int RCH = (TY + 2) * NCH, RPT = (RCH + 255) / 256;    // raw chunks per plane, per thread
    constexpr int ECH = TY * (TZ / 4), EPT = (ECH + 255) / 256;     // epilogue chunks
    extern __shared__ __align__(16) float async_sm[];
    float* rr = async_sm;                    // [RS][NR][RPos]
    float* ee = async_sm + RS * NR * RPos;   // [ES][NE][EPos]
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const long long plane = (long long)d.ny * d.nz;
    // the centre coefficient of the three directions, applied once
    const float cc = (cf.c[0][1] + cf.c[1][1]) + cf.c[2][1];
    for (long long t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int tz = (int)(t % tl.ntz);
        const long long r2 = t / tl.ntz;
        const int tyy = (int)(r2 % tl.nty), txx = (int)(r2 / tl.nty);
        const int k0 = tz * TZ, j0 = tyy * TY, i0 = txx * tl.xc;
        const int i1 = min(i0 + tl.xc, d.nx);
        const int ey = min(TY, d.ny - j0);
        // This thread's copies are the same in every plane of the tile:
        // in-plane source offsets and shared-memory positions, computed once.
        // A single wrap suffices for the halo rows unless the grid is
        // shorter than a tile in y; nz is a multiple of TZ >= 32, so the halo
        // chunks k0 - 4 and k0 + TZ need one.
        const int kl = wrap(k0 - 4, d.nz), kr = wrap(k0 + TZ, d.nz);
        long long rg[RPT], eg[EPT];
        int rs[RPT], es[EPT];
        bool rv[RPT], ev[EPT];
#pragma unroll
        for (int m = 0; m < RPT; ++m) {
            const int p = tid + 256 * m;
            rv[m] = p < RCH;
            const int yy = rv[m] ? p / NCH : 0, ch = rv[m] ? p - yy * NCH : 0;
            const int j = j0 + yy - 1;
            const int jj = d.ny <= TY ? pmod(j, d.ny) : wrap(j, d.ny);
            const int k = ch == 0 ? kl : (ch == NCH - 1 ? kr : k0 + 4 * (ch - 1));
            rg[m] = (long long)jj * d.nz + k;
            rs[m] = yy * SZ + 4 * ch;
        }
#pragma unroll
        for (int m = 0; m < EPT; ++m) {
            const int p = tid + 256 * m;
            const int yy = p / (TZ / 4), ch = p - yy * (TZ / 4);
            ev[m] = p < ECH && yy < ey;
            eg[m] = (long long)(j0 + yy) * d.nz + k0 + 4 * ch;
            es[m] = yy * TZ + 4 * ch;
        }
        auto load_raw = [&](int xp, int slot) {
            const long long base = (long long)pmod(xp, d.nx) * plane;
#pragma unroll
            for (int f = 0; f < NR; ++f) {
                float* dst = rr + (slot * NR + f) * RPos;
                const float* src = ph.rf[f] + base;
#pragma unroll
                for (int m = 0; m < RPT; ++m)
                    if (rv[m]) cp_async_sm<16>(dst + rs[m], src + rg[m]);
            }
        };
        auto load_ext = [&](int xp, int slot) {
            const long long base = (long long)xp * plane;
#pragma unroll
            for (int f = 0; f < NE; ++f) {
                float* dst = ee + (slot * NE + f) * EPos;
                const float* src = ph.ef[f] + base;
#pragma unroll
                for (int m = 0; m < EPT; ++m)
                    if (ev[m]) cp_async_sm<16>(dst + es[m], src + eg[m]);
            }
        };
        auto rslot = [&](int xp) { return (xp - i0 + 1 + 4 * RS) % RS; };
        auto eslot = [&](int xp) { return (xp - i0 + 4 * ES) % ES; };
        load_raw(i0 - 1, rslot(i0 - 1));
        load_raw(i0, rslot(i0));
        load_raw(i0 + 1, rslot(i0 + 1));
        load_ext(i0, eslot(i0));
        cp_async_commit_group();
#pragma unroll
        for (int a = 1; a <= kAsyncDep; ++a) {
            if (i0 + a < i1) { load_raw(i0 + a + 1, rslot(i0 + a + 1)); load_ext(i0 + a, eslot(i0 + a)); }
            cp_async_commit_group();
        }
        const long long orow = (long long)(j0 + ty) * d.nz + k0 + tx;
        for (int i = i0; i < i1; ++i) {
            cp_async_wait_groups<kAsyncDep>();
            __syncthreads();
            if (i + kAsyncDep + 1 < i1) {
                load_raw(i + kAsyncDep + 2, rslot(i + kAsyncDep + 2));
                load_ext(i + kAsyncDep + 1, eslot(i + kAsyncDep + 1));
            }
            cp_async_commit_group();
            const float* pm = rr + rslot(i - 1) * NR * RPos;
            const float* pc = rr + rslot(i) * NR * RPos;
            const float* pp = rr + rslot(i + 1) * NR * RPos;
            const float* eb = ee + eslot(i) * NE * EPos;
            const long long bi = (long long)i * plane + orow;
            auto opat = [&](const float* pl, int c) {
                float r[NR];
#pragma unroll
                for (int f = 0; f < NR; ++f) r[f] = pl[f * RPos + c];
                return ph.op(r);
            };
#pragma unroll
            for (int r = 0; r < TY / 8; ++r) {
                const int yl = ty + 8 * r;
                if (yl >= ey) continue;
#pragma unroll
                for (int v = 0; v < TZ / 32; ++v) {
                    const int zl = tx + 32 * v;
                    const int c = (yl + 1) * SZ + zl + 4;
                    const float oc = opat(pc, c);
                    float b = oc * cc;
                    b = fmaf(opat(pm, c), cf.c[0][0], b);
                    b = fmaf(opat(pp, c), cf.c[0][2], b);
                    b = fmaf(opat(pc, c - SZ), cf.c[1][0], b);
                    b = fmaf(opat(pc, c + SZ), cf.c[1][2], b);
                    b = fmaf(opat(pc, c - 1), cf.c[2][0], b);
                    b = fmaf(opat(pc, c + 1), cf.c[2][2], b);
                    float e[NE > 0 ? NE : 1];
#pragma unroll
                    for (int f = 0; f < NE; ++f) e[f] = eb[f * EPos + yl * TZ + zl];
                    ph.epi(bi + (long long)(8 * r) * d.nz + 32 * v, oc, b, e);
                }
            }
        }
        cp_async_wait_groups<0>();
        __syncthreads();
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

__device__ __forceinline__ bool tid0() { return threadIdx.x == 0 && threadIdx.y == 0; }

static inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Programmatic dependent launch: the kernel may be launched while its
// predecessor in the stream is still finishing (launch latency and the
// predecessor's tail overlap); it must call pdl_wait() before touching any
// memory, which blocks until the predecessor has completed and its writes
// are visible.  Without the launch attribute pdl_wait() is a no-op.
__device__ __forceinline__ void pdl_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <typename... KArgs, typename... Args>
static inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block,
                                     size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

}  // namespace pf
