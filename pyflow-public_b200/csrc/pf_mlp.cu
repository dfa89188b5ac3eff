// pf_mlp.cu -- the SGS MLP closure on the 5th-generation tensor cores.
//
// Per cell: the nine cell-centred velocity gradients (grad_vel_center,
// src/metric/metric_staggered.py:215-268) scaled by 1/g_rms are the inputs of
// a 9 -> 128 -> 128 -> 6 MLP with tanh hidden layers, BF16 weights and FP32
// accumulation; its six outputs times out_scale are the stresses FXX, FYY, FZZ,
// FXY, FXZ, FYZ of the 'tensor' SFS slot (src/solver/velocity.py:262-267,...).
//
// One CTA of 512 threads per SM: four warpgroups, each with its own H tile,
// mbarrier and 128 of the SM's 512 TMEM columns, walk tiles of 128
// consecutive cells independently (named barriers per warpgroup) and share
// one copy of the weights; cell m of a warpgroup's tile is accumulator row /
// TMEM lane m and belongs to the warpgroup's thread m:
//   1. each thread computes its cell's gradients and writes 16 BF16 features
//      (9 + 7 zero pads) into the X tile in shared memory (the first 4 KB of
//      the H tile);
//   2. the warpgroup's thread 0 issues tcgen05.mma (M=128, N=128, K=16):
//      D1 = X W1^T;
//   3. each thread reads its D1 row from TMEM (tcgen05.ld, 32 columns per
//      wait), adds b1, truncates pairs of pre-activations to BF16, applies
//      the packed BF16 tanh and writes them into the H tile;
//   4. 8 tcgen05.mma (K=16 each): D2 = H W2^T; same epilogue back into H;
//   5. 8 tcgen05.mma with N=16: D3 = H W3^T; each thread adds b3 and writes
//      its six stresses (FP64) to global memory.
// The three layers accumulate one after another into the warpgroup's 128
// TMEM columns (each epilogue has read its accumulator before the next layer
// is issued).
// Completion of each MMA group is signalled by tcgen05.commit to an mbarrier;
// every wait on it is bounded and reports a timeout through an error flag.
//
// Shared-memory operands use the K-major, no-swizzle canonical layout of the
// UMMA descriptors: 8-row x 16-byte core matrices, K chunks 128 B apart
// (leading byte offset), 8-row groups 256 B apart (stride byte offset), one
// 4 KiB (128 rows) or 512 B (16 rows) block per 16-wide K slice.  The weights
// arrive pre-packed in exactly this layout (see pf_mlp_pack_bytes).
#include <cuda_bf16.h>
#include <stdint.h>

#include <algorithm>

#include "pf_common.cuh"
#include "pf_kernels.cuh"
#include "pf_profile.cuh"
#include "pf_umma.cuh"

namespace pf {

namespace mlp {

using namespace umma;

constexpr int kHidden = 128;
constexpr int kTile = 128;
constexpr int kThreads = 512;      // four warpgroups, one tile each
constexpr int kCtasPerSm = 1;      // four tiles in flight per SM
constexpr int kGroups = 4;
constexpr int kW1Bytes = 4096;      // 128 x 16 bf16
constexpr int kW2Bytes = 32768;     // 128 x 128 bf16
constexpr int kW3Bytes = 4096;      // 16 x 128 bf16
constexpr int kBiasBytes = (128 + 128 + 16) * 4;
constexpr int kPackBytes = kW1Bytes + kW2Bytes + kW3Bytes + kBiasBytes;
constexpr int kHBytes = 32768;      // 128 x 128 bf16; its first 4 KB hold the 128 x 16 X tile
constexpr unsigned kTmemCols = 512; // 128 columns per warpgroup

// byte offset of element (row r, col k) in a K-major no-swizzle tile whose
// 16-wide K slices are `slice` bytes apart
__device__ __forceinline__ uint32_t kmajor_off(int r, int k, int slice) {
    return (uint32_t)((k >> 4) * slice + (r >> 3) * 256 + ((k >> 3) & 1) * 128 + (r & 7) * 16 +
                      (k & 7) * 2);
}

// tanh of two FP32 pre-activations as one packed BF16 pair (a in the low
// half): both are truncated to BF16 by one byte permutation (their high
// halves), then the hardware tanh of the pair (tanh.approx.bf16x2) gives the
// two BF16 activations the next layer reads.  The epilogue is bound by the
// special-function unit; the permutation runs on the integer pipe, so a
// pair costs that unit one instruction.
__device__ __forceinline__ uint32_t tanh_pack_bf16x2(float a, float b) {
    const uint32_t x = __byte_perm(__float_as_uint(a), __float_as_uint(b), 0x7632);
    uint32_t y;
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(y) : "r"(x));
    return y;
}

__device__ __forceinline__ uint16_t bf16_bits(float x) {
    return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}

// The 30 velocity values the nine gradients of one cell need, loaded ahead
// of their use so the loads of the next tile overlap this tile's layers.
struct CellNb {
    double u[10], v[10], w[10];
};

__device__ inline void load_nb(const Dims& d, const double* __restrict__ u,
                               const double* __restrict__ v, const double* __restrict__ w,
                               long long cell, CellNb& nb) {
    int i, j, k;
    if (d.n < (1LL << 31)) {
        const unsigned c = (unsigned)cell, nz = (unsigned)d.nz, ny = (unsigned)d.ny;
        const unsigned r = c / nz;
        k = (int)(c - r * nz);
        i = (int)(r / ny);
        j = (int)(r - (unsigned)i * ny);
    } else {
        k = (int)(cell % d.nz);
        const long long r = cell / d.nz;
        j = (int)(r % d.ny);
        i = (int)(r / d.ny);
    }
    const int ip = wrap(i + 1, d.nx), im = wrap(i - 1, d.nx);
    const int jp = wrap(j + 1, d.ny), jm = wrap(j - 1, d.ny);
    const int kp = wrap(k + 1, d.nz), km = wrap(k - 1, d.nz);
    auto L = [&](const double* f, int a, int b, int c) { return __ldg(f + idx(d, a, b, c)); };
    // u: faces i, i+1 at (j,k), (j-1,k), (j+1,k), (j,k-1), (j,k+1)
    nb.u[0] = L(u, ip, j, k);  nb.u[1] = L(u, i, j, k);
    nb.u[2] = L(u, ip, jm, k); nb.u[3] = L(u, i, jm, k);
    nb.u[4] = L(u, ip, jp, k); nb.u[5] = L(u, i, jp, k);
    nb.u[6] = L(u, ip, j, km); nb.u[7] = L(u, i, j, km);
    nb.u[8] = L(u, ip, j, kp); nb.u[9] = L(u, i, j, kp);
    // v: faces j, j+1 at (i,k), (i-1,k), (i+1,k), (i,k-1), (i,k+1)
    nb.v[0] = L(v, i, jp, k);  nb.v[1] = L(v, i, j, k);
    nb.v[2] = L(v, im, jp, k); nb.v[3] = L(v, im, j, k);
    nb.v[4] = L(v, ip, jp, k); nb.v[5] = L(v, ip, j, k);
    nb.v[6] = L(v, i, jp, km); nb.v[7] = L(v, i, j, km);
    nb.v[8] = L(v, i, jp, kp); nb.v[9] = L(v, i, j, kp);
    // w: faces k, k+1 at (i,j), (i-1,j), (i+1,j), (i,j-1), (i,j+1)
    nb.w[0] = L(w, i, j, kp);  nb.w[1] = L(w, i, j, k);
    nb.w[2] = L(w, im, j, kp); nb.w[3] = L(w, im, j, k);
    nb.w[4] = L(w, ip, j, kp); nb.w[5] = L(w, ip, j, k);
    nb.w[6] = L(w, i, jm, kp); nb.w[7] = L(w, i, jm, k);
    nb.w[8] = L(w, i, jp, kp); nb.w[9] = L(w, i, jp, k);
}

// The nine cell-centred gradients (the arithmetic of pf_sgs_closure model 2)
__device__ inline void nb_gradients(const CellNb& nb, double dxi, double dyi, double dzi,
                                    double* g) {
    {
        const double* a = nb.u;
        const double c0 = 0.5 * (a[0] + a[1]);
        const double cym = 0.5 * (a[2] + a[3]);
        const double cyp = 0.5 * (a[4] + a[5]);
        const double czm = 0.5 * (a[6] + a[7]);
        const double czp = 0.5 * (a[8] + a[9]);
        g[0] = (a[0] - a[1]) * dxi;
        g[1] = (0.5 * (cyp + c0) - 0.5 * (c0 + cym)) * dyi;
        g[2] = (0.5 * (czp + c0) - 0.5 * (c0 + czm)) * dzi;
    }
    {
        const double* a = nb.v;
        const double c0 = 0.5 * (a[0] + a[1]);
        const double cxm = 0.5 * (a[2] + a[3]);
        const double cxp = 0.5 * (a[4] + a[5]);
        const double czm = 0.5 * (a[6] + a[7]);
        const double czp = 0.5 * (a[8] + a[9]);
        g[3] = (0.5 * (cxp + c0) - 0.5 * (c0 + cxm)) * dxi;
        g[4] = (a[0] - a[1]) * dyi;
        g[5] = (0.5 * (czp + c0) - 0.5 * (c0 + czm)) * dzi;
    }
    {
        const double* a = nb.w;
        const double c0 = 0.5 * (a[0] + a[1]);
        const double cxm = 0.5 * (a[2] + a[3]);
        const double cxp = 0.5 * (a[4] + a[5]);
        const double cym = 0.5 * (a[6] + a[7]);
        const double cyp = 0.5 * (a[8] + a[9]);
        g[6] = (0.5 * (cxp + c0) - 0.5 * (c0 + cxm)) * dxi;
        g[7] = (0.5 * (cyp + c0) - 0.5 * (c0 + cym)) * dyi;
        g[8] = (a[0] - a[1]) * dzi;
    }
}

// Writes the 128 hidden values of this thread's row: tanh(acc + bias) as
// BF16 (c_begin = 0).
__device__ __forceinline__ void hidden_epilogue(uint32_t taddr, const float* bias,
                                                uint8_t* H, int row, int c_begin) {
    // 32 columns per TMEM load and wait (the second warpgroup's loads and the
    // other CTA's work cover the wait)
#pragma unroll 1
    for (int c0 = c_begin; c0 < c_begin + kHidden; c0 += 32) {
        uint32_t r[32];
        tmem_ld32_issue(taddr + c0, r);
        tmem_wait_ld();
        // the bias of these 32 columns as 16-byte shared-memory loads
        const float4* b4 = reinterpret_cast<const float4*>(bias + c0);
#pragma unroll
        for (int q = 0; q < 32; q += 8) {
            const float4 ba = b4[q / 4], bb = b4[q / 4 + 1];
            const float bq[8] = {ba.x, ba.y, ba.z, ba.w, bb.x, bb.y, bb.z, bb.w};
            uint32_t packed[4];
#pragma unroll
            for (int e = 0; e < 4; ++e)
                packed[e] = tanh_pack_bf16x2(__uint_as_float(r[q + 2 * e]) + bq[2 * e],
                                             __uint_as_float(r[q + 2 * e + 1]) + bq[2 * e + 1]);
            // 8 consecutive k of one row are one 16-byte chunk
            *reinterpret_cast<uint4*>(H + kmajor_off(row, c0 + q, 4096)) =
                make_uint4(packed[0], packed[1], packed[2], packed[3]);
        }
    }
}

}  // namespace mlp

// scales[0] = 1/g_rms (input normalisation), scales[1] = output scale
__global__ void __launch_bounds__(mlp::kThreads, mlp::kCtasPerSm)
mlp_closure_kernel(Dims d, const double* __restrict__ u, const double* __restrict__ v,
                   const double* __restrict__ w, double dxi, double dyi, double dzi,
                   const uint8_t* __restrict__ wpack, const float* __restrict__ scales,
                   double* __restrict__ out, int* __restrict__ err) {
    using namespace mlp;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* sW1 = smem;
    uint8_t* sW2 = sW1 + kW1Bytes;
    uint8_t* sW3 = sW2 + kW2Bytes;
    float* sB = reinterpret_cast<float*>(sW3 + kW3Bytes);  // b1[128] b2[128] b3[16]
    // X shares the first 4 KB of the H tile: layer 1 reads X before the
    // epilogue that writes H, and the next tile writes X after layer 3 has
    // read H
    uint8_t* sH0 = reinterpret_cast<uint8_t*>(sB) + kBiasBytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sH0 + kGroups * kHBytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + kGroups);

    // thread `row` owns accumulator row / TMEM lane `row`: its features, its
    // 128 hidden columns in the epilogues and its outputs.  Warp w reads TMEM
    // lanes 32 w .. 32 w + 31.
    const int tid = threadIdx.x, warp = tid >> 5, grp = tid >> 7;
    const int row = tid & 127;  // the warpgroup's thread / TMEM lane
    uint8_t* sH = sH0 + grp * kHBytes;
    uint8_t* sX = sH;
    uint64_t* bar = bars + grp;
    auto gsync = [&]() { asm volatile("bar.sync %0, 128;" :: "r"(grp + 1) : "memory"); };
    auto gsync_and = [&](bool v) -> bool {
        int r;
        asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.b32 p, %1, 0;\n\t"
                     "bar.red.and.pred q, %2, 128, p;\n\tselp.b32 %0, 1, 0, q;\n\t}"
                     : "=r"(r) : "r"((int)v), "r"(grp + 1) : "memory");
        return r != 0;
    };
    // weights: a straight copy of the packed image
    {
        const uint4* src = reinterpret_cast<const uint4*>(wpack);
        uint4* dst = reinterpret_cast<uint4*>(smem);
        for (int q = tid; q < kPackBytes / 16; q += blockDim.x) dst[q] = src[q];
    }
    if (tid < kGroups) {
        mbar_init(&bars[tid], 1);
        mbar_init_fence();
    }
    if (warp == 0) tmem_alloc(tmem_slot, kTmemCols);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot + (uint32_t)(grp * 128);
    const uint32_t d1 = tmem, d2 = tmem, d3 = tmem;  // one 128-column accumulator
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
    const float in_scale = scales[0], out_scale = scales[1];
    const uint32_t id128 = instr_desc(kFmtBF16, 128, 128), id16 = instr_desc(kFmtBF16, 128, 16);
    uint32_t phase = 0;
    bool ok = true;
    const long long ntiles = (d.n + kTile - 1) / kTile;
    CellNb nb;
    const long long t0 = (long long)blockIdx.x * kGroups + grp, stride = (long long)gridDim.x * kGroups;
    {
        const long long c0 = t0 * kTile + row;
        if (t0 < ntiles && c0 < d.n) load_nb(d, u, v, w, c0, nb);
    }
    for (long long t = t0; t < ntiles && ok; t += stride) {
        const long long cell = t * kTile + row;
        const bool valid = cell < d.n;
        // ---- features -> X (row `row`)
        {
            double g[9];
            if (valid) nb_gradients(nb, dxi, dyi, dzi, g);
            uint32_t p[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const int k0 = 2 * e, k1 = 2 * e + 1;
                const float a = (valid && k0 < 9) ? float(g[k0]) * in_scale : 0.f;
                const float b = (valid && k1 < 9) ? float(g[k1]) * in_scale : 0.f;
                p[e] = (uint32_t)bf16_bits(a) | ((uint32_t)bf16_bits(b) << 16);
            }
            *reinterpret_cast<uint4*>(sX + kmajor_off(row, 0, 4096)) = make_uint4(p[0], p[1], p[2], p[3]);
            *reinterpret_cast<uint4*>(sX + kmajor_off(row, 8, 4096)) = make_uint4(p[4], p[5], p[6], p[7]);
        }
        fence_async_smem();
        tc_fence_before();
        gsync();
        // ---- layer 1
        if (row == 0) {
            tc_fence_after();
            mma_bf16(d1, smem_desc(smem_u32(sX)), smem_desc(smem_u32(sW1)), id128, 0u);
            commit(bar);
        }
        // the next tile's neighbourhood loads run under this tile's layers
        {
            const long long cn = (t + stride) * kTile + row;
            if (t + stride < ntiles && cn < d.n) load_nb(d, u, v, w, cn, nb);
        }
        ok = gsync_and(wait_phase(bar, phase));
        phase ^= 1u;
        if (!ok) break;
        tc_fence_after();
        hidden_epilogue(lane_base + d1, sB, sH, row, 0);
        fence_async_smem();
        tc_fence_before();
        gsync();
        // ---- layer 2
        if (row == 0) {
            tc_fence_after();
#pragma unroll 1
            for (int kb = 0; kb < 8; ++kb)
                mma_bf16(d2, smem_desc(smem_u32(sH) + kb * 4096), smem_desc(smem_u32(sW2) + kb * 4096),
                         id128, kb > 0 ? 1u : 0u);
            commit(bar);
        }
        ok = gsync_and(wait_phase(bar, phase));
        phase ^= 1u;
        if (!ok) break;
        tc_fence_after();
        hidden_epilogue(lane_base + d2, sB + 128, sH, row, 0);
        fence_async_smem();
        tc_fence_before();
        gsync();
        // ---- layer 3
        if (row == 0) {
            tc_fence_after();
#pragma unroll 1
            for (int kb = 0; kb < 8; ++kb)
                mma_bf16(d3, smem_desc(smem_u32(sH) + kb * 4096), smem_desc(smem_u32(sW3) + kb * 512),
                         id16, kb > 0 ? 1u : 0u);
            commit(bar);
        }
        ok = gsync_and(wait_phase(bar, phase));
        phase ^= 1u;
        if (!ok) break;
        tc_fence_after();
        {
            float y[16];
            mlp::tmem_ld16(lane_base + d3, y);
            if (valid) {
                const float* b3 = sB + 256;
#pragma unroll
                for (int c = 0; c < 6; ++c)
                    out[(long long)c * d.n + cell] = double(y[c] + b3[c]) * double(out_scale);
            }
        }
        tc_fence_before();
        gsync();
    }
    if (!ok) {
        // an MMA group did not signal completion: record it, and give the
        // tensor core one more bounded wait before the TMEM is released
        if (row == 0) atomicExch(err, 1);
        wait_phase(bar, phase ^ 1u);  // the phase whose wait gave up
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, kTmemCols);
    }
}

size_t mlp_smem_bytes() {
    return (size_t)mlp::kPackBytes + mlp::kGroups * mlp::kHBytes + 64;
}

static cudaError_t mlp_attrs() {
    cudaError_t e = cudaFuncSetAttribute(mlp_closure_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)mlp_smem_bytes());
    if (e != cudaSuccess) return e;
    // the largest shared-memory carveout (170 KB per CTA)
    return cudaFuncSetAttribute(mlp_closure_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared);
}

cudaError_t mlp_prepare() { return once_per_context((const void*)&mlp_attrs, &mlp_attrs); }

cudaError_t launch_mlp(const pf_grid* g, const double* u, const double* v,
                       const double* w, const void* wpack, const float* scales,
                       double* out, int* err, cudaStream_t s) {
    Dims d{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    const size_t smem = mlp_smem_bytes();
    {   // once per CUDA context (function attributes belong to the context)
        const cudaError_t e = once_per_context((const void*)&mlp_attrs, &mlp_attrs);
        if (e != cudaSuccess) return e;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long ntiles = (d.n + mlp::kTile - 1) / mlp::kTile;
    // one CTA per SM (four tiles in flight, the layers of some overlapping
    // the epilogues of the others; the weights are shared, 170 KB of shared
    // memory and all 512 TMEM columns per CTA)
    const int grid = (int)std::min<long long>((ntiles + mlp::kGroups - 1) / mlp::kGroups,
                                              (long long)mlp::kCtasPerSm * sms);
    PF_LAUNCH("mlp_closure", s, mlp_closure_kernel<<<grid, mlp::kThreads, smem, s>>>(
        d, u, v, w, 1.0 / g->dx, 1.0 / g->dy, 1.0 / g->dz, (const uint8_t*)wpack, scales,
        out, err));
    return cudaGetLastError();
}

}  // namespace pf

extern "C" size_t pf_mlp_pack_bytes(void) { return (size_t)pf::mlp::kPackBytes; }

extern "C" int pf_mlp_closure(const pf_grid* g, const double* u, const double* v,
                              const double* w, const void* wpack,
                              const float* scales, double* out, int* err,
                              void* stream) {
    if (!g || g->nx < 2 || g->ny < 2 || g->nz < 2 || !(g->dx > 0) || !(g->dy > 0) ||
        !(g->dz > 0) || !u || !v || !w || !wpack || !scales || !out || !err)
        return PF_ERR_BAD_ARG;
    if (((uintptr_t)wpack & 15) != 0) return PF_ERR_BAD_ARG;
    return pf::launch_mlp(g, u, v, w, wpack, scales, out, err, (cudaStream_t)stream) == cudaSuccess
               ? PF_OK : PF_ERR_CUDA;
}
