// pf_mlsrc.cu -- the reference's 'source'-type ML closure on the 5th-generation
// tensor cores.
//
// The closure is sfsmodel_ML.residual_stress.update
// (src/sfsmodel/sfsmodel_ML.py:354-401): 21 features per cell (:407-460), the
// features of the cell and of its 12 neighbours at +-1, +-2 along each axis
// divided by the normalisation constants (:464-510, 273 inputs), the gated
// network NeuralNetworkModel2 (:77-116)
//     H1 = tanh(fc1 x),  H2 = tanh(fc2 H1) * tanh(fcG x),
//     H4 = tanh(fc3 H2) * tanh(fcG2 x),  out = fc4 H4   (273 -> 200 -> 18),
// and the closure terms GX/GY/GZ as sums of central differences of outputs
// 0-8 (:513-590), whose face interpolants the RHS subtracts
// (src/solver/velocity.py:374-383, interp_sc_x/y/z,
// src/metric/metric_staggered.py:112-124).  The reference computes in FP32.
//
// Launches:
//   1. mlsrc_features: one thread per cell.  Cell-centred u, v, w (FP64
//      interpolation, rounded to FP32), their central first and second
//      differences in FP32 (every direction with the x spacing, as the
//      reference), divided by the normalisation constants.  Each value is
//      stored as a TF32 pair, hi = value rounded to TF32 and lo = value - hi
//      (exact), in rows of 24 floats (21 features + 3 zeros) per cell.
//   2. mlsrc_layer: one CTA of 512 threads per (tile of 128 cells, weight
//      matrix), two CTAs per SM (256 TMEM columns each), so one CTA's
//      epilogue overlaps the other's products.  A loop over K steps of 8
//      streams the A rows (layer 1: eight features of one of the 13 stencil
//      neighbours' feature rows; later layers: eight columns of the previous
//      layer's activations) and the weight rows into shared memory with
//      cp.async, four stages deep, while one thread issues three
//      tcgen05.mma kind::tf32 per K step,
//          D += A_lo B_hi + A_hi B_lo + A_hi B_hi,
//      which keeps about 21 bits of every FP32 product (the dropped A_lo B_lo
//      term and the TF32 truncation of the lo parts are below 2^-21 of the
//      product), into an FP32 accumulator in TMEM.  The epilogue (four warps per
//      TMEM lane quarter, each taking every fourth 16-column group; TMEM lane
//      m is cell m of the tile) adds the bias and applies
//      the layer's activation: tanh split into a TF32 pair (fc1); tanh stored
//      as FP32 (the gates fcG, fcG2); tanh times the gate, split into a pair
//      (fc2, fc3); the affine output (fc4, outputs 0-15, of which 0-8 are
//      used).  Layer 1 runs fc1, fcG and fcG2 as one launch (grid y = 3).
//   3. mlsrc_terms: one thread per cell; GX, GY, GZ (FP32 central
//      differences, stored as FP64 like the reference's GX/GY/GZ) and the
//      face sources 0.5 (G[i] + G[i-1]) in FP64.
// The weights are packed once per parameter update (mlsrc_pack*): TF32 pairs
// of fc1, fcG, fcG2 (rows padded to 208, K laid out as 13 x 24), fc2, fc3
// (208 x 200) and fc4 (16 x 200), the biases padded to 208 / 16, and the 21
// normalisation constants.
#include <stdint.h>

#include <algorithm>

#include "pf_common.cuh"
#include "pf_kernels.cuh"
#include "pf_profile.cuh"
#include "pf_sweep.cuh"
#include "pf_umma.cuh"

namespace pf {
namespace mlsrc {

using namespace umma;

constexpr int kF = 21;              // features per cell
constexpr int kFP = 24;             // feature row (3 K steps of 8)
constexpr int kPts = 13;            // stencil points of the network input
constexpr int kK1 = kPts * kFP;     // layer-1 K (312)
constexpr int kH = 200;             // hidden width, K of layers 2-4
constexpr int kNP = 208;            // hidden width padded to the MMA's N granule
constexpr int kNO = 16;             // outputs computed by fc4 (0-8 used)
constexpr int kTile = 128;          // cells per tile = MMA M = TMEM lanes
constexpr int kThreads = 512;       // 16 warps: four per TMEM lane quarter
constexpr long long kSpin = 1LL << 20;   // polls of one bounded mbarrier wait

enum Epi { kEpiTanhSplit = 0, kEpiTanh = 1, kEpiGatedSplit = 2, kEpiLinear = 3 };

// --- pack layout (in floats) ------------------------------------------------
// matrices 0 fc1, 1 fcG, 2 fcG2, 3 fc2, 4 fc3, 5 fc4
__host__ __device__ constexpr int mat_rows(int m) { return m == 5 ? kNO : kNP; }
__host__ __device__ constexpr int mat_k(int m) { return m < 3 ? kK1 : kH; }
__host__ __device__ constexpr long long mat_floats(int m) {
    return (long long)mat_rows(m) * mat_k(m);
}
// hi part of matrix m, its lo part follows immediately
__host__ __device__ constexpr long long w_off(int m) {
    return m == 0 ? 0 : w_off(m - 1) + 2 * mat_floats(m - 1);
}
__host__ __device__ constexpr long long bias_off(int m) {
    return m == 0 ? w_off(6) : bias_off(m - 1) + mat_rows(m - 1);
}
constexpr long long kNormOff = bias_off(6);
constexpr long long kPackFloats = (kNormOff + 32 + 63) / 64 * 64;

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// --- packing ------------------------------------------------------------------
// K values per chunk of the layers' K loops: one MMA K step (8)
__host__ __device__ constexpr int chunk_k(int) { return 8; }

// W (rows x cols, row-major as torch stores nn.Linear.weight) into matrix m of
// the pack: per K chunk, the TF32 hi parts of all rows and then the lo parts,
// each in the K-major core-matrix order of the MMA's shared-memory operand,
// so a chunk is one flat copy.  Layer-1 K index s*24 + f takes input column
// s*21 + f.
__global__ void pack_matrix(const float* __restrict__ W, int rows, int cols, int m,
                            float* __restrict__ pack) {
    const int R = mat_rows(m), K = mat_k(m), CK = chunk_k(m);
    const int total = R * K;
    const int part = R * CK;  // floats of one part of a chunk
    float* base = pack + w_off(m);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int r = e / K, k = e - r * K;
        int c = k;
        if (m < 3) {
            const int s = k / kFP, f = k - s * kFP;
            c = f < kF ? s * kF + f : cols;
        }
        const float x = (r < rows && c < cols) ? W[(long long)r * cols + c] : 0.f;
        const int ch = k / CK, kk = k - ch * CK;
        float* dst = base + (long long)ch * 2 * part + piece_off(r, kk >> 2, R) / 4 + (kk & 3);
        const float h = tf32_rna(x);
        dst[0] = h;
        dst[part] = x - h;
    }
}

__global__ void pack_vector(const float* __restrict__ b, int n, int npad,
                            float* __restrict__ dst) {
    for (int e = threadIdx.x; e < npad; e += blockDim.x) dst[e] = e < n ? b[e] : 0.f;
}

// --- features -------------------------------------------------------------------
// cell-centred value of the face field at cell (i, j, k), rounded to FP32
__device__ __forceinline__ float centre(const Dims& d, const double* f, int axis, int i, int j,
                                        int k) {
    const double a = f[idx(d, i, j, k)];
    const double b = axis == 0 ? f[idx(d, wrap(i + 1, d.nx), j, k)]
                   : axis == 1 ? f[idx(d, i, wrap(j + 1, d.ny), k)]
                               : f[idx(d, i, j, wrap(k + 1, d.nz))];
    return (float)(0.5 * (b + a));
}

__global__ void __launch_bounds__(256)
mlsrc_features(Dims d, const double* __restrict__ u, const double* __restrict__ v,
               const double* __restrict__ w, float two_dx, float dx2,
               const float* __restrict__ norm, float* __restrict__ f_hi,
               float* __restrict__ f_lo) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;  // cells < 2^31 (checked)
    if (c >= d.n) return;
    const int k = c % d.nz, r = c / d.nz;
    const int j = r % d.ny, i = r / d.ny;
    const int ip = wrap(i + 1, d.nx), im = wrap(i - 1, d.nx);
    const int jp = wrap(j + 1, d.ny), jm = wrap(j - 1, d.ny);
    const int kp = wrap(k + 1, d.nz), km = wrap(k - 1, d.nz);
    float x[kFP];
    const double* fld[3] = {u, v, w};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const double* f = fld[q];
        const float a = centre(d, f, q, i, j, k);
        const float xp = centre(d, f, q, ip, j, k), xm = centre(d, f, q, im, j, k);
        const float yp = centre(d, f, q, i, jp, k), ym = centre(d, f, q, i, jm, k);
        const float zp = centre(d, f, q, i, j, kp), zm = centre(d, f, q, i, j, km);
        x[q] = a;
        x[3 + 3 * q + 0] = (xp - xm) / two_dx;
        x[3 + 3 * q + 1] = (yp - ym) / two_dx;
        x[3 + 3 * q + 2] = (zp - zm) / two_dx;
        x[12 + 3 * q + 0] = (xp - 2.f * a + xm) / dx2;
        x[12 + 3 * q + 1] = (yp - 2.f * a + ym) / dx2;
        x[12 + 3 * q + 2] = (zp - 2.f * a + zm) / dx2;
    }
    float4* oh = reinterpret_cast<float4*>(f_hi + (long long)c * kFP);
    float4* ol = reinterpret_cast<float4*>(f_lo + (long long)c * kFP);
#pragma unroll
    for (int q = 0; q < kFP / 4; ++q) {
        float h[4], l[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int fi = 4 * q + e;
            const float val = fi < kF ? x[fi] / norm[fi] : 0.f;
            h[e] = tf32_rna(val);
            l[e] = val - h[e];
        }
        oh[q] = make_float4(h[0], h[1], h[2], h[3]);
        ol[q] = make_float4(l[0], l[1], l[2], l[3]);
    }
}

// --- layers ---------------------------------------------------------------------
// Activation tiles (the A operand of layers 2-4): per tile of 128 cells, per K
// step of 8, the hi parts of the 128 rows and then the lo parts, each in the
// core-matrix order of the shared-memory operand (one flat copy per chunk).
constexpr int kActK = 8;                        // K values per chunk (one MMA K step)
constexpr int kActChunk = 2 * kTile * kActK;    // floats of one chunk (both parts)
constexpr int kActTile = (kH / kActK) * kActChunk;  // floats of one tile (K = 200)
// Gate tiles: per tile, column-major [208][128] FP32, so the lanes of a warp
// (consecutive cells) touch consecutive addresses in the epilogues.
constexpr int kGateTile = kNP * kTile;

struct LayerMat {
    const float* w;       // the matrix in the pack (chunk-tiled TF32 pairs)
    const float* bias;
    const float* gate;    // kEpiGatedSplit: gate tiles
    float* out;           // activation tiles, gate tiles or (kEpiLinear) (n, 16) rows
    int epi;
};

struct LayerArgs {
    LayerMat m[3];        // blockIdx.y selects
    const float* a_hi;    // layer 1: feature rows (hi, lo); later: activation tiles
    const float* a_lo;
    Dims d;
};

// layer-1 stencil: the cell, then +1/-1 along x, y, z, then +2/-2
__device__ __forceinline__ int stencil_cell(const Dims& d, int c, int s) {
    if (s == 0) return c;
    const int k = c % d.nz, r = c / d.nz;
    const int j = r % d.ny, i = r / d.ny;
    const int sh = s <= 6 ? 1 : 2;
    const int t = (s - 1) % 6;           // 0 +x, 1 -x, 2 +y, 3 -y, 4 +z, 5 -z
    const int dlt = (t & 1) ? -sh : sh;
    const int ax = t >> 1;
    const int ii = ax == 0 ? pmod(i + dlt, d.nx) : i;
    const int jj = ax == 1 ? pmod(j + dlt, d.ny) : j;
    const int kk = ax == 2 ? pmod(k + dlt, d.nz) : k;
    return (int)idx(d, ii, jj, kk);
}

template <int KC, int NP>
struct LayerGeom {
    static constexpr int kAPart = kTile * KC * 32;  // bytes of one TF32 part of A
    static constexpr int kBPart = NP * KC * 32;
    static constexpr int kStage = 2 * (kAPart + kBPart);
    static constexpr int kTmemCols = NP <= 32 ? 32 : NP <= 64 ? 64 : NP <= 128 ? 128 : 256;
};

// NS stages, barriers, bias, layer-1 neighbour table
template <int KC, int NP, bool GATHER, int NS>
constexpr size_t layer_smem() {
    return NS * LayerGeom<KC, NP>::kStage + 64 + kNP * 4 + (GATHER ? kPts * kTile * 4 : 0);
}

// flat 16-byte copy of `bytes` (a multiple of 16) by all threads
__device__ __forceinline__ void copy_flat(uint8_t* dst, const float* src, int bytes, int tid) {
    const uint8_t* s8 = reinterpret_cast<const uint8_t*>(src);
#pragma unroll 4
    for (int o = tid * 16; o < bytes; o += kThreads * 16) cp_async_sm<16>(dst + o, s8 + o);
}

// KC K steps of 8 per chunk, NCH chunks, MMA N = NP, NS shared-memory
// stages (the copies of chunk c + NS - 1 are issued while chunk c is
// multiplied).  GATHER: A rows are the feature rows of the stencil neighbours
// (chunk c = K step c % 3 of stencil point c / 3).
template <int KC, int NCH, int NP, bool GATHER, int NS>
__global__ void __launch_bounds__(kThreads, 2)
mlsrc_layer(LayerArgs args, int* __restrict__ err) {
    using G = LayerGeom<KC, NP>;
    constexpr int K = NCH * KC * 8;       // B row length
    constexpr int QA = 2 * KC;            // 16-byte pieces of one row per chunk
    static_assert(!GATHER || (KC == 1 && K == kK1), "layer-1 chunking");
    static_assert(GATHER || (K == kH && KC * 8 == kActK), "dense chunking");
    static_assert(NS >= 2 && NS <= 6 && NCH >= NS, "stages");
    extern __shared__ __align__(1024) uint8_t smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + NS * G::kStage);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + NS);
    float* sbias = reinterpret_cast<float*>(smem + NS * G::kStage + 64);
    int* nbr = reinterpret_cast<int*>(sbias + kNP);

    const LayerMat& M = args.m[blockIdx.y];
    const Dims d = args.d;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int tile = blockIdx.x;
    const int tile0 = tile * kTile;
    const int last = (int)d.n - 1;

    if (GATHER) {
#pragma unroll 1
        for (int e = tid; e < kPts * kTile; e += kThreads) {
            const int s = e / kTile, r = e - s * kTile;
            nbr[e] = stencil_cell(d, min(tile0 + r, last), s);
        }
    }
    for (int e = tid; e < NP; e += kThreads) sbias[e] = M.bias[e];
    if (tid == 0) {
        for (int q = 0; q < NS; ++q) mbar_init(&bar[q], 1);
        mbar_init_fence();
    }
    if (warp == 0) tmem_alloc(tmem_slot, G::kTmemCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    auto load_chunk = [&](int c, int stage) {
        uint8_t* sA = smem + stage * G::kStage;
        if (GATHER) {
#pragma unroll 4
            for (int e = tid; e < 2 * kTile * QA; e += kThreads) {
                const int q = e % QA, r = (e / QA) % kTile, part = e / (QA * kTile);
                // chunk c: K step c % 3 of stencil point c / 3
                const int sp = c / 3, sub = c - 3 * sp;
                const float* src = (part ? args.a_lo : args.a_hi) +
                                   (long long)nbr[sp * kTile + r] * kFP + sub * 8 + q * 4;
                cp_async_sm<16>(sA + part * G::kAPart + piece_off(r, q, kTile), src);
            }
        } else {
            copy_flat(sA, args.a_hi + (long long)tile * kActTile + c * kActChunk, 2 * G::kAPart,
                      tid);
        }
        copy_flat(sA + 2 * G::kAPart, M.w + (long long)c * (2 * NP * KC * 8), 2 * G::kBPart, tid);
    };

    constexpr uint32_t idesc = instr_desc(kFmtTF32, kTile, NP);
    bool ok = true;
#pragma unroll
    for (int q = 0; q < NS - 1; ++q) {  // one copy group per chunk
        load_chunk(q, q);
        cp_async_commit_group();
    }
#pragma unroll 1
    for (int c = 0; c < NCH; ++c) {
        const int stage = c % NS;
        const int nxt = c + NS - 1;
        if (nxt < NCH) {
            // the stage of chunk nxt last held chunk c - 1: wait for its MMAs
            if (c >= 1) ok = ok && wait_phase(&bar[(c - 1) % NS], ((c - 1) / NS) & 1, kSpin);
            if (ok) load_chunk(nxt, nxt % NS);
        }
        cp_async_commit_group();
        cp_async_wait_groups<NS - 1>();  // chunk c's copies have landed
        fence_async_smem();
        ok = __syncthreads_and(ok);
        if (!ok) break;
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(smem + stage * G::kStage);
            const uint32_t b0 = a0 + 2 * G::kAPart;
#pragma unroll
            for (int j = 0; j < KC; ++j) {
                const uint64_t ah = smem_desc(a0 + j * kTile * 32);
                const uint64_t al = smem_desc(a0 + G::kAPart + j * kTile * 32);
                const uint64_t bh = smem_desc(b0 + j * NP * 32);
                const uint64_t bl = smem_desc(b0 + G::kBPart + j * NP * 32);
                mma_tf32(tmem, al, bh, idesc, (c | j) ? 1u : 0u);
                mma_tf32(tmem, ah, bl, idesc, 1u);
                mma_tf32(tmem, ah, bh, idesc, 1u);
            }
            commit(&bar[stage]);
        }
    }
    // MMAs complete in order: the last chunk's commit covers all of them
    if (ok) ok = wait_phase(&bar[(NCH - 1) % NS], ((NCH - 1) / NS) & 1, kSpin);
    ok = __syncthreads_and(ok);
    if (ok) {
        tc_fence_after();
        // warp w reads TMEM lane quarter w % 4 (cells 32 (w % 4) ..) and
        // every fourth 16-column group from group w / 4
        const int row = (warp & 3) * 32 + (tid & 31);
        const int cell = tile0 + row;
        const uint32_t taddr = tmem + ((uint32_t)((warp & 3) * 32) << 16);
        const int ncol = M.epi == kEpiLinear ? kNO : kH;
        float* const act = M.out + (long long)tile * kActTile;     // split outputs
        float* const gto = M.out + (long long)tile * kGateTile;    // gate outputs
        const float* const gti = M.gate + (long long)tile * kGateTile;
#pragma unroll 1
        for (int c0 = 16 * (warp >> 2); c0 < NP; c0 += 64) {
            float y[16];
            tmem_ld16(taddr + c0, y);  // every lane of the warp takes part
            const int cn = min(16, ncol - c0);
            if (cn <= 0) continue;
            if (M.epi == kEpiLinear) {
                if (cell > last) continue;
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    *reinterpret_cast<float4*>(M.out + (long long)cell * kNO + c0 + 4 * q) =
                        make_float4(y[4 * q] + sbias[c0 + 4 * q], y[4 * q + 1] + sbias[c0 + 4 * q + 1],
                                    y[4 * q + 2] + sbias[c0 + 4 * q + 2],
                                    y[4 * q + 3] + sbias[c0 + 4 * q + 3]);
            } else if (M.epi == kEpiTanh) {
#pragma unroll
                for (int e = 0; e < 16; ++e)
                    if (e < cn) gto[(c0 + e) * kTile + row] = tanhf(y[e] + sbias[c0 + e]);
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (4 * q >= cn) break;
                    float hv[4], lv[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const int col = c0 + 4 * q + e;
                        float h = tanhf(y[4 * q + e] + sbias[col]);
                        if (M.epi == kEpiGatedSplit) h = h * gti[col * kTile + row];
                        hv[e] = tf32_rna(h);
                        lv[e] = h - hv[e];
                    }
                    // column col = c0 + 4q .. +3 is K piece (col % 8) / 4 of chunk col / 8
                    const int col = c0 + 4 * q, ch = col / kActK, kk = col - ch * kActK;
                    float* dst = act + ch * kActChunk + piece_off(row, kk >> 2, kTile) / 4;
                    *reinterpret_cast<float4*>(dst) = make_float4(hv[0], hv[1], hv[2], hv[3]);
                    *reinterpret_cast<float4*>(dst + kTile * kActK) =
                        make_float4(lv[0], lv[1], lv[2], lv[3]);
                }
            }
        }
    } else {
        // a wait gave up: record it, and give the tensor core one more
        // bounded wait for each stage before the TMEM is released
        if (tid == 0) atomicExch(err, 1);
        for (int q = 0; q < NS; ++q) wait_phase(&bar[q], 0, kSpin);
        cp_async_wait_groups<0>();
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, G::kTmemCols);
    }
}

// --- closure terms and face sources ---------------------------------------------
__device__ __forceinline__ float pch(const float* P, long long c, int ch) {
    return P[c * kNO + ch];
}

// sum over axes of the central difference of output channel ch0 + axis
__device__ __forceinline__ float div_term(const Dims& d, const float* P, int i, int j, int k,
                                          int ch0, float two_dx) {
    const float gx = (pch(P, idx(d, wrap(i + 1, d.nx), j, k), ch0) -
                      pch(P, idx(d, wrap(i - 1, d.nx), j, k), ch0)) / two_dx;
    const float gy = (pch(P, idx(d, i, wrap(j + 1, d.ny), k), ch0 + 1) -
                      pch(P, idx(d, i, wrap(j - 1, d.ny), k), ch0 + 1)) / two_dx;
    const float gz = (pch(P, idx(d, i, j, wrap(k + 1, d.nz)), ch0 + 2) -
                      pch(P, idx(d, i, j, wrap(k - 1, d.nz)), ch0 + 2)) / two_dx;
    return gx + gy + gz;
}

__global__ void __launch_bounds__(256)
mlsrc_terms(Dims d, const float* __restrict__ P, float two_dx, double* __restrict__ G,
            double* __restrict__ S) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d.n) return;
    const int k = c % d.nz, r = c / d.nz;
    const int j = r % d.ny, i = r / d.ny;
    const double gx = (double)div_term(d, P, i, j, k, 0, two_dx);
    const double gy = (double)div_term(d, P, i, j, k, 3, two_dx);
    const double gz = (double)div_term(d, P, i, j, k, 6, two_dx);
    const double gxm = (double)div_term(d, P, wrap(i - 1, d.nx), j, k, 0, two_dx);
    const double gym = (double)div_term(d, P, i, wrap(j - 1, d.ny), k, 3, two_dx);
    const double gzm = (double)div_term(d, P, i, j, wrap(k - 1, d.nz), 6, two_dx);
    G[c] = gx;
    G[d.n + c] = gy;
    G[2 * d.n + c] = gz;
    S[c] = 0.5 * (gx + gxm);
    S[d.n + c] = 0.5 * (gy + gym);
    S[2 * d.n + c] = 0.5 * (gz + gzm);
}

// --- workspace --------------------------------------------------------------------
struct Ws {
    float *f_hi, *f_lo, *act_a, *act_b, *g1, *g2, *p;
};

static size_t ws_layout(long long n, char* base, Ws* w) {
    const long long ntiles = (n + kTile - 1) / kTile;
    size_t off = 0;
    auto take = [&](long long floats) {
        float* p = base ? reinterpret_cast<float*>(base + off) : nullptr;
        off += ((size_t)floats * sizeof(float) + 255) & ~(size_t)255;
        return p;
    };
    Ws t;
    t.f_hi = take(n * kFP);
    t.f_lo = take(n * kFP);
    t.act_a = take(ntiles * kActTile);
    t.act_b = take(ntiles * kActTile);
    t.g1 = take(ntiles * kGateTile);
    t.g2 = take(ntiles * kGateTile);
    t.p = take(n * kNO);
    if (w) *w = t;
    return off;
}

template <int KC, int NCH, int NP, bool GATHER, int NS>
static cudaError_t layer_attrs() {
    return cudaFuncSetAttribute(mlsrc_layer<KC, NCH, NP, GATHER, NS>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)layer_smem<KC, NP, GATHER, NS>());
}

template <int KC, int NCH, int NP, bool GATHER, int NS>
static cudaError_t launch_layer(const LayerArgs& a, int nmat, long long ntiles, int* err,
                                cudaStream_t s, const char* name) {
    auto kern = mlsrc_layer<KC, NCH, NP, GATHER, NS>;
    const size_t smem = layer_smem<KC, NP, GATHER, NS>();
    // once per CUDA context (function attributes belong to the context)
    cudaError_t e = once_per_context((const void*)&layer_attrs<KC, NCH, NP, GATHER, NS>,
                                     &layer_attrs<KC, NCH, NP, GATHER, NS>);
    if (e != cudaSuccess) return e;
    const dim3 grid((unsigned)ntiles, (unsigned)nmat);
    PF_LAUNCH(name, s, kern<<<grid, kThreads, smem, s>>>(a, err));
    return cudaGetLastError();
}

}  // namespace mlsrc

size_t mlsrc_ws_bytes(const pf_grid* g) {
    const long long n = (long long)g->nx * g->ny * g->nz;
    return mlsrc::ws_layout(n, nullptr, nullptr);
}

cudaError_t launch_mlsrc_pack(const float* const* p, void* pack, cudaStream_t s) {
    using namespace mlsrc;
    float* dst = reinterpret_cast<float*>(pack);
    const int rows[6] = {kH, kH, kH, kH, kH, 18};
    const int cols[6] = {kPts * kF, kPts * kF, kPts * kF, kH, kH, kH};
    for (int m = 0; m < 6; ++m) {
        PF_LAUNCH("mlsrc_pack", s,
                  pack_matrix<<<148, 256, 0, s>>>(p[2 * m], rows[m], cols[m], m, dst));
        PF_LAUNCH("mlsrc_pack", s,
                  pack_vector<<<1, 256, 0, s>>>(p[2 * m + 1], rows[m], mat_rows(m),
                                                dst + bias_off(m)));
    }
    PF_LAUNCH("mlsrc_pack", s, pack_vector<<<1, 32, 0, s>>>(p[12], kF, 32, dst + kNormOff));
    return cudaGetLastError();
}

cudaError_t launch_mlsrc(const pf_grid* g, const double* u, const double* v, const double* w,
                         const void* pack, double* G, double* S, void* ws, int* err,
                         cudaStream_t s) {
    using namespace mlsrc;
    const Dims d{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    Ws W;
    ws_layout(d.n, reinterpret_cast<char*>(ws), &W);
    const float* pk = reinterpret_cast<const float*>(pack);
    const float two_dx = (float)(2.0 * g->dx), dx2 = (float)(g->dx * g->dx);
    const unsigned pts = (unsigned)((d.n + 255) / 256);
    PF_LAUNCH("mlsrc_features", s,
              mlsrc_features<<<pts, 256, 0, s>>>(d, u, v, w, two_dx, dx2, pk + kNormOff,
                                                 W.f_hi, W.f_lo));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const long long ntiles = (d.n + kTile - 1) / kTile;
    auto mat = [&](int m, const float* gate, float* out, int epi) {
        LayerMat M;
        M.w = pk + w_off(m);
        M.bias = pk + bias_off(m);
        M.gate = gate;
        M.out = out;
        M.epi = epi;
        return M;
    };
    // layer 1: H1 = tanh(fc1 x) (pairs), gates tanh(fcG x), tanh(fcG2 x)
    LayerArgs a{};
    a.m[0] = mat(0, nullptr, W.act_a, kEpiTanhSplit);
    a.m[1] = mat(1, nullptr, W.g1, kEpiTanh);
    a.m[2] = mat(2, nullptr, W.g2, kEpiTanh);
    a.a_hi = W.f_hi;
    a.a_lo = W.f_lo;
    a.d = d;
    if ((e = launch_layer<1, kK1 / 8, kNP, true, 4>(a, 3, ntiles, err, s, "mlsrc_layer1")))
        return e;
    // H2 = tanh(fc2 H1) * G1
    a.m[0] = mat(3, W.g1, W.act_b, kEpiGatedSplit);
    a.a_hi = W.act_a;
    a.a_lo = nullptr;
    if ((e = launch_layer<1, kH / 8, kNP, false, 4>(a, 1, ntiles, err, s, "mlsrc_layer2"))) return e;
    // H4 = tanh(fc3 H2) * G2
    a.m[0] = mat(4, W.g2, W.act_a, kEpiGatedSplit);
    a.a_hi = W.act_b;
    if ((e = launch_layer<1, kH / 8, kNP, false, 4>(a, 1, ntiles, err, s, "mlsrc_layer3"))) return e;
    // out = fc4 H4 (outputs 0-15)
    a.m[0] = mat(5, nullptr, W.p, kEpiLinear);
    a.a_hi = W.act_a;
    if ((e = launch_layer<1, kH / 8, kNO, false, 4>(a, 1, ntiles, err, s, "mlsrc_layer4"))) return e;
    PF_LAUNCH("mlsrc_terms", s,
              mlsrc_terms<<<pts, 256, 0, s>>>(d, W.p, two_dx, G, S));
    return cudaGetLastError();
}

}  // namespace pf

extern "C" size_t pf_mlsrc_pack_bytes(void) {
    return (size_t)pf::mlsrc::kPackFloats * sizeof(float);
}

extern "C" size_t pf_mlsrc_workspace_bytes(const pf_grid* g) {
    if (!g || g->nx < 1 || g->ny < 1 || g->nz < 1) return 0;
    return pf::mlsrc_ws_bytes(g);
}

extern "C" int pf_mlsrc_pack(const float* const* params, void* pack, void* stream) {
    if (!params || !pack || ((uintptr_t)pack & 15) != 0) return PF_ERR_BAD_ARG;
    for (int q = 0; q < 13; ++q)
        if (!params[q]) return PF_ERR_BAD_ARG;
    return pf::launch_mlsrc_pack(params, pack, (cudaStream_t)stream) == cudaSuccess
               ? PF_OK : PF_ERR_CUDA;
}

extern "C" int pf_mlsrc_closure(const pf_grid* g, const double* u, const double* v,
                                const double* w, const void* pack, double* G, double* S,
                                void* ws, size_t ws_bytes, int* err, void* stream) {
    if (!g || g->nx < 5 || g->ny < 5 || g->nz < 5 || !(g->dx > 0) || !u || !v || !w ||
        !pack || !G || !S || !ws || !err)
        return PF_ERR_BAD_ARG;
    if ((long long)g->nx * g->ny * g->nz >= (1LL << 31)) return PF_ERR_TOO_LARGE;
    if (((uintptr_t)pack & 15) != 0 || ((uintptr_t)ws & 255) != 0 ||
        ws_bytes < pf::mlsrc_ws_bytes(g))
        return PF_ERR_BAD_ARG;
    return pf::launch_mlsrc(g, u, v, w, pack, G, S, ws, err, (cudaStream_t)stream) == cudaSuccess
               ? PF_OK : PF_ERR_CUDA;
}
