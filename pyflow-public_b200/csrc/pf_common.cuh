// pf_common.cuh -- shared definitions of the pyflow_b200 CUDA library.
//
// Field layout: every field is a ghost-free [nx][ny][nz] array with z
// contiguous (the interior of the reference's state_P.var,
// src/data/state.py:142-146).  The reference's 2-deep periodic ghost exchange
// (src/library/parallel.py:301-414) becomes index wrap inside the kernels.
//
// Arithmetic: the library is compiled with --fmad=false, so every multiply and
// add rounds separately like torch's elementwise ops; fma() appears exactly
// where the reference calls torch's add_(alpha, x) / sub_(alpha, x), which
// torch evaluates as one fused multiply-add.  FP64 kernels therefore reproduce
// the reference bit for bit except for reductions (summation order).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/pyflow_b200.h"

namespace pf {

constexpr int kBlock = 256;        // threads per block of the pointwise kernels
constexpr int kTileZ = 32;         // stencil tile: z extent (one warp)
constexpr int kTileY = 16;         // stencil tile: y extent
constexpr int kRowsPerThread = 2;  // block is 32 x 8 threads, 2 rows each
constexpr int kMaxPartials = 4096; // per-reduction partial slots (>= grid size)

struct Dims {
    int nx, ny, nz;
    long long n;  // nx*ny*nz
};

__host__ __device__ inline int wrap(int a, int n) {
    return a < 0 ? a + n : (a >= n ? a - n : a);
}

// full periodic wrap (any distance)
__host__ __device__ inline int pmod(int a, int n) {
    const int r = a % n;
    return r < 0 ? r + n : r;
}

__host__ __device__ inline long long idx(const Dims& d, int i, int j, int k) {
    return ((long long)i * d.ny + j) * d.nz + k;
}

// --------------------------------------------------------------------------
// Block reductions with a fixed combination order (deterministic).
// --------------------------------------------------------------------------
template <int NT>
__device__ inline double block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    (void)lane;
    if ((tid & 31) == 0) sh[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (tid < 32) {
        r = (tid < NT / 32) ? sh[tid] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;  // valid in thread 0
}

// max that propagates NaN (a NaN residual must stop the solver, not hide)
__device__ inline double nanmax(double a, double b) {
    return (a != a || b != b) ? __longlong_as_double(0x7ff8000000000000LL) : fmax(a, b);
}

// block-wide max of non-negative values; a NaN anywhere gives NaN
template <int NT>
__device__ inline double block_max(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_down_sync(0xffffffffu, v, o));
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int wid = tid >> 5;
    if ((tid & 31) == 0) sh[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (tid < 32) {
        r = (tid < NT / 32) ? sh[tid] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r = nanmax(r, __shfl_down_sync(0xffffffffu, r, o));
    }
    __syncthreads();
    return r;
}

}  // namespace pf
