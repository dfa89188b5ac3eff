// pf_io.cu -- NGA restart fields straight from and to device memory.
//
// A restart file (src/data/dataReader.py:119-208) stores each variable as an
// nx*ny*nz FP64 array in Fortran order (x fastest); the device fields are
// [nx][ny][nz] with z fastest.  The two layouts are transposes of each other
// in (x, z) at fixed y, so writing and reading a restart is one tiled
// transpose on the device (32 x 32 tiles of (x, z) through shared memory,
// both sides coalesced) plus a contiguous copy to or from the file.
#include "pf_common.cuh"
#include "pf_profile.cuh"

namespace pf {

// B[c][b][a] = A[a][b][c] for an n0 x n1 x n2 array A (C order).
__global__ void __launch_bounds__(256)
transpose02(const double* __restrict__ A, double* __restrict__ B, int n0, int n1, int n2) {
    __shared__ double tile[32][33];
    const int c0 = blockIdx.x * 32, a0 = blockIdx.y * 32, b = blockIdx.z;
    const int tx = threadIdx.x, ty = threadIdx.y;
    // read rows a of A (c contiguous)
#pragma unroll
    for (int r = 0; r < 32; r += 8) {
        const int a = a0 + ty + r, c = c0 + tx;
        if (a < n0 && c < n2) tile[ty + r][tx] = A[((long long)a * n1 + b) * n2 + c];
    }
    __syncthreads();
    // write rows c of B (a contiguous)
#pragma unroll
    for (int r = 0; r < 32; r += 8) {
        const int c = c0 + ty + r, a = a0 + tx;
        if (a < n0 && c < n2) B[((long long)c * n1 + b) * n0 + a] = tile[tx][ty + r];
    }
}

static cudaError_t launch_transpose(const double* A, double* B, int n0, int n1, int n2,
                                    cudaStream_t s) {
    dim3 grid((n2 + 31) / 32, (n0 + 31) / 32, n1), blk(32, 8);
    PF_LAUNCH("restart_transpose", s, transpose02<<<grid, blk, 0, s>>>(A, B, n0, n1, n2));
    return cudaGetLastError();
}

}  // namespace pf

static bool io_grid_ok(const pf_grid* g) {
    return g && g->nx >= 1 && g->ny >= 1 && g->nz >= 1 && g->ny <= 65535;
}

extern "C" int pf_restart_pack(const pf_grid* g, const double* field, double* file_order,
                               void* stream) {
    if (!io_grid_ok(g) || !field || !file_order || field == file_order) return PF_ERR_BAD_ARG;
    return pf::launch_transpose(field, file_order, g->nx, g->ny, g->nz, (cudaStream_t)stream) ==
                   cudaSuccess ? PF_OK : PF_ERR_CUDA;
}

extern "C" int pf_restart_unpack(const pf_grid* g, const double* file_order, double* field,
                                 void* stream) {
    if (!io_grid_ok(g) || !field || !file_order || field == file_order) return PF_ERR_BAD_ARG;
    // the file order is a [nz][ny][nx] C-order array
    return pf::launch_transpose(file_order, field, g->nz, g->ny, g->nx, (cudaStream_t)stream) ==
                   cudaSuccess ? PF_OK : PF_ERR_CUDA;
}
