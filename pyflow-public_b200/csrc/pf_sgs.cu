// pf_sgs.cu -- cell-centred SGS closures: velocity-gradient tensor, Smagorinsky
// eddy viscosity and the gradient-model stress tensor, fused per cell.
//
// The nine cell-centred gradients follow metric_uniform.grad_vel_center
// (src/metric/metric_staggered.py:215-268): the normal derivative of a
// component is the one-sided difference of its two face values; a transverse
// derivative is the difference of the face-to-centre interpolant averaged back
// to the two neighbouring faces, e.g. for u in y
//   c(j)  = 0.5 (u[i+1,j] + u[i,j]),   f(j) = 0.5 (c(j) + c(j-1)),
//   du/dy = (f(j+1) - f(j)) / dy.
// Indices wrap periodically everywhere (the reference reads stale values in
// its outermost ghost layer instead; interior values agree bit for bit).
#include <algorithm>

#include "pf_common.cuh"
#include "pf_grad.cuh"
#include "pf_kernels.cuh"
#include "pf_profile.cuh"

namespace pf {

// model 0: Smagorinsky mu_t = coef |S| (sfsmodel_smagorinsky.py:72-88), plus
//          `add` (the molecular viscosity when the field is the total one)
// model 1: gradient model, six stresses (sfsmodel_gradient.py:77-148)
// model 2: the nine gradients themselves (ux,uy,uz,vx,...,wz)
// Every value is formed in FP64 and rounded once to T: for T = float that is
// the FP64 closure field converted to the mixed forms' stage type.
template <typename T>
__global__ void __launch_bounds__(256)
sgs_kernel(Dims d, int model, const double* __restrict__ u,
           const double* __restrict__ v, const double* __restrict__ w,
           double dxi, double dyi, double dzi, double coef, double add,
           T* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    const Grad9 g = grad_center(d, u, v, w, i, j, k, dxi, dyi, dzi);
    const long long q = idx(d, i, j, k), n = d.n;
    if (model == 0) {
        const double div3 = ((g.ux + g.vy) + g.wz) / 3.0;
        const double s11 = g.ux - div3, s22 = g.vy - div3, s33 = g.wz - div3;
        const double s12 = 0.5 * (g.uy + g.vx);
        const double s13 = 0.5 * (g.uz + g.wx);
        const double s23 = 0.5 * (g.vz + g.wy);
        const double smag = sqrt(((s11 * s11 + s22 * s22) + s33 * s33) +
                                 2.0 * ((s12 * s12 + s13 * s13) + s23 * s23));
        out[q] = (T)(coef * smag + add);
    } else if (model == 1) {
        out[q] = (T)(((g.ux * g.ux + g.uy * g.uy) + g.uz * g.uz) * coef);
        out[n + q] = (T)(((g.vx * g.vx + g.vy * g.vy) + g.vz * g.vz) * coef);
        out[2 * n + q] = (T)(((g.wx * g.wx + g.wy * g.wy) + g.wz * g.wz) * coef);
        out[3 * n + q] = (T)(((g.ux * g.vx + g.uy * g.vy) + g.uz * g.vz) * coef);
        out[4 * n + q] = (T)(((g.ux * g.wx + g.uy * g.wy) + g.uz * g.wz) * coef);
        out[5 * n + q] = (T)(((g.vx * g.wx + g.vy * g.wy) + g.vz * g.wz) * coef);
    } else {
        const double a[9] = {g.ux, g.uy, g.uz, g.vx, g.vy, g.vz, g.wx, g.wy, g.wz};
#pragma unroll
        for (int c = 0; c < 9; ++c) out[c * n + q] = (T)a[c];
    }
}

cudaError_t launch_sgs(const pf_grid* g, int model, const double* u,
                       const double* v, const double* w, double coef,
                       double add, void* out, bool f32, cudaStream_t s) {
    Dims d{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    dim3 blk(32, 8), grd((d.nz + 31) / 32, (d.ny + 7) / 8, d.nx);
    const double dxi = 1.0 / g->dx, dyi = 1.0 / g->dy, dzi = 1.0 / g->dz;
    if (f32)
        PF_LAUNCH("sgs_closure_f32", s, sgs_kernel<float><<<grd, blk, 0, s>>>(
            d, model, u, v, w, dxi, dyi, dzi, coef, add, (float*)out));
    else
        PF_LAUNCH("sgs_closure", s, sgs_kernel<double><<<grd, blk, 0, s>>>(
            d, model, u, v, w, dxi, dyi, dzi, coef, add, (double*)out));
    return cudaGetLastError();
}

// g2 = the mean over cells of the nine squared cell-centred gradients (FP64,
// cells summed per block in a fixed order, blocks by the last block in
// block order), then the MLP closure's scales [1/sqrt(g2), delta2 g2],
// each formed in FP64 and rounded once to float (sfsmodel_mlp.closure).
// ws: the arrival counter (one unsigned, zeroed by the launcher) at byte 0,
// block partials from byte 256.
__global__ void __launch_bounds__(256)
grad_sq_kernel(Dims d, const double* __restrict__ u, const double* __restrict__ v,
               const double* __restrict__ w, double dxi, double dyi, double dzi,
               double delta2, unsigned char* ws, float* __restrict__ scales) {
    __shared__ double sh[32];
    __shared__ bool last;
    unsigned* counter = (unsigned*)ws;
    double* part = (double*)(ws + 256);
    const int tz = (d.nz + 31) / 32, ty = (d.ny + 7) / 8;
    const long long ntiles = (long long)tz * ty * d.nx;
    double acc = 0.0;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int k = (int)(t % tz) * 32 + threadIdx.x;
        const int j = (int)((t / tz) % ty) * 8 + threadIdx.y;
        const int i = (int)(t / ((long long)tz * ty));
        if (k >= d.nz || j >= d.ny) continue;
        const Grad9 g = grad_center(d, u, v, w, i, j, k, dxi, dyi, dzi);
        const double a[9] = {g.ux, g.uy, g.uz, g.vx, g.vy, g.vz, g.wx, g.wy, g.wz};
        double c = 0.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) c += a[q] * a[q];
        acc += c;
    }
    const double bs = block_sum<256>(acc, sh);
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if (tid == 0) part[blockIdx.x] = bs;
    __threadfence();
    __syncthreads();
    if (tid == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    double v2 = 0.0;
    for (int b = tid; b < (int)gridDim.x; b += 256) v2 += ((volatile const double*)part)[b];
    const double tot = block_sum<256>(v2, sh);
    if (tid == 0) {
        const double g2 = tot / (9.0 * (double)d.n);
        scales[0] = (float)(1.0 / sqrt(g2));
        scales[1] = (float)(delta2 * g2);
        *counter = 0u;
    }
}

constexpr int kGradSqBlocks = 1024;

size_t mlp_scales_ws_bytes() { return 256 + kGradSqBlocks * sizeof(double); }

cudaError_t launch_mlp_scales(const pf_grid* g, const double* u, const double* v,
                              const double* w, double delta2, float* scales, void* ws,
                              cudaStream_t s) {
    Dims d{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    const long long ntiles = (long long)((d.nz + 31) / 32) * ((d.ny + 7) / 8) * d.nx;
    const int nb = (int)std::min<long long>(ntiles, kGradSqBlocks);
    cudaError_t e = cudaMemsetAsync(ws, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    PF_LAUNCH("mlp_scales", s, grad_sq_kernel<<<nb, dim3(32, 8), 0, s>>>(
        d, u, v, w, 1.0 / g->dx, 1.0 / g->dy, 1.0 / g->dz, delta2, (unsigned char*)ws, scales));
    return cudaGetLastError();
}

__global__ void __launch_bounds__(256)
to_float_kernel(const double* __restrict__ in, float* __restrict__ out, long long n) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x)
        out[q] = (float)in[q];
}

cudaError_t launch_to_float(const double* in, float* out, long long n, cudaStream_t s) {
    const int nb = (int)std::max<long long>(1, std::min<long long>((n + 1023) / 1024, 4096));
    PF_LAUNCH("to_float", s, to_float_kernel<<<nb, 256, 0, s>>>(in, out, n));
    return cudaGetLastError();
}

}  // namespace pf

extern "C" size_t pf_mlp_scales_workspace_bytes(void) { return pf::mlp_scales_ws_bytes(); }

extern "C" int pf_mlp_scales(const pf_grid* g, const double* u, const double* v,
                             const double* w, double delta2, float* scales, void* ws,
                             size_t ws_bytes, void* stream) {
    if (!g || g->nx < 2 || g->ny < 2 || g->nz < 2 || !(g->dx > 0) || !(g->dy > 0) ||
        !(g->dz > 0) || !u || !v || !w || !scales || !ws || ((uintptr_t)ws & 255) ||
        ws_bytes < pf::mlp_scales_ws_bytes())
        return PF_ERR_BAD_ARG;
    const cudaError_t e =
        pf::launch_mlp_scales(g, u, v, w, delta2, scales, ws, (cudaStream_t)stream);
    return e == cudaSuccess ? PF_OK : PF_ERR_CUDA;
}

extern "C" int pf_sgs_closure(const pf_grid* g, int model, const double* u,
                              const double* v, const double* w, double coef,
                              double* out, void* stream) {
    if (!g || g->nx < 2 || g->ny < 2 || g->nz < 2 || !(g->dx > 0) || !(g->dy > 0) ||
        !(g->dz > 0) || !u || !v || !w || !out || model < 0 || model > 2)
        return PF_ERR_BAD_ARG;
    const cudaError_t e =
        pf::launch_sgs(g, model, u, v, w, coef, 0.0, out, false, (cudaStream_t)stream);
    return e == cudaSuccess ? PF_OK : PF_ERR_CUDA;
}
