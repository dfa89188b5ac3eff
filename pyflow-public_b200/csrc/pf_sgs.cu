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

}  // namespace pf

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
