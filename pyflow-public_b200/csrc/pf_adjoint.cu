// pf_adjoint.cu -- exact discrete adjoint (vector-Jacobian product) of the
// staggered Navier-Stokes right-hand side, and of its 'tensor' SFS term.
//
// The forward RHS (rhs_NavierStokes.evaluate, src/solver/velocity.py:221-355)
// is a sum of conservative differences of face/edge fluxes:
//   rhs_u +=  dxi (FX[i] - FX[i-1]) + dyi (FXY[j] - FXY[j-1]) + dzi (FXZ[k] - FXZ[k-1])
//   rhs_u -=  dxi (Cxx[i] - Cxx[i-1]) + dyi (Cxy[j+1] - Cxy[j]) + dzi (Cxz[k+1] - Cxz[k])
// (and likewise for v, w), where the viscous fluxes are linear in the
// velocity and the convective ones are products of face averages
// (Cxx = cu^2, Cxy = uy vx, ...; metric_staggered.py:149-188,458-526).  The
// transpose of a flux difference is a difference of the adjoint field, so for
// a given adjoint mu the kernel first forms each flux's adjoint
//   lam_Cxx(p) = dxi (mu_u(p+x) - mu_u(p)),
//   lam_Cxy(p) = dyi (mu_u(p) - mu_u(p-y)) + dxi (mu_v(p) - mu_v(p-x)), ...
// and then gathers lam * dFlux/du over every flux that reads the cell.  The
// result is J(u)^T mu exactly (to round-off), computed per cell from a 3x3x3
// neighbourhood of u and mu: deterministic, no atomics.
//
// The reference's own adjoint (src/solver/adjoint.py:94-227,
// src/metric/metric_staggered.py:537-799) evaluates the same transpose with
// the viscous operator applied as-is (it is symmetric) and its discrete-exact
// convective terms; tests/test_gpu_adjoint.py compares the two.
#include "pf_common.cuh"
#include "pf_kernels.cuh"
#include "pf_profile.cuh"

namespace pf {

struct AdjArgs {
    const double *u, *v, *w;     // forward state at which J is evaluated
    const double *mu, *mv, *mw;  // adjoint input
    double dxi, dyi, dzi;
    double a;   // 2 mu / rho   (diagonal viscous flux factor)
    double e;   // mu_edge / rho (off-diagonal viscous flux factor)
};

__global__ void __launch_bounds__(256)
rhs_adjoint_kernel(Dims d, AdjArgs A, double* __restrict__ ou,
                   double* __restrict__ ov, double* __restrict__ ow) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    const double dxi = A.dxi, dyi = A.dyi, dzi = A.dzi;
    auto at = [&](const double* f, int di, int dj, int dk) -> double {
        return __ldg(f + idx(d, wrap(i + di, d.nx), wrap(j + dj, d.ny), wrap(k + dk, d.nz)));
    };
    // ---- convective flux adjoints (at flux position p = c + (di,dj,dk))
    auto lamCxx = [&](int di, int dj, int dk) { return dxi * (at(A.mu, di + 1, dj, dk) - at(A.mu, di, dj, dk)); };
    auto lamCyy = [&](int di, int dj, int dk) { return dyi * (at(A.mv, di, dj + 1, dk) - at(A.mv, di, dj, dk)); };
    auto lamCzz = [&](int di, int dj, int dk) { return dzi * (at(A.mw, di, dj, dk + 1) - at(A.mw, di, dj, dk)); };
    auto lamCxy = [&](int di, int dj, int dk) {
        return dyi * (at(A.mu, di, dj, dk) - at(A.mu, di, dj - 1, dk)) +
               dxi * (at(A.mv, di, dj, dk) - at(A.mv, di - 1, dj, dk));
    };
    auto lamCxz = [&](int di, int dj, int dk) {
        return dzi * (at(A.mu, di, dj, dk) - at(A.mu, di, dj, dk - 1)) +
               dxi * (at(A.mw, di, dj, dk) - at(A.mw, di - 1, dj, dk));
    };
    auto lamCyz = [&](int di, int dj, int dk) {
        return dzi * (at(A.mv, di, dj, dk) - at(A.mv, di, dj, dk - 1)) +
               dyi * (at(A.mw, di, dj, dk) - at(A.mw, di, dj - 1, dk));
    };
    // face averages of the state entering the products
    auto cu = [&](int di, int dj, int dk) { return 0.5 * (at(A.u, di + 1, dj, dk) + at(A.u, di, dj, dk)); };
    auto cv = [&](int di, int dj, int dk) { return 0.5 * (at(A.v, di, dj + 1, dk) + at(A.v, di, dj, dk)); };
    auto cw = [&](int di, int dj, int dk) { return 0.5 * (at(A.w, di, dj, dk + 1) + at(A.w, di, dj, dk)); };
    auto uy = [&](int di, int dj, int dk) { return 0.5 * (at(A.u, di, dj, dk) + at(A.u, di, dj - 1, dk)); };
    auto uz = [&](int di, int dj, int dk) { return 0.5 * (at(A.u, di, dj, dk) + at(A.u, di, dj, dk - 1)); };
    auto vx = [&](int di, int dj, int dk) { return 0.5 * (at(A.v, di, dj, dk) + at(A.v, di - 1, dj, dk)); };
    auto vz = [&](int di, int dj, int dk) { return 0.5 * (at(A.v, di, dj, dk) + at(A.v, di, dj, dk - 1)); };
    auto wx = [&](int di, int dj, int dk) { return 0.5 * (at(A.w, di, dj, dk) + at(A.w, di - 1, dj, dk)); };
    auto wy = [&](int di, int dj, int dk) { return 0.5 * (at(A.w, di, dj, dk) + at(A.w, di, dj - 1, dk)); };

    double au = 0.0, av = 0.0, aw = 0.0;
    // Cxx(p) = cu(p)^2 reads u(p), u(p+x): cell c is read by p = c, c-x
    au += lamCxx(0, 0, 0) * cu(0, 0, 0) + lamCxx(-1, 0, 0) * cu(-1, 0, 0);
    // Cxy(p) = uy(p) vx(p): u(c) in uy at p = c, c+y; v(c) in vx at p = c, c+x
    au += 0.5 * (lamCxy(0, 0, 0) * vx(0, 0, 0) + lamCxy(0, 1, 0) * vx(0, 1, 0));
    av += 0.5 * (lamCxy(0, 0, 0) * uy(0, 0, 0) + lamCxy(1, 0, 0) * uy(1, 0, 0));
    // Cxz(p) = uz(p) wx(p)
    au += 0.5 * (lamCxz(0, 0, 0) * wx(0, 0, 0) + lamCxz(0, 0, 1) * wx(0, 0, 1));
    aw += 0.5 * (lamCxz(0, 0, 0) * uz(0, 0, 0) + lamCxz(1, 0, 0) * uz(1, 0, 0));
    // Cyy(p) = cv(p)^2
    av += lamCyy(0, 0, 0) * cv(0, 0, 0) + lamCyy(0, -1, 0) * cv(0, -1, 0);
    // Cyz(p) = vz(p) wy(p)
    av += 0.5 * (lamCyz(0, 0, 0) * wy(0, 0, 0) + lamCyz(0, 0, 1) * wy(0, 0, 1));
    aw += 0.5 * (lamCyz(0, 0, 0) * vz(0, 0, 0) + lamCyz(0, 1, 0) * vz(0, 1, 0));
    // Czz(p) = cw(p)^2
    aw += lamCzz(0, 0, 0) * cw(0, 0, 0) + lamCzz(0, 0, -1) * cw(0, 0, -1);

    // ---- viscous (constant viscosity): diagonal fluxes at centres
    // FX = (ux - D/3) a, FY = (vy - D/3) a, FZ = (wz - D/3) a with D = ux+vy+wz;
    // their adjoints lX = dxi (mu_u(p) - mu_u(p+x)), ...
    auto lX = [&](int di, int dj, int dk) { return dxi * (at(A.mu, di, dj, dk) - at(A.mu, di + 1, dj, dk)); };
    auto lY = [&](int di, int dj, int dk) { return dyi * (at(A.mv, di, dj, dk) - at(A.mv, di, dj + 1, dk)); };
    auto lZ = [&](int di, int dj, int dk) { return dzi * (at(A.mw, di, dj, dk) - at(A.mw, di, dj, dk + 1)); };
    auto sx = [&](int di, int dj, int dk) {
        return A.a * (2.0 * lX(di, dj, dk) - lY(di, dj, dk) - lZ(di, dj, dk)) / 3.0;
    };
    auto sy = [&](int di, int dj, int dk) {
        return A.a * (2.0 * lY(di, dj, dk) - lX(di, dj, dk) - lZ(di, dj, dk)) / 3.0;
    };
    auto sz = [&](int di, int dj, int dk) {
        return A.a * (2.0 * lZ(di, dj, dk) - lX(di, dj, dk) - lY(di, dj, dk)) / 3.0;
    };
    // ux(p) = (u(p+x) - u(p)) dxi reads u(c) at p = c-x (+), c (-)
    au += dxi * (sx(-1, 0, 0) - sx(0, 0, 0));
    av += dyi * (sy(0, -1, 0) - sy(0, 0, 0));
    aw += dzi * (sz(0, 0, -1) - sz(0, 0, 0));
    // off-diagonal fluxes on edges: FXY = ((u(p+y)-u(p)) dyi + (v(p+x)-v(p)) dxi) e
    auto txy = [&](int di, int dj, int dk) {
        return A.e * (dyi * (at(A.mu, di, dj, dk) - at(A.mu, di, dj + 1, dk)) +
                      dxi * (at(A.mv, di, dj, dk) - at(A.mv, di + 1, dj, dk)));
    };
    auto txz = [&](int di, int dj, int dk) {
        return A.e * (dzi * (at(A.mu, di, dj, dk) - at(A.mu, di, dj, dk + 1)) +
                      dxi * (at(A.mw, di, dj, dk) - at(A.mw, di + 1, dj, dk)));
    };
    auto tyz = [&](int di, int dj, int dk) {
        return A.e * (dzi * (at(A.mv, di, dj, dk) - at(A.mv, di, dj, dk + 1)) +
                      dyi * (at(A.mw, di, dj, dk) - at(A.mw, di, dj + 1, dk)));
    };
    au += dyi * (txy(0, -1, 0) - txy(0, 0, 0)) + dzi * (txz(0, 0, -1) - txz(0, 0, 0));
    av += dxi * (txy(-1, 0, 0) - txy(0, 0, 0)) + dzi * (tyz(0, 0, -1) - tyz(0, 0, 0));
    aw += dxi * (txz(-1, 0, 0) - txz(0, 0, 0)) + dyi * (tyz(0, -1, 0) - tyz(0, 0, 0));

    const long long q = idx(d, i, j, k);
    ou[q] = au;
    ov[q] = av;
    ow[q] = aw;
}

// Adjoint of the 'tensor' SFS stresses: the stresses are added to the viscous
// fluxes before the divergence (src/solver/velocity.py:262-267,...), the
// diagonal ones at cell centres and the off-diagonal ones edge-averaged from
// centres one cell below (interp_sc_xy, metric_staggered.py:127-144).
// out[0..5] += adjoint of FXX, FYY, FZZ, FXY, FXZ, FYZ for adjoint mu (scaled
// by `weight`, accumulated so that RK4 stages can be summed).
__global__ void __launch_bounds__(256)
sfs_adjoint_kernel(Dims d, const double* __restrict__ mu, const double* __restrict__ mv,
                   const double* __restrict__ mw, double dxi, double dyi, double dzi,
                   double weight, double* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    auto at = [&](const double* f, int di, int dj, int dk) -> double {
        return __ldg(f + idx(d, wrap(i + di, d.nx), wrap(j + dj, d.ny), wrap(k + dk, d.nz)));
    };
    // flux adjoints at edge positions p
    auto lxy = [&](int di, int dj) {
        return dyi * (at(mu, di, dj, 0) - at(mu, di, dj + 1, 0)) + dxi * (at(mv, di, dj, 0) - at(mv, di + 1, dj, 0));
    };
    auto lxz = [&](int di, int dk) {
        return dzi * (at(mu, di, 0, dk) - at(mu, di, 0, dk + 1)) + dxi * (at(mw, di, 0, dk) - at(mw, di + 1, 0, dk));
    };
    auto lyz = [&](int dj, int dk) {
        return dzi * (at(mv, 0, dj, dk) - at(mv, 0, dj, dk + 1)) + dyi * (at(mw, 0, dj, dk) - at(mw, 0, dj + 1, dk));
    };
    const long long q = idx(d, i, j, k), n = d.n;
    const double fxx = dxi * (at(mu, 0, 0, 0) - at(mu, 1, 0, 0));
    const double fyy = dyi * (at(mv, 0, 0, 0) - at(mv, 0, 1, 0));
    const double fzz = dzi * (at(mw, 0, 0, 0) - at(mw, 0, 0, 1));
    // S(p) = 0.25 (F(p) + F(p-x) + F(p-y) + F(p-x-y)): F(c) feeds p = c, c+x, c+y, c+x+y
    const double fxy = 0.25 * (lxy(0, 0) + lxy(1, 0) + lxy(0, 1) + lxy(1, 1));
    const double fxz = 0.25 * (lxz(0, 0) + lxz(1, 0) + lxz(0, 1) + lxz(1, 1));
    const double fyz = 0.25 * (lyz(0, 0) + lyz(1, 0) + lyz(0, 1) + lyz(1, 1));
    out[q] += weight * fxx;
    out[n + q] += weight * fyy;
    out[2 * n + q] += weight * fzz;
    out[3 * n + q] += weight * fxy;
    out[4 * n + q] += weight * fxz;
    out[5 * n + q] += weight * fyz;
}

}  // namespace pf

extern "C" int pf_rhs_adjoint(const pf_grid* g, const double* u, const double* v,
                              const double* w, const double* mu_u,
                              const double* mu_v, const double* mu_w, double mu,
                              double rho, double* out_u, double* out_v,
                              double* out_w, void* stream) {
    if (!g || g->nx < 2 || g->ny < 2 || g->nz < 2 || !(g->dx > 0) || !(g->dy > 0) ||
        !(g->dz > 0) || !u || !v || !w || !mu_u || !mu_v || !mu_w || !out_u || !out_v ||
        !out_w || !(rho != 0.0))
        return PF_ERR_BAD_ARG;
    pf::Dims d{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    pf::AdjArgs A{u, v, w, mu_u, mu_v, mu_w, 1.0 / g->dx, 1.0 / g->dy, 1.0 / g->dz,
                  (2.0 * mu) / rho, (0.25 * (((mu + mu) + mu) + mu)) / rho};
    cudaStream_t s = (cudaStream_t)stream;
    dim3 blk(32, 8), grd((d.nz + 31) / 32, (d.ny + 7) / 8, d.nx);
    PF_LAUNCH("rhs_adjoint", s, pf::rhs_adjoint_kernel<<<grd, blk, 0, s>>>(d, A, out_u, out_v, out_w));
    return cudaGetLastError() == cudaSuccess ? PF_OK : PF_ERR_CUDA;
}

extern "C" int pf_sfs_adjoint(const pf_grid* g, const double* mu_u,
                              const double* mu_v, const double* mu_w,
                              double weight, double* out, void* stream) {
    if (!g || g->nx < 2 || g->ny < 2 || g->nz < 2 || !(g->dx > 0) || !(g->dy > 0) ||
        !(g->dz > 0) || !mu_u || !mu_v || !mu_w || !out)
        return PF_ERR_BAD_ARG;
    pf::Dims d{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    cudaStream_t s = (cudaStream_t)stream;
    dim3 blk(32, 8), grd((d.nz + 31) / 32, (d.ny + 7) / 8, d.nx);
    PF_LAUNCH("sfs_adjoint", s, pf::sfs_adjoint_kernel<<<grd, blk, 0, s>>>(
        d, mu_u, mu_v, mu_w, 1.0 / g->dx, 1.0 / g->dy, 1.0 / g->dz, weight, out));
    return cudaGetLastError() == cudaSuccess ? PF_OK : PF_ERR_CUDA;
}
