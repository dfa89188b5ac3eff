// pf_grad.cuh -- cell-centred velocity-gradient tensor of the staggered field.
//
// metric_uniform.grad_vel_center (src/metric/metric_staggered.py:215-268): the
// normal derivative of a component is the one-sided difference of its two face
// values; a transverse derivative is the difference of the face-to-centre
// interpolant averaged back to the two neighbouring faces, e.g. for u in y
//   c(j)  = 0.5 (u[i+1,j] + u[i,j]),   f(j) = 0.5 (c(j) + c(j-1)),
//   du/dy = (f(j+1) - f(j)) / dy.
// Indices wrap periodically everywhere.
#pragma once
#include "pf_common.cuh"

namespace pf {

struct Grad9 {
    double ux, uy, uz, vx, vy, vz, wx, wy, wz;
};

__device__ inline Grad9 grad_center(const Dims& d, const double* __restrict__ u,
                                    const double* __restrict__ v,
                                    const double* __restrict__ w, int i, int j,
                                    int k, double dxi, double dyi, double dzi) {
    const int ip = wrap(i + 1, d.nx), im = wrap(i - 1, d.nx);
    const int jp = wrap(j + 1, d.ny), jm = wrap(j - 1, d.ny);
    const int kp = wrap(k + 1, d.nz), km = wrap(k - 1, d.nz);
    auto L = [&](const double* f, int a, int b, int c) { return __ldg(f + idx(d, a, b, c)); };
    Grad9 g;
    // u: centre values along x at the needed (j,k) offsets
    {
        const double c0 = 0.5 * (L(u, ip, j, k) + L(u, i, j, k));
        const double cym = 0.5 * (L(u, ip, jm, k) + L(u, i, jm, k));
        const double cyp = 0.5 * (L(u, ip, jp, k) + L(u, i, jp, k));
        const double czm = 0.5 * (L(u, ip, j, km) + L(u, i, j, km));
        const double czp = 0.5 * (L(u, ip, j, kp) + L(u, i, j, kp));
        g.ux = (L(u, ip, j, k) - L(u, i, j, k)) * dxi;
        g.uy = (0.5 * (cyp + c0) - 0.5 * (c0 + cym)) * dyi;
        g.uz = (0.5 * (czp + c0) - 0.5 * (c0 + czm)) * dzi;
    }
    {
        const double c0 = 0.5 * (L(v, i, jp, k) + L(v, i, j, k));
        const double cxm = 0.5 * (L(v, im, jp, k) + L(v, im, j, k));
        const double cxp = 0.5 * (L(v, ip, jp, k) + L(v, ip, j, k));
        const double czm = 0.5 * (L(v, i, jp, km) + L(v, i, j, km));
        const double czp = 0.5 * (L(v, i, jp, kp) + L(v, i, j, kp));
        g.vx = (0.5 * (cxp + c0) - 0.5 * (c0 + cxm)) * dxi;
        g.vy = (L(v, i, jp, k) - L(v, i, j, k)) * dyi;
        g.vz = (0.5 * (czp + c0) - 0.5 * (c0 + czm)) * dzi;
    }
    {
        const double c0 = 0.5 * (L(w, i, j, kp) + L(w, i, j, k));
        const double cxm = 0.5 * (L(w, im, j, kp) + L(w, im, j, k));
        const double cxp = 0.5 * (L(w, ip, j, kp) + L(w, ip, j, k));
        const double cym = 0.5 * (L(w, i, jm, kp) + L(w, i, jm, k));
        const double cyp = 0.5 * (L(w, i, jp, kp) + L(w, i, jp, k));
        g.wx = (0.5 * (cxp + c0) - 0.5 * (c0 + cxm)) * dxi;
        g.wy = (0.5 * (cyp + c0) - 0.5 * (c0 + cym)) * dyi;
        g.wz = (L(w, i, j, kp) - L(w, i, j, k)) * dzi;
    }
    return g;
}

}  // namespace pf
