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
#include "pf_common.cuh"
#include "pf_kernels.cuh"
#include "pf_profile.cuh"

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

template <typename T>
__device__ inline T edge4(T a, T b, T c, T d) {
    return T(0.25) * (((a + b) + c) + d);
}

// Computes (ru, rv, rw) at cell (i, j, k).
template <typename T, typename TI>
__device__ inline void rhs_cell(const Dims& d, const RhsArgs<T, TI>& a, int i,
                                int j, int k, T& ru_o, T& rv_o, T& rw_o) {
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const T dxi = a.dxi, dyi = a.dyi, dzi = a.dzi, rho = a.rho;
    // wrapped plane / row / column offsets of the neighbours i-2 .. i+1
    // (computed once; every load is then two adds)
    const long long P = (long long)ny * nz;
    long long xo[4];
    int yo[4], zo[4];
#pragma unroll
    for (int o = 0; o < 4; ++o) {
        xo[o] = (long long)wrap(i + o - 2, nx) * P;
        yo[o] = wrap(j + o - 2, ny) * nz;
        zo[o] = wrap(k + o - 2, nz);
    }
    auto off = [&](int di, int dj, int dk) -> long long {
        return xo[di + 2] + (long long)(yo[dj + 2] + zo[dk + 2]);
    };
    auto L = [&](const TI* f, int di, int dj, int dk) -> T {
        return T(__ldg(f + off(di, dj, dk)));
    };
    auto LV = [&](int di, int dj, int dk) -> T {
        return a.visc ? __ldg(a.visc + off(di, dj, dk)) : a.mu;
    };
    const long long n = d.n;
    auto LS = [&](int c, int di, int dj, int dk) -> T {
        return __ldg(a.sfs + (long long)c * n + off(di, dj, dk));
    };
    // velocity neighbourhood
    const T u_c = L(a.u, 0, 0, 0), u_xp = L(a.u, 1, 0, 0), u_xm = L(a.u, -1, 0, 0);
    const T u_yp = L(a.u, 0, 1, 0), u_ym = L(a.u, 0, -1, 0), u_zp = L(a.u, 0, 0, 1);
    const T u_zm = L(a.u, 0, 0, -1), u_xm_yp = L(a.u, -1, 1, 0), u_xp_ym = L(a.u, 1, -1, 0);
    const T u_xm_zp = L(a.u, -1, 0, 1), u_xp_zm = L(a.u, 1, 0, -1);
    const T v_c = L(a.v, 0, 0, 0), v_xp = L(a.v, 1, 0, 0), v_xm = L(a.v, -1, 0, 0);
    const T v_yp = L(a.v, 0, 1, 0), v_ym = L(a.v, 0, -1, 0), v_zp = L(a.v, 0, 0, 1);
    const T v_zm = L(a.v, 0, 0, -1), v_xm_yp = L(a.v, -1, 1, 0), v_xp_ym = L(a.v, 1, -1, 0);
    const T v_ym_zp = L(a.v, 0, -1, 1), v_yp_zm = L(a.v, 0, 1, -1);
    const T w_c = L(a.w, 0, 0, 0), w_xp = L(a.w, 1, 0, 0), w_xm = L(a.w, -1, 0, 0);
    const T w_yp = L(a.w, 0, 1, 0), w_ym = L(a.w, 0, -1, 0), w_zp = L(a.w, 0, 0, 1);
    const T w_zm = L(a.w, 0, 0, -1), w_xm_zp = L(a.w, -1, 0, 1), w_xp_zm = L(a.w, 1, 0, -1);
    const T w_ym_zp = L(a.w, 0, -1, 1), w_yp_zm = L(a.w, 0, 1, -1);

    // divergence / 3 at centres (div_vel_over, metric_staggered.py:424-433)
    auto div3 = [&](T ue, T uw, T vn, T vs, T wt, T wb) -> T {
        return ((((ue - uw) * dxi) + ((vn - vs) * dyi)) + ((wt - wb) * dzi)) / T(3.0);
    };
    const T D_c = div3(u_xp, u_c, v_yp, v_c, w_zp, w_c);
    const T D_xm = div3(u_c, u_xm, v_xm_yp, v_xm, w_xm_zp, w_xm);
    const T D_ym = div3(u_xp_ym, u_ym, v_c, v_ym, w_ym_zp, w_ym);
    const T D_zm = div3(u_xp_zm, u_zm, v_yp_zm, v_zm, w_c, w_zm);

    const T two = T(2.0);
    // diagonal viscous fluxes at centres
    const T fxx_c = ((u_xp - u_c) * dxi - D_c) * ((two * LV(0, 0, 0)) / rho);
    const T fxx_m = ((u_c - u_xm) * dxi - D_xm) * ((two * LV(-1, 0, 0)) / rho);
    const T fyy_c = ((v_yp - v_c) * dyi - D_c) * ((two * LV(0, 0, 0)) / rho);
    const T fyy_m = ((v_c - v_ym) * dyi - D_ym) * ((two * LV(0, -1, 0)) / rho);
    const T fzz_c = ((w_zp - w_c) * dzi - D_c) * ((two * LV(0, 0, 0)) / rho);
    const T fzz_m = ((w_c - w_zm) * dzi - D_zm) * ((two * LV(0, 0, -1)) / rho);

    // edge viscosities (one cell below the flux, as in the reference)
    T vxy_c, vxy_ym, vxy_xm, vxz_c, vxz_zm, vxz_xm, vyz_c, vyz_zm, vyz_ym;
    if (a.visc) {
        vxy_c = edge4(LV(0, 0, 0), LV(-1, 0, 0), LV(0, -1, 0), LV(-1, -1, 0));
        vxy_ym = edge4(LV(0, -1, 0), LV(-1, -1, 0), LV(0, -2, 0), LV(-1, -2, 0));
        vxy_xm = edge4(LV(-1, 0, 0), LV(-2, 0, 0), LV(-1, -1, 0), LV(-2, -1, 0));
        vxz_c = edge4(LV(0, 0, 0), LV(-1, 0, 0), LV(0, 0, -1), LV(-1, 0, -1));
        vxz_zm = edge4(LV(0, 0, -1), LV(-1, 0, -1), LV(0, 0, -2), LV(-1, 0, -2));
        vxz_xm = edge4(LV(-1, 0, 0), LV(-2, 0, 0), LV(-1, 0, -1), LV(-2, 0, -1));
        vyz_c = edge4(LV(0, 0, 0), LV(0, -1, 0), LV(0, 0, -1), LV(0, -1, -1));
        vyz_zm = edge4(LV(0, 0, -1), LV(0, -1, -1), LV(0, 0, -2), LV(0, -1, -2));
        vyz_ym = edge4(LV(0, -1, 0), LV(0, -2, 0), LV(0, -1, -1), LV(0, -2, -1));
    } else {
        const T m = a.mu;
        const T e = edge4(m, m, m, m);
        vxy_c = vxy_ym = vxy_xm = vxz_c = vxz_zm = vxz_xm = vyz_c = vyz_zm = vyz_ym = e;
    }
    // off-diagonal viscous fluxes on edges: (grad_y u + grad_x v) * (Vxy / rho)
    const T fxy_c = (((u_yp - u_c) * dyi) + ((v_xp - v_c) * dxi)) * (vxy_c / rho);
    const T fxy_ym = (((u_c - u_ym) * dyi) + ((v_xp_ym - v_ym) * dxi)) * (vxy_ym / rho);
    const T fxy_xm = (((u_xm_yp - u_xm) * dyi) + ((v_c - v_xm) * dxi)) * (vxy_xm / rho);
    const T fxz_c = (((u_zp - u_c) * dzi) + ((w_xp - w_c) * dxi)) * (vxz_c / rho);
    const T fxz_zm = (((u_c - u_zm) * dzi) + ((w_xp_zm - w_zm) * dxi)) * (vxz_zm / rho);
    const T fxz_xm = (((u_xm_zp - u_xm) * dzi) + ((w_c - w_xm) * dxi)) * (vxz_xm / rho);
    const T fyz_c = (((v_zp - v_c) * dzi) + ((w_yp - w_c) * dyi)) * (vyz_c / rho);
    const T fyz_zm = (((v_c - v_zm) * dzi) + ((w_yp_zm - w_zm) * dyi)) * (vyz_zm / rho);
    const T fyz_ym = (((v_ym_zp - v_ym) * dzi) + ((w_c - w_ym) * dyi)) * (vyz_ym / rho);

    T ux_p = fxx_c, ux_m = fxx_m, uy_p = fxy_c, uy_m = fxy_ym, uz_p = fxz_c, uz_m = fxz_zm;
    T vx_p = fxy_c, vx_m = fxy_xm, vy_p = fyy_c, vy_m = fyy_m, vz_p = fyz_c, vz_m = fyz_zm;
    T wx_p = fxz_c, wx_m = fxz_xm, wy_p = fyz_c, wy_m = fyz_ym, wz_p = fzz_c, wz_m = fzz_m;
    if (a.sfs) {
        // 'tensor' SFS stresses, off-diagonals edge-averaged (interp_sc_xy/xz/yz)
        const T sxy_c = edge4(LS(3, 0, 0, 0), LS(3, -1, 0, 0), LS(3, 0, -1, 0), LS(3, -1, -1, 0));
        const T sxy_ym = edge4(LS(3, 0, -1, 0), LS(3, -1, -1, 0), LS(3, 0, -2, 0), LS(3, -1, -2, 0));
        const T sxy_xm = edge4(LS(3, -1, 0, 0), LS(3, -2, 0, 0), LS(3, -1, -1, 0), LS(3, -2, -1, 0));
        const T sxz_c = edge4(LS(4, 0, 0, 0), LS(4, -1, 0, 0), LS(4, 0, 0, -1), LS(4, -1, 0, -1));
        const T sxz_zm = edge4(LS(4, 0, 0, -1), LS(4, -1, 0, -1), LS(4, 0, 0, -2), LS(4, -1, 0, -2));
        const T sxz_xm = edge4(LS(4, -1, 0, 0), LS(4, -2, 0, 0), LS(4, -1, 0, -1), LS(4, -2, 0, -1));
        const T syz_c = edge4(LS(5, 0, 0, 0), LS(5, 0, -1, 0), LS(5, 0, 0, -1), LS(5, 0, -1, -1));
        const T syz_zm = edge4(LS(5, 0, 0, -1), LS(5, 0, -1, -1), LS(5, 0, 0, -2), LS(5, 0, -1, -2));
        const T syz_ym = edge4(LS(5, 0, -1, 0), LS(5, 0, -2, 0), LS(5, 0, -1, -1), LS(5, 0, -2, -1));
        ux_p += LS(0, 0, 0, 0); ux_m += LS(0, -1, 0, 0);
        uy_p += sxy_c;          uy_m += sxy_ym;
        uz_p += sxz_c;          uz_m += sxz_zm;
        vx_p += sxy_c;          vx_m += sxy_xm;
        vy_p += LS(1, 0, 0, 0); vy_m += LS(1, 0, -1, 0);
        vz_p += syz_c;          vz_m += syz_zm;
        wx_p += sxz_c;          wx_m += sxz_xm;
        wy_p += syz_c;          wy_m += syz_ym;
        wz_p += LS(2, 0, 0, 0); wz_m += LS(2, 0, 0, -1);
    }
    // div_visc (metric_staggered.py:406-418): rhs.add_(dxi, F) is one fma
    T ru = T(0), rv = T(0), rw = T(0);
    ru = fma(dxi, ux_p, ru); ru = fma(-dxi, ux_m, ru);
    ru = fma(dyi, uy_p, ru); ru = fma(-dyi, uy_m, ru);
    ru = fma(dzi, uz_p, ru); ru = fma(-dzi, uz_m, ru);
    rv = fma(dxi, vx_p, rv); rv = fma(-dxi, vx_m, rv);
    rv = fma(dyi, vy_p, rv); rv = fma(-dyi, vy_m, rv);
    rv = fma(dzi, vz_p, rv); rv = fma(-dzi, vz_m, rv);
    rw = fma(dxi, wx_p, rw); rw = fma(-dxi, wx_m, rw);
    rw = fma(dyi, wy_p, rw); rw = fma(-dyi, wy_m, rw);
    rw = fma(dzi, wz_p, rw); rw = fma(-dzi, wz_m, rw);

    // convective fluxes (vel_conv_*, metric_staggered.py:458-526)
    const T h = T(0.5), one = T(1.0);
    {
        const T cp = h * (u_xp + u_c), cm = h * (u_c + u_xm);
        ru -= (cp * cp - cm * cm) * dxi * one;
        const T uyp = h * (u_yp + u_c), uym = h * (u_c + u_ym);
        const T vxp = h * (v_yp + v_xm_yp), vxm = h * (v_c + v_xm);
        ru -= (uyp * vxp - uym * vxm) * dyi * one;
        const T uzp = h * (u_zp + u_c), uzm = h * (u_c + u_zm);
        const T wxp = h * (w_zp + w_xm_zp), wxm = h * (w_c + w_xm);
        ru -= (uzp * wxp - uzm * wxm) * dzi * one;
    }
    {
        const T vxp = h * (v_xp + v_c), vxm = h * (v_c + v_xm);
        const T uyp = h * (u_xp + u_xp_ym), uym = h * (u_c + u_ym);
        rv -= (vxp * uyp - vxm * uym) * dxi * one;
        const T cp = h * (v_yp + v_c), cm = h * (v_c + v_ym);
        rv -= (cp * cp - cm * cm) * dyi * one;
        const T vzp = h * (v_zp + v_c), vzm = h * (v_c + v_zm);
        const T wyp = h * (w_zp + w_ym_zp), wym = h * (w_c + w_ym);
        rv -= (vzp * wyp - vzm * wym) * dzi * one;
    }
    {
        const T wxp = h * (w_xp + w_c), wxm = h * (w_c + w_xm);
        const T uzp = h * (u_xp + u_xp_zm), uzm = h * (u_c + u_zm);
        rw -= (wxp * uzp - wxm * uzm) * dxi * one;
        const T wyp = h * (w_yp + w_c), wym = h * (w_c + w_ym);
        const T vzp = h * (v_yp + v_yp_zm), vzm = h * (v_c + v_zm);
        rw -= (wyp * vzp - wym * vzm) * dyi * one;
        const T cp = h * (w_zp + w_c), cm = h * (w_c + w_zm);
        rw -= (cp * cp - cm * cm) * dzi * one;
    }
    ru_o = ru; rv_o = rv; rw_o = rw;
}

enum StageMode { kModeRhs = 0, kModeFirst = 1, kModeMid = 2, kModeLast = 3, kModeEuler = 4 };

// TS: stage-state storage type; TA: k-sum storage type.
template <typename T, typename TI, typename TS, typename TA, int MODE>
__global__ void __launch_bounds__(256)
rhs_stage_kernel(Dims d, RhsArgs<T, TI> a, double* __restrict__ u,
                 double* __restrict__ v, double* __restrict__ w,
                 TS* __restrict__ su, TS* __restrict__ sv, TS* __restrict__ sw,
                 TA* __restrict__ au, TA* __restrict__ av, TA* __restrict__ aw,
                 T* __restrict__ ru, T* __restrict__ rv, T* __restrict__ rw,
                 double hdt, double c6, double dt) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    T ku, kv, kw;
    rhs_cell<T, TI>(d, a, i, j, k, ku, kv, kw);
    const long long q = idx(d, i, j, k);
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
    } else {  // Euler
        u[q] = u[q] + double(ku) * dt;
        v[q] = v[q] + double(kv) * dt;
        w[q] = w[q] + double(kw) * dt;
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
            (double*)ru, (double*)rv, (double*)rw, 0.0, 0.0, 0.0));
    } else {
        auto a = make_args<float, float>(g, (const float*)u, (const float*)v, (const float*)w,
                                         (const float*)visc, (const float*)sfs, mu, rho);
        PF_LAUNCH("rhs_rhs_f32", s, rhs_stage_kernel<float, float, float, float, kModeRhs><<<cell_grid(d), blk, 0, s>>>(
            d, a, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
            (float*)ru, (float*)rv, (float*)rw, 0.0, 0.0, 0.0));
    }
    return cudaGetLastError();
}

// Predictor step.  Workspace: stage states (2 ping-pong sets) and the k-sum,
// each 3 fields of the stage type (double for PF_FP64, float for PF_MIXED).
template <typename T>
static cudaError_t predictor_impl(const pf_grid* g, int rk4, double* u,
                                  double* v, double* w, const T* visc,
                                  double mu, double rho, const T* sfs,
                                  double dt, T* ws, cudaStream_t s) {
    Dims d{g->nx, g->ny, g->nz, (long long)g->nx * g->ny * g->nz};
    const long long n = d.n;
    dim3 blk(32, 8), grd = cell_grid(d);
    T *sa = ws, *sb = ws + 3 * n, *acc = ws + 6 * n;
    const double hdt = 0.5 * dt, c6 = dt / 6.0;
    auto a0 = make_args<T, double>(g, u, v, w, visc, sfs, mu, rho);
    if (!rk4) {
        PF_LAUNCH((sizeof(T) == 8 ? "rhs_euler_f64" : "rhs_euler_f32"), s, rhs_stage_kernel<T, double, T, T, kModeEuler><<<grd, blk, 0, s>>>(
            d, a0, u, v, w, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
            nullptr, nullptr, nullptr, hdt, c6, dt));
        return cudaGetLastError();
    }
    PF_LAUNCH((sizeof(T) == 8 ? "rhs_first_f64" : "rhs_first_f32"), s, rhs_stage_kernel<T, double, T, T, kModeFirst><<<grd, blk, 0, s>>>(
        d, a0, u, v, w, sa, sa + n, sa + 2 * n, acc, acc + n, acc + 2 * n,
        nullptr, nullptr, nullptr, hdt, c6, dt));
    auto a1 = make_args<T, T>(g, sa, sa + n, sa + 2 * n, visc, sfs, mu, rho);
    PF_LAUNCH((sizeof(T) == 8 ? "rhs_mid_f64" : "rhs_mid_f32"), s, rhs_stage_kernel<T, T, T, T, kModeMid><<<grd, blk, 0, s>>>(
        d, a1, u, v, w, sb, sb + n, sb + 2 * n, acc, acc + n, acc + 2 * n,
        nullptr, nullptr, nullptr, hdt, c6, dt));
    auto a2 = make_args<T, T>(g, sb, sb + n, sb + 2 * n, visc, sfs, mu, rho);
    PF_LAUNCH((sizeof(T) == 8 ? "rhs_mid_f64" : "rhs_mid_f32"), s, rhs_stage_kernel<T, T, T, T, kModeMid><<<grd, blk, 0, s>>>(
        d, a2, u, v, w, sa, sa + n, sa + 2 * n, acc, acc + n, acc + 2 * n,
        nullptr, nullptr, nullptr, hdt, c6, dt));
    PF_LAUNCH((sizeof(T) == 8 ? "rhs_last_f64" : "rhs_last_f32"), s, rhs_stage_kernel<T, T, T, T, kModeLast><<<grd, blk, 0, s>>>(
        d, a1, u, v, w, nullptr, nullptr, nullptr, acc, acc + n, acc + 2 * n,
        nullptr, nullptr, nullptr, hdt, c6, dt));
    return cudaGetLastError();
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
