// pf_flux.cuh -- the staggered Navier-Stokes right-hand side of one cell.
//
// rhs_NavierStokes.evaluate (src/solver/velocity.py:221-355) for one cell from
// its 3x3x3 neighbourhood: viscous fluxes (grad_vel_visc, div_vel_over,
// div_visc, src/metric/metric_staggered.py:373-433) and convective fluxes
// (vel_conv_*, :458-526) in the reference's operation order, including the
// edge-averaged viscosity one cell below the off-diagonal flux
// (:127-144 vs :378-384).  Host and device code: the same routine runs in the
// kernels and in a host check of the x-face carry (tests/flux_carry_check.cpp).
#pragma once
#include <cmath>

#if defined(__CUDACC__)
#define PF_HD __host__ __device__
#else
#define PF_HD
#endif

namespace pf {

#if !defined(__CUDACC__)
using std::fma;  // the float overload in host builds
#endif

template <typename T>
PF_HD inline T edge4(T a, T b, T c, T d) {
    return T(0.25) * (((a + b) + c) + d);
}

// The six x-face terms of a cell that the cell at i+1 reuses as its x-minus
// terms: the viscous fluxes fxx (centre), fxy, fxz (x-edges) and the
// convective products u u, v u, w u on the x-plus side.  Each is the same
// expression, with the same operands in the same order, as the x-minus term
// of the next cell, so reusing it changes no rounding.
template <typename T>
struct XFace {
    T fxx, fxy, fxz, cuu, cvu, cwu;
};

// Computes (ru, rv, rw) of one cell from its neighbourhood S (velocity at
// offsets -1..1, viscosity / SFS stresses at offsets -2..0 when present).
// With CARRY, the x-minus terms come from *xin (the x-plus terms of the cell
// at i-1: constant viscosity, no SFS stresses) and u at i-1 is not read;
// *xout, when given, receives this cell's x-plus terms.
template <typename T, bool CARRY = false, class Src>
PF_HD inline void rhs_core(const Src& S, T mu, T rho, T dxi, T dyi, T dzi,
                                bool has_visc, bool has_sfs, T& ru_o, T& rv_o, T& rw_o,
                                const XFace<T>* xin = nullptr, XFace<T>* xout = nullptr) {
    auto LV = [&](int di, int dj, int dk) -> T { return has_visc ? S.visc(di, dj, dk) : mu; };
    auto LS = [&](int c, int di, int dj, int dk) -> T { return S.sfs(c, di, dj, dk); };
    // velocity neighbourhood
    // (u at i-1 enters only the x-minus terms, which CARRY supplies; v and w
    // at i-1 also enter the y and z convective fluxes of u)
    const T u_c = S.u(0, 0, 0), u_xp = S.u(1, 0, 0), u_xm = CARRY ? T(0) : S.u(-1, 0, 0);
    const T u_yp = S.u(0, 1, 0), u_ym = S.u(0, -1, 0), u_zp = S.u(0, 0, 1);
    const T u_zm = S.u(0, 0, -1), u_xm_yp = CARRY ? T(0) : S.u(-1, 1, 0), u_xp_ym = S.u(1, -1, 0);
    const T u_xm_zp = CARRY ? T(0) : S.u(-1, 0, 1), u_xp_zm = S.u(1, 0, -1);
    const T v_c = S.v(0, 0, 0), v_xp = S.v(1, 0, 0), v_xm = S.v(-1, 0, 0);
    const T v_yp = S.v(0, 1, 0), v_ym = S.v(0, -1, 0), v_zp = S.v(0, 0, 1);
    const T v_zm = S.v(0, 0, -1), v_xm_yp = S.v(-1, 1, 0), v_xp_ym = S.v(1, -1, 0);
    const T v_ym_zp = S.v(0, -1, 1), v_yp_zm = S.v(0, 1, -1);
    const T w_c = S.w(0, 0, 0), w_xp = S.w(1, 0, 0), w_xm = S.w(-1, 0, 0);
    const T w_yp = S.w(0, 1, 0), w_ym = S.w(0, -1, 0), w_zp = S.w(0, 0, 1);
    const T w_zm = S.w(0, 0, -1), w_xm_zp = S.w(-1, 0, 1), w_xp_zm = S.w(1, 0, -1);
    const T w_ym_zp = S.w(0, -1, 1), w_yp_zm = S.w(0, 1, -1);

    // FP64 keeps the reference's divisions (bit-exact parity); the FP32 stage
    // of the mixed forms multiplies by the reciprocals instead (one rounding
    // more, no IEEE division sequence per use)
    constexpr bool f32 = sizeof(T) == 4;
    const T irho = T(1) / rho;
    auto over_rho = [&](T a) -> T { if constexpr (f32) return a * irho; else return a / rho; };
    // divergence / 3 at centres (div_vel_over, metric_staggered.py:424-433)
    auto div3 = [&](T ue, T uw, T vn, T vs, T wt, T wb) -> T {
        const T s = (((ue - uw) * dxi) + ((vn - vs) * dyi)) + ((wt - wb) * dzi);
        if constexpr (f32) return s * T(1.0f / 3.0f); else return s / T(3.0);
    };
    const T D_c = div3(u_xp, u_c, v_yp, v_c, w_zp, w_c);
    const T D_xm = CARRY ? T(0) : div3(u_c, u_xm, v_xm_yp, v_xm, w_xm_zp, w_xm);
    const T D_ym = div3(u_xp_ym, u_ym, v_c, v_ym, w_ym_zp, w_ym);
    const T D_zm = div3(u_xp_zm, u_zm, v_yp_zm, v_zm, w_c, w_zm);

    const T two = T(2.0);
    // diagonal viscous fluxes at centres
    const T fxx_c = ((u_xp - u_c) * dxi - D_c) * over_rho(two * LV(0, 0, 0));
    const T fxx_m = CARRY ? xin->fxx : ((u_c - u_xm) * dxi - D_xm) * over_rho(two * LV(-1, 0, 0));
    const T fyy_c = ((v_yp - v_c) * dyi - D_c) * over_rho(two * LV(0, 0, 0));
    const T fyy_m = ((v_c - v_ym) * dyi - D_ym) * over_rho(two * LV(0, -1, 0));
    const T fzz_c = ((w_zp - w_c) * dzi - D_c) * over_rho(two * LV(0, 0, 0));
    const T fzz_m = ((w_c - w_zm) * dzi - D_zm) * over_rho(two * LV(0, 0, -1));

    // edge viscosities (one cell below the flux, as in the reference)
    T vxy_c, vxy_ym, vxy_xm, vxz_c, vxz_zm, vxz_xm, vyz_c, vyz_zm, vyz_ym;
    if (has_visc) {
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
        const T m = mu;
        const T e = edge4(m, m, m, m);
        vxy_c = vxy_ym = vxy_xm = vxz_c = vxz_zm = vxz_xm = vyz_c = vyz_zm = vyz_ym = e;
    }
    // off-diagonal viscous fluxes on edges: (grad_y u + grad_x v) * (Vxy / rho)
    const T fxy_c = (((u_yp - u_c) * dyi) + ((v_xp - v_c) * dxi)) * over_rho(vxy_c);
    const T fxy_ym = (((u_c - u_ym) * dyi) + ((v_xp_ym - v_ym) * dxi)) * over_rho(vxy_ym);
    const T fxy_xm = CARRY ? xin->fxy
                           : (((u_xm_yp - u_xm) * dyi) + ((v_c - v_xm) * dxi)) * over_rho(vxy_xm);
    const T fxz_c = (((u_zp - u_c) * dzi) + ((w_xp - w_c) * dxi)) * over_rho(vxz_c);
    const T fxz_zm = (((u_c - u_zm) * dzi) + ((w_xp_zm - w_zm) * dxi)) * over_rho(vxz_zm);
    const T fxz_xm = CARRY ? xin->fxz
                           : (((u_xm_zp - u_xm) * dzi) + ((w_c - w_xm) * dxi)) * over_rho(vxz_xm);
    const T fyz_c = (((v_zp - v_c) * dzi) + ((w_yp - w_c) * dyi)) * over_rho(vyz_c);
    const T fyz_zm = (((v_c - v_zm) * dzi) + ((w_yp_zm - w_zm) * dyi)) * over_rho(vyz_zm);
    const T fyz_ym = (((v_ym_zp - v_ym) * dzi) + ((w_c - w_ym) * dyi)) * over_rho(vyz_ym);

    T ux_p = fxx_c, ux_m = fxx_m, uy_p = fxy_c, uy_m = fxy_ym, uz_p = fxz_c, uz_m = fxz_zm;
    T vx_p = fxy_c, vx_m = fxy_xm, vy_p = fyy_c, vy_m = fyy_m, vz_p = fyz_c, vz_m = fyz_zm;
    T wx_p = fxz_c, wx_m = fxz_xm, wy_p = fyz_c, wy_m = fyz_ym, wz_p = fzz_c, wz_m = fzz_m;
    if (has_sfs) {
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
    T cuu_p, cvu_p, cwu_p;  // this cell's x-plus convective products
    {
        const T cp = h * (u_xp + u_c);
        cuu_p = cp * cp;
        T cmm;
        if constexpr (CARRY) cmm = xin->cuu;
        else { const T cm = h * (u_c + u_xm); cmm = cm * cm; }
        ru -= (cuu_p - cmm) * dxi * one;
        const T uyp = h * (u_yp + u_c), uym = h * (u_c + u_ym);
        const T vxp = h * (v_yp + v_xm_yp), vxm = h * (v_c + v_xm);
        ru -= (uyp * vxp - uym * vxm) * dyi * one;
        const T uzp = h * (u_zp + u_c), uzm = h * (u_c + u_zm);
        const T wxp = h * (w_zp + w_xm_zp), wxm = h * (w_c + w_xm);
        ru -= (uzp * wxp - uzm * wxm) * dzi * one;
    }
    {
        const T vxp = h * (v_xp + v_c);
        const T uyp = h * (u_xp + u_xp_ym);
        cvu_p = vxp * uyp;
        T mm;
        if constexpr (CARRY) mm = xin->cvu;
        else { const T vxm = h * (v_c + v_xm), uym = h * (u_c + u_ym); mm = vxm * uym; }
        rv -= (cvu_p - mm) * dxi * one;
        const T cp = h * (v_yp + v_c), cm = h * (v_c + v_ym);
        rv -= (cp * cp - cm * cm) * dyi * one;
        const T vzp = h * (v_zp + v_c), vzm = h * (v_c + v_zm);
        const T wyp = h * (w_zp + w_ym_zp), wym = h * (w_c + w_ym);
        rv -= (vzp * wyp - vzm * wym) * dzi * one;
    }
    {
        const T wxp = h * (w_xp + w_c);
        const T uzp = h * (u_xp + u_xp_zm);
        cwu_p = wxp * uzp;
        T mm;
        if constexpr (CARRY) mm = xin->cwu;
        else { const T wxm = h * (w_c + w_xm), uzm = h * (u_c + u_zm); mm = wxm * uzm; }
        rw -= (cwu_p - mm) * dxi * one;
        const T wyp = h * (w_yp + w_c), wym = h * (w_c + w_ym);
        const T vzp = h * (v_yp + v_yp_zm), vzm = h * (v_c + v_zm);
        rw -= (wyp * vzp - wym * vzm) * dyi * one;
        const T cp = h * (w_zp + w_c), cm = h * (w_c + w_zm);
        rw -= (cp * cp - cm * cm) * dzi * one;
    }
    ru_o = ru; rv_o = rv; rw_o = rw;
    if (xout) *xout = XFace<T>{fxx_c, fxy_c, fxz_c, cuu_p, cvu_p, cwu_p};
}

// ---------------------------------------------------------------------------
// Face form of the same right-hand side (constant viscosity, no SFS stresses):
// each cell computes the terms on its three plus faces once, and a cell's
// minus-face terms are the plus-face terms of its neighbours at i-1, j-1 and
// k-1 -- the same expressions on the same operands as rhs_core's minus terms,
// so assembling them in rhs_core's order gives its result bit for bit.
//   x-plus (XFace): fxx, fxy, fxz and the products u u, v u, w u
//   y-plus (YFace): fxy, fyy, fyz and the products of u, v, w on the y face
//   z-plus (ZFace): fxz, fyz, fzz and the products of u, v, w on the z face
template <typename T>
struct YFace {
    T fxy, fyy, fyz, cuv, cvv, cwv;
};

template <typename T>
struct ZFace {
    T fxz, fyz, fzz, cuw, cvw, cww;
};

template <typename T>
struct PlusFaces {
    XFace<T> x;
    YFace<T> y;
    ZFace<T> z;
};

template <typename T>
struct FluxCoef {
    T dxi, dyi, dzi;
    T two_mu_r;   // over_rho(2 mu): the diagonal fluxes' factor
    T edge_r;     // over_rho(edge4(mu, mu, mu, mu)): the off-diagonal fluxes' factor
};

// rhs_core's scalar factors for constant viscosity (over_rho of the FP32 form
// multiplies by 1/rho, the FP64 form divides)
template <typename T>
PF_HD inline FluxCoef<T> flux_coef(T mu, T rho, T dxi, T dyi, T dzi) {
    constexpr bool f32 = sizeof(T) == 4;
    const T irho = T(1) / rho;
    auto over_rho = [&](T a) -> T { if constexpr (f32) return a * irho; else return a / rho; };
    return FluxCoef<T>{dxi, dyi, dzi, over_rho(T(2.0) * mu), over_rho(edge4(mu, mu, mu, mu))};
}

template <typename T>
PF_HD inline T div3_c(T ue, T uw, T vn, T vs, T wt, T wb, const FluxCoef<T>& c) {
    const T s = (((ue - uw) * c.dxi) + ((vn - vs) * c.dyi)) + ((wt - wb) * c.dzi);
    if constexpr (sizeof(T) == 4) return s * T(1.0f / 3.0f); else return s / T(3.0);
}

// Plus-face terms of one cell; with Y / Z false the y / z set is skipped (the
// halo cells of a tile need only one set).  Uses the velocity at x, y, z
// offsets 0 and +1 and, for the products, -1 in the other two directions.
template <typename T, bool X = true, bool Y = true, bool Z = true, class Src>
PF_HD inline PlusFaces<T> plus_faces(const Src& S, const FluxCoef<T>& c) {
    const T h = T(0.5);
    const T u_c = S.u(0, 0, 0), v_c = S.v(0, 0, 0), w_c = S.w(0, 0, 0);
    const T u_xp = S.u(1, 0, 0), v_yp = S.v(0, 1, 0), w_zp = S.w(0, 0, 1);
    const T D_c = div3_c(u_xp, u_c, v_yp, v_c, w_zp, w_c, c);
    PlusFaces<T> f;
    T fxy = T(0), fxz = T(0), fyz = T(0);
    if (X || Y) {
        const T u_yp = S.u(0, 1, 0), v_xp = S.v(1, 0, 0);
        fxy = (((u_yp - u_c) * c.dyi) + ((v_xp - v_c) * c.dxi)) * c.edge_r;
    }
    if (X || Z) {
        const T u_zp = S.u(0, 0, 1), w_xp = S.w(1, 0, 0);
        fxz = (((u_zp - u_c) * c.dzi) + ((w_xp - w_c) * c.dxi)) * c.edge_r;
    }
    if (Y || Z) {
        const T v_zp = S.v(0, 0, 1), w_yp = S.w(0, 1, 0);
        fyz = (((v_zp - v_c) * c.dzi) + ((w_yp - w_c) * c.dyi)) * c.edge_r;
    }
    if (X) {
        const T v_xp = S.v(1, 0, 0), w_xp = S.w(1, 0, 0);
        const T cp = h * (u_xp + u_c);
        const T vxp = h * (v_xp + v_c), uyp = h * (u_xp + S.u(1, -1, 0));
        const T wxp = h * (w_xp + w_c), uzp = h * (u_xp + S.u(1, 0, -1));
        f.x = XFace<T>{((u_xp - u_c) * c.dxi - D_c) * c.two_mu_r, fxy, fxz, cp * cp, vxp * uyp,
                       wxp * uzp};
    }
    if (Y) {
        const T u_yp = S.u(0, 1, 0), w_yp = S.w(0, 1, 0);
        const T uyp = h * (u_yp + u_c), vxp = h * (v_yp + S.v(-1, 1, 0));
        const T cp = h * (v_yp + v_c);
        const T wyp = h * (w_yp + w_c), vzp = h * (v_yp + S.v(0, 1, -1));
        f.y = YFace<T>{fxy, ((v_yp - v_c) * c.dyi - D_c) * c.two_mu_r, fyz, uyp * vxp, cp * cp,
                       wyp * vzp};
    }
    if (Z) {
        const T u_zp = S.u(0, 0, 1), v_zp = S.v(0, 0, 1);
        const T uzp = h * (u_zp + u_c), wxp = h * (w_zp + S.w(-1, 0, 1));
        const T vzp = h * (v_zp + v_c), wyp = h * (w_zp + S.w(0, -1, 1));
        const T cp = h * (w_zp + w_c);
        f.z = ZFace<T>{fxz, fyz, ((w_zp - w_c) * c.dzi - D_c) * c.two_mu_r, uzp * wxp, vzp * wyp,
                       cp * cp};
    }
    return f;
}

// (ru, rv, rw) of a cell from its plus-face terms p and the plus-face terms of
// its neighbours at i-1 (xm), j-1 (ym), k-1 (zm), in rhs_core's order
template <typename T>
PF_HD inline void assemble_faces(const PlusFaces<T>& p, const XFace<T>& xm, const YFace<T>& ym,
                                 const ZFace<T>& zm, const FluxCoef<T>& c, T& ru_o, T& rv_o,
                                 T& rw_o) {
    const T dxi = c.dxi, dyi = c.dyi, dzi = c.dzi, one = T(1.0);
    T ru = T(0), rv = T(0), rw = T(0);
    ru = fma(dxi, p.x.fxx, ru); ru = fma(-dxi, xm.fxx, ru);
    ru = fma(dyi, p.y.fxy, ru); ru = fma(-dyi, ym.fxy, ru);
    ru = fma(dzi, p.z.fxz, ru); ru = fma(-dzi, zm.fxz, ru);
    rv = fma(dxi, p.x.fxy, rv); rv = fma(-dxi, xm.fxy, rv);
    rv = fma(dyi, p.y.fyy, rv); rv = fma(-dyi, ym.fyy, rv);
    rv = fma(dzi, p.z.fyz, rv); rv = fma(-dzi, zm.fyz, rv);
    rw = fma(dxi, p.x.fxz, rw); rw = fma(-dxi, xm.fxz, rw);
    rw = fma(dyi, p.y.fyz, rw); rw = fma(-dyi, ym.fyz, rw);
    rw = fma(dzi, p.z.fzz, rw); rw = fma(-dzi, zm.fzz, rw);
    ru -= (p.x.cuu - xm.cuu) * dxi * one;
    ru -= (p.y.cuv - ym.cuv) * dyi * one;
    ru -= (p.z.cuw - zm.cuw) * dzi * one;
    rv -= (p.x.cvu - xm.cvu) * dxi * one;
    rv -= (p.y.cvv - ym.cvv) * dyi * one;
    rv -= (p.z.cvw - zm.cvw) * dzi * one;
    rw -= (p.x.cwu - xm.cwu) * dxi * one;
    rw -= (p.y.cwv - ym.cwv) * dyi * one;
    rw -= (p.z.cww - zm.cww) * dzi * one;
    ru_o = ru; rv_o = rv; rw_o = rw;
}

// A source shifted by (a, b, c) cells: the neighbour's view of the same data
template <class Src>
struct Shifted {
    const Src& s;
    int a, b, c;
    PF_HD auto u(int di, int dj, int dk) const { return s.u(di + a, dj + b, dk + c); }
    PF_HD auto v(int di, int dj, int dk) const { return s.v(di + a, dj + b, dk + c); }
    PF_HD auto w(int di, int dj, int dk) const { return s.w(di + a, dj + b, dk + c); }
};

}  // namespace pf
