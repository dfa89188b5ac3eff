/*
 * pf_oracle.c -- CPU restatement (FP64, OpenMP) of PyFlow's time-advance hot
 * path.  TEST INFRASTRUCTURE ONLY: the CUDA product never links or calls this
 * file; tests/, the smoke check and bench.py's CPU-baseline / reference arm use
 * it as the checker.  Parity of this restatement with the reference itself is
 * pinned by tests/test_oracle_golden.py against fixtures generated by running
 * the unmodified reference (tests/golden/make_golden.py).
 *
 * Fields are ghost-free [nx][ny][nz] arrays (z contiguous), i.e. the
 * reference's state_P.interior() (src/data/state.py:142-146); the reference's
 * periodic 2-deep ghost exchange (src/library/parallel.py:301-414) becomes
 * index wrap.
 *
 * Rounding follows the reference operation by operation: the file is compiled
 * with -ffp-contract=off, and an explicit fma() appears exactly where the
 * reference calls torch's add_(alpha, x) / sub_(alpha, x), which torch
 * evaluates as one fused multiply-add.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int nx, ny, nz;
    double dx, dy, dz;
} or_grid;

#define IDX(i, j, k) (((size_t)(i) * ny + (size_t)(j)) * nz + (size_t)(k))
#define WRAP(a, n) ((a) < 0 ? (a) + (n) : ((a) >= (n) ? (a) - (n) : (a)))

static size_t ncell(const or_grid* g) { return (size_t)g->nx * g->ny * g->nz; }

/* 0.25*(((a+b)+c)+d): interp_sc_xy/xz/yz, src/metric/metric_staggered.py:127-144 */
static inline double edge4(double a, double b, double c, double d) {
    return 0.25 * (((a + b) + c) + d);
}

/* ------------------------------------------------------------------------ *
 * rhs_NavierStokes.evaluate  (src/solver/velocity.py:221-355)
 *   visc == NULL : VISC_P is the constant mu everywhere
 *                  (src/data/domain.py:130-131)
 *   sfs  != NULL : 'tensor' SFS model stresses FXX,FYY,FZZ,FXY,FXZ,FYZ at cell
 *                  centres (six consecutive fields), added to the viscous flux
 *                  (src/solver/velocity.py:262-267,286-291,310-315)
 * ------------------------------------------------------------------------ */
void or_rhs_ns(const or_grid* g, const double* u, const double* v,
               const double* w, const double* visc, double mu, double rho,
               const double* sfs, double* ru, double* rv, double* rw) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const double dxi = 1.0 / g->dx, dyi = 1.0 / g->dy, dzi = 1.0 / g->dz;
    const size_t n = ncell(g);
    const double *FXX = 0, *FYY = 0, *FZZ = 0, *FXY = 0, *FXZ = 0, *FYZ = 0;
    if (sfs) {
        FXX = sfs; FYY = sfs + n; FZZ = sfs + 2 * n;
        FXY = sfs + 3 * n; FXZ = sfs + 4 * n; FYZ = sfs + 5 * n;
    }
#define V(i, j, k) (visc ? visc[IDX(WRAP(i, nx), WRAP(j, ny), WRAP(k, nz))] : mu)
#define F(a, i, j, k) (a[IDX(WRAP(i, nx), WRAP(j, ny), WRAP(k, nz))])
#define U(i, j, k) F(u, i, j, k)
#define VV(i, j, k) F(v, i, j, k)
#define W(i, j, k) F(w, i, j, k)
/* div_vel_over / 3 at a cell centre: metric_staggered.py:424-433, velocity.py:240-241 */
#define DIV3(i, j, k)                                                     \
    (((((U(i + 1, j, k) - U(i, j, k)) * dxi) +                           \
       ((VV(i, j + 1, k) - VV(i, j, k)) * dyi)) +                         \
      ((W(i, j, k + 1) - W(i, j, k)) * dzi)) / 3.0)
/* diagonal viscous flux of component c: (grad - div/3) * (2 VISC / rho) */
#define DIAG_X(i, j, k) (((U(i + 1, j, k) - U(i, j, k)) * dxi - DIV3(i, j, k)) * ((2.0 * V(i, j, k)) / rho))
#define DIAG_Y(i, j, k) (((VV(i, j + 1, k) - VV(i, j, k)) * dyi - DIV3(i, j, k)) * ((2.0 * V(i, j, k)) / rho))
#define DIAG_Z(i, j, k) (((W(i, j, k + 1) - W(i, j, k)) * dzi - DIV3(i, j, k)) * ((2.0 * V(i, j, k)) / rho))
/* off-diagonal viscous fluxes (grad_vel_visc forward differences, edge-averaged
   VISC one cell below: quirk of interp_sc_xy/xz/yz) */
#define VXY(i, j, k) edge4(V(i, j, k), V(i - 1, j, k), V(i, j - 1, k), V(i - 1, j - 1, k))
#define VXZ(i, j, k) edge4(V(i, j, k), V(i - 1, j, k), V(i, j, k - 1), V(i - 1, j, k - 1))
#define VYZ(i, j, k) edge4(V(i, j, k), V(i, j - 1, k), V(i, j, k - 1), V(i, j - 1, k - 1))
#define OFF_XY(i, j, k) ((((U(i, j + 1, k) - U(i, j, k)) * dyi) + ((VV(i + 1, j, k) - VV(i, j, k)) * dxi)) * (VXY(i, j, k) / rho))
#define OFF_XZ(i, j, k) ((((U(i, j, k + 1) - U(i, j, k)) * dzi) + ((W(i + 1, j, k) - W(i, j, k)) * dxi)) * (VXZ(i, j, k) / rho))
#define OFF_YZ(i, j, k) ((((VV(i, j, k + 1) - VV(i, j, k)) * dzi) + ((W(i, j + 1, k) - W(i, j, k)) * dyi)) * (VYZ(i, j, k) / rho))
#define SXY(i, j, k) edge4(F(FXY, i, j, k), F(FXY, i - 1, j, k), F(FXY, i, j - 1, k), F(FXY, i - 1, j - 1, k))
#define SXZ(i, j, k) edge4(F(FXZ, i, j, k), F(FXZ, i - 1, j, k), F(FXZ, i, j, k - 1), F(FXZ, i - 1, j, k - 1))
#define SYZ(i, j, k) edge4(F(FYZ, i, j, k), F(FYZ, i, j - 1, k), F(FYZ, i, j, k - 1), F(FYZ, i, j - 1, k - 1))
    int i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < nx; ++i) {
        for (int j = 0; j < ny; ++j) {
            for (int k = 0; k < nz; ++k) {
                double fxp, fxm, fyp, fym, fzp, fzm, r;
                /* ---- u: viscous ---- */
                fxp = DIAG_X(i, j, k);     fxm = DIAG_X(i - 1, j, k);
                fyp = OFF_XY(i, j, k);     fym = OFF_XY(i, j - 1, k);
                fzp = OFF_XZ(i, j, k);     fzm = OFF_XZ(i, j, k - 1);
                if (sfs) {
                    fxp += F(FXX, i, j, k); fxm += F(FXX, i - 1, j, k);
                    fyp += SXY(i, j, k);    fym += SXY(i, j - 1, k);
                    fzp += SXZ(i, j, k);    fzm += SXZ(i, j, k - 1);
                }
                r = 0.0;
                r = fma(dxi, fxp, r); r = fma(-dxi, fxm, r);
                r = fma(dyi, fyp, r); r = fma(-dyi, fym, r);
                r = fma(dzi, fzp, r); r = fma(-dzi, fzm, r);
                /* ---- u: convective (metric_staggered.py:458-526) ---- */
                {
                    double cp = 0.5 * (U(i + 1, j, k) + U(i, j, k));
                    double cm = 0.5 * (U(i, j, k) + U(i - 1, j, k));
                    r -= (cp * cp - cm * cm) * dxi * 1.0;
                    double uyp = 0.5 * (U(i, j + 1, k) + U(i, j, k));
                    double uym = 0.5 * (U(i, j, k) + U(i, j - 1, k));
                    double vxp = 0.5 * (VV(i, j + 1, k) + VV(i - 1, j + 1, k));
                    double vxm = 0.5 * (VV(i, j, k) + VV(i - 1, j, k));
                    r -= (uyp * vxp - uym * vxm) * dyi * 1.0;
                    double uzp = 0.5 * (U(i, j, k + 1) + U(i, j, k));
                    double uzm = 0.5 * (U(i, j, k) + U(i, j, k - 1));
                    double wxp = 0.5 * (W(i, j, k + 1) + W(i - 1, j, k + 1));
                    double wxm = 0.5 * (W(i, j, k) + W(i - 1, j, k));
                    r -= (uzp * wxp - uzm * wxm) * dzi * 1.0;
                }
                ru[IDX(i, j, k)] = r;

                /* ---- v: viscous ---- */
                fxp = OFF_XY(i, j, k);     fxm = OFF_XY(i - 1, j, k);
                fyp = DIAG_Y(i, j, k);     fym = DIAG_Y(i, j - 1, k);
                fzp = OFF_YZ(i, j, k);     fzm = OFF_YZ(i, j, k - 1);
                if (sfs) {
                    fxp += SXY(i, j, k);    fxm += SXY(i - 1, j, k);
                    fyp += F(FYY, i, j, k); fym += F(FYY, i, j - 1, k);
                    fzp += SYZ(i, j, k);    fzm += SYZ(i, j, k - 1);
                }
                r = 0.0;
                r = fma(dxi, fxp, r); r = fma(-dxi, fxm, r);
                r = fma(dyi, fyp, r); r = fma(-dyi, fym, r);
                r = fma(dzi, fzp, r); r = fma(-dzi, fzm, r);
                {
                    double vxp = 0.5 * (VV(i + 1, j, k) + VV(i, j, k));
                    double vxm = 0.5 * (VV(i, j, k) + VV(i - 1, j, k));
                    double uyp = 0.5 * (U(i + 1, j, k) + U(i + 1, j - 1, k));
                    double uym = 0.5 * (U(i, j, k) + U(i, j - 1, k));
                    r -= (vxp * uyp - vxm * uym) * dxi * 1.0;
                    double cp = 0.5 * (VV(i, j + 1, k) + VV(i, j, k));
                    double cm = 0.5 * (VV(i, j, k) + VV(i, j - 1, k));
                    r -= (cp * cp - cm * cm) * dyi * 1.0;
                    double vzp = 0.5 * (VV(i, j, k + 1) + VV(i, j, k));
                    double vzm = 0.5 * (VV(i, j, k) + VV(i, j, k - 1));
                    double wyp = 0.5 * (W(i, j, k + 1) + W(i, j - 1, k + 1));
                    double wym = 0.5 * (W(i, j, k) + W(i, j - 1, k));
                    r -= (vzp * wyp - vzm * wym) * dzi * 1.0;
                }
                rv[IDX(i, j, k)] = r;

                /* ---- w: viscous ---- */
                fxp = OFF_XZ(i, j, k);     fxm = OFF_XZ(i - 1, j, k);
                fyp = OFF_YZ(i, j, k);     fym = OFF_YZ(i, j - 1, k);
                fzp = DIAG_Z(i, j, k);     fzm = DIAG_Z(i, j, k - 1);
                if (sfs) {
                    fxp += SXZ(i, j, k);    fxm += SXZ(i - 1, j, k);
                    fyp += SYZ(i, j, k);    fym += SYZ(i, j - 1, k);
                    fzp += F(FZZ, i, j, k); fzm += F(FZZ, i, j, k - 1);
                }
                r = 0.0;
                r = fma(dxi, fxp, r); r = fma(-dxi, fxm, r);
                r = fma(dyi, fyp, r); r = fma(-dyi, fym, r);
                r = fma(dzi, fzp, r); r = fma(-dzi, fzm, r);
                {
                    double wxp = 0.5 * (W(i + 1, j, k) + W(i, j, k));
                    double wxm = 0.5 * (W(i, j, k) + W(i - 1, j, k));
                    double uzp = 0.5 * (U(i + 1, j, k) + U(i + 1, j, k - 1));
                    double uzm = 0.5 * (U(i, j, k) + U(i, j, k - 1));
                    r -= (wxp * uzp - wxm * uzm) * dxi * 1.0;
                    double wyp = 0.5 * (W(i, j + 1, k) + W(i, j, k));
                    double wym = 0.5 * (W(i, j, k) + W(i, j - 1, k));
                    double vzp = 0.5 * (VV(i, j + 1, k) + VV(i, j + 1, k - 1));
                    double vzm = 0.5 * (VV(i, j, k) + VV(i, j, k - 1));
                    r -= (wyp * vzp - wym * vzm) * dyi * 1.0;
                    double cp = 0.5 * (W(i, j, k + 1) + W(i, j, k));
                    double cm = 0.5 * (W(i, j, k) + W(i, j, k - 1));
                    r -= (cp * cp - cm * cm) * dzi * 1.0;
                }
                rw[IDX(i, j, k)] = r;
            }
        }
    }
#undef V
#undef F
#undef U
#undef VV
#undef W
#undef DIV3
#undef DIAG_X
#undef DIAG_Y
#undef DIAG_Z
#undef VXY
#undef VXZ
#undef VYZ
#undef OFF_XY
#undef OFF_XZ
#undef OFF_YZ
#undef SXY
#undef SXZ
#undef SYZ
}

/* ------------------------------------------------------------------------ *
 * RK4.step (src/solver/advancer.py:75-113), including the reference's stage-4
 * state u + 0.5*dt*k3.  Updates u, v, w in place.
 * ------------------------------------------------------------------------ */
void or_rk4_step(const or_grid* g, double* u, double* v, double* w,
                 const double* visc, double mu, double rho, const double* sfs,
                 double dt) {
    const size_t n = ncell(g);
    double* buf = (double*)malloc(sizeof(double) * n * 12);
    double *ut = buf, *vt = buf + n, *wt = buf + 2 * n;
    double *k[4][3];
    for (int s = 0; s < 3; ++s)
        for (int c = 0; c < 3; ++c) k[s][c] = buf + (3 + 3 * s + c) * n;
    double *ku = 0, *kv = 0, *kw = 0;
    const double h = 0.5 * dt;
    /* stage 1 */
    or_rhs_ns(g, u, v, w, visc, mu, rho, sfs, k[0][0], k[0][1], k[0][2]);
    for (int s = 1; s < 4; ++s) {
        size_t q;
#pragma omp parallel for schedule(static)
        for (q = 0; q < n; ++q) {
            ut[q] = h * k[s - 1][0][q] + u[q]; /* ZAXPY: A*X + Y, state.py:157-165 */
            vt[q] = h * k[s - 1][1][q] + v[q];
            wt[q] = h * k[s - 1][2][q] + w[q];
        }
        if (s < 3) {
            ku = k[s][0]; kv = k[s][1]; kw = k[s][2];
        } else {
            /* stage-4 rhs: reuse the stage-1 .. 3 storage only after the
               combination below has consumed them, so use fresh buffers */
            ku = (double*)malloc(sizeof(double) * n * 3);
            kv = ku + n; kw = ku + 2 * n;
        }
        or_rhs_ns(g, ut, vt, wt, visc, mu, rho, sfs, ku, kv, kw);
    }
    {
        const double c6 = dt / 6.0;
        size_t q;
#pragma omp parallel for schedule(static)
        for (q = 0; q < n; ++q) {
            double su = ((k[0][0][q] + 2.0 * k[1][0][q]) + 2.0 * k[2][0][q]) + ku[q];
            double sv = ((k[0][1][q] + 2.0 * k[1][1][q]) + 2.0 * k[2][1][q]) + kv[q];
            double sw = ((k[0][2][q] + 2.0 * k[1][2][q]) + 2.0 * k[2][2][q]) + kw[q];
            u[q] = u[q] + c6 * su;
            v[q] = v[q] + c6 * sv;
            w[q] = w[q] + c6 * sw;
        }
    }
    free(ku);
    free(buf);
}

/* Euler.step (src/solver/advancer.py:49-57) */
void or_euler_step(const or_grid* g, double* u, double* v, double* w,
                   const double* visc, double mu, double rho, const double* sfs,
                   double dt) {
    const size_t n = ncell(g);
    double* k = (double*)malloc(sizeof(double) * n * 3);
    or_rhs_ns(g, u, v, w, visc, mu, rho, sfs, k, k + n, k + 2 * n);
    size_t q;
#pragma omp parallel for schedule(static)
    for (q = 0; q < n; ++q) {
        u[q] = u[q] + k[q] * dt;
        v[q] = v[q] + k[n + q] * dt;
        w[q] = w[q] + k[2 * n + q] * dt;
    }
    free(k);
}

/* metric_uniform.div_vel (src/metric/metric_staggered.py:438-453) */
void or_div_vel(const or_grid* g, const double* u, const double* v,
                const double* w, double* divg) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const double dxi = 1.0 / g->dx, dyi = 1.0 / g->dy, dzi = 1.0 / g->dz;
    int i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < nx; ++i) {
        const int ip = WRAP(i + 1, nx);
        for (int j = 0; j < ny; ++j) {
            const int jp = WRAP(j + 1, ny);
            for (int k = 0; k < nz; ++k) {
                const int kp = WRAP(k + 1, nz);
                double d = (u[IDX(ip, j, k)] - u[IDX(i, j, k)]) * dxi;
                d += (v[IDX(i, jp, k)] - v[IDX(i, j, k)]) * dyi;
                d += (w[IDX(i, j, kp)] - w[IDX(i, j, k)]) * dzi;
                divg[IDX(i, j, k)] = d;
            }
        }
    }
}

/* Laplace coefficients of metric_uniform.__init__ (metric_staggered.py:84-102):
   c[d][0..2] = {dxi^2, -2 dxi^2, dxi^2} * (-vol) */
static void lap_coeffs(const or_grid* g, double c[3][3]) {
    const double dxi = 1.0 / g->dx, dyi = 1.0 / g->dy, dzi = 1.0 / g->dz;
    const double vol = (g->dx * g->dy) * g->dz;
    const double di[3] = {dxi, dyi, dzi};
    for (int d = 0; d < 3; ++d) {
        c[d][0] = (di[d] * di[d]) * (-1.0 * vol);
        c[d][1] = ((-2.0 * di[d]) * di[d]) * (-1.0 * vol);
        c[d][2] = (di[d] * di[d]) * (-1.0 * vol);
    }
}

/* Pressure_Base.applyOperator (src/solver/pressure.py:54-84): B = (-vol L) A */
void or_laplace_apply(const or_grid* g, const double* A, double* B) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    double c[3][3];
    lap_coeffs(g, c);
    int i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < nx; ++i) {
        const int im = WRAP(i - 1, nx), ip = WRAP(i + 1, nx);
        for (int j = 0; j < ny; ++j) {
            const int jm = WRAP(j - 1, ny), jp = WRAP(j + 1, ny);
            for (int k = 0; k < nz; ++k) {
                const int km = WRAP(k - 1, nz), kp = WRAP(k + 1, nz);
                double b = 0.0;
                b += A[IDX(im, j, k)] * c[0][0];
                b += A[IDX(i, j, k)] * c[0][1];
                b += A[IDX(ip, j, k)] * c[0][2];
                b += A[IDX(i, jm, k)] * c[1][0];
                b += A[IDX(i, j, k)] * c[1][1];
                b += A[IDX(i, jp, k)] * c[1][2];
                b += A[IDX(i, j, km)] * c[2][0];
                b += A[IDX(i, j, k)] * c[2][1];
                b += A[IDX(i, j, kp)] * c[2][2];
                B[IDX(i, j, k)] = b;
            }
        }
    }
}

/* Deterministic sums: one partial per x-plane in (j,k) order, planes summed
   in order.  Independent of the OpenMP thread count. */
static double dot(const or_grid* g, const double* a, const double* b) {
    const int nx = g->nx;
    const size_t plane = (size_t)g->ny * g->nz;
    double* part = (double*)malloc(sizeof(double) * nx);
    int i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < nx; ++i) {
        double s = 0.0;
        const double* pa = a + i * plane;
        const double* pb = b + i * plane;
        for (size_t q = 0; q < plane; ++q) s += pa[q] * pb[q];
        part[i] = s;
    }
    double s = 0.0;
    for (i = 0; i < nx; ++i) s += part[i];
    free(part);
    return s;
}

static double absmax(size_t n, const double* a) {
    double m = 0.0;
    size_t q;
#pragma omp parallel for reduction(max : m) schedule(static)
    for (q = 0; q < n; ++q) {
        double t = fabs(a[q]);
        if (t > m || t != t) m = t;
    }
    return m;
}

/* ------------------------------------------------------------------------ *
 * solver_bicgstab.solve (src/solver/pressure.py:196-297).  source is scaled in
 * place by rho/dt and -vol exactly as the reference does; DP is zeroed and
 * overwritten; p += DP.  Returns max_res; *iters gets the iteration count and
 * *status 0 (done), 1 (gamma == 0 breakdown), 2 (buf2 == 0 breakdown).
 * ------------------------------------------------------------------------ */
double or_bicgstab(const or_grid* g, double rho, double dt, double min_res,
                   int max_it, double* DP, double* p, double* source,
                   int* iters, int* status) {
    const size_t n = ncell(g);
    const double vol = (g->dx * g->dy) * g->dz;
    double* buf = (double*)calloc(n * 6, sizeof(double));
    double *pp = buf, *s = buf + n, *vv = buf + 2 * n, *t = buf + 3 * n,
           *res = buf + 4 * n, *res0 = buf + 5 * n;
    size_t q;
    memset(DP, 0, sizeof(double) * n);
    const double sc = rho / dt, sv = -1.0 * vol;
#pragma omp parallel for schedule(static)
    for (q = 0; q < n; ++q) {
        source[q] = source[q] * sc;
        source[q] = source[q] * sv;
        res[q] = source[q];
        res0[q] = source[q];
    }
    const double max_res0 = absmax(n, res);
    double rho1 = 1.0, rho2 = 1.0, alpha = 0.0, omega = 1.0, max_res = 0.0;
    int it = 0, st = 0;
    for (;;) {
        rho1 = dot(g, res, res0);
        const double beta = alpha * rho1 / (rho2 * omega);
#pragma omp parallel for schedule(static)
        for (q = 0; q < n; ++q) {
            double x = fma(-omega, vv[q], pp[q]);
            x = x * beta;
            pp[q] = x + res[q];
        }
        or_laplace_apply(g, pp, vv);
        const double gamma = dot(g, vv, res0);
        if (gamma == 0.0) { st = 1; break; }
        alpha = rho1 / gamma;
#pragma omp parallel for schedule(static)
        for (q = 0; q < n; ++q) {
            DP[q] = fma(alpha, pp[q], DP[q]);
            s[q] = fma(-alpha, vv[q], res[q]);
        }
        or_laplace_apply(g, s, t);
        const double buf1 = dot(g, s, t);
        const double buf2 = dot(g, t, t);
        if (buf2 == 0.0) { st = 2; break; }
        omega = buf1 / buf2;
#pragma omp parallel for schedule(static)
        for (q = 0; q < n; ++q) {
            DP[q] = fma(omega, s[q], DP[q]);
            res[q] = fma(-omega, t[q], s[q]);
        }
        rho2 = rho1;
        max_res = absmax(n, res) / max_res0;
        ++it;
        if (it >= max_it) break;
        if (max_res <= min_res) break;
    }
#pragma omp parallel for schedule(static)
    for (q = 0; q < n; ++q) p[q] = p[q] + DP[q];
    free(buf);
    if (iters) *iters = it;
    if (status) *status = st;
    return max_res;
}

/* ------------------------------------------------------------------------ *
 * solver_jacobi.solve (src/solver/pressure.py:115-161).  p is zeroed and holds
 * the last iterate; pold (the domain's DP) holds the one before it; the
 * returned residual is the reference's (source - (-vol L) p) max-norm ratio.
 * ------------------------------------------------------------------------ */
double or_jacobi(const or_grid* g, double rho, double dt, int n_it,
                 double* pold, double* p, double* source) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const size_t n = ncell(g);
    const double dx = g->dx;
    double* res = (double*)malloc(sizeof(double) * n);
    size_t q;
    memset(p, 0, sizeof(double) * n);
    const double sc = rho / dt;
#pragma omp parallel for schedule(static)
    for (q = 0; q < n; ++q) source[q] = source[q] * sc;
    const double max_res0 = absmax(n, source);
    const double DInv = -1.0 / 6.0;
    const double dx2 = pow(dx, 2.0);
#pragma omp parallel for schedule(static)
    for (q = 0; q < n; ++q) source[q] = source[q] * dx2;
    for (int it = 0; it < n_it; ++it) {
        memcpy(pold, p, sizeof(double) * n);
        int i;
#pragma omp parallel for schedule(static)
        for (i = 0; i < nx; ++i) {
            const int im = WRAP(i - 1, nx), ip = WRAP(i + 1, nx);
            for (int j = 0; j < ny; ++j) {
                const int jm = WRAP(j - 1, ny), jp = WRAP(j + 1, ny);
                for (int k = 0; k < nz; ++k) {
                    const int km = WRAP(k - 1, nz), kp = WRAP(k + 1, nz);
                    double x = -pold[IDX(ip, j, k)];
                    x = x - pold[IDX(im, j, k)];
                    x = x - pold[IDX(i, jp, k)];
                    x = x - pold[IDX(i, jm, k)];
                    x = x - pold[IDX(i, j, kp)];
                    x = x - pold[IDX(i, j, km)];
                    x = x + source[IDX(i, j, k)];
                    p[IDX(i, j, k)] = x * DInv;
                }
            }
        }
    }
#pragma omp parallel for schedule(static)
    for (q = 0; q < n; ++q) source[q] = source[q] / dx2;
    or_laplace_apply(g, p, res);
#pragma omp parallel for schedule(static)
    for (q = 0; q < n; ++q) res[q] = res[q] * -1.0 + source[q];
    double r = absmax(n, res) / max_res0;
    free(res);
    return r;
}

/* grad_P + vel_corr (src/metric/metric_staggered.py:390-401,
   src/data/state.py:198-211, src/data/domain.py:397-402) */
void or_vel_corr(const or_grid* g, const double* DP, double scale, double* u,
                 double* v, double* w) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const double dxi = 1.0 / g->dx, dyi = 1.0 / g->dy, dzi = 1.0 / g->dz;
    int i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < nx; ++i) {
        const int im = WRAP(i - 1, nx);
        for (int j = 0; j < ny; ++j) {
            const int jm = WRAP(j - 1, ny);
            for (int k = 0; k < nz; ++k) {
                const int km = WRAP(k - 1, nz);
                const double c = DP[IDX(i, j, k)];
                const double gx = (c - DP[IDX(im, j, k)]) * dxi;
                const double gy = (c - DP[IDX(i, jm, k)]) * dyi;
                const double gz = (c - DP[IDX(i, j, km)]) * dzi;
                u[IDX(i, j, k)] = fma(-scale, gx, u[IDX(i, j, k)]);
                v[IDX(i, j, k)] = fma(-scale, gy, v[IDX(i, j, k)]);
                w[IDX(i, j, k)] = fma(-scale, gz, w[IDX(i, j, k)]);
            }
        }
    }
}

/* ------------------------------------------------------------------------ *
 * Domain.forwardStep with SFS off or 'tensor' (src/data/domain.py:342-367) and
 * velCorr (:373-402).  solver: 0 = bicgstab, 1 = Jacobi (n_it = max_it).
 * Returns the solver's max residual; *iters gets the BiCGStab iteration count.
 * ------------------------------------------------------------------------ */
double or_forward_step(const or_grid* g, double* u, double* v, double* w,
                       double* p, double* DP, const double* visc, double mu,
                       double rho, const double* sfs, double dt, int rk4,
                       int solver, double min_res, int max_it, int* iters) {
    const size_t n = ncell(g);
    if (rk4) or_rk4_step(g, u, v, w, visc, mu, rho, sfs, dt);
    else or_euler_step(g, u, v, w, visc, mu, rho, sfs, dt);
    double* src = (double*)malloc(sizeof(double) * n);
    or_div_vel(g, u, v, w, src);
    double r;
    int st = 0;
    if (solver == 0) {
        r = or_bicgstab(g, rho, dt, min_res, max_it, DP, p, src, iters, &st);
    } else {
        r = or_jacobi(g, rho, dt, max_it, DP, p, src);
        if (iters) *iters = max_it;
    }
    or_vel_corr(g, DP, dt / rho, u, v, w);
    free(src);
    return r;
}

/* Per-step statistics of PyFlow.run (src/core/PyFlow.py:379-395):
   out = {max|u|, max|v|, max|w|, TKE, max|div u|} */
void or_stats(const or_grid* g, const double* u, const double* v,
              const double* w, double* out) {
    const size_t n = ncell(g);
    const int nx = g->nx;
    const size_t plane = (size_t)g->ny * g->nz;
    out[0] = absmax(n, u);
    out[1] = absmax(n, v);
    out[2] = absmax(n, w);
    double* part = (double*)malloc(sizeof(double) * nx);
    int i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < nx; ++i) {
        double s = 0.0;
        for (size_t q = i * plane; q < (i + 1) * plane; ++q)
            s += (u[q] * u[q] + v[q] * v[q]) + w[q] * w[q];
        part[i] = s;
    }
    double s = 0.0;
    for (i = 0; i < nx; ++i) s += part[i];
    free(part);
    out[3] = s / (double)n * 0.5;
    double* d = (double*)malloc(sizeof(double) * n);
    or_div_vel(g, u, v, w, d);
    out[4] = absmax(n, d);
    free(d);
}
