// pf_api.cu -- extern "C" entry points of libpyflow_b200.so (include/pyflow_b200.h).
//
// Argument checking and workspace sizing live here; the kernels are in
// pf_rhs.cu and pf_poisson.cu.  No entry point allocates device memory and no
// C++ exception crosses the ABI.
#include <algorithm>
#include <cstdint>

#include "pf_common.cuh"
#include "pf_kernels.cuh"

using namespace pf;

namespace {

bool grid_ok(const pf_grid* g) {
    // stencils reach two cells back (edge viscosity one cell below the flux);
    // the periodic wrap handles one period, so every extent must be >= 2
    return g && g->nx >= 2 && g->ny >= 2 && g->nz >= 2 && g->dx > 0 && g->dy > 0 && g->dz > 0 &&
           (long long)g->nx * g->ny * g->nz < (1LL << 40);
}

bool prec_ok(int p) { return p == PF_FP64 || p == PF_MIXED || p == PF_MIXED_MG; }

// prec with the optional PF_WARM_START flag of the solving entry points
bool prec_flags_ok(int p) { return prec_ok(p & 0xFF) && (p & ~0xFF & ~PF_WARM_START) == 0; }

cudaStream_t S(void* s) { return (cudaStream_t)s; }

int cuda_rc(cudaError_t e) { return e == cudaSuccess ? PF_OK : PF_ERR_CUDA; }

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

extern "C" {

int pf_version(void) { return 100; }

const char* pf_status_string(int status) {
    switch (status) {
        case PF_OK: return "ok";
        case PF_ERR_BAD_ARG: return "bad argument";
        case PF_ERR_CUDA: return "CUDA error";
        case PF_BREAKDOWN: return "BiCGStab breakdown";
        case PF_MAXIT: return "iteration limit reached";
        case PF_NONFINITE: return "non-finite residual";
        case PF_STAGNATION: return "refinement stagnated";
        case PF_ERR_TOO_LARGE: return "grid exceeds the no-allocation scratch limit (64^3 cells)";
        default: return "unknown status";
    }
}

size_t pf_workspace_bytes(const pf_grid* g, int prec) {
    if (!grid_ok(g) || !prec_ok(prec)) return 0;
    const size_t n = (size_t)g->nx * g->ny * g->nz;
    // the forward step needs the predictor scratch and the Poisson scratch at
    // different times, plus one FP64 field for the divergence
    size_t b = std::max(predictor_ws_bytes(g, prec), poisson_ws_bytes(g, prec));
    b = std::max(b, stats_ws_bytes(g));
    return align256(b) + align256(n * sizeof(double));
}

int pf_rhs_ns(const pf_grid* g, int prec, const void* u, const void* v,
              const void* w, const void* visc, double mu, double rho,
              const void* sfs, void* ru, void* rv, void* rw, void* stream) {
    if (!grid_ok(g) || !prec_ok(prec) || !u || !v || !w || !ru || !rv || !rw || !(rho != 0.0))
        return PF_ERR_BAD_ARG;
    return cuda_rc(launch_rhs(g, prec, u, v, w, visc, mu, rho, sfs, ru, rv, rw, S(stream)));
}

int pf_div_vel(const pf_grid* g, const double* u, const double* v,
               const double* w, double* div, void* stream) {
    if (!grid_ok(g) || !u || !v || !w || !div) return PF_ERR_BAD_ARG;
    return cuda_rc(launch_div(g, u, v, w, div, S(stream)));
}

int pf_laplace_apply(const pf_grid* g, const double* A, double* B, void* stream) {
    if (!grid_ok(g) || !A || !B) return PF_ERR_BAD_ARG;
    return cuda_rc(launch_laplace(g, A, B, S(stream)));
}

int pf_predictor_step(const pf_grid* g, int prec, int rk4, double* u,
                      double* v, double* w, const void* visc, double mu,
                      double rho, const void* sfs, double dt, void* ws,
                      size_t ws_bytes, void* stream) {
    if (!grid_ok(g) || !prec_ok(prec) || !u || !v || !w || !(rho != 0.0)) return PF_ERR_BAD_ARG;
    if (!ws || ws_bytes < predictor_ws_bytes(g, prec)) return PF_ERR_BAD_ARG;
    // variable viscosity / SFS fields are given in the stage precision
    return cuda_rc(launch_predictor(g, prec, rk4, u, v, w, visc, mu, rho, sfs, dt, ws, S(stream)));
}

int pf_bicgstab_solve(const pf_grid* g, int prec, double rho, double dt,
                      double min_res, int max_it, const double* source,
                      double* DP, double* p, void* ws, size_t ws_bytes,
                      void* stream, pf_solve_info* info) {
    if (!grid_ok(g) || !prec_flags_ok(prec) || !source || !DP || !p || !(dt != 0.0))
        return PF_ERR_BAD_ARG;
    if (!ws || ws_bytes < poisson_ws_bytes(g, prec & 0xFF)) return PF_ERR_BAD_ARG;
    return bicgstab_solve(g, prec, rho, dt, min_res, max_it, source, DP, p, ws, S(stream), info);
}

int pf_jacobi_solve(const pf_grid* g, double rho, double dt, int n_it,
                    const double* source, double* pold, double* p, void* ws,
                    size_t ws_bytes, void* stream, double* max_res) {
    if (!grid_ok(g) || !source || !pold || !p || n_it < 0 || !(dt != 0.0)) return PF_ERR_BAD_ARG;
    if (!ws || ws_bytes < poisson_ws_bytes(g, PF_FP64)) return PF_ERR_BAD_ARG;
    return jacobi_solve(g, rho, dt, n_it, source, pold, p, ws, S(stream), max_res);
}

int pf_vel_corr(const pf_grid* g, const double* DP, double scale, double* u,
                double* v, double* w, void* stream) {
    if (!grid_ok(g) || !DP || !u || !v || !w) return PF_ERR_BAD_ARG;
    return cuda_rc(launch_vel_corr(g, DP, scale, u, v, w, S(stream)));
}

int pf_forward_step(const pf_grid* g, int prec, int rk4, int solver,
                    double* u, double* v, double* w, double* p, double* DP,
                    const void* visc, double mu, double rho,
                    const void* sfs, double dt, double min_res, int max_it,
                    void* ws, size_t ws_bytes, void* stream,
                    pf_solve_info* info) {
    if (!grid_ok(g) || !prec_flags_ok(prec) || !u || !v || !w || !p || !DP || !(rho != 0.0) ||
        !(dt != 0.0) || (solver != 0 && solver != 1))
        return PF_ERR_BAD_ARG;
    const int flags = prec & ~0xFF;
    prec &= 0xFF;
    if (!ws || ws_bytes < pf_workspace_bytes(g, prec)) return PF_ERR_BAD_ARG;
    const size_t n = (size_t)g->nx * g->ny * g->nz;
    double* div = (double*)ws;
    void* rest = (char*)ws + align256(n * sizeof(double));
    cudaStream_t s = S(stream);
    int rc = cuda_rc(launch_predictor(g, prec, rk4, u, v, w, visc, mu, rho, sfs, dt, rest, s));
    if (rc) return rc;
    rc = cuda_rc(launch_div(g, u, v, w, div, s));
    if (rc) return rc;
    pf_solve_info si{0.0, 0, 1, PF_OK};
    if (solver == 0) {
        rc = bicgstab_solve(g, prec | flags, rho, dt, min_res, max_it, div, DP, p, rest, s, &si);
    } else {
        // the Jacobi solver zeroes and overwrites p (src/solver/pressure.py:121)
        rc = jacobi_solve(g, rho, dt, max_it, div, DP, p, rest, s, &si.max_res);
        si.iterations = max_it;
    }
    if (rc) return rc;
    rc = cuda_rc(launch_vel_corr(g, DP, dt / rho, u, v, w, s));
    if (rc) return rc;
    if (info) *info = si;
    return PF_OK;
}

int pf_stats(const pf_grid* g, const double* u, const double* v,
             const double* w, double* out_dev, void* ws, size_t ws_bytes,
             void* stream) {
    if (!grid_ok(g) || !u || !v || !w || !out_dev) return PF_ERR_BAD_ARG;
    if (!ws || ws_bytes < stats_ws_bytes(g)) return PF_ERR_BAD_ARG;
    return cuda_rc(launch_stats(g, u, v, w, out_dev, ws, S(stream)));
}

int pf_flow_stats(const pf_grid* g, const double* u, const double* v,
                  const double* w, double nu, double* out_dev, void* ws,
                  size_t ws_bytes, void* stream) {
    if (!grid_ok(g) || !u || !v || !w || !out_dev || !(nu >= 0.0)) return PF_ERR_BAD_ARG;
    if (!ws || ws_bytes < stats_ws_bytes(g)) return PF_ERR_BAD_ARG;
    return cuda_rc(launch_flow_stats(g, u, v, w, nu, out_dev, ws, S(stream)));
}

size_t pf_step_plan_workspace_bytes(const pf_grid* g, int prec) {
    if (!grid_ok(g) || !prec_ok(prec)) return 0;
    return step_plan_ws_bytes(g, prec);
}

int pf_step_plan_create(const pf_grid* g, int prec, int rk4, double* u, double* v,
                        double* w, double* p, double* DP, double mu, double rho,
                        double dt, double min_res, int max_it, void* ws,
                        size_t ws_bytes, double* stats, pf_step_plan** plan) {
    if (!grid_ok(g) || !prec_ok(prec) || !u || !v || !w || !p || !DP || !stats || !plan ||
        !(rho != 0.0) || !(dt != 0.0) || max_it < 1)
        return PF_ERR_BAD_ARG;
    if (!ws || ws_bytes < step_plan_ws_bytes(g, prec) || ((uintptr_t)ws & 255) != 0)
        return PF_ERR_BAD_ARG;
    void* h = nullptr;
    const int rc = step_plan_create(g, prec, rk4, u, v, w, p, DP, mu, rho, dt, min_res, max_it,
                                    nullptr, ws, stats, &h);
    if (rc == PF_OK) *plan = (pf_step_plan*)h;
    return rc;
}

static bool closure_kind_ok(int kind) {
    return kind == PF_CLOSURE_SMAGORINSKY || kind == PF_CLOSURE_GRADIENT || kind == PF_CLOSURE_MLP;
}

size_t pf_step_closure_bytes(const pf_grid* g, int prec, int kind) {
    if (!grid_ok(g) || !prec_ok(prec) || !closure_kind_ok(kind)) return 0;
    return closure_layout(g, prec, kind).bytes;
}

size_t pf_step_closure_stage_offset(const pf_grid* g, int prec, int kind) {
    if (!grid_ok(g) || !prec_ok(prec) || !closure_kind_ok(kind)) return 0;
    return closure_layout(g, prec, kind).stage;
}

int pf_step_plan_create_sfs(const pf_grid* g, int prec, int rk4, double* u, double* v,
                            double* w, double* p, double* DP, double mu, double rho,
                            double dt, double min_res, int max_it, const pf_step_closure* c,
                            void* ws, size_t ws_bytes, double* stats, pf_step_plan** plan) {
    if (!grid_ok(g) || !prec_ok(prec) || !u || !v || !w || !p || !DP || !stats || !plan ||
        !(rho != 0.0) || !(dt != 0.0) || max_it < 1 || !c || !closure_kind_ok(c->kind) ||
        !c->field || ((uintptr_t)c->field & 255) ||
        c->field_bytes < closure_layout(g, prec, c->kind).bytes)
        return PF_ERR_BAD_ARG;
    if (c->kind == PF_CLOSURE_MLP &&
        (!c->wpack || ((uintptr_t)c->wpack & 15) || !c->err || g->nx < 2 || g->ny < 2 || g->nz < 2))
        return PF_ERR_BAD_ARG;
    if (!ws || ws_bytes < step_plan_ws_bytes(g, prec) || ((uintptr_t)ws & 255) != 0)
        return PF_ERR_BAD_ARG;
    void* h = nullptr;
    const int rc = step_plan_create(g, prec, rk4, u, v, w, p, DP, mu, rho, dt, min_res, max_it,
                                    c, ws, stats, &h);
    if (rc == PF_OK) *plan = (pf_step_plan*)h;
    return rc;
}

size_t pf_batch_table_bytes(int count) {
    if (count < 1 || count > kMaxBatch) return 0;
    return grouped_predictor_table_bytes(count);
}

int pf_batch_plan_create(int prec, int rk4, const pf_batch_member* m, int count, void* table,
                         size_t table_bytes, pf_step_plan** plan) {
    if (!prec_ok(prec) || !m || count < 1 || count > kMaxBatch || !plan || !table ||
        ((uintptr_t)table & 255) || table_bytes < grouped_predictor_table_bytes(count))
        return PF_ERR_BAD_ARG;
    for (int r = 0; r < count; ++r) {
        const pf_batch_member& b = m[r];
        if (!grid_ok(&b.grid) || !b.u || !b.v || !b.w || !b.p || !b.DP || !b.stats || !b.ws ||
            ((uintptr_t)b.ws & 255) || b.ws_bytes < step_plan_ws_bytes(&b.grid, prec) ||
            !(b.dt != 0.0) || !(b.rho != 0.0) || b.max_it < 1)
            return PF_ERR_BAD_ARG;
    }
    void* p = nullptr;
    const int rc = batch_plan_create(prec, rk4 ? 1 : 0, m, count, table, &p);
    if (rc == PF_OK) *plan = (pf_step_plan*)p;
    return rc;
}

int pf_step_plan_launch(pf_step_plan* plan, int nsteps, void* stream) {
    if (!plan || nsteps < 0) return PF_ERR_BAD_ARG;
    return step_plan_launch(plan, nsteps, S(stream));
}

int pf_step_plan_destroy(pf_step_plan* plan) { return step_plan_destroy(plan); }

}  // extern "C"
