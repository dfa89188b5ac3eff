// pf_kernels.cuh -- host-side launchers shared between the library's .cu files.
#pragma once
#include <cuda_runtime.h>

#include "../../include/pyflow_b200.h"

namespace pf {

// Unique id of the CUDA context current on this thread (0 when none is).
int context_id(unsigned long long* id);
// Runs setup() once per (key, current CUDA context): kernel attributes and
// symbol addresses belong to a context, not to a device (pf_ctx.cu).
cudaError_t once_per_context(const void* key, cudaError_t (*setup)());


cudaError_t launch_rhs(const pf_grid* g, int prec, const void* u,
                       const void* v, const void* w, const void* visc,
                       double mu, double rho, const void* sfs, void* ru,
                       void* rv, void* rw, cudaStream_t s);

size_t predictor_ws_bytes(const pf_grid* g, int prec);
// One-time per-device kernel attributes of the predictor (call before any
// stream capture that contains predictor launches).
cudaError_t predictor_prepare(int prec);
cudaError_t launch_predictor(const pf_grid* g, int prec, int rk4, double* u,
                             double* v, double* w, const void* visc,
                             double mu, double rho, const void* sfs,
                             double dt, void* ws, cudaStream_t s);

// One request of a grouped predictor: its grid, state, constants and the
// stage-buffer region of its workspace (predictor_ws_bytes of it).
struct GroupMember {
    pf_grid grid;
    double *u, *v, *w;
    double mu, rho, dt;
    void* R;
};
constexpr int kMaxBatch = 64;  // requests of one grouped launch
// Kernel attributes of the grouped stage kernels (before any capture).
int grouped_predictor_prepare(int prec);
// Device bytes of the grouped stages' job tables for `count` members.
size_t grouped_predictor_table_bytes(int count);
// Writes the job tables into `table` (synchronous on s, clears the error
// flag in its first word) and prepares the kernels; before any capture of
// launch_grouped_predictor with the same members and table.
int grouped_predictor_tables(int prec, int rk4, const GroupMember* m, int count,
                             void* table, cudaStream_t s);
// The predictor of every member, one launch per RK4 stage (constant
// viscosity, no SFS stresses); same results as launch_predictor per member.
cudaError_t launch_grouped_predictor(int prec, int rk4, const GroupMember* m, int count,
                                     void* table, cudaStream_t s);

size_t poisson_ws_bytes(const pf_grid* g, int prec);
int bicgstab_solve(const pf_grid* g, int prec, double rho, double dt,
                   double min_res, int max_it, const double* source,
                   double* DP, double* p, void* ws, cudaStream_t s,
                   pf_solve_info* info);
int jacobi_solve(const pf_grid* g, double rho, double dt, int n_it,
                 const double* source, double* pold, double* p, void* ws,
                 cudaStream_t s, double* max_res);

cudaError_t launch_div(const pf_grid* g, const double* u, const double* v,
                       const double* w, double* div, cudaStream_t s);
cudaError_t launch_laplace(const pf_grid* g, const double* A, double* B,
                           cudaStream_t s);
cudaError_t launch_vel_corr(const pf_grid* g, const double* DP, double scale,
                            double* u, double* v, double* w, cudaStream_t s);
size_t stats_ws_bytes(const pf_grid* g);
cudaError_t launch_stats(const pf_grid* g, const double* u, const double* v,
                         const double* w, double* out, void* ws,
                         cudaStream_t s);
cudaError_t launch_flow_stats(const pf_grid* g, const double* u, const double* v,
                              const double* w, double nu, double* out, void* ws,
                              cudaStream_t s);

size_t step_plan_ws_bytes(const pf_grid* g, int prec);
// SGS closure fields (pf_sgs_closure models 0-2) as FP64 (f32 false) or
// float; model 0 adds `add` to coef |S|
cudaError_t launch_sgs(const pf_grid* g, int model, const double* u,
                       const double* v, const double* w, double coef,
                       double add, void* out, bool f32, cudaStream_t s);

// the MLP closure's input and output scales (pf_mlp_scales); ws of
// mlp_scales_ws_bytes(), 256-byte aligned
size_t mlp_scales_ws_bytes();
cudaError_t launch_mlp_scales(const pf_grid* g, const double* u, const double* v,
                              const double* w, double delta2, float* scales, void* ws,
                              cudaStream_t s);
cudaError_t launch_to_float(const double* in, float* out, long long n, cudaStream_t s);
cudaError_t launch_mlp(const pf_grid* g, const double* u, const double* v,
                       const double* w, const void* wpack, const float* scales,
                       double* out, int* err, cudaStream_t s);
cudaError_t mlp_prepare();

// byte layout of a plan's closure buffer (pf_step_closure.field)
struct ClosureLayout {
    size_t scratch;    // MLP: scales (2 floats) at 0, the reduction scratch at 256
    size_t f64;        // MLP: the six FP64 stresses
    size_t stage;      // the field the stages read (stage type)
    size_t bytes;      // total
};
ClosureLayout closure_layout(const pf_grid* g, int prec, int kind);

// c: NULL for a plan without SFS closure
int step_plan_create(const pf_grid* g, int prec, int rk4, double* u, double* v,
                     double* w, double* p, double* DP, double mu, double rho,
                     double dt, double min_res, int max_it, const pf_step_closure* c,
                     void* ws, double* stats, void** out);
int step_plan_launch(void* plan, int nsteps, cudaStream_t s);
int batch_plan_create(int prec, int rk4, const pf_batch_member* m, int count, void* table,
                      void** out);
int step_plan_destroy(void* plan);

}  // namespace pf
