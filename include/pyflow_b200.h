/*
 * pyflow_b200.h -- C ABI of the B200-native PyFlow time-advance hot path.
 *
 * All field pointers are DEVICE pointers to ghost-free [nx][ny][nz] arrays
 * (z contiguous): the interior of the reference's state_P.var
 * (src/data/state.py:142-146).  Periodic boundaries are index wraps inside the
 * kernels (the reference's decomp.communicate_border, src/library/parallel.py:301-414).
 *
 * Conventions
 *  - Every entry point is asynchronous on the given stream unless stated.
 *  - The library never allocates device memory: scratch space is a caller
 *    buffer of at least pf_workspace_bytes() bytes, 256-byte aligned.
 *  - Return value: PF_OK or a pf_status code; no C++ exception crosses the ABI.
 *  - prec: PF_FP64 computes every operator in FP64 in the reference's
 *    operation order; PF_MIXED keeps the velocity/pressure state in FP64, runs
 *    fluxes, RK4 stages and the Poisson matvec in FP32, and keeps FP64 for the
 *    Poisson residual recomputation, the BiCGStab inner products, the
 *    iterative-refinement outer loop and all global sums.  PF_MIXED_MG is
 *    PF_MIXED whose FP32 refinement passes run BiCGStab right-preconditioned
 *    by a geometric multigrid V-cycle (no counterpart in the reference, whose
 *    BiCGStab is unpreconditioned); it needs the grid to halve in every
 *    dimension (while all are even) down to at most 4096 cells, and otherwise
 *    runs the PF_MIXED passes.  Both mixed forms converge to the same FP64
 *    tolerance.
 */
#ifndef PYFLOW_B200_H
#define PYFLOW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pf_grid {
    int nx, ny, nz;     /* interior cells */
    double dx, dy, dz;  /* uniform spacings (geometry.uniform, src/geometry/geometry.py:97-99) */
} pf_grid;

enum pf_status {
    PF_OK = 0,
    PF_ERR_BAD_ARG = 1,     /* null pointer, bad size, workspace too small */
    PF_ERR_CUDA = 2,        /* a CUDA runtime call failed */
    PF_BREAKDOWN = 3,       /* BiCGStab gamma == 0 or (t,t) == 0 (src/solver/pressure.py:247-248,266-267) */
    PF_MAXIT = 4,           /* iteration limit reached before the tolerance */
    PF_NONFINITE = 5,       /* NaN/Inf seen in a residual */
    PF_STAGNATION = 6,      /* mixed-precision refinement stopped improving */
    PF_ERR_TOO_LARGE = 7    /* grid exceeds the fixed scratch of pf_bicgstab_solve_noalloc */
};

enum pf_prec { PF_FP64 = 0, PF_MIXED = 1, PF_MIXED_MG = 2 };

/* Flag OR-ed into prec of pf_bicgstab_solve / pf_forward_step: in the mixed
 * forms the solve starts from the DP it is given (for example the previous
 * step's) instead of zero, as the mixed step plans do; the stop criterion is
 * unchanged (max|b - A DP| <= min_res max|b|).  Ignored for PF_FP64, which
 * always starts from DP = 0 like the reference. */
enum pf_flags { PF_WARM_START = 0x100 };

/* Result of a Poisson solve (host struct, filled by the synchronous calls). */
typedef struct pf_solve_info {
    double max_res;      /* max|r| / max|r0|, the reference's return value */
    int iterations;      /* BiCGStab iterations (inner iterations for the mixed forms) */
    int outer;           /* refinement passes (mixed forms), 1 for PF_FP64 */
    int status;          /* pf_status */
} pf_solve_info;

int pf_version(void);
const char* pf_status_string(int status);

/* Scratch bytes needed by pf_rk4_step / pf_bicgstab_solve / pf_forward_step
 * for this grid and precision. */
size_t pf_workspace_bytes(const pf_grid* g, int prec);

/* rhs_NavierStokes.evaluate (src/solver/velocity.py:221-355): viscous +
 * convective staggered fluxes.  visc: NULL for the constant mu
 * (src/data/domain.py:130-131) or a cell-centred viscosity field; sfs: NULL or
 * six consecutive cell-centred fields FXX,FYY,FZZ,FXY,FXZ,FYZ of a 'tensor'
 * SFS model (src/solver/velocity.py:262-267,286-291,310-315).  Fields are
 * double for PF_FP64, float for the mixed forms (u,v,w,visc,sfs,rhs all
 * float). */
int pf_rhs_ns(const pf_grid* g, int prec, const void* u, const void* v,
              const void* w, const void* visc, double mu, double rho,
              const void* sfs, void* ru, void* rv, void* rw, void* stream);

/* metric_uniform.div_vel (src/metric/metric_staggered.py:438-453), FP64. */
int pf_div_vel(const pf_grid* g, const double* u, const double* v,
               const double* w, double* div, void* stream);

/* Pressure_Base.applyOperator (src/solver/pressure.py:54-84): B = (-vol L) A,
 * FP64. */
int pf_laplace_apply(const pf_grid* g, const double* A, double* B,
                     void* stream);

/* RK4.step (src/solver/advancer.py:75-113) including the reference's stage-4
 * state u + dt/2 k3; u, v, w (FP64) updated in place.  Euler.step
 * (src/solver/advancer.py:49-57) when rk4 == 0.  visc / sfs (NULL or as for
 * pf_rhs_ns) are in the stage type: double for PF_FP64, float for the mixed
 * forms. */
int pf_predictor_step(const pf_grid* g, int prec, int rk4, double* u,
                      double* v, double* w, const void* visc, double mu,
                      double rho, const void* sfs, double dt, void* ws,
                      size_t ws_bytes, void* stream);

/* solver_bicgstab.solve (src/solver/pressure.py:196-297) on
 * (-vol L) DP = -vol rho/dt source, DP0 = 0, stop on max|r|/max|r0| <= min_res
 * or iterations >= max_it; then p += DP.  source (FP64, the divergence) is not
 * modified.  Synchronous: returns after the solve with *info filled. */
int pf_bicgstab_solve(const pf_grid* g, int prec, double rho, double dt,
                      double min_res, int max_it, const double* source,
                      double* DP, double* p, void* ws, size_t ws_bytes,
                      void* stream, pf_solve_info* info);

/* solver_jacobi.solve (src/solver/pressure.py:115-161): n_it sweeps of
 * p <- (sum of neighbours - dx^2 rho/dt source)/6 from p = 0; p holds the last
 * iterate and pold the one before it; *max_res gets the reference's residual
 * ratio.  FP64, synchronous. */
int pf_jacobi_solve(const pf_grid* g, double rho, double dt, int n_it,
                    const double* source, double* pold, double* p,
                    void* ws, size_t ws_bytes, void* stream, double* max_res);

/* grad_P + vel_corr (src/metric/metric_staggered.py:390-401,
 * src/data/state.py:198-211): u_d -= scale * backward difference of DP. */
int pf_vel_corr(const pf_grid* g, const double* DP, double scale, double* u,
                double* v, double* w, void* stream);

/* Domain.forwardStep with the SFS model off, 'eddyVisc' (visc = mu + mu_t)
 * or 'tensor' (src/data/domain.py:342-402): predictor, divergence, Poisson
 * solve (solver 0 = BiCGStab, 1 = Jacobi with max_it sweeps), projection.
 * visc / sfs as for pf_predictor_step (stage type).  Synchronous; *info gets
 * the solve result. */
int pf_forward_step(const pf_grid* g, int prec, int rk4, int solver,
                    double* u, double* v, double* w, double* p, double* DP,
                    const void* visc, double mu, double rho,
                    const void* sfs, double dt, double min_res, int max_it,
                    void* ws, size_t ws_bytes, void* stream,
                    pf_solve_info* info);

/* Per-step monitor statistics (src/core/PyFlow.py:379-395), FP64:
 * out_dev[0..4] = max|u|, max|v|, max|w|, TKE, max|div u| written to DEVICE
 * memory (5 doubles) asynchronously. */
int pf_stats(const pf_grid* g, const double* u, const double* v,
             const double* w, double* out_dev, void* ws, size_t ws_bytes,
             void* stream);

/* pf_stats plus the dissipation rate: out_dev[0..5] = max|u|, max|v|, max|w|,
 * TKE, max|div u| (as pf_stats, src/core/PyFlow.py:379-395) and
 * eps = 2 nu <S_ij S_ij>, the mean over cells of the cell-centred strain rate
 * of metric_uniform.grad_vel_center (src/metric/metric_staggered.py:215-268)
 * with periodic wrap.  The reference computes no dissipation; this is the
 * quantity its monitor would need for the energy budget dKE/dt = -eps.
 * FP64, 6 doubles of DEVICE memory, asynchronous; ws as for pf_stats. */
int pf_flow_stats(const pf_grid* g, const double* u, const double* v,
                  const double* w, double nu, double* out_dev, void* ws,
                  size_t ws_bytes, void* stream);

/* Cell-centred SGS closures (FP64), computed from the cell-centred velocity
 * gradients of metric_uniform.grad_vel_center
 * (src/metric/metric_staggered.py:215-268) with periodic wrap:
 *   model 0: Smagorinsky eddy viscosity out[0] = coef * |S|
 *            (stress_constCs.eddyVisc, src/sfsmodel/sfsmodel_smagorinsky.py:65-88;
 *            coef = rho (Cs Delta)^2);
 *   model 1: gradient-model stresses out[0..5] = coef du_i/dx_k du_j/dx_k for
 *            ij = xx, yy, zz, xy, xz, yz (residual_stress.update,
 *            src/sfsmodel/sfsmodel_gradient.py:70-148; coef = dx^2/12);
 *   model 2: the nine gradients out[0..8] = du/dx, du/dy, du/dz, dv/dx, ...
 * out holds 1, 6 or 9 consecutive fields. */
int pf_sgs_closure(const pf_grid* g, int model, const double* u,
                   const double* v, const double* w, double coef, double* out,
                   void* stream);

/* SGS MLP closure on the tensor cores (tcgen05, BF16 operands, FP32
 * accumulation in TMEM): out[c*n + cell], c = 0..5 (FXX, FYY, FZZ, FXY, FXZ,
 * FYZ, FP64) = scales[1] * MLP(scales[0] * grad u), where grad u are the nine
 * cell-centred gradients of pf_sgs_closure model 2 and MLP is
 * 9 -> 128 (tanh) -> 128 (tanh) -> 6.  The stresses go to the 'tensor' SFS
 * slot (src/solver/velocity.py:262-267,286-291,310-315); the model itself has
 * no reference code (the reference's ML closure, src/sfsmodel/sfsmodel_ML.py,
 * is a different 'source'-type network).  wpack: device buffer of
 * pf_mlp_pack_bytes() bytes, 16-byte aligned, holding W1 (128x16), W2
 * (128x128), W3 (16x128) as BF16 in the K-major no-swizzle UMMA layout
 * followed by b1[128], b2[128], b3[16] as float (see sfsmodel_mlp.pack);
 * scales: 2 device floats; err: device int set to 1 if a tensor-core wait
 * timed out. */
size_t pf_mlp_pack_bytes(void);
/* The MLP closure's scales from the nine cell-centred gradients:
 * g2 = their mean square (FP64, fixed summation order), scales[0] =
 * 1/sqrt(g2), scales[1] = delta2 g2, each rounded once to float (device).
 * ws: pf_mlp_scales_workspace_bytes() bytes, 256-byte aligned. */
size_t pf_mlp_scales_workspace_bytes(void);
int pf_mlp_scales(const pf_grid* g, const double* u, const double* v,
                  const double* w, double delta2, float* scales, void* ws,
                  size_t ws_bytes, void* stream);
int pf_mlp_closure(const pf_grid* g, const double* u, const double* v,
                   const double* w, const void* wpack, const float* scales,
                   double* out, int* err, void* stream);

/* The reference's 'source'-type ML closure on the tensor cores: replaces
 * residual_stress.update (src/sfsmodel/sfsmodel_ML.py:354-401; features
 * :407-460, stencil input :464-510, network NeuralNetworkModel2 :77-116,
 * closure terms :513-590) and the face interpolation the RHS subtracts
 * (src/solver/velocity.py:374-383).  Inputs: the staggered FP64 velocity;
 * the spacing used in every direction is g->dx, as in the reference.
 * Outputs (FP64, 3n each): G = GX, GY, GZ at cell centres and S = the face
 * sources 0.5 (G[i] + G[i-1]) along x, y, z.  The network runs as three
 * TF32 MMAs per product (hi/lo split of both operands, FP32 accumulation in
 * TMEM), close to the reference's FP32.
 *   pf_mlsrc_pack: params = 13 device float pointers, the torch layouts of
 *     fc1.weight (200x273), fc1.bias, fcG.weight, fcG.bias, fcG2.weight,
 *     fcG2.bias, fc2.weight (200x200), fc2.bias, fc3.weight, fc3.bias,
 *     fc4.weight (18x200), fc4.bias, then the 21 feature normalisation
 *     constants; pack: device buffer of pf_mlsrc_pack_bytes(), 16-byte
 *     aligned.  Repack after every parameter update.
 *   pf_mlsrc_closure: ws: device buffer of pf_mlsrc_workspace_bytes(g)
 *     (about 5 KB per cell), 256-byte aligned; err: device int set to 1 if a
 *     tensor-core wait timed out.  Grids need at least 5 cells per axis. */
size_t pf_mlsrc_pack_bytes(void);
size_t pf_mlsrc_workspace_bytes(const pf_grid* g);
int pf_mlsrc_pack(const float* const* params, void* pack, void* stream);
int pf_mlsrc_closure(const pf_grid* g, const double* u, const double* v,
                     const double* w, const void* pack, double* G, double* S,
                     void* ws, size_t ws_bytes, int* err, void* stream);

/* Exact discrete adjoint of the constant-viscosity RHS: out = J(u)^T mu where
 * J is the Jacobian of pf_rhs_ns (rhs_NavierStokes.evaluate,
 * src/solver/velocity.py:221-355) at state (u, v, w).  Replaces the
 * reference's adjoint RHS (rhs_adjPredictor.evaluate, src/solver/adjoint.py:94-227,
 * adj_conv_*, src/metric/metric_staggered.py:537-799).  FP64. */
int pf_rhs_adjoint(const pf_grid* g, const double* u, const double* v,
                   const double* w, const double* mu_u, const double* mu_v,
                   const double* mu_w, double mu, double rho, double* out_u,
                   double* out_v, double* out_w, void* stream);

/* Adjoint of the 'tensor' SFS stresses in the RHS
 * (src/solver/velocity.py:262-267,286-291,310-315): out[0..5] += weight *
 * dL/d(FXX, FYY, FZZ, FXY, FXZ, FYZ) for the RHS adjoint mu.  FP64. */
int pf_sfs_adjoint(const pf_grid* g, const double* mu_u, const double* mu_v,
                   const double* mu_w, double weight, double* out, void* stream);

/* No counterpart in the reference: the pf_bicgstab_solve solve (FP64) for
 * callers that cannot allocate device memory or pass a workspace (for example
 * a plugin whose host application owns the whole device-memory budget, or a
 * loop that must not allocate after start-up).  Scratch is a fixed 16.25 MiB
 * array inside the library (held by every GPU that loads it); grids above
 * 64^3 = 262144 cells return PF_ERR_TOO_LARGE.  The array's device address
 * is looked up once per CUDA context (keyed by the context's unique id), at
 * the first call in that context, so make that call before any stream
 * capture.
 * All calls share the array: calls that overlap on the GPU race.  Allocates
 * nothing.  Synchronous, like pf_bicgstab_solve. */
int pf_bicgstab_solve_noalloc(const pf_grid* g, double rho, double dt,
                              double min_res, int max_it, const double* source,
                              double* DP, double* p, void* stream,
                              pf_solve_info* info);

/* A whole Domain.forwardStep (src/data/domain.py:342-402; constant viscosity,
 * no SFS model) captured once as a CUDA graph bound to the given fields and
 * workspace: predictor, divergence, Poisson solve with device-side
 * convergence loops (conditional WHILE nodes), p += DP, projection and the
 * monitor statistics (src/core/PyFlow.py:379-395).  Each launch advances one
 * step with no host synchronisation; stats (device, 10 doubles) receives
 * max|u|, max|v|, max|w|, TKE, max|div u|, max_res, iterations, status after
 * every step, and accumulates the iterations and the step count in
 * stats[8], stats[9].  The workspace (pf_step_plan_workspace_bytes, 256-byte aligned)
 * belongs to the plan.  Plans of different fields may run concurrently on
 * different streams.  PF_FP64 solves from DP = 0 like the reference
 * (src/solver/pressure.py:202); the mixed forms start each solve from the DP
 * that the previous step left (so DP must hold finite values -- zeros --
 * before the first launch) and stop on the reference's criterion applied to
 * the true residual, max|b - A DP| <= min_res max|b|. */
typedef struct pf_step_plan pf_step_plan;
size_t pf_step_plan_workspace_bytes(const pf_grid* g, int prec);
int pf_step_plan_create(const pf_grid* g, int prec, int rk4, double* u,
                        double* v, double* w, double* p, double* DP, double mu,
                        double rho, double dt, double min_res, int max_it,
                        void* ws, size_t ws_bytes, double* stats,
                        pf_step_plan** plan);
int pf_step_plan_launch(pf_step_plan* plan, int nsteps, void* stream);
int pf_step_plan_destroy(pf_step_plan* plan);

/* pf_step_plan_create for LES: an SFS closure runs inside the graph at the
 * start of every step, as the SFS pre-step of Domain.forwardStep
 * (src/data/domain.py:347-355), and the RK4 stages read its field:
 *   PF_CLOSURE_SMAGORINSKY: the viscosity field mu + coef |S|
 *     (stress_constCs.eddyVisc, src/sfsmodel/sfsmodel_smagorinsky.py:65-88,
 *     added to the molecular viscosity as src/data/domain.py:352 does;
 *     coef = rho (Cs Delta)^2);
 *   PF_CLOSURE_GRADIENT: the six 'tensor' stresses coef du_i/dx_k du_j/dx_k
 *     (src/sfsmodel/sfsmodel_gradient.py:70-148; coef = dx^2/12);
 *   PF_CLOSURE_MLP: the tensor-core MLP's six stresses (pf_mlp_scales with
 *     delta2 = coef = Delta^2, then pf_mlp_closure with wpack and err).
 * field: device buffer of pf_step_closure_bytes(g, prec, kind) bytes,
 * 256-byte aligned, owned by the plan.  The field the stages read is in
 * their type (double for PF_FP64, float for the mixed forms; the stresses as
 * consecutive fields FXX,FYY,FZZ,FXY,FXZ,FYZ) at byte
 * pf_step_closure_stage_offset(g, prec, kind) of it; for the MLP the buffer
 * also holds the scales (2 floats at byte 0) and the six FP64 stresses.
 * Every step computes what the host-driven closure (pf_sgs_closure; or
 * pf_mlp_scales and pf_mlp_closure), the FP64 addition of mu, the conversion
 * to the stage type and pf_forward_step with that visc or sfs compute, bit
 * for bit (the mixed forms from a warm start, as pf_step_plan_create). */
enum { PF_CLOSURE_SMAGORINSKY = 1, PF_CLOSURE_GRADIENT = 2, PF_CLOSURE_MLP = 3 };
typedef struct pf_step_closure {
    int kind;            /* PF_CLOSURE_* */
    double coef;
    const void* wpack;   /* PF_CLOSURE_MLP: as for pf_mlp_closure */
    int* err;            /* PF_CLOSURE_MLP: as for pf_mlp_closure */
    void* field;
    size_t field_bytes;
} pf_step_closure;
size_t pf_step_closure_bytes(const pf_grid* g, int prec, int kind);
size_t pf_step_closure_stage_offset(const pf_grid* g, int prec, int kind);
int pf_step_plan_create_sfs(const pf_grid* g, int prec, int rk4, double* u,
                            double* v, double* w, double* p, double* DP,
                            double mu, double rho, double dt, double min_res,
                            int max_it, const pf_step_closure* closure, void* ws,
                            size_t ws_bytes, double* stats, pf_step_plan** plan);

/* x-slab decomposition (replaces decomp and communicate_border,
 * src/library/parallel.py:118-414, and comms.parallel_sum / parallel_max,
 * :60-94, for a periodic box split along x over ranks).  A rank's fields are
 * a LOCAL EXTENDED grid g: g->nx = halo + interior planes + halo, ny and nz
 * the global ones, z fastest; plane `halo` is the first interior plane.  The
 * caller moves ghost planes between neighbours (planes are contiguous) and
 * gathers every rank's 2-double `send` buffer, in rank order, into `recv`
 * (world x 2 doubles, device) -- the only communication of the solve.
 * Kernels without reductions (pf_predictor_step, pf_div_vel, pf_vel_corr)
 * run unchanged on g: with halo >= 4 ghost planes exchanged, a whole RK4
 * predictor is exact on the interior.
 *
 * The pressure solve is solver_bicgstab.solve (src/solver/pressure.py:196-297)
 * in FP64 with the reference's three reductions per iteration; scalars stay
 * on the device and every rank folds the gathered values in rank order, so
 * all ranks take the same branches.  One rank's loop:
 *   pf_slab_bicg_init -> gather -> phase START;
 *   repeat { exchange(pp, 1 plane) -> APPLY_P -> gather -> S ->
 *            exchange(s, 1 plane) -> APPLY_S -> gather -> FINAL -> gather ->
 *            NEXT }   until pf_slab_bicg_info reports done (after NEXT);
 *   then pf_slab_add (p += DP), exchange(DP, 1 plane), pf_vel_corr.
 * pp and s (the exchanged vectors) live in the workspace
 * (pf_slab_bicg_vectors).  info: 4 device doubles [max_res, iterations,
 * status, done].  After `done` the phases return at once, so ranks may poll
 * every few iterations.  halo >= 1 for the solve. */
enum {
    PF_SLAB_START = 0,    /* fold the init gather; pp = res */
    PF_SLAB_NEXT = 1,     /* fold the stop test and rho1; pp = (pp - w vv) b + res */
    PF_SLAB_APPLY_P = 2,  /* vv = A pp; send = [(vv, res0), 0] */
    PF_SLAB_S = 3,        /* fold gamma; DP += a pp; s = res - a vv */
    PF_SLAB_APPLY_S = 4,  /* t = A s; send = [(s, t), (t, t)] */
    PF_SLAB_FINAL = 5     /* fold omega; DP += w s; res = s - w t; send = [(res, res0), max|res|] */
};
size_t pf_slab_workspace_bytes(const pf_grid* g);
int pf_slab_bicg_vectors(const pf_grid* g, void* ws, double** pp, double** s);
int pf_slab_bicg_init(const pf_grid* g, int halo, double rho, double dt,
                      double min_res, int max_it, const double* div, double* DP,
                      void* ws, size_t ws_bytes, double* send, void* stream);
int pf_slab_bicg_phase(const pf_grid* g, int halo, int phase, const double* recv,
                       int world, double* DP, void* ws, double* send, void* stream);
int pf_slab_bicg_info(const pf_grid* g, void* ws, double* info, void* stream);
int pf_slab_add(const pf_grid* g, int halo, const double* DP, double* p, void* stream);

/* NGA restart I/O from device memory (readNGArestart / writeNGArestart,
 * src/data/dataReader.py:119-208, whose MPI-IO path is :215-390): a restart
 * file stores each variable as an FP64 array in Fortran order (x fastest).
 * pf_restart_pack writes a device field ([nx][ny][nz], z fastest) in the
 * file's order into the device buffer file_order (nx*ny*nz doubles), ready
 * for one contiguous copy to the file; pf_restart_unpack is the inverse.
 * Asynchronous; the two buffers must not overlap; ny <= 65535. */
int pf_restart_pack(const pf_grid* g, const double* field, double* file_order,
                    void* stream);
int pf_restart_unpack(const pf_grid* g, const double* file_order, double* field,
                      void* stream);

/* A batch of independent time steps (the serving loop's active requests,
 * any grid sizes, one precision form) captured as ONE CUDA graph: each
 * replay advances every member by one Domain.forwardStep
 * (src/data/domain.py:342-402; constant viscosity, no SFS model).  The RK4
 * stages of all members run as one grouped launch per stage (a persistent
 * kernel walking the members' tiles, src/solver/advancer.py:75-113), then
 * each member's divergence, pressure solve (device-side WHILE loops),
 * projection and statistics run as independent branches of the graph, so
 * the members' solves overlap on the device.  Every member computes exactly
 * what its own pf_step_plan would: results are the same alone and in any
 * batch.  A member's fields, workspace (pf_step_plan_workspace_bytes) and
 * stats (10 doubles, the layout of pf_step_plan_create) belong to the plan
 * while it exists.  table is a caller device buffer of
 * pf_batch_table_bytes(count) bytes, 256-byte aligned, that holds the grouped
 * launches' per-member arguments (written at creation) and, in its first int,
 * an error flag that a grouped launch sets to 1 if it finds a tile outside
 * every member's range (it then skips the tile).  At most 64 members.  A member
 * with fresh != 0 joins a plan for the first time: creation initialises its
 * solver state (synchronously, on a stream of its own).  A member with
 * fresh == 0 is carried over from an earlier plan, whose launches may still
 * be running: creation does not touch its memory, and launches of the new
 * plan on the same stream follow the old plan's in stream order. */
typedef struct pf_batch_member {
    pf_grid grid;
    double *u, *v, *w, *p, *DP;
    double mu, rho, dt, min_res;
    int max_it;
    int fresh;
    void* ws;
    size_t ws_bytes;
    double* stats;
} pf_batch_member;
size_t pf_batch_table_bytes(int count);
int pf_batch_plan_create(int prec, int rk4, const pf_batch_member* members,
                         int count, void* table, size_t table_bytes,
                         pf_step_plan** plan);

/* Optional per-kernel device-time accounting: when enabled, each kernel launch
 * of the library is bracketed by CUDA events on its stream.  pf_profile_read
 * waits for pending events and fills up to max_entries records (per kernel
 * name: launches and summed milliseconds); *count gets the number of names. */
typedef struct pf_kernel_time {
    char name[48];
    long long launches;
    double ms;
} pf_kernel_time;

int pf_profile_enable(int enable);
int pf_profile_read(pf_kernel_time* out, int max_entries, int* count);

#ifdef __cplusplus
}
#endif

#endif /* PYFLOW_B200_H */
