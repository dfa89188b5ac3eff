// pf_mg.cuh -- FP32 BiCGStab right-preconditioned by a geometric multigrid
// V-cycle: the inner solver of the PF_MIXED_MG pressure refinement.
#pragma once
#include "pf_sweep.cuh"

namespace pf {

constexpr int kMgMaxLevels = 16;
constexpr long long kMgCoarseTarget = 512;  // stop coarsening at or below this
constexpr long long kMgCoarseMax = 4096;    // largest coarsest level (one CTA)

struct MgLevel {
    Dims d;
    LapCoef<float> cf;  // the scaled operator -vol L with this level's spacing
    float wd;           // omega / diag(A)
    float *b, *x, *t;   // right-hand side, iterate, smoothing buffer
    Tiling tl;
};

struct MgPlan {
    int L = 0;  // number of levels; 0 = multigrid does not apply to the grid
    MgLevel lv[kMgMaxLevels];
    // Krylov vectors (FP32, finest grid); p is double-buffered
    float *res, *res0, *p[2], *v, *s, *t, *ph, *sh, *e;
};

// Level hierarchy of grid g (no memory touched).  Returns the number of
// levels, 0 when the grid cannot be coarsened to a coarsest level of at most
// kMgCoarseMax cells.
int mg_levels(const pf_grid* g, MgLevel* lv);
// FP32 bytes of the Krylov vectors and the coarse levels (0 if L == 0).
size_t mg_region_bytes(const pf_grid* g);
// Carve the vectors from `region` (mg_region_bytes long, 256-byte aligned).
int mg_setup(const pf_grid* g, void* region, MgPlan* P);
// One inner solve: A e = rhs / sc->scale to relative max-norm `tol` (host
// polls between chunks).  Leaves the iteration count and status in sc.
int mg_inner_solve(const MgPlan& P, BicgScalars* sc, double* part,
                   const double* rhs, double tol, int max_it, cudaStream_t s,
                   BicgScalars* hs);
// Kernels of the inner solve, for graph capture: initialisation and one
// iteration with parity k & 1 (kernels of a finished solve return at once).
int mg_enqueue_init(const MgPlan& P, BicgScalars* sc, double* part,
                    const double* rhs, double tol, int max_it, cudaStream_t s);
int mg_enqueue_iteration(const MgPlan& P, BicgScalars* sc, double* part, int k,
                         cudaStream_t s, int use_cond = 0,
                         cudaGraphConditionalHandle cond = 0);

}  // namespace pf
