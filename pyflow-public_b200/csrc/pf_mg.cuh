// pf_mg.cuh -- FP32 BiCGStab right-preconditioned by a geometric multigrid
// V-cycle: the inner solver of the PF_MIXED_MG pressure refinement.
#pragma once
#include "pf_sweep.cuh"

namespace pf {

constexpr int kMgMaxLevels = 16;
constexpr long long kMgCoarseTarget = 64;     // coarsen down to at most this many cells
constexpr long long kMgBottomMax = 4096;      // largest coarsest level (solved in one CTA)
constexpr long long kMgBottomLevel = 512;     // levels this small run inside that CTA
constexpr long long kMgSweepMin = 1LL << 20;  // levels this large use the tiled sweep
constexpr long long kMgClusterMax = 4096;     // levels this small may run in the cluster kernel
constexpr int kClusterCtas = 8;               // CTAs of that cluster (x planes split among them)
constexpr int kMgPinvMax = 64;                // largest coarsest level solved with a pseudo-inverse

// How a level's kernels run: the tiled sweep (the finest level always, and
// every level of at least kMgSweepMin cells), one thread per cell, inside
// the single-CTA bottom kernel (every level of at most kMgBottomLevel cells,
// and the coarsest level, which must have at most kMgBottomMax cells), or
// split by x planes across the CTAs of the cluster kernel, which also runs
// the bottom levels (the levels just above the bottom ones with at most
// kMgClusterMax cells and an x extent that kClusterCtas divides).
enum MgKind { kMgSwept = 0, kMgPointwise = 1, kMgBottom = 2, kMgCluster = 3 };

struct MgLevel {
    Dims d;
    LapCoef<float> cf;  // the scaled operator -vol L with this level's spacing
    float wd;           // omega / diag(A)
    float *b, *x, *t;   // right-hand side, iterate, smoothing buffer
    Tiling tl, tl8;     // tilings of the 4- and 8-row register sweeps
    int az;             // cp.async sweep tile width (64, 32; 0: none, nz not a multiple of 32)
    Tiling ta1, tan;    // cp.async tilings: one input field (32 rows), several (16 rows)
    int kind;
    double cq[3];       // vol / h_q^2: the operator's off-diagonal magnitudes
};

struct MgPlan {
    int L = 0;  // number of levels; 0 = multigrid does not apply to the grid
    int B = 0;  // first level handled by the bottom kernel
    int C = 0;  // first level of the cluster kernel (C == B: the bottom kernel alone)
    MgLevel lv[kMgMaxLevels];
    // Krylov vectors (FP32, finest grid); p is double-buffered
    float *res, *res0, *p[2], *v, *s, *t, *ph, *sh, *e;
    float* pinv = nullptr;  // coarsest-level pseudo-inverse (small coarsest levels)
    // one-thread-per-cell levels G .. C-1 (G < C) run as two cooperative
    // launches per V-cycle with grid barriers (coop != 0, opt-in through
    // PF_MG_COOP=1; bit-identical to the per-level kernels): coop_grid blocks,
    // barrier words gbar[0..3] (arrivals, generation, failure; zeroed by
    // mg_enqueue_setup and restored by every barrier)
    int G = 0;
    int coop = 0;
    int coop_grid = 0;
    unsigned* gbar = nullptr;
};

// Bytes of the grid-barrier words (a slot of their own).
constexpr size_t kMgBarrierBytes = 256;

// Level hierarchy of grid g (no memory touched).  Returns the number of
// levels and sets *bottom; 0 when the finest level is itself at most
// kMgBottomMax cells or the grid stops coarsening (an odd dimension) above
// that size.
int mg_levels(const pf_grid* g, MgLevel* lv, int* bottom);
// FP32 bytes of the Krylov vectors and the coarse levels (0 if L == 0).
size_t mg_region_bytes(const pf_grid* g);
// Carve the vectors from `region` (mg_region_bytes long, 256-byte aligned).
int mg_setup(const pf_grid* g, void* region, MgPlan* P);
// One inner solve: A e = rhs / sc->scale to relative max-norm `tol`, or
// looser when the refinement (outer tolerance `outer_tol`, current true
// residual sc->true_res of max|b| sc->max_b) needs less; the host polls
// between chunks.  Leaves the iteration count and status in sc.
int mg_inner_solve(const MgPlan& P, BicgScalars* sc, double* part,
                   const double* rhs, double tol, int max_it, cudaStream_t s,
                   BicgScalars* hs, double outer_tol = 0.0);
// Per-solve set-up kernels (the coarsest level's pseudo-inverse); enqueue
// once before the first inner solve that uses the vectors of `region`.
int mg_enqueue_setup(const MgPlan& P, cudaStream_t s);
// Kernels of the inner solve, for graph capture: initialisation and one
// iteration with parity k & 1 (kernels of a finished solve return at once).
int mg_enqueue_init(const MgPlan& P, BicgScalars* sc, double* part,
                    const double* rhs, double tol, int max_it, cudaStream_t s,
                    double outer_tol = 0.0);
int mg_enqueue_iteration(const MgPlan& P, BicgScalars* sc, double* part, int k,
                         cudaStream_t s, int use_cond = 0,
                         cudaGraphConditionalHandle cond = 0);

}  // namespace pf
