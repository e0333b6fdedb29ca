// ggb_solver.h — device descriptors of the multigrid-preconditioned CG solve.
#pragma once

#include "ggb_stencil.cuh"

namespace ggb {

constexpr int kMaxLev = 12;

// One multigrid level on the device.  The level vectors are float in the
// plain solve and __half in the mixed-precision solve (SolveParams::mixed).
struct LevelDev {
    StencilDev S;
    const float *dinv;  // [n] 1 / sum of link weights
    void *x;            // [n] iterate (pre-smoothed, then corrected)
    void *xo;           // [n] V-cycle output of this level
    void *b;            // [n] right-hand side (restricted residual)
    void *r;            // [n] residual after the pre-smooth
    // transfer to the next coarser level
    const int *ptap;    // [4n] coarse taps of each cell of this level
    const float *pw;    // [4n] their bilinear weights
    const int *rstart;  // [n_coarse+1] rows of R = P^T
    const int *ridx;    // fine cells of each row (ascending)
    const float *rw;    // weights of each row
    int structured;     // 1: interior rows of R / P follow the 4x4 / 2x2 index pattern (verified at setup)
    const float *rw16;  // [16][n_coarse] weights of the structured R rows (coarse-major), or nullptr
};

// Status bits of a solve (SolveResult::flags; also ggb_solve_flags).
enum {
    kSolveTimeout = 1,    // a grid barrier timed out (the solve was abandoned)
    kSolveNonFinite = 2,  // a NaN or Inf reached b.b, r.r, r.z or p.Ap
    kSolveBreakdown = 4,  // p.Ap <= 0: CG stopped early (upstream src/fluid.c:329-330 stops silently)
    kSolveMaxit = 8,      // maxit iterations without reaching the tolerance
};

struct SolveResult {
    int iters;
    int status;      // 0 ok, 1 barrier timeout
    double relres;
    int r_final;     // which r buffer holds the final residual (0: r, 1: r2)
    int flags;       // kSolve* bits
    unsigned long long ns;  // device time of the solve (%globaltimer, block 0 of the solve)
};

struct SolveParams {
    int mixed;           // 1: V-cycle vectors (and coarse slot weights) in FP16 with FP32 accumulation,
                         //    flexible (Polak-Ribiere) CG; 0: FP32 vectors, FP64 accumulation
    int nlev;            // >= 1 when multigrid, 0 for the Jacobi preconditioner
    int nlev_grid;       // non-coarsest levels 0..nlev_grid-1 run grid-wide
    int coarse_on_grid;  // coarsest level swept grid-wide (else by block 0)
    int coarse_sweeps;   // Jacobi sweeps on the coarsest level (upstream: 60)
    int remove_mean;     // project the mean out of omega first
    int maxit;
    double tol;
    double total_area;
    LevelDev L[kMaxLev];
    const float *area;   // level-0 cell areas
    float *omega, *psi;
    float *r, *r2, *p, *p2, *Ap, *z;  // level-0 CG vectors (r / p ping-pong)
    float *z2;           // mixed: the previous z (z / z2 ping-pong for the flexible beta)
    double *part;        // [RED_N][gridDim.x] per-block partial sums
    unsigned long long *trace;  // optional: block 0 stamps %globaltimer at phase marks
    int trace_cap;
    GridBarrier *bar;
    SolveResult *res;
    // dense form of the V-cycle below the grid levels: xo_G = D b_G
    const double *dense;  // [nd][nd] row-major, or nullptr
    int nd;               // cells of level nlev_grid
};

}  // namespace ggb
