/* CPU restatement of the reference's pressure-solve path — TEST INFRASTRUCTURE ONLY.
 *
 * The oracle is the checker of the CUDA path: only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load it.  Each function names the reference lines it
 * restates (paths inside the Voluma project).  Pinned by tests/test_oracle.py against the
 * reference itself compiled from its sources (oracle/_ref, see oracle/Makefile) and against
 * the committed fixtures in tests/golden/.
 */
#ifndef VLM_ORACLE_H
#define VLM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* par::ExactSum add/value (src/fvm/parallel/Comm.h:65-93, Comm.cpp:114-164) */
double vo_exact_sum(const double* v, long n);

/* amul (src/fvm/linalg/LinearSolver.cpp:121-133); lower == NULL: symmetric */
void vo_amul(int n, int nf, const int* own, const int* nei, const double* diag, const double* upper,
             const double* lower, const double* x, double* y);

/* buildHierarchy (src/fvm/linalg/GAMG.cpp:15-94, 206-261), serial */
typedef struct vo_hier vo_hier;
/* the device agglomeration's parallel matching (voluma_b200/csrc/aggl.cu), restated */
vo_hier* vo_hier_build_matching(int n, int nf, const int* own, const int* nei, const double* magSf,
                                const double* ndc, int mergeLevels, int nCoarsest);
vo_hier* vo_hier_build(int n, int nf, const int* own, const int* nei, const double* magSf, const double* ndc,
                       int mergeLevels, int nCoarsest);
void vo_hier_free(vo_hier* h);
int vo_hier_nlevels(const vo_hier* h);
/* sizes[0]=n, sizes[1]=nFaces, sizes[2]=len(agg); outputs may be NULL */
void vo_hier_level(const vo_hier* h, int lev, int* sizes, int* l, int* u, double* weight, int* agg, int* faceMap,
                   signed char* faceFlip);
/* greedy natural-order colouring of a level (the device smoother's colouring) */
int vo_hier_colour(const vo_hier* h, int lev, int* colour);

/* GAMG options: smoother 0 = natural-order Gauss-Seidel (the reference, GAMG.cpp:363-385),
 * 1 = the device's Gauss-Seidel schedule: level 0 multicolour GS (forward colours pre, reversed
 *     post) when its greedy colouring has <= 4 colours, block-hybrid GS (512-row blocks,
 *     block-local colours, out-of-block neighbours from the previous sweep) on the other levels,
 * 2 = Jacobi(omega) on every level,
 * 3 = level 0 as in 1, Jacobi(omega) on the coarser levels;
 * coarse 0 = LU substitution (GAMG.cpp:406-420), 1 = explicit inverse from the LU. */
typedef struct {
    int smoother;
    double omega;
    int coarse;
    int mergeLevels;
    int matching;  /* 1: the hierarchy of the device agglomeration's parallel matching */
} vo_gamg_opts;

/* One V-cycle w = M^-1 r (GamgPreconditioner ctor + apply, GAMG.cpp:263-353, 403-449).
 * Returns 0, or 4 for a singular coarsest matrix. */
int vo_gamg_apply(int n, int nf, const int* own, const int* nei, const double* magSf, const double* ndc,
                  const double* diag, const double* upper, const double* lower, const double* r, double* w,
                  const vo_gamg_opts* opt);

/* solveLdu (src/fvm/linalg/LinearSolver.cpp:135-284) for PCG and PBiCGStab with the
 * preconditioners none / diagonal / GAMG.  exactSums: ExactSum instead of plain double sums
 * (CFD_REPRODUCIBLE).  perf: initialResidual, finalResidual, residualSum, normFactor,
 * iterations, converged.  Returns 0, 4 (singular coarsest), 7 (unsupported). */
int vo_solve(int n, int nf, const int* own, const int* nei, const double* magSf, const double* ndc,
             const double* diag, const double* upper, const double* lower, const double* b, double* x,
             const char* solver, const char* precond, double tol, double relTol, int maxIter, int minIter,
             int exactSums, const vo_gamg_opts* opt, double* perf);

/* vo_solve with the relaxation solvers GaussSeidel / symGaussSeidel / Jacobi (nSweeps sweeps per
 * residual evaluation, LinearSolver.cpp:238-278) and the DIC / DILU preconditioners
 * (LinearSolver.cpp:56-107).  Returns 1 for nSweeps < 1 with a relaxation solver. */
int vo_solve_ex(int n, int nf, const int* own, const int* nei, const double* magSf, const double* ndc,
                const double* diag, const double* upper, const double* lower, const double* b, double* x,
                const char* solver, const char* precond, double tol, double relTol, int maxIter, int minIter,
                int nSweeps, int exactSums, const vo_gamg_opts* opt, double* perf);

/* w = M^-1 r for "none", "diagonal", "DIC", "DILU" (Preconditioner, LinearSolver.cpp:56-107). */
int vo_precond_apply(int n, int nf, const int* own, const int* nei, const double* diag, const double* upper,
                     const double* lower, const char* precond, const double* r, double* w);

#ifdef __cplusplus
}
#endif
#endif
