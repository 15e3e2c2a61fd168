/*
 * claw_oracle.h -- CPU oracle for the classic Clawpack 2D wave-propagation step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path is
 * compared against; the product package never links, loads or calls it.  Only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use it.
 *
 * It restates, loop for loop and in the same floating-point operation order,
 * the reference's FP64 kernels:
 *   step2    src/pyclaw/classic/step2.f90:2-250     (unsplit step)
 *   step2ds  src/pyclaw/classic/step2ds.f90:2-264   (dimensionally split step)
 *   flux2    src/pyclaw/classic/flux2.f90:1-207
 *   limiter  src/pyclaw/classic/limiter.f90:1-57
 *   philim   src/pyclaw/classic/philim.f90:1-37
 *   BC fill  src/pyclaw/solver.py:351-519          (extrap / periodic / wall)
 * and the Riemann solvers of the external clawpack/riemann package (not
 * vendored in the reference; restated from the published mathematics, see
 * claw_oracle.cpp for each).
 *
 * Array layouts are the reference's: qbc is Fortran-ordered
 * (num_eqn, mx+2*num_ghost, my+2*num_ghost), i.e. component fastest.
 *
 * Parity pins: tests/golden/ holds the reference's own regression goldens
 * (advection_2d, acoustics_2d_homogeneous, euler_2d quadrants, shallow_2d
 * radial dam break), which this oracle reproduces through the host driver.
 */
#ifndef CLAW_ORACLE_H
#define CLAW_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Riemann solver ids (shared numbering with include/claw2.h). */
enum {
    ORC_RP_ADVECTION = 1,   /* advection_2D           cparam: u, v            */
    ORC_RP_ACOUSTICS = 2,   /* acoustics_2D           cparam: rho,bulk,cc,zz  */
    ORC_RP_EULER_ROE = 3,   /* euler_4wave_2D         cparam: gamma, efix     */
    ORC_RP_SHALLOW_ROE = 4, /* shallow_roe_with_efix_2D cparam: grav, efix    */
    ORC_RP_EULER_EXACT = 5, /* exact Euler (new)      cparam: gamma, tol      */
    ORC_RP_VC_ACOUSTICS = 6, /* vc_acoustics_2D       aux: rho, c; no cparam  */
    ORC_RP_VC_ADVECTION = 7, /* vc_advection_2D       aux: u, v edge velocities */
    ORC_RP_PSYSTEM = 8,      /* psystem_2D (f-waves)  aux: rho, K, relation, eps */
    ORC_RP_VC_ADVECTION_VEC = 9, /* advection_reaction's vector vc advection, split only */
    ORC_RP_EULER_5WAVE = 10,     /* euler_5wave_2D (Roe + tracer) cparam: gamma, efix */
    ORC_RP_SHALLOW_HLLE = 12     /* shallow_hlle_2D, no rpt2       cparam: grav        */
};

/* One unsplit step (step2.f90).  qold, qnew: (meqn, mx+2mbc, my+2mbc) F-order;
 * qnew must equal qold on entry.  aux may be NULL when maux == 0.
 * method[7] and mthlim[mwaves] exactly as the reference builds them
 * (classic/solver.py:173-193).  Returns 0 on success. */
int oracle_step2(int maxm, int meqn, int mwaves, int maux, int mbc, int mx, int my,
                 const double* qold, double* qnew, const double* aux,
                 double dx, double dy, double dt, const int* method,
                 const int* mthlim, double* cfl, int use_fwave, int rp_id,
                 const double* cparam);

/* One sweep of the dimensionally split step (step2ds.f90); ids = 1 (x) or 2 (y).
 * qold may alias qnew (the reference's second call passes qbc twice). */
int oracle_step2ds(int maxm, int meqn, int mwaves, int maux, int mbc, int mx, int my,
                   const double* qold, double* qnew, const double* aux,
                   double dx, double dy, double dt, const int* method,
                   const int* mthlim, double* cfl, int ids, int use_fwave,
                   int rp_id, const double* cparam);

/* Ghost-cell fill of qbc (solver.py:351-519, q only).  bc codes follow
 * pyclaw.BC: 1 extrap, 2 periodic, 3 wall; -1 leaves that side to the caller
 * (a halo filled by a neighbouring rank).  reflect_index = {1,2}. */
int oracle_bc_fill(int meqn, int mbc, int mx, int my, double* qbc,
                   const int* bc_lower, const int* bc_upper);

/* Ghost-cell fill of an aux array (solver.py:439-519 with name != 'q'): as
 * oracle_bc_fill, but a wall mirrors without negating any component. */
int oracle_bc_fill_aux(int maux, int mbc, int mx, int my, double* auxbc,
                       const int* bc_lower, const int* bc_upper);

/* Riemann solvers with aux slices for unit tests: aux (maux, 1-mbc:mx+mbc)
 * for the slice itself (auxl = auxr), aux1/aux3 for the slices below/above
 * (rpt2 only), Fortran ABI. */
int oracle_rpn2_aux(int rp_id, int ixy, int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
                    const double* q, const double* aux, double* wave, double* s, double* amdq,
                    double* apdq, const double* cparam);
int oracle_rpt2_aux(int rp_id, int ixy, int imp, int maxm, int meqn, int mwaves, int maux, int mbc,
                    int mx, const double* q, const double* aux1, const double* aux2,
                    const double* aux3, const double* asdq, double* bmasdq, double* bpasdq,
                    const double* cparam);

/* Direct Riemann-solver access for unit tests: one slice, Fortran ABI. */
int oracle_rpn2(int rp_id, int ixy, int maxm, int meqn, int mwaves, int mbc, int mx,
                const double* ql, const double* qr, double* wave, double* s,
                double* amdq, double* apdq, const double* cparam);
int oracle_rpt2(int rp_id, int ixy, int imp, int maxm, int meqn, int mwaves, int mbc,
                int mx, const double* ql, const double* qr, const double* asdq,
                double* bmasdq, double* bpasdq, const double* cparam);

/* Exact Euler Riemann problem in the normal direction (Toro ch. 4):
 * returns p*, u* and the Newton iteration count for one interface. */
int oracle_exact_star(double gamma, double rl, double ul, double pl,
                      double rr, double ur, double pr, double tol, int guess,
                      double* pstar, double* ustar, int* iters);

/* Threads used by oracle_step2 (OpenMP over slices when built with it). */
void oracle_set_threads(int n);
int oracle_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
