/*
 * claw2.h -- C ABI of the B200 (sm_100a) classic Clawpack 2D step.
 *
 * Drop-in boundary.  In the reference, ClawSolver2D.step_hyperbolic
 * (src/pyclaw/classic/solver.py:498-549) calls the f2py-wrapped Fortran
 * routines step2 (src/pyclaw/classic/step2.f90:2-5) and step2ds
 * (src/pyclaw/classic/step2ds.f90:2-6), which call the Riemann solvers through
 * raw Fortran function pointers (classic/solver.py:516-521).  This library
 * replaces those routines.  Plain C types only; every function returns an
 * int status (CLAW2_OK = 0) and never aborts; claw2_last_error() describes
 * the last failure on the calling thread.
 *
 * Riemann solvers cannot cross the ABI as host function pointers, so they are
 * selected by id (CLAW2_RP_*) and their parameters (the reference's COMMON
 * /cparam/, src/pyclaw/state.py:206-231) are passed as a double array.
 *
 * Layouts.  Host arrays use the reference's Fortran order:
 *   qbc  (num_eqn, mx+2*num_ghost, my+2*num_ghost)   for claw2_step2/_step2ds
 *   q    (num_eqn, mx, my)                            for the patch upload/download
 * (src/pyclaw/state.py:330-335, solver.py:343-345).  On the device the library
 * keeps structure-of-arrays planes with a 2-cell ghost ring and a padded pitch.
 */
#ifndef CLAW2_H
#define CLAW2_H

#ifdef __cplusplus
extern "C" {
#endif

#define CLAW2_MAX_PARAMS 8
#define CLAW2_MAX_WAVES 8

/* Riemann solver ids and their cparam layouts. */
enum {
    CLAW2_RP_ADVECTION = 1,    /* advection_2D:               {u, v}                 */
    CLAW2_RP_ACOUSTICS = 2,    /* acoustics_2D:               {rho, bulk, cc, zz}    */
    CLAW2_RP_EULER_ROE = 3,    /* euler_4wave_2D:             {gamma, efix}          */
    CLAW2_RP_SHALLOW_ROE = 4,  /* shallow_roe_with_efix_2D:   {grav, efix}           */
    CLAW2_RP_EULER_EXACT = 5,  /* exact Euler (no reference counterpart): {gamma, tol, guess} */
    CLAW2_RP_VC_ACOUSTICS = 6, /* vc_acoustics_2D: no cparam; aux = {rho, c} per cell        */
    CLAW2_RP_VC_ADVECTION = 7, /* vc_advection_2D: no cparam; aux = {u left edge, v bottom edge} */
    CLAW2_RP_PSYSTEM = 8,      /* psystem_2D (f-waves): no cparam; aux = {rho, K, relation, strain} */
    CLAW2_RP_VC_ADVECTION_VEC = 9, /* examples/advection_reaction_2d's own solver, num_eqn 2: aux =
                                  {u left edge, v bottom edge}; no transverse solve */
    CLAW2_RP_EULER_5WAVE = 10, /* euler_5wave_2D (Roe + tracer):  {gamma, efix}          */
    CLAW2_RP_SHALLOW_HLLE = 12 /* shallow_hlle_2D: {grav}; no transverse solve           */
};

/* Boundary-condition codes: pyclaw.BC (src/pyclaw/solver.py:13-19), plus
 * CLAW2_BC_NONE for a side whose ghost rows the caller fills (a neighbour's
 * halo in a domain split across ranks, as petclaw's DMDA globalToLocal does,
 * src/petclaw/state.py:223-229); only the x rule is applied to its corners. */
enum { CLAW2_BC_NONE = -1, CLAW2_BC_CUSTOM = 0, CLAW2_BC_EXTRAP = 1, CLAW2_BC_PERIODIC = 2,
       CLAW2_BC_WALL = 3 };

/* Status codes. */
enum {
    CLAW2_OK = 0,
    CLAW2_EINVAL = 1,      /* bad argument (sizes, ids, null pointers)           */
    CLAW2_ECUDA = 2,       /* a CUDA runtime call failed                         */
    CLAW2_ENONFINITE = 3,  /* the step produced a non-finite value               */
    CLAW2_ETIMEOUT = 4,    /* a bounded device-side wait gave up                 */
    CLAW2_ENOMEM = 5,      /* device allocation failed                           */
    CLAW2_EUNSUPPORTED = 6 /* valid request this build does not implement        */
};

/* Patch description: the state of one ClawSolver2D after setup()
 * (classic/solver.py:195-234, solver.py:158-242). */
typedef struct claw2_desc {
    int mx, my;               /* interior cells                                        */
    int num_eqn, num_waves;   /* must match the Riemann solver                         */
    int num_aux;              /* aux components per cell on the device: at least the ones the
                                 solver reads (2 for vc_acoustics_2D, vc_advection_2D) and the
                                 capacity's; 0 when neither needs aux          */
    int num_ghost;            /* must be 2                                              */
    int riemann;              /* CLAW2_RP_*                                             */
    int order;                /* method(2): 1 or 2                                      */
    int transverse;           /* method(3): 0, 1, 2 (unsplit)                           */
    int dimensional_split;    /* 1: step2ds x then y (method(3) = -1)                   */
    int fwave;                /* use_fwave                                              */
    int mthlim[CLAW2_MAX_WAVES];
    int bc_lower[2], bc_upper[2];
    double dx, dy;
    double cparam[CLAW2_MAX_PARAMS];
    int ncparam;
    int device;               /* CUDA device ordinal                                    */
    int mcapa;                /* method(6): 0, or 1 + the aux component holding the
                                 capacity function kappa (state.index_capa + 1)      */
} claw2_desc;

typedef struct claw2_patch claw2_patch;

/* ---- stateless drop-ins for the f2py routines (host buffers) ------------- */

/* Replaces step2 (src/pyclaw/classic/step2.f90:2-5; called at
 * classic/solver.py:539-541).  qold/qnew: qbc layout, ghost cells already
 * filled; qnew must equal qold on entry.  method[7] and mthlim[num_waves] as
 * built by classic/solver.py:162-193.  On return the interior cells of qnew
 * hold the updated solution and *cfl the Courant number over the same
 * interfaces as the reference (flux2.f90:111-119 over step2.f90:92,172
 * slices).  Ghost cells of qnew are left as they were on entry (the next BC
 * fill overwrites them; the reference's partial ghost updates are never read). */
int claw2_step2(int maxm, int num_eqn, int num_waves, int num_aux, int num_ghost,
                int mx, int my, const double* qold, double* qnew, const double* aux,
                double dx, double dy, double dt, const int* method, const int* mthlim,
                double* cfl, int use_fwave, int riemann, const double* cparam,
                int ncparam);

/* Replaces step2ds (src/pyclaw/classic/step2ds.f90:2-6; called twice at
 * classic/solver.py:527-535).  ids = 1: x-sweep over every row including the
 * ghost rows; ids = 2: y-sweep.  qold may alias qnew. */
int claw2_step2ds(int maxm, int num_eqn, int num_waves, int num_aux, int num_ghost,
                  int mx, int my, const double* qold, double* qnew, const double* aux,
                  double dx, double dy, double dt, const int* method, const int* mthlim,
                  double* cfl, int ids, int use_fwave, int riemann,
                  const double* cparam, int ncparam);

/* Replaces Solver._apply_bcs for q (src/pyclaw/solver.py:351-519) on a host
 * qbc array: extrap / periodic / wall, dimension 0 then 1. */
int claw2_bc_fill(int num_eqn, int num_ghost, int mx, int my, double* qbc,
                  const int* bc_lower, const int* bc_upper);

/* ---- device-resident patch (the fast path) ------------------------------- */

/* Allocates the device state (two q buffers, CFL and status words) for one
 * ClawSolver2D (replaces ClawSolver2D._allocate_workspace and
 * Solver._allocate_bc_arrays, classic/solver.py:466-494, solver.py:321-349). */
int claw2_patch_create(const claw2_desc* desc, claw2_patch** out);
int claw2_patch_destroy(claw2_patch* p);

/* Replaces state.set_cparam (state.py:206-231). */
int claw2_patch_set_cparam(claw2_patch* p, const double* cparam, int ncparam);

/* Host <-> device copies of State.q, shape (num_eqn, mx, my), Fortran order. */
int claw2_patch_upload_q(claw2_patch* p, const double* q);
int claw2_patch_download_q(claw2_patch* p, double* q);

/* Source step on the current state (no step pending): q <- q + dt M q_old in
 * every interior cell, M row-major n x n with n = num_eqn (a linear
 * step_source of classic/solver.py:126-144 without leaving the device). */
int claw2_patch_linear_source(claw2_patch* p, const double* m, int n, double dt);

/* Source step on the current state (no step pending): the geometric source
 * of the Euler equations in r-z coordinates with cylindrical symmetry, r the
 * aux component radius_aux, by a two-stage Runge-Kutta step (the step_source
 * of examples/euler_2d/shock_bubble_interaction.py:113-146, bit for bit). */
int claw2_patch_euler_axisymmetric_source(claw2_patch* p, double gamma, int radius_aux, double dt);

/* PyClaw's ascii frame files (src/pyclaw/fileio/ascii.py:17-123).
 * claw2_write_ascii writes `header` (the patch header lines) and the array
 * q (nvar, mx, my), Fortran order, one line of nvar "%18.8e" values per cell,
 * a blank line after each row; rows are formatted by nthreads threads
 * (0: all cores).  append: add to the file instead of replacing it.
 * claw2_patch_write_ascii_async does the same for the patch's current state:
 * the copy to the host is queued behind the steps already issued, and a host
 * thread formats and writes the file while later steps run;
 * claw2_patch_wait_output waits for it and returns its status (one frame in
 * flight: the next write call waits for the previous one). */
int claw2_write_ascii(const char* path, int append, const char* header, const double* q, int nvar, int mx,
                      int my, int nthreads);
int claw2_patch_write_ascii_async(claw2_patch* p, const char* path, int append, const char* header,
                                  int nthreads);
int claw2_patch_wait_output(claw2_patch* p);

/* q of the current state at n interior cells: ij holds n (i, j) pairs
 * (0-based), out receives n * num_eqn values, cell by cell.  The gauge
 * values of Solver.write_gauge_values (solver.py:680-715) without
 * downloading the whole array. */
int claw2_patch_gather_q(claw2_patch* p, int n, const int* ij, double* out);

/* State.aux, shape (num_aux, mx, my), Fortran order, and its ghost cells from
 * the aux BCs (solver.py:351-519 with name 'aux': a wall mirrors without
 * changing sign).  aux is constant in time on the device: upload it again
 * after changing it. */
int claw2_patch_upload_aux(claw2_patch* p, const double* aux, const int* aux_bc_lower,
                           const int* aux_bc_upper);

/* qbc as the host filled it, shape (num_eqn, mx+4, my+4), Fortran order,
 * ghost cells included, into the current state; the next step keeps these
 * ghost cells instead of filling them (custom BCs: the user_bc_lower/upper
 * functions that solver.py:378-427 calls). */
int claw2_patch_upload_qbc(claw2_patch* p, const double* qbc);

/* auxbc as the host filled it, shape (num_aux, mx+4, my+4), Fortran order,
 * ghost cells included: for aux BCs the host applies itself (BC.custom, the
 * user_aux_bc_lower/upper functions that solver.py:378-427 calls). */
int claw2_patch_upload_auxbc(claw2_patch* p, const double* auxbc);

/* Device-resident time loop: Solver.evolve_to_time (src/pyclaw/solver.py:
 * 554-666) for a solver without host callbacks, with get_dt, the CFL test,
 * accept/reject and the clipping to tend done on the GPU after every step, so
 * the host waits only every few dozen steps.  In: t (solution.t), tstart,
 * tend, dt (solver.dt), cfl (the solver's cached Courant number), cfl_desired,
 * cfl_max, dt_max, dtmin/dtmax/cflmax (solver.status), dt_variable,
 * dt_old_set (solver.dt_old is not None), max_steps (attempts allowed).  Out:
 * the same fields after the loop, num_steps (accepted), attempts (accepted +
 * rejected), cfl_error (a fixed-dt step exceeded cfl_max: the reference
 * raises CFLError).  The current state is the loop's result; a step that
 * produced a non-finite value ends the loop with that step undone and
 * CLAW2_ENONFINITE.  Same steps, dt sequence and results as the host loop. */
typedef struct claw2_evolve_state {
    double t, tstart, tend, dt, cfl;
    double cfl_desired, cfl_max, dt_max;
    double dtmin, dtmax, cflmax;
    int dt_variable, dt_old_set, max_steps;
    int num_steps, attempts, cfl_error;
} claw2_evolve_state;
int claw2_patch_evolve(claw2_patch* p, claw2_evolve_state* s);

/* One hyperbolic step from the current q: ghost fill on the device, then the
 * unsplit (or split) step into the pending buffer.  If cfl is non-NULL the
 * call waits and returns the Courant number; with NULL it only enqueues. */
int claw2_patch_step(claw2_patch* p, double dt, double* cfl);

/* The same step in two parts around a halo exchange (no counterpart in the
 * reference; petclaw exchanges before its step, src/petclaw/state.py:223-229):
 * part 1 enqueues the ghost fill of every cell but the ghost rows of sides
 * marked CLAW2_BC_NONE, and the step of the row blocks that read no ghost row;
 * the caller then fills those ghost rows (the exchange may run on another
 * stream meanwhile: part 1 neither reads nor writes them); part 2, enqueued
 * after the exchange, fills their ghost columns and steps the first and last
 * row blocks, and with cfl non-NULL waits and returns the Courant number.
 * The result equals claw2_patch_step's.  A split step, the exact solver, host
 * ghost cells or fewer than three row blocks run whole in part 2. */
int claw2_patch_step_part(claw2_patch* p, double dt, int part, double* cfl);

/* Many independent steps from host buffers (no counterpart in the reference,
 * whose step2 call moves one host qbc per step through f2py): for k < nsteps,
 * q_out[k] = one step (ghost fill, step, CFL) of q_in[k] with dt[k], each
 * accepted, cfl_out[k] its Courant number.  q_in/q_out are host arrays of
 * shape (num_eqn, mx, my), Fortran order (pinned memory for overlap).  The
 * upload of step k+1 and the download of step k overlap step k+1's compute
 * (an upload and a download stream, two staging buffers per direction), so the
 * input of a step must not be the output buffer of an earlier step of the
 * same call (chained steps stay on the device: claw2_patch_step).  Afterwards
 * the patch holds the last result.  Returns CLAW2_ENONFINITE if any step
 * produced a non-finite value. */
int claw2_patch_run_host(claw2_patch* p, int nsteps, const double* const* q_in, double* const* q_out,
                         const double* dt, double* cfl_out);

/* Accept (1) or reject (0) the pending step (solver.py:619-651): accept makes
 * it the current q; reject keeps the old q.  No copy either way. */
int claw2_patch_accept(claw2_patch* p, int accept);

/* Courant number of the last step (waits for it). */
int claw2_patch_cfl(claw2_patch* p, double* cfl);

/* Waits for the patch's stream and reports device-side error flags. */
int claw2_patch_sync(claw2_patch* p);

/* Raw device pointer of the current q planes and the layout, for callers that
 * share the device buffers (layout[0..3] = mx+4, my+4, pitch, plane). */
int claw2_patch_device_q(claw2_patch* p, double** q, long long* layout);

/* Run the patch's work on a caller-owned CUDA stream (a cudaStream_t passed
 * as void*); NULL returns to the patch's own stream. */
int claw2_patch_set_stream(claw2_patch* p, void* stream);

/* Kernel timing with CUDA events recorded on the patch's stream around the
 * step kernel(s) of each claw2_patch_step (ghost fill excluded).  After a
 * step, claw2_patch_kernel_ms waits for it and returns the elapsed time. */
int claw2_patch_set_timing(claw2_patch* p, int on);
int claw2_patch_kernel_ms(claw2_patch* p, float* ms);

/* Instrumentation, no counterpart in the reference: the kernels enqueued so
 * far by the patch's steps (claw2_patch_step and the host pipeline): ghost
 * fill, step kernel(s), learned-guess pre-pass, tile schedule sort.  Read it
 * before and after a run to count the run's launches. */
int claw2_patch_launch_count(claw2_patch* p, long long* n);

/* Launch shape of the unsplit step kernel for one Riemann solver: variant 0
 * compiles for 2 blocks per SM (no register cap), 1 for 3 blocks per SM,
 * 2 and 3 the same with rows staged by TMA, 4 the two-barrier tile, 8 the
 * direction-split tile (two threads per column: one for the y-interfaces, one
 * for the x-interfaces; solvers without aux data, no capacity form, others
 * run variant 0); rows = row-block height (0 = heuristic).  Process-wide; set by an autotuner
 * (pyclaw_b200.tune) or by hand. */
int claw2_tune_set(int riemann, int variant, int rows);
int claw2_tune_get(int riemann, int* variant, int* rows);

/* FP64 FMA throughput of the current device, TFLOP/s (2 flops per FMA): a
 * roofline denominator for the FP64-bound Riemann solvers. */
int claw2_probe_fp64(int device, double* tflops);

/* Self-test of the reciprocal the step kernels use in place of IEEE division
 * (no counterpart in the reference; Newton-Raphson refinement of the hardware
 * approximation): over n seeded values a = +-(1+u)*2^e, e uniform in
 * [-1000, 1000], *max_ulp = the largest distance in units in the last place
 * between it and CUDA's IEEE quotient 1.0/a.  Special values (+-0, +-inf,
 * NaN, a subnormal, 1e308) that do not give the documented results make
 * *max_ulp huge. */
int claw2_selftest_rcp(int device, int n, unsigned long long seed, double* max_ulp);
/* The same for the square root the solvers use per cell and per interface
 * (no counterpart in the reference; Goldschmidt iteration from the hardware's
 * reciprocal square root): x = (1+u)*2^e, against CUDA's IEEE sqrt(x). */
int claw2_selftest_sqrt(int device, int n, unsigned long long seed, double* max_ulp);
/* The same for the reciprocal square root of the Roe averages (no counterpart
 * in the reference; Newton steps from the hardware approximation), against
 * CUDA's 1.0 / sqrt(x): two roundings there, so up to 2 ulps apart. */
int claw2_selftest_rsqrt(int device, int n, unsigned long long seed, double* max_ulp);

/* Self-test (no counterpart in the reference) of the longest-first tile
 * schedule's sort: n (1..8192) seeded tile costs with many ties, sorted on the
 * device; *mismatches = positions where the order differs from a stable
 * descending sort on the host (cost descending, ties by lower tile first). */
int claw2_selftest_lpt(int device, int n, unsigned long long seed, int* mismatches);

/* ---- no counterpart in the reference ------------------------------------
 * The split step (x-sweep then y-sweep, as claw2_step2ds with ids = 1 then 2)
 * for callers that cannot allocate device memory: frameworks that reserve the
 * GPU's memory in their own pool, where a library cudaMalloc would fail or
 * fragment it, and loops that cannot take cudaMalloc's implicit device
 * synchronisation.  It allocates nothing: the caller passes the device q
 * planes (qold with its ghost cells filled, qnew; element (m, c, r) at
 * q[m*plane + r*pitch + c], padded column c in [0, mx+4), row r in [0, my+4)),
 * and the intermediate state plus the CFL/status words live in one fixed
 * device array of CLAW2_NOALLOC_SCRATCH_BYTES held by every GPU that loads
 * the library until exit.  Grids needing more than that (256 bytes +
 * num_eqn*plane*8 bytes), or with mx or my above 2^28, are rejected with
 * CLAW2_EINVAL before any GPU work.  Every
 * call reuses that array: the call clears the words that must start at zero;
 * calls whose GPU work overlaps race and must be serialised.  The first call
 * on a device looks up the array's address; make it before any stream
 * capture.  The call runs on `stream` (NULL: the legacy default stream),
 * waits for it, writes the Courant number to *cfl (host memory) and writes
 * the interior cells of qnew only. */
#define CLAW2_NOALLOC_SCRATCH_BYTES (32ll << 20)
int claw2_step2ds_noalloc(const claw2_desc* desc, const double* qold, double* qnew, long long pitch,
                          long long plane, double dt, double* cfl, void* stream);

/* ---- batches of independent problems (the batched form) ------------------
 * n problems of different sizes with the same solver, method, BCs and
 * parameters (the unsplit step), each with its own dt and time.  One batch
 * step = ghost fill of every instance + one persistent kernel over a flat
 * list of (instance, strip, row block) tiles + a per-instance accept/reject
 * and dt update on the device (solver.py:524-552, 619-651).  Replaces a host
 * loop of ClawSolver2D.evolve_to_time calls, one per problem. */
typedef struct claw2_batch claw2_batch;
int claw2_batch_create(const claw2_desc* descs, int n, claw2_batch** out);
int claw2_batch_destroy(claw2_batch* b);
/* Row-block height per instance (0 = heuristic); rebuilds the tile list. */
int claw2_batch_set_rows(claw2_batch* b, const int* rows);
int claw2_batch_upload_q(claw2_batch* b, int i, const double* q);
int claw2_batch_download_q(claw2_batch* b, int i, double* q);
/* Initial dt per instance, start/end time and the dt rule's constants. */
int claw2_batch_set_time(claw2_batch* b, const double* dt0, double t0, double tend, double cfl_desired,
                         double cfl_max, double dt_max);
/* nsteps batch steps; mode 0: the steps captured in one CUDA graph (captured
 * on first use for that nsteps), 1: the same launches issued directly,
 * 2: the plain loop -- one ghost-fill / step / finalize launch sequence per
 * instance.  *ms = device time of the whole run (CUDA events). */
int claw2_batch_run(claw2_batch* b, int nsteps, int mode, float* ms);
/* Per-instance state (arrays of n; any pointer may be NULL).  status bit 0:
 * a step produced a non-finite value; that step was discarded and the
 * instance retired at its last good state (the others go on). */
int claw2_batch_get_state(claw2_batch* b, double* t, double* dt, int* nsteps, int* nreject, double* cfl_last,
                          int* status);
int claw2_batch_tiles(claw2_batch* b, int* ntiles, int* persistent_grid);

/* ---- the exact Euler solver's learned Newton guess (no reference counterpart)
 * A 6-32-32-1 tanh network predicting log(p_star / p_pvrs) / w from the normalised
 * left/right states (w = J^2/(1+J^2), J a normalised jump size), trained on
 * the device by the library's own forward/backward kernels and Adam, and
 * evaluated in BF16 on the tensor cores (FP32 accumulation) for every
 * interface before each exact-solver step. */
typedef struct claw2_mlp claw2_mlp;
int claw2_mlp_create(int device, unsigned long long seed, claw2_mlp** out);
int claw2_mlp_destroy(claw2_mlp* m);
int claw2_mlp_set_params(claw2_mlp* m, const float* p, int n);  /* n = 1313 */
int claw2_mlp_get_params(claw2_mlp* m, float* p, int n);
/* n seeded Riemann problems (rho, p log-uniform in [1e-2, 1e2], u in [-3, 3])
 * solved to tol by FP64 Newton; *nvalid = problems without vacuum. */
int claw2_mlp_generate(claw2_mlp* m, unsigned long long seed, long long n, double gamma, double tol,
                       long long* nvalid);
/* Host copies of samples [first, first+count): 8 floats of features each
 * (6 inputs, jump weight, 0), the target and the validity flag. */
int claw2_mlp_samples(claw2_mlp* m, long long first, int count, float* x8, float* y, int* ok);
/* Gradient of 0.5 * mean squared error over samples [first, first+count). */
int claw2_mlp_gradient(claw2_mlp* m, long long first, int count, float* grad, float* loss);
/* Adam over all samples in minibatches; *last_loss = mean loss of the last epoch. */
int claw2_mlp_train(claw2_mlp* m, int epochs, int batch, float lr, float* last_loss);
/* Network outputs for n rows of 8 floats (BF16 tensor cores, FP32 accumulation). */
int claw2_mlp_infer(claw2_mlp* m, const float* x8, int n, float* y);
/* The tensor-core path of claw2_mlp_infer and of the exact solver's guess
 * pass: tcgen05.mma with TMEM accumulators (the default), or the warp-level
 * mma.sync form kept for comparison.  Both round operands to BF16 and
 * accumulate in FP32. */
enum { CLAW2_MLP_TCGEN05 = 0, CLAW2_MLP_MMA_SYNC = 1 };
int claw2_mlp_set_engine(claw2_mlp* m, int engine);
/* Exact-solver patches: start Newton from the network's guesses (NULL: the
 * adaptive PVRS guess); Newton updates and Riemann solves since the last reset. */
int claw2_patch_set_mlp(claw2_patch* p, claw2_mlp* m);
int claw2_patch_counters(claw2_patch* p, unsigned long long* iters_and_solves, int reset);
/* Newton counts since the last reset: out[0] steps needed (a final step below
 * the tolerance is applied but not counted), out[1] steps applied (the needed
 * ones plus that final step, for every interface whose two states differ),
 * out[2] Riemann solves. */
int claw2_patch_newton_counts(claw2_patch* p, unsigned long long* out, int reset);
/* Measurement aid for exact-solver patches (unsplit steps): mode 1 runs a
 * pre-pass before every step that solves each interface to the tolerance and
 * hands the converged p* to the step as its Newton guess, outside the
 * kernel timing (claw2_patch_kernel_ms): the step kernel's time with perfect
 * guesses, the floor for any guess.  Mode 0 (default) turns it off; the
 * device time loop ignores it. */
int claw2_patch_set_exact_guess(claw2_patch* p, int mode);
/* With mode 1 and rel > 0 (0 <= rel < 0.5): where the adaptive guess needs
 * Newton steps, start from the converged p* carrying a relative error of at
 * most rel (p* (1 + rel u), u in [-1, 1) fixed per interface), elsewhere
 * from the adaptive guess, so the step measures the most a guess of that
 * precision can save with the adaptive guess as fallback; 0 (default) keeps
 * the exact converged values everywhere. */
int claw2_patch_set_exact_guess_error(claw2_patch* p, double rel);

/* Description of the last error on this thread (never NULL). */
const char* claw2_last_error(void);

/* Library version string. */
const char* claw2_version(void);

#ifdef __cplusplus
}
#endif
#endif
