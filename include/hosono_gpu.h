/*
 * hosono_gpu.h -- C ABI of the B200 (sm_100a, FP64) time-step path of
 * hosono-2DMHD.
 *
 * The library replaces the reference's hot path behind its module
 * interfaces:
 *   cfl_computedt(blk, state)                 src/cfl.f90:14-52
 *   timeStep_advanceSolution(dt, blk, state)  src/timeStep.f90:22-43
 * and, inside it, reconstruct_faceValsWithGP (src/reconstruct.f90:18-175),
 * getFluxes_ (src/getFluxes.f90:16-90), riemannSolver_* (src/riemannSolver.f90),
 * FLICDdivB_fluxCorrections (src/FLICDdivB.f90:13-70), detect_ALL
 * (src/detect.f90:18-236), gridBlock_lowerOrder (src/gridBlock.f90:194-235),
 * boundaryConditions_applyBlk/applyMOOD (src/boundaryConditions.f90) and
 * timeStep_RK3/forwardEuler (src/timeStep.f90:45-171).
 *
 * All entry points are extern "C", take plain pointers and sizes, return an
 * int status (HOSONO_OK = 0) and never abort the process.  Host arrays use
 * the reference's Fortran order with guard cells:
 *     U(var=1..8, i=1..nx+2*NGC, j=1..ny+2*NGC), var fastest,
 *     V(var=1..10, i, j), scheme(i, j) (int).
 * One host thread per handle.
 */
#ifndef HOSONO_GPU_H
#define HOSONO_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define HOSONO_OK 0
#define HOSONO_EINVAL 1     /* bad argument (sizes, radius, boundary id)          */
#define HOSONO_ENOMEM 2     /* device allocation failed                           */
#define HOSONO_ECUDA 3      /* a CUDA call failed (message in last_error)         */
#define HOSONO_ENANDT 4     /* dt is NaN, infinite or negative (validTimeStep)    */
#define HOSONO_EMOODCAP 5   /* MOOD loop exceeded its pass cap                    */
#define HOSONO_ETIMEOUT 6   /* a bounded device wait gave up                      */
#define HOSONO_EPAR 7       /* .par file missing a key or holding a bad value     */
#define HOSONO_ENOTBUILT 8  /* library loaded without device code for this GPU    */
#define HOSONO_ECANCELED 9  /* served solve ended by the server's shutdown        */

/* boundary ids (sim_BC, src/simulation.f90:62) */
#define HOSONO_BC_OUTFLOW 0
#define HOSONO_BC_PERIODIC 1

/* arithmetic modes */
#define HOSONO_FP_STRICT 0  /* no FMA contraction: bit-identical to the oracle   */
#define HOSONO_FP_FAST 1    /* FMA contraction allowed                            */

/* POD copy of the run settings: sim_* of src/simulation.f90:9-31 and the
 * index/geometry fields of gridBlock_t (src/gridBlock.f90:36-45). */
typedef struct hosono_params {
    int nx, ny;            /* interior cells (grid_Nx, grid_Ny)                  */
    int ngc;               /* guard cells, must be max_radius + 2 (grid.f90:71)  */
    int max_radius;        /* GP_maxRadius, 1..3                                  */
    int bc;                /* HOSONO_BC_*                                         */
    int force_hydro;       /* sim_forceHydro                                      */
    int riemann_solver;    /* sim_riemannSolverID; 1 = HLLC-MHD                   */
    int fp_mode;           /* HOSONO_FP_*                                         */
    double dx, dy;         /* blk%dl                                              */
    double mindxdy, maxdxdy;
    double gamma;          /* sim_gamma                                           */
    double small_pressure, small_density, small_energy, small_b;
    double cfl;            /* sim_cfl                                             */
} hosono_params;

typedef struct hosono_handle hosono_handle;

/* Per-handle counters of the last advance (MOOD activity). */
typedef struct hosono_stats {
    int stages;            /* forward-Euler stages run                           */
    int mood_passes;       /* MOOD passes summed over the stages                  */
    int max_passes;        /* largest pass count of one stage                     */
    long long detect_lowered;  /* cells lowered by detect_ALL                      */
    long long inner_lowered;   /* cells lowered by the reconstruct face cascade    */
    int cascade_iters;     /* inner cascade iterations                            */
} hosono_stats;

/* ---------------------------------------------------------------- set-up */

/* GP_init (src/GP.f90:37-200): quad-precision GP prediction vectors and
 * quadrature weights, rounded to FP64.  Real inputs are decimal strings
 * parsed in quad precision like readParamFile_quadPrecisionReal
 * (src/readParamFile.f90:67-84).  Outputs in Fortran order:
 *   pv(nsMax, nqMax, 4, R), qw(nqMax, R), stenc(2, nsMax, R),
 * nsMax = 1+2R(R+1), nqMax = R+1. */
int hosono_gp_build(int max_radius, const char* x_beg, const char* x_end, int nx,
                    const char* y_beg, const char* y_end, int ny, const char* ell_over_delta,
                    double* pv, double* qw, int* stenc);
/* hosono_gp_build keeps the tables of the last 256 distinct (R, dx, dy, ell)
 * (the quad values it computes from its inputs) and returns them again for
 * the same values: the same bits as a fresh build, without the quad-precision
 * solve.  No counterpart in the reference (GP_init runs once per process). */
int hosono_gp_cache_info(long long* hits, long long* misses, int* entries);
int hosono_gp_cache_clear(void);

/* Run settings of a .par file that are not part of hosono_params. */
typedef struct hosono_run_info {
    double tmax;               /* sim_tmax                                      */
    int nstepmax;              /* sim_nstepmax                                  */
    int output_freq_step;      /* sim_outputFreqStep                            */
    double output_freq_time;   /* sim_outputFreqTime                            */
    double ell_over_delta;     /* GP_ellOverDelta                               */
    double x_beg, x_end, y_beg, y_end;  /* grid_xBeg .. grid_yEnd               */
    int nx_tot, ny_tot;        /* nx + 2*NGC, ny + 2*NGC (host array extents)   */
    char ic_type[32];          /* IC_type                                       */
    char data_file_base[256];  /* sim_dataFileBaseName                          */
} hosono_run_info;

/* simulation_init + grid_init (src/simulation.f90:35-78, src/grid.f90:31-103):
 * read a .par file (format of src/readParamFile.f90:1-9, first matching line
 * wins) into params and run settings.  fp_mode is set to HOSONO_FP_STRICT. */
int hosono_par_load(const char* parfile, hosono_params* p, hosono_run_info* run, char* err, int errlen);

/* GP_init from a .par file (grid_* and GP_* keys read in quad precision). */
int hosono_par_gp(const char* parfile, double* pv, double* qw, int* stenc, char* err, int errlen);

/* initialCondition_set (src/initialCondition.f90:23-84): fills U and V
 * (Fortran order, nx_tot*ny_tot cells, guards by the boundary condition).
 * IC types explosion2d, sedov2d, OrszagTang2d.  Optional keys beyond the
 * reference, whose defaults reproduce it: IC_B0 and IC_pres for
 * OrszagTang2d (default 1/gamma), IC_magx/IC_magy/IC_magz for explosion2d
 * (default 0). */
int hosono_ic_set(const char* parfile, const hosono_params* p, double* U, double* V, char* err, int errlen);

/* initialCondition_set for the device: a problem's initial state as a few
 * constants and per-row / per-column tables (the only libm terms, sines of
 * the Orszag-Tang state, are evaluated here on the host), from which
 * hosono_gpu_ic / hosono_batch_ic / hosono_serve_submit_ic build U and V on
 * the GPU with the same bits as hosono_ic_set (src/initialCondition.f90:
 * 86-226, then the boundary fill).  O(nx+ny) host work and transfer instead
 * of O(nx*ny).  xtab: 3*(nx+2*ngc) doubles, ytab: 2*(ny+2*ngc) doubles. */
#define HOSONO_IC_EXPLOSION 1   /* explosion2d (plus IC_magx/y/z) */
#define HOSONO_IC_SEDOV 2       /* sedov2d */
#define HOSONO_IC_ORSZAG_TANG 3 /* OrszagTang2d (plus IC_B0, IC_pres) */
typedef struct hosono_ic_desc {
    int type;    /* HOSONO_IC_* */
    int pad;
    double c[16]; /* the problem's constants (centre, radius, inside/outside states, ...) */
} hosono_ic_desc;
int hosono_ic_describe(const char* parfile, const hosono_params* p, hosono_ic_desc* ic, double* xtab, double* ytab,
                       char* err, int errlen);

/* ---------------------------------------------------------------- solver */

/* Allocate a device instance (gridBlock_t + gridState_t of grid.f90:88-89
 * and the GP tables of GP.f90:99-101).  pv/qw/stenc as produced by
 * hosono_gp_build.  The handle owns its device buffers and CUDA stream. */
int hosono_gpu_create(const hosono_params* p, const double* pv, const double* qw, const int* stenc,
                      hosono_handle** out);
int hosono_gpu_destroy(hosono_handle* h);

/* Host <-> device state (Fortran order, guards included).  V may be NULL
 * on upload (then V = cons2prim(U) on every cell).  Any download pointer
 * may be NULL. */
int hosono_gpu_upload(hosono_handle* h, const double* U, const double* V);
/* the initial state built on the device from hosono_ic_describe's output */
int hosono_gpu_ic(hosono_handle* h, const hosono_ic_desc* ic, const double* xtab, const double* ytab);
int hosono_gpu_download(hosono_handle* h, double* U, double* V, int* scheme);

/* cfl_computedt (src/cfl.f90:14-52) on the resident state. */
int hosono_gpu_cfl(hosono_handle* h, double* dt);

/* timeStep_advanceSolution (src/timeStep.f90:22-43) on the resident state. */
int hosono_gpu_advance(hosono_handle* h, double dt);

/* The mhd_driver time loop (src/mhd_driver.f90:76-95 with validTimeStep
 * :117-144) on the resident state, without output: steps until t >= tmax,
 * nstep >= nstepmax or max_steps steps (max_steps <= 0: no extra limit). */
int hosono_gpu_run(hosono_handle* h, double tmax, int nstepmax, int max_steps, double* t_out, int* nstep_out);

/* Set the instance's time-loop position (t, nstep) and limits (tmax, nstepmax). */
int hosono_gpu_set_time(hosono_handle* h, double t, double tmax, int nstep, int nstepmax);

/* MOOD pass cap.  The reference's forward-Euler MOOD loop
 * (src/timeStep.f90:86-128) has no limit; every pass that does not end it
 * lowers at least one cell by one order, so it ends after at most
 * R*nx*ny + 1 passes -- 8.4 M at 2048^2, R=2, which on a device that never
 * converged would spin for hours.  A stage that reaches `cap` passes without
 * converging stops its instance with HOSONO_EMOODCAP instead (the state
 * stays at the start of that step; other instances of a batch go on).
 * Default HOSONO_MOOD_CAP_DEFAULT(R, nx, ny) passes per stage: linear in the
 * grid's extent (a troubled region spreads by a few cells a pass), where the
 * proven bound is quadratic; a small multiple of R+1 is not enough (Orszag-
 * Tang 512^2, R=2, needs more than 48 passes in some stages once its shocks
 * form).  cap <= 0 restores the proven bound R*nx*ny + 1.  No counterpart in
 * the reference. */
#define HOSONO_MOOD_CAP_DEFAULT(R, nx, ny) (((R) + 1) * ((nx) + (ny)))
int hosono_gpu_set_mood_cap(hosono_handle* h, int cap);

/* Continue the driver's time loop from the current t/nstep: up to max_steps
 * steps of cfl_computedt + validTimeStep + timeStep_advanceSolution, each one
 * taken on the device without a host round trip (max_steps <= 0: to tmax). */
int hosono_gpu_step(hosono_handle* h, int max_steps, double* t_out, int* nstep_out);

/* Run the MOOD loops from a captured CUDA graph (on, the default) or from
 * host-driven launches (off; always the case while tracing). */
int hosono_gpu_set_graphs(hosono_handle* h, int on);

/* Drop-in with host buffers: upload U, advance by dt, download U (and V if
 * not NULL).  The form a Fortran caller that keeps grid_state on the host
 * binds (timeStep_advanceSolution with state%U/state%V).  V is output only:
 * like timeStep_advanceSolution, the step reads U and recomputes V from the
 * new U.  On large grids (hosono_tuning.upload_bands) U goes up in row bands
 * on a second stream, and the first stage's MOOD pass 1 computes each band's
 * tiles as soon as their rows and halo have landed, so the upload and that
 * kernel overlap; results are the same bits either way. */
int hosono_gpu_advance_host(hosono_handle* h, double dt, double* U, double* V);

int hosono_gpu_stats(hosono_handle* h, hosono_stats* s);

/* Copies the last error message into buf; returns its status code. */
int hosono_gpu_last_error(hosono_handle* h, char* buf, int len);

/* MOOD trace for parity tests: one record per MOOD pass.  meta[0..3] =
 * stage, pass, inner-cascade lowerings, detect lowerings; masks hold
 * per-cell lowering counts of that pass (nxTot*nyTot bytes, may be NULL). */
int hosono_gpu_trace_enable(hosono_handle* h, int on);
int hosono_gpu_trace_count(hosono_handle* h);
int hosono_gpu_trace_get(hosono_handle* h, int k, int* meta, unsigned char* inner_mask,
                         unsigned char* detect_mask);
int hosono_gpu_trace_clear(hosono_handle* h);

/* ------------------------------------------------------- stage modules
 * The reference's stage modules one at a time on the handle's block, for a
 * host that keeps its own forward-Euler MOOD loop (src/timeStep.f90:76-128)
 * and for unit parity of each module.  They work on the handle's module
 * state, the arrays of gridBlock_t (src/gridBlock.f90:51-88): scheme,
 * recompute, recomputeFLICD, faceVals, flux and fluxRaw, with U = the
 * resident state and Unew = the handle's stage buffer.  faceVals and flux
 * (8*nqMax*4 + 16 doubles a cell: 3.8 GB at 2048^2, R=2) are allocated on
 * the handle's first module call and freed with it; the fused time step
 * (hosono_gpu_advance / _step) never reads them, and it overwrites the flags,
 * fluxRaw and Unew.  Each call returns when its kernels are done.
 *
 * Host arrays in the reference's Fortran order with guard cells:
 *   scheme, recompute, recomputeFLICD: (nxTot, nyTot) int (logicals 0/1)
 *   faceVals (8, nqMax, 4, nxTot, nyTot), faces north, south, east, west
 *   fluxRaw, flux (8, 2, nxTot, nyTot); Unew (8, nxTot, nyTot)
 * Any pointer may be NULL (that array is left alone / not copied). */
int hosono_gpu_module_set(hosono_handle* h, const int* scheme, const int* recompute, const int* recompute_flicd);
int hosono_gpu_module_get(hosono_handle* h, double* faceVals, double* fluxRaw, double* flux, double* Unew,
                          int* scheme, int* recompute, int* recompute_flicd);
/* reconstruct_faceValsWithGP(blk, state%U) (src/reconstruct.f90:18-175):
 * faceVals of the recompute cells of [strt-2, stop+2]^2 at the EDP1 radius,
 * with the inner CAD/PAD cascade (failing cells lowered until every face
 * state is admissible) */
int hosono_gpu_reconstruct(hosono_handle* h);
/* getFluxes_(blk) (src/getFluxes.f90:16-90, riemannSolver_getFaceFlux
 * src/riemannSolver.f90:23-47): fluxRaw and flux of the faces next to a
 * recompute cell, on [strt-1, stop+2]^2 */
int hosono_gpu_getfluxes(hosono_handle* h);
/* FLICDdivB_fluxCorrections(blk) (src/FLICDdivB.f90:13-70) */
int hosono_gpu_flicd(hosono_handle* h);
/* the unsplit update of timeStep_forwardEuler (src/timeStep.f90:105-118):
 * Unew = U - dt/dx (F(i+1)-F(i)) - dt/dy (G(j+1)-G(j)) where recomputeFLICD */
int hosono_gpu_update(hosono_handle* h, double dt);
/* detect_ALL(blk, U, Unew, exit_mood_loop) (src/detect.f90:18-236) */
int hosono_gpu_detect(hosono_handle* h, int* exit_mood_loop);
/* boundaryConditions_applyBlk (src/boundaryConditions.f90:53-77) on the
 * resident U (which = 0), V (1) or Unew (2) */
int hosono_gpu_bc(hosono_handle* h, int which);
/* boundaryConditions_applyMOOD(blk) (src/boundaryConditions.f90:16-51) */
int hosono_gpu_bc_mood(hosono_handle* h);
/* MOOD activity of the last hosono_gpu_advance / _step: passes summed over
 * its stages, and troubled cells (lowerings by detect_ALL plus by the
 * reconstruct cascade) */
int hosono_gpu_mood_pass_stats(hosono_handle* h, int* npasses, long long* ntroubled);
/* riemannSolver_fromConsHllcMHD (src/riemannSolver.f90:68-221) on n faces
 * of caller-owned device arrays uL, uR, flux, each (8, n) (the 8 conserved
 * variables of a face together), direction 0 (x) or 1 (y), with the
 * handle's gamma, floors and sim_forceHydro; returns when flux is written */
int hosono_gpu_riemann(hosono_handle* h, int n, const double* uL_dev, const double* uR_dev, int dir, double* flux_dev);
/* eigen_vecsFromPrim (src/eigen.f90:20-255) on n primitive states of a
 * caller-owned device array V (10, n), direction 0 (x) or 1 (y): the left
 * and right eigenvectors of the 7 MHD waves into L and R, each (8, 8, n),
 * column w (1..7) = wave w, column 8 zero, in primitive variables
 * (cons = 0, 'prim') or conserved ones (cons = 1, 'cons'); the handle's
 * gamma floors and sim_smallB.  No .par option of the reference reaches this
 * routine (it is not on the time-step path). */
int hosono_gpu_eigenvecs(hosono_handle* h, int n, const double* V_dev, int dir, int cons, double* L_dev,
                         double* R_dev);

/* Device-resident access for callers that manage their own buffers
 * (benchmarks, batching): device pointer of the first U plane; planes are
 * pitch*nyTot doubles apart, rows pitch doubles apart. */
int hosono_gpu_state_layout(hosono_handle* h, double** U_dev, int* pitch, long long* plane);

/* Library identification: fills the compiled device architecture (e.g. 100
 * for sm_100a) and returns HOSONO_OK. */
int hosono_gpu_build_info(int* sm_arch, int* has_fast_mode);

/* Select the CUDA device for handles created afterwards on this thread. */
int hosono_gpu_set_device(int device);

/* The cudaStream_t every kernel of this handle runs on (for events). */
int hosono_gpu_stream(hosono_handle* h, void** stream);

/* Launch choices of the time-step kernels (no counterpart in the reference,
 * whose loops are OpenMP regions).  Results do not depend on them: every
 * choice gives the same bits.  Setting them rebuilds the handle's step
 * graphs on the next step.  A new handle or batch starts with TMA staging,
 * the dynamic schedule, two blocks per SM and one box per block (the fastest
 * choice on the 2048^2 Orszag-Tang and Sedov workloads). */
#define HOSONO_STAGE_CP_ASYNC 0  /* pass-1 stencil box staged by per-thread cp.async copies */
#define HOSONO_STAGE_TMA 1       /* ... by one TMA tensor copy (cp.async.bulk.tensor) per box */
#define HOSONO_SCHED_STATIC 0    /* pass-1 blocks walk the tile list grid-stride */
#define HOSONO_SCHED_DYNAMIC 1   /* ... take their next tile from a launch-wide counter */
#define HOSONO_LATER_KERNELS 0     /* later MOOD passes: a chain of kernels per pass (graph nodes) */
#define HOSONO_LATER_PERSISTENT 1  /* ... all of a stage's later passes in one persistent launch */
typedef struct hosono_tuning {
    int pass1_staging;        /* HOSONO_STAGE_* */
    int pass1_schedule;       /* HOSONO_SCHED_* */
    int pass1_blocks_per_sm;  /* resident pass-1 blocks per SM the register budget aims at: 2 (0 = 2;
                                 128 registers), 3 or 4 (80 / 64 registers, one stencil box per
                                 block, cp.async staging only) */
    int later_passes;         /* HOSONO_LATER_*; the autotuner keeps the caller's choice */
    int pass1_boxes;          /* stencil boxes per pass-1 block at two blocks per SM: 1 (0 = 1; load,
                                 compute, load the next; the shared memory saved goes to L1) or 2 (the
                                 next tile's box loads while the current one is computed) */
    int upload_bands;         /* hosono_gpu_advance_host: row bands of the overlapped upload (0 = by size:
                                 16 from 2048 array rows, 8 from 1024, else 1; 1 = upload, then step;
                                 at most HOSONO_UPLOAD_BANDS_MAX) */
    int pdl;                  /* 1: the step's kernels are launched as programmatic dependent launches
                                 (each may be scheduled while its predecessor drains and waits on
                                 the GPU for its completion); 0: plain stream order */
    int update_staging;       /* the pass-1 update (FLICD, update, detect): HOSONO_STAGE_CP_ASYNC (0) reads
                                 the planes through the caches, HOSONO_STAGE_TMA (1) stages the tile's
                                 boxes of U, FX and FY in shared memory with TMA copies first */
} hosono_tuning;
#define HOSONO_UPLOAD_BANDS_MAX 16
int hosono_gpu_set_tuning(hosono_handle* h, const hosono_tuning* t);
int hosono_gpu_get_tuning(hosono_handle* h, hosono_tuning* t);

/* Autotuner.  Times every candidate hosono_tuning on the instances the
 * handle or batch holds now -- `trials` launches of the MOOD pass-1 kernels
 * (83 % of a time step; they only write scratch that every stage rewrites,
 * so the solution is untouched) per candidate, after one untimed launch --
 * and applies the fastest.  The choice is kept in a process-wide cache keyed
 * by (arithmetic mode, GP radii present, size class = floor(log2(interior
 * cells)), floor(log2(instances))); a later call with the same key applies
 * the cached choice without timing unless `force` is set. */
#define HOSONO_TUNE_MAX 12
typedef struct hosono_tune_report {
    int candidates;                    /* entries of tried/ms filled                  */
    int cached;                        /* 1: taken from the cache, nothing was timed  */
    int size_class, instances;         /* the cache key's size class; instances held  */
    hosono_tuning tried[HOSONO_TUNE_MAX];
    double ms[HOSONO_TUNE_MAX];        /* mean ms of one pass-1 launch (all radii)    */
    hosono_tuning best;
} hosono_tune_report;
int hosono_gpu_autotune(hosono_handle* h, int trials, int force, hosono_tune_report* report);

/* Launch geometry of the handle's kernels: every per-tile kernel walks the
 * tile list grid-stride with a grid sized to the GPU, so a grid smaller than
 * `tiles` makes each block take several tiles in turn.  No counterpart in
 * the reference (its loops are OpenMP regions). */
typedef struct hosono_launch_info {
    int tiles;          /* 32x8 cell tiles of the instance, guard cells included */
    int sms;            /* multiprocessors of the device                          */
    int pass1_grid;     /* blocks of the MOOD pass-1 kernel (radius R)            */
    int tile_grid_max;  /* the largest grid of the other per-tile kernels          */
} hosono_launch_info;
int hosono_gpu_launch_info(hosono_handle* h, hosono_launch_info* info);

/* ---------------------------------------------------------------- batches
 * Many independent blocks (any sizes, radii, boundary conditions, problems)
 * advanced together: every kernel launch covers all instances' tiles, each
 * instance keeps its own t, dt (its own cfl_computedt), MOOD loop and time
 * limits, and hosono_batch_run takes them all to their tmax in one graph
 * launch.  Instances can be added and removed between runs (continuous
 * batching); capacity is fixed at creation in slots and 32x8 tiles. */
typedef struct hosono_batch hosono_batch;

int hosono_batch_create(int max_instances, int max_tiles, int fp_mode, hosono_batch** out);
int hosono_batch_destroy(hosono_batch* b);
/* tiles and device bytes one instance with these parameters needs */
int hosono_batch_tiles_for(const hosono_params* p);
long long hosono_batch_instance_bytes(const hosono_params* p);
int hosono_batch_add(hosono_batch* b, const hosono_params* p, const double* pv, const double* qw, const int* stenc,
                     int* slot);
int hosono_batch_remove(hosono_batch* b, int slot);
int hosono_batch_upload(hosono_batch* b, int slot, const double* U, const double* V);
int hosono_batch_ic(hosono_batch* b, int slot, const hosono_ic_desc* ic, const double* xtab, const double* ytab);
int hosono_batch_download(hosono_batch* b, int slot, double* U, double* V, int* scheme);
int hosono_batch_set_time(hosono_batch* b, int slot, double t, double tmax, int nstep, int nstepmax);
int hosono_batch_set_tuning(hosono_batch* b, const hosono_tuning* t);
int hosono_batch_get_tuning(hosono_batch* b, hosono_tuning* t);
int hosono_batch_autotune(hosono_batch* b, int trials, int force, hosono_tune_report* report);
/* hosono_gpu_set_mood_cap for one instance of the batch */
int hosono_batch_set_mood_cap(hosono_batch* b, int slot, int cap);
/* every live, unfinished instance steps until its tmax/nstepmax, or at most
 * max_steps steps (max_steps <= 0: no limit) */
int hosono_batch_run(hosono_batch* b, int max_steps);
int hosono_batch_status(hosono_batch* b, int slot, double* t, double* dt, int* nstep, int* done, int* error);
/* cumulative MOOD counters of one instance */
int hosono_batch_stats(hosono_batch* b, int slot, hosono_stats* s);
int hosono_batch_stream(hosono_batch* b, void** stream);
int hosono_batch_set_graphs(hosono_batch* b, int on);
int hosono_batch_last_error(hosono_batch* b, char* buf, int len);
int hosono_batch_capacity(hosono_batch* b, int* max_instances, int* max_tiles, int* used_tiles, int* live);

/* CFL time step that allocates nothing.  No counterpart in the reference:
 * it exists for callers that cannot call cudaMalloc when they need dt (code
 * inside a CUDA stream capture, where allocation fails; hosts whose device
 * memory is wholly owned by their own pool allocator; loops that must not
 * enter the allocator, which may synchronise the device).
 * Computes dt = cfl * min(dx/max(|u|+c_f), dy/max(|v|+c_f)) over the interior
 * of a caller-owned device V (10 SoA planes, rows `pitch` doubles apart,
 * planes `plane` doubles apart, ngc guard cells; the layout of the handle's
 * own V) and writes it to the caller-owned device double *dt_dev, on
 * `stream` (NULL = default stream).  Result equal to hosono_gpu_cfl's on an
 * HOSONO_FP_STRICT handle (this entry point is built without FMA contraction;
 * a HOSONO_FP_FAST handle's dt may differ in the last bits).
 * Scratch: a file-scope device array of 2*HOSONO_NOALLOC_MAX_ROWS doubles
 * (256 KiB) per GPU, held until process exit; ny > HOSONO_NOALLOC_MAX_ROWS
 * returns HOSONO_EINVAL.  All calls on a device share that array, so calls
 * whose kernels overlap on the GPU race.  Every call outside a stream capture
 * looks up the array's address afresh (so it survives a cudaDeviceReset);
 * calls inside a capture reuse the last address found, so make the first
 * call on each device before any stream capture (a first call inside one
 * returns HOSONO_EINVAL).  Only this call's own launch errors are returned;
 * an earlier error pending on the thread is left as it was. */
#define HOSONO_NOALLOC_MAX_ROWS 16384
int hosono_cfl_noalloc(const double* V_dev, int nx, int ny, int ngc, int pitch, long long plane, double dx, double dy,
                       double cfl, int force_hydro, double* dt_dev, void* stream);

/* The derived fields output_writeHdf5 writes (src/output.f90:230-274),
 * computed on the device from the resident state for the interior cells, in
 * the HDF5 datasets' order (nx*ny, x fastest): `fields` holds 13 planes --
 * dens velx vely velz pres eint gama ener magp divb magx magy magz --, and
 * `scheme`, `ordr` (= 2*scheme+1) one int plane each; any of them may be
 * NULL.  divb_l1 = mean |div B| and divb_linf = max |div B| over the interior
 * (same bits on every call).  Allocates and frees device scratch. */
int hosono_gpu_diagnostics(hosono_handle* h, double* fields, int* scheme, int* ordr, double* divb_l1,
                           double* divb_linf);
int hosono_batch_diagnostics(hosono_batch* b, int slot, double* fields, int* scheme, int* ordr, double* divb_l1,
                             double* divb_linf);

/* Kernel timing: when on, CUDA events bracket every launch of the MOOD
 * pass-1 kernel; times[0] = summed milliseconds, counts[0] = launches since
 * the last reset.  launches = kernels launched by this handle since reset. */
int hosono_gpu_profile(hosono_handle* h, int on);
int hosono_gpu_profile_read(hosono_handle* h, double* pass1_ms, long long* pass1_launches, long long* launches,
                            int reset);

/* ---------------------------------------------------------------- serving
 * No counterpart in the reference, which runs one solve per process.  A
 * server owns one batch on the current GPU and a scheduler thread.  Solves
 * are submitted at any time from any thread and wait in a queue.  A queued
 * solve is admitted (in the order of the server's policy, HOSONO_SERVE_*)
 * when an instance slot, tile capacity and a
 * free range of the server's device-memory budget are available: the budget
 * is one device allocation made at start-up, so admission and retirement
 * never call cudaMalloc.  An admitted solve advances with every other
 * resident solve in the same batched launches (continuous batching), each at
 * its own dt, until its tmax or nstepmax; then its final state is copied to
 * the caller's buffers and its memory returns to the budget.  A solve's
 * result does not depend on what else is resident.  Between launches the
 * scheduler admits, retires and serves snapshots. */
typedef struct hosono_server hosono_server;

/* Scheduling policies.  FIFO: the queue head is admitted first and every
 * resident solve takes every time step of every launch.  SHORTEST: queued
 * solves are admitted shortest estimated work first (interior cells x
 * tmax / min(dx, dy); a solve that does not fit is passed over), and each
 * launch steps the resident solves with the least estimated remaining work
 * (cells x (tmax - t) / dt) until they cover fill_tiles tiles, while the
 * others sit out that launch with their state untouched; any solve that has
 * waited (queued or sitting out) for aging_s seconds goes first.  A solve's
 * result is the same bits under either policy. */
#define HOSONO_SERVE_FIFO 0
#define HOSONO_SERVE_SHORTEST 1
typedef struct hosono_serve_config {
    long long memory_budget; /* device bytes for resident solves; <= 0: 55% of free memory  */
    int max_resident;        /* instance slots; <= 0: 1024                                  */
    int fp_mode;             /* HOSONO_FP_*                                                 */
    double chunk_ms;         /* target GPU time of one batched launch; <= 0: 25 ms          */
    int max_chunk_steps;     /* time steps per batched launch at most; <= 0: 64             */
    int policy;              /* HOSONO_SERVE_*                                              */
    double aging_s;          /* SHORTEST: wait after which a solve goes first; <= 0: 5 s     */
    int fill_tiles;          /* SHORTEST: tiles a launch steps at least; <= 0: 40 per SM    */
    int pad;
} hosono_serve_config;

#define HOSONO_REQ_QUEUED 0
#define HOSONO_REQ_RUNNING 1
#define HOSONO_REQ_DONE 2

typedef struct hosono_request_info {
    long long id;
    int state;                /* HOSONO_REQ_*                                                */
    int status;               /* HOSONO_OK, or what ended it (ENANDT, EMOODCAP, ECANCELED...) */
    int nstep;                /* time steps taken                                            */
    int slot;                 /* batch slot while resident, else -1                          */
    double t;                 /* simulation time reached                                     */
    long long zone_updates;   /* nx*ny*nstep                                                 */
    long long device_bytes;   /* budget bytes held while resident                            */
    double submit_s, admit_s, finish_s; /* hosono_serve_clock() at each event; 0 = not yet    */
    hosono_stats mood;        /* MOOD counters over the solve                                */
} hosono_request_info;

typedef struct hosono_serve_totals {
    long long submitted, completed, failed, queued, resident;
    long long zone_updates;   /* of completed solves                                         */
    long long chunks, steps;  /* batched launches; batch time steps                          */
    long long peak_resident;
    long long budget_bytes, used_bytes, peak_bytes;
    long long head_blocked;   /* admission rounds that stopped at a head that did not fit    */
    double busy_s;            /* wall time inside batched launches                           */
    double admin_s;           /* wall time admitting, retiring and snapshotting              */
} hosono_serve_totals;

/* seconds on the server clock (steady, shared by all servers of the process) */
double hosono_serve_clock(void);
int hosono_serve_create(const hosono_serve_config* cfg, hosono_server** out);
/* stops the scheduler after its current launch; queued and resident solves
 * end with HOSONO_ECANCELED.  Threads blocked in hosono_serve_wait, _drain
 * or _snapshot on this server return before it is freed; no other call on
 * it may overlap this one. */
int hosono_serve_destroy(hosono_server* s);
/* Queue one solve: parameters, GP tables (as hosono_gpu_create), the initial
 * U and V (host, Fortran order with guards, as initialCondition_set leaves
 * them; copied, so they may be freed on return; V may be NULL: then
 * V = cons2prim(U) on the device, as hosono_gpu_upload), its tmax and
 * nstepmax.  U_out (8 doubles/cell), V_out (10) and scheme_out
 * (int) are filled with the final state when the solve ends; each may be
 * NULL and must stay valid until hosono_serve_wait/poll reports the solve
 * done.  A solve larger than the whole budget or the tile capacity is
 * refused with HOSONO_ENOMEM. */
int hosono_serve_submit(hosono_server* s, const hosono_params* p, const double* pv, const double* qw, const int* stenc,
                        const double* U, const double* V, double tmax, int nstepmax, double* U_out, double* V_out,
                        int* scheme_out, long long* id);
/* the same with the initial state described by hosono_ic_describe (tables
 * copied): the server builds it on the device at admission */
int hosono_serve_submit_ic(hosono_server* s, const hosono_params* p, const double* pv, const double* qw,
                           const int* stenc, const hosono_ic_desc* ic, const double* xtab, const double* ytab,
                           double tmax, int nstepmax, double* U_out, double* V_out, int* scheme_out, long long* id);
/* block until the solve is done (HOSONO_ETIMEOUT after timeout_s; < 0: no limit) */
int hosono_serve_wait(hosono_server* s, long long id, double timeout_s, hosono_request_info* info);
/* Forget a finished solve: its id becomes unknown to wait/info.  The server
 * keeps the record of every solve (its info) until this call or the
 * server's end, one entry per submitted solve; a long-running server's
 * callers release each solve once they have read its result. */
int hosono_serve_release(hosono_server* s, long long id);
/* ids of solves finished since the last poll (up to cap) */
int hosono_serve_poll(hosono_server* s, long long* ids, int cap, int* n);
int hosono_serve_info(hosono_server* s, long long id, hosono_request_info* info);
/* current state of a resident solve, taken between batched launches */
int hosono_serve_snapshot(hosono_server* s, long long id, double* U, double* V, int* scheme, double* t, int* nstep);
/* block until no solve is queued or resident (HOSONO_ETIMEOUT after timeout_s) */
int hosono_serve_drain(hosono_server* s, double timeout_s);
int hosono_serve_stats(hosono_server* s, hosono_serve_totals* st);
int hosono_serve_last_error(hosono_server* s, char* buf, int len);

#ifdef __cplusplus
}
#endif
#endif
