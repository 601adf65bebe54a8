/*
 * hosono_oracle.h -- C interface of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is a line-by-line CPU restatement of
 * the hosono-2DMHD Fortran time-step path (src/timeStep.f90, reconstruct.f90,
 * getFluxes.f90, riemannSolver.f90, FLICDdivB.f90, detect.f90, cfl.f90,
 * boundaryConditions.f90, GP.f90, ...).  It is the checker that the CUDA
 * path is compared against.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it; the product library never does.
 *
 * Arrays crossing this interface use the reference's Fortran order, guard
 * cells included:  U(var=1..8, i=1..nx+2*NGC, j=1..ny+2*NGC)  with var
 * fastest, i.e. element (v,i,j) (1-based) sits at
 *     (v-1) + nvar*((i-1) + nxTot*(j-1)).
 */
#ifndef HOSONO_ORACLE_H
#define HOSONO_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_handle orc_handle;

/* Build an instance from a .par file (simulation_init + GP_init + grid_init
 * + initialCondition_set of mhd_driver.f90:40-58).  Returns NULL on error
 * and writes a message into err. */
orc_handle* orc_create_from_par(const char* parfile, char* err, int errlen);
void orc_destroy(orc_handle* h);

/* ints[0..9]  = nx, ny, NGC, R, nxTot, nyTot, nqMax, nsMax, bc(0 outflow,1 periodic), forceHydro
 * dbls[0..9]  = dx, dy, mindxdy, maxdxdy, gamma, cfl, tmax, smallPressure, smallDensity, ellOverDelta */
int orc_info(const orc_handle* h, int* ints, double* dbls);

/* GP tables in Fortran order: pv(nsMax,nqMax,4,R), qw(nqMax,R), stenc(2,nsMax,R) */
int orc_get_gp(const orc_handle* h, double* pv, double* qw, int* stenc);

int orc_get_U(const orc_handle* h, double* U);
int orc_get_V(const orc_handle* h, double* V);
int orc_set_U(orc_handle* h, const double* U);
int orc_set_V(orc_handle* h, const double* V);
int orc_get_scheme(const orc_handle* h, int* scheme);

/* cfl_computedt (cfl.f90:14-52) */
double orc_cfl(const orc_handle* h);
/* timeStep_advanceSolution (timeStep.f90:22-43) */
int orc_advance(orc_handle* h, double dt);
/* mhd_driver main loop (mhd_driver.f90:64-95) without output; stops after
 * max_steps steps (<=0: no extra limit).  Returns 0 or a nonzero status. */
int orc_run(orc_handle* h, int max_steps, double* t_out, int* nstep_out);

/* reconstruct_faceValsWithGP on every cell at one radius (the set-up of
 * test/test_reconstruct_faceValsWithGP.f90:31-34).  faceVals in Fortran
 * order (8, nqMax, 4, nxTot, nyTot). */
int orc_reconstruct_all(orc_handle* h, int radius, double* faceVals);

/* The stage modules one at a time on the instance's block, for unit parity
 * of the CUDA library's per-module entry points.  Arrays in the reference's
 * Fortran order: scheme/recompute/recomputeFLICD (nxTot, nyTot) (logicals as
 * 0/1 ints), faceVals (8, nqMax, 4, nxTot, nyTot), fluxRaw/flux (8, 2, nxTot,
 * nyTot), Unew like U.  NULL arguments are skipped.
 *   orc_mod_reconstruct  reconstruct_faceValsWithGP(blk, U)  reconstruct.f90:18-175
 *   orc_mod_getfluxes    getFluxes_(blk)                     getFluxes.f90:16-90
 *   orc_mod_flicd        FLICDdivB_fluxCorrections(blk)      FLICDdivB.f90:13-70
 *   orc_mod_update       Unew where recomputeFLICD           timeStep.f90:105-118
 *   orc_mod_detect       detect_ALL(blk, U, Unew, exit)      detect.f90:18-236; returns exit_mood_loop
 *   orc_mod_bc           boundaryConditions_applyBlk on U (0), V (1), Unew (2)
 *   orc_mod_bc_mood      boundaryConditions_applyMOOD(blk)   boundaryConditions.f90:16-51 */
int orc_mod_set(orc_handle* h, const int* scheme, const int* recompute, const int* recomputeFLICD);
int orc_mod_get(orc_handle* h, double* faceVals, double* fluxRaw, double* flux, double* Unew, int* scheme,
                int* recompute, int* recomputeFLICD);
int orc_mod_reconstruct(orc_handle* h);
int orc_mod_getfluxes(orc_handle* h);
int orc_mod_flicd(orc_handle* h);
int orc_mod_update(orc_handle* h, double dt);
int orc_mod_detect(orc_handle* h);
int orc_mod_bc(orc_handle* h, int which);
int orc_mod_bc_mood(orc_handle* h);

/* MOOD trace: one record per MOOD pass of every forward-Euler stage. */
int orc_trace_enable(orc_handle* h, int on);
int orc_trace_count(const orc_handle* h);
/* meta[0..3] = stage index (counted from the first traced stage), pass,
 *              cells lowered by the inner face cascade, cells lowered by
 *              detect.  Masks (nxTot*nyTot bytes, may be NULL) count
 *              lowerings per cell in that pass. */
int orc_trace_get(const orc_handle* h, int k, int* meta,
                  unsigned char* inner_mask, unsigned char* detect_mask);
void orc_trace_clear(orc_handle* h);

/* Pointwise physics on one state, with the instance's parameters. */
void orc_cons2prim(const orc_handle* h, const double* U, double* V);
double orc_cons2pres(const orc_handle* h, const double* U);
void orc_cons2flux(const orc_handle* h, const double* U, int dir, double* F);
void orc_hllc(const orc_handle* h, const double* uL, const double* uR, int dir, double* F);
double orc_c_fs(double gam, double rho, double p, double BB, double BN, double pm);
/* eigen_vecsFromPrim (eigen.f90:20-255): left (L) and right (R) eigenvectors
 * of the 7 MHD waves of the primitive state V(10) in direction dir (0 x, 1 y),
 * each 8x8 column-major (column = wave 1..7, column 8 zero); cons != 0: in
 * conserved variables ('cons'), else primitive ('prim'). */
void orc_eigenvecs(const orc_handle* h, const double* V, int dir, int cons, double* L, double* R);

/* Standalone GP set-up (GP.f90:37-200) for given par strings.
 * Real values are passed as decimal strings and parsed in quad precision,
 * as readParamFile_quadPrecisionReal does. */
int orc_gp_build(int R, const char* x_beg, const char* x_end, int nx,
                 const char* y_beg, const char* y_end, int ny,
                 const char* ell_over_delta,
                 double* pv, double* qw, int* stenc);

/* Number of OpenMP threads the oracle uses (0 = runtime default). */
void orc_set_threads(int n);
int orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
