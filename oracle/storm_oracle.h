/*
 * storm_oracle.h -- CPU FP64 oracle for the SToRM FVT time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * Fortran (scharlton2/storm, Source_xsy-64bit/) routines on the solverFVT path,
 * written routine by routine with the reference file:line each follows.  It is
 * the checker for the CUDA library, never part of it: only tests/, the smoke
 * check and bench.py's CPU-baseline leg load it.
 *
 * Parity status: the reference publishes no numeric golden vectors (its only
 * test, tests/Tutorial_1, checks the exit code) and no Fortran compiler exists
 * on the build or GPU machines, so numeric parity is UNPINNED against a reference
 * run.  The topology builders are pinned against the counts of the reference's
 * own Tutorial_1 fixture (.edge/.v.edge files).
 */
#ifndef STORM_ORACLE_H
#define STORM_ORACLE_H

#include "../include/storm_fvt.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc orc_t;

/* Build the prepared mesh (read_data topology + dataprepFVT).  Returns 0 or a
 * negative code; the message is in orc_last_error(). */
int orc_create(const StormFvtProblem* prob, const StormFvtOptions* opt, orc_t** out);
void orc_destroy(orc_t* o);
const char* orc_last_error(void);

/* View of the prepared mesh in the StormFvtMesh layout (pointers into `o`). */
int orc_export_mesh(const orc_t* o, StormFvtMesh* m);

/* Number of OpenMP threads used by the cell/node/edge loops (1 = serial).  The
 * results are bitwise identical for every thread count. */
void orc_set_threads(orc_t* o, int n);

int orc_set_state(orc_t* o, const double* h, const double* u, const double* v);
int orc_step(orc_t* o, int nsteps, StormFvtStepStats* st);
int orc_get_state(const orc_t* o, double* h, double* u, double* v, double* rkh,
                  double* rku, double* rkv, double* hvtx);
/* drycell as find_dry_cells would set it for the next stage (int32 0/1). */
int orc_get_drycell(orc_t* o, int32_t* dry);

/* The output step of solverFVT (to_vertices, ctr2vtx(cd), error_est(2)) after the
 * last completed iteration; zeroes u,v of wet cells with a dry vertex as the reference
 * does.  Output pointers may be NULL. */
int orc_output_vertices(orc_t* o, const StormFvtOutputBoundary* ob, int in_loop, double* hvtx, double* uvtx,
                        double* vvtx, double* cdvtx, double* e_est);

/* Debug hooks: run only the first `upto` phases of one RK stage (rkstep) from the
 * current state and copy out intermediates.  Phases: 1 = dry cells, 2 = gradients
 * + hgradfix2, 3 = to_vertices, 4 = fluxes + bed slope.  Pointers may be NULL.
 * The state is left untouched (the stage works on copies). */
int orc_stage_probe(orc_t* o, int rkstep, int upto, int32_t* dry, double* grads6,
                    double* uv2, double* hvtx, double* phi3);

/* One iteration of orc_step in steps, for one part of a mesh split over processes
 * (the caller exchanges halo values and reduces dt and sums between the calls):
 * orc_iter_begin (level copy, this part's CFL dt), orc_iter_set_dt (the global dt),
 * orc_iter_stage for each RK stage, orc_iter_fric (friction with the whole mesh's
 * friction dt, this part's sums over its owned elements), orc_iter_finish (scalars
 * and stop test from the sums of all parts).  orc_get_level / orc_put_level move h,
 * u, v and one RK level ([6][n] blocks). */
int orc_iter_begin(orc_t* o, double* dt_local);
void orc_iter_set_dt(orc_t* o, double delt);
int orc_iter_stage(orc_t* o, int rkstep, double* delt_out, int* bad);
int orc_iter_fric(orc_t* o, double delt, const uint8_t* owned, double* sums);
int orc_iter_finish(orc_t* o, const double* sums, StormFvtStepStats* st);
int orc_get_level(const orc_t* o, int level, double* out6);
int orc_put_level(orc_t* o, int level, int32_t n, const int32_t* elems, const double* in6);
void orc_set_bch_max(orc_t* o, double v);
double orc_get_bch_max(const orc_t* o);

#ifdef __cplusplus
}
#endif
#endif
