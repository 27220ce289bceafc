/*
 * storm_fvt.h -- C-ABI of the B200 finite-volume (FVT) time step for SToRM.
 *
 * This library replaces one call of the SToRM Fortran program:
 *
 *     CALL solverFVT(iter,ttime,rmax,fn,title)      Source_xsy-64bit/solver.f90:57
 *
 * whose body is Source_xsy-64bit/solverFVT.f90:129-478 (the SSP-RK loop and the
 * ~45 routines it calls).  The Fortran host keeps mesh/option input, boundary
 * set-up (read_data, dataprepFVT) and output; at the call site it passes the
 * module arrays it already holds (geometry, dep_vars, options, vbc_arrays) through
 * the StormFvtMesh struct below, then steps the solution on the GPU.
 *
 * Conventions (identical to the Fortran module arrays, so a BIND(C) shim can pass
 * them unchanged):
 *   - node, element and edge ids are 1-based INTEGER(4);
 *   - 2-D arrays are column-major with the leading dimension stated per field;
 *   - LOGICAL(4) arrays are int32 (0 = .FALSE., non-zero = .TRUE.);
 *   - every real is REAL(KIND=8).
 *
 * Every entry point returns 0 on success or a negative STORM_ERR_* code; the
 * message of the most recent failure on the calling thread is returned by
 * storm_fvt_last_error().  Device-side checks (non-finite depth, a bounded wait
 * that ran out) are reported by the next call on the handle.
 *
 * Threading: one handle may be used by one host thread at a time; each handle owns
 * one CUDA stream on the device named in StormFvtOptions.device.
 */
#ifndef STORM_FVT_H
#define STORM_FVT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define STORM_FVT_ABI_VERSION 2

#if defined(__GNUC__)
#define STORM_FVT_API __attribute__((visibility("default")))
#else
#define STORM_FVT_API
#endif

/* ---- status codes ------------------------------------------------------- */
enum {
  STORM_OK = 0,
  STORM_ERR_ARG = -1,         /* invalid argument or option value              */
  STORM_ERR_MESH = -2,        /* mesh/boundary data inconsistent (byebye cases)*/
  STORM_ERR_CUDA = -3,        /* CUDA runtime error                            */
  STORM_ERR_NOMEM = -4,       /* host or device allocation failed              */
  STORM_ERR_DEVICE = -5,      /* device-side check tripped (see message)       */
  STORM_ERR_UNSUPPORTED = -6  /* option not implemented by this library         */
};

/* ---- choices ------------------------------------------------------------ */
enum { STORM_FLUX_ROE = 0, STORM_FLUX_HLL = 1, STORM_FLUX_RUSANOV = 2 };
enum { STORM_PREC_FP64 = 0, STORM_PREC_MIXED = 1 };

/*
 * Solver options: the fields of MODULE options (Source_xsy-64bit/options.f90) that
 * solverFVT reads, with the defaults of initialize_options.f90:23-141 listed.
 * `flux` and `precision` have no counterpart in the reference (it hard-wires Roe,
 * invisc_fluxes.f90:137, and FP64).
 */
typedef struct StormFvtOptions {
  double h_dry;        /* dry threshold, default 0.001            (options.f90:39) */
  double h_wet;        /* wet threshold = coef*h_dry, default h_dry                */
  double cfl;          /* CFL number; with steady=0 and dt_op=0 it is dt in s     */
  double vceiling;     /* velocity clip ceiling, default 35                       */
  double rstop;        /* steady stop threshold on rmax                            */
  double visc;         /* kinematic viscosity (opt_friction 3), viscosity(18 C)   */
  int32_t steady;      /* 1 = local-time-step pseudo-time march (default 1)       */
  int32_t dt_op;       /* unsteady: 0 = fixed dt (=cfl), 1 = CFL dt reduction     */
  int32_t rkorder;     /* 1, 2 or 3 (SSP-RK), default 2                           */
  int32_t opt_limiter; /* 0 = zero gradients, 1 = LSQ, 2 = LSQ + Barth-Jespersen   */
  int32_t btype;       /* walls: 0 = no-slip (wenslp3), 1 = slip (weslp2)          */
  int32_t hvalve;      /* numerical valve at stage boundaries, default 1           */
  int32_t vclip;       /* velocity clipping, default 0                             */
  int32_t opt_friction;/* 0 Manning, 1 Chezy, 2 drag, 3 Colebrook, 4 Strickler     */
  int32_t stop_cr;     /* steady stop criterion: 0 max|phi|, 1 RMS relative dh     */
  int32_t flux;        /* interior-edge flux: STORM_FLUX_ROE|HLL|RUSANOV           */
  int32_t precision;   /* STORM_PREC_FP64, or STORM_PREC_MIXED (FP32 gradient, flux
                          and source arithmetic; FP64 state, reconstruction, mass)  */
  int32_t device;      /* CUDA device ordinal                                      */
  int32_t rsavg_passes;/* residual smoothing (activateRSAVG, solverFVT.f90:238-256):
                          Gauss-Seidel passes nRSAVG, 0 = off (the default)        */
  int32_t rsavg_order; /* 0: cells in index order, as the reference (oracle only);
                          1: by colour of the smoothing stencil (a documented
                          variant: same steady state, parallel on the GPU)         */
  double rsavg_eps;    /* epsRSAVG, 0 < eps <= 1                                   */
  int32_t reserved[2]; /* must be zero                                             */
} StormFvtOptions;

/* Fill `opt` with the defaults of initialize_options.f90:23-141 (+ ROE, FP64). */
STORM_FVT_API void storm_fvt_default_options(StormFvtOptions* opt);

/*
 * One boundary-condition node string (ioflow.f90 / read_cgns.f90:433-552 input):
 *   inflow  strings: type = vtype (1 = Q by depth, 4 = stage, 5 = Q by depth on wet
 *                    cells only); value = qin (m^3/s) or inflow stage (vtype 4);
 *   outflow strings: type = htype (0 = free, 1 = stage, 2 = critical); value = hbc.
 * A time series (n_series > 0) replaces `value` through get_time_bcs
 * (get_time_bcs.f90:31-77).
 */
typedef struct StormFvtBoundary {
  int32_t type;
  int32_t n_nodes;
  const int32_t* nodes;      /* [n_nodes], 1-based, consecutive nodes share an edge */
  double value;
  int32_t n_series;
  const double* series_t;    /* [n_series] times (s), increasing                  */
  const double* series_v;    /* [n_series] values                                  */
} StormFvtBoundary;

/*
 * Raw problem description, the input of read_data (mesh, bed, roughness, BC
 * strings).  storm_fvt_mesh_build() turns it into the prepared StormFvtMesh the
 * way find_edges / t_areas / walls / ibc_arrays / node_db / elemnt_db and
 * dataprepFVT do.  Callers that already hold the Fortran module arrays skip it.
 */
typedef struct StormFvtProblem {
  int32_t n_pts, n_elems;
  const double* x;           /* [n_pts] node coordinates                           */
  const double* y;
  const int32_t* tri;        /* [3*n_elems] 1-based vertices, counter-clockwise   */
  int32_t n_edges;           /* 0: edges are derived (find_edges.f90:41-54);       */
  const int32_t* edge_p;     /*  else Triangle .edge endpoints [2*n_edges]         */
  const int32_t* edge_e;     /*  and .v.edge elements [2*n_edges] (-1 = ray)       */
  const double* zb;          /* bed elevation                                      */
  int32_t zb_at_vertices;    /*  1: zb is [n_pts] (datav(3)); 0: [n_elems]         */
  const double* cd;          /* roughness coefficient                              */
  int32_t cd_at_vertices;    /*  1: cd is [n_pts] (datav(7)); 0: [n_elems]         */
  int32_t n_inflow;
  const StormFvtBoundary* inflow;
  int32_t n_outflow;
  const StormFvtBoundary* outflow;
  /* wind forcing (the text input of windforcing.f90: drag coefficient and wind
     velocity components), NULL = no wind terms */
  const double* wind_c0;
  const double* wind_x;
  const double* wind_y;
  int32_t wind_at_vertices;  /*  1: the three arrays are [n_pts]; 0: [n_elems]     */
  /* culverts (the data file of ioculvert.f90), n_culvert = 0: none */
  int32_t n_culvert;
  int32_t cv_ld;             /* rows of the performance tables (>= every ncvtable) */
  const double* cvptoin;     /* (3,n_culvert) inlet x, y and invert elevation      */
  const double* cvptoout;    /* (2,n_culvert) outlet x, y                          */
  const int32_t* ncvtable;   /* [n_culvert] rows of each performance curve (>= 1)  */
  const double* cvhead;      /* (cv_ld,n_culvert) headwater elevations, ascending  */
  const double* cvq;         /* (cv_ld,n_culvert) discharges                       */
} StormFvtProblem;

/*
 * Prepared mesh: the module state at the solverFVT call site (after dataprepFVT).
 * Field names follow the Fortran arrays; array shapes are given as Fortran
 * declarations, stored column-major.
 */
typedef struct StormFvtMesh {
  int32_t n_pts, n_elems, n_edges;
  /* geometry.f90 */
  const double* node_x;          /* nodes(:)%x                 [n_pts]             */
  const double* node_y;          /* nodes(:)%y                 [n_pts]             */
  const int32_t* tri_vertex;     /* grid(:)%vertex             (3,n_elems)         */
  const int32_t* tri_edge;       /* grid(:)%edge, signed       (3,n_elems)         */
  const double* tri_area;        /* grid(:)%area               [n_elems]           */
  const double* tri_perim;       /* grid(:)%perim              [n_elems]           */
  const double* tri_xc;          /* grid(:)%xc                 [n_elems]           */
  const double* tri_yc;          /* grid(:)%yc                 [n_elems]           */
  const int32_t* edge_p;         /* edges(:)%p                 (2,n_edges)         */
  const int32_t* edge_e;         /* edges(:)%e (<1: no element)(2,n_edges)         */
  const double* edge_normal;     /* edges(:)%normal, unit      (2,n_edges)         */
  const double* edge_tang;       /* edges(:)%tang, unit        (2,n_edges)         */
  const double* edge_length;     /* edges(:)%length            [n_edges]           */
  const double* rc_x;            /* rc(:,:)%x                  (n_elems,3)         */
  const double* rc_y;            /* rc(:,:)%y                  (n_elems,3)         */
  int32_t t2t_ncol;              /* SIZE(t2t,2) = maxdim                            */
  const int32_t* t2t;            /* t2t                        (n_elems,t2t_ncol)  */
  const double* lsq_dx;          /* dx                         (n_elems,t2t_ncol-1)*/
  const double* lsq_dy;          /* dy                         (n_elems,t2t_ncol-1)*/
  const double* lsq_w;           /* lsqweight                  (n_elems,t2t_ncol-1)*/
  const double* lsq_a;           /* ai  [n_elems] */
  const double* lsq_b;           /* bi  [n_elems] */
  const double* lsq_c;           /* ci  [n_elems] */
  const double* lsq_det;         /* det [n_elems] */
  const int32_t* t2t3;           /* t2t3                       (3,n_elems)         */
  int32_t n2t_ncol;              /* SIZE(n2t,2)                                     */
  const int32_t* n2t;            /* n2t                        (n_pts,n2t_ncol)    */
  int32_t c2v_ncol;              /* SIZE(c2v_weights_id,2) (>= n2t_ncol-1)          */
  const double* c2v_w;           /* c2v_weights_id             (n_pts,c2v_ncol)    */
  const int32_t* csortedz;       /* csortedz(:)%p              (3,n_elems)         */
  int32_t flow_edges1;           /* interior edges                                  */
  const int32_t* flowedg1;       /* [flow_edges1]                                   */
  int32_t wall_edges1;           /* wall edges with a flux (walls.f90:132-136)      */
  const int32_t* walledg1;       /* [wall_edges1]                                   */
  int32_t n_bcedges;
  const int32_t* bcedges;        /* [n_bcedges]                                     */
  const int32_t* hbar;           /* LOGICAL [n_bcedges]: stage-boundary edge        */
  /* dep_vars.f90 */
  const double* z;               /* cell bed elevation         [n_elems]           */
  const double* zvtx;            /* vertex bed elevation       [n_pts]             */
  const double* cd;              /* roughness                  [n_elems]           */
  /* vbc_arrays.f90 / dep_vars.f90: inflow boundaries */
  int32_t n_inflowbdr;
  const int32_t* vtype;          /* [n_inflowbdr]                                   */
  const double* qin;             /* [n_inflowbdr]                                   */
  int32_t bcin_ld;               /* SIZE(bcedgesinflow,1) = d1+1                    */
  const int32_t* bcedgesinflow;  /* (0:d1,n_inflowbdr); row 0 holds the count       */
  int32_t tsq_ld;                /* SIZE(timelocq,1)                                */
  const int32_t* n_timeserq;     /* [n_inflowbdr]                                   */
  const double* timelocq;        /* (tsq_ld,n_inflowbdr)                            */
  const double* timeserq;        /* (tsq_ld,n_inflowbdr)                            */
  /* outflow boundaries */
  int32_t n_outflowbdr;
  const int32_t* htype;          /* [n_outflowbdr]                                  */
  const double* hbc;             /* [n_outflowbdr]                                  */
  int32_t bcout_ld;              /* SIZE(bcedgesoutflow,1) = d1+1                   */
  const int32_t* bcedgesoutflow; /* (0:d1,n_outflowbdr)                             */
  int32_t hbc_ld;                /* SIZE(hbc_nodes,1)                               */
  const int32_t* n_hbc;          /* [n_outflowbdr]                                  */
  const int32_t* hbc_nodes;      /* (hbc_ld,n_outflowbdr)                           */
  int32_t tsh_ld;                /* SIZE(timeloch,1)                                */
  const int32_t* n_timeserh;     /* [n_outflowbdr]                                  */
  const double* timeloch;        /* (tsh_ld,n_outflowbdr)                           */
  const double* timeserh;        /* (tsh_ld,n_outflowbdr)                           */
  double bch_max;                /* dataprepFVT.f90:278-286                         */
  const double* wcoef1;          /* [n_elems] wind terms added to phi(:,2:3) of wet */
  const double* wcoef2;          /*  cells (dep_vars.f90:33), NULL: no wind terms   */
  /* culverts (dep_vars.f90:68-82; cvprep.f90 placed the ends), n_culvert = 0: none */
  int32_t n_culvert;
  int32_t cv_ld;                 /* SIZE(cvhead,1)                                  */
  const int32_t* cvtrigin;       /* [n_culvert] 1-based triangle of the inlet       */
  const int32_t* cvtrigout;      /* [n_culvert] 1-based triangle of the outlet      */
  const double* cvptoin;         /* (3,n_culvert) inlet x, y, invert elevation      */
  const double* cvrin;           /* (2,n_culvert) inlet minus the inlet centroid    */
  const int32_t* ncvtable;       /* [n_culvert] rows of each performance curve      */
  const double* cvhead;          /* (cv_ld,n_culvert) headwater elevations          */
  const double* cvq;             /* (cv_ld,n_culvert) discharges                    */
} StormFvtMesh;

/* Per-call statistics, the scalars solverFVT prints per iteration
 * (solverFVT.f90:407-449).  cqin3/cqout3 are those of the last RK stage. */
#define STORM_MAX_BDR 16
typedef struct StormFvtStepStats {
  int32_t iter;        /* iterations done so far on this handle                    */
  int32_t converged;   /* steady: rmax < rstop was reached (solverFVT.f90:431)     */
  double ttime;        /* sum of delt (solverFVT.f90:155)                          */
  double stime;        /* simulated time (unsteady) or iter (steady)               */
  double delt;         /* last dt (steady: local dt of the last cell, as the ref.) */
  double rmax;         /* stopping quantity (steady) / max|phi| (unsteady)         */
  double rms_dh;       /* SQRT(sumtop/sumbot)                                      */
  double tmass;        /* SUM(h*area)                                              */
  double cqin3[STORM_MAX_BDR];
  double cqout3[STORM_MAX_BDR];
  int32_t device_status; /* 0, or the device-side check code                      */
  int32_t reserved[7];
} StormFvtStepStats;

typedef struct StormFvtHandle StormFvtHandle;

/* Message of the last failure on this thread ("" if none). */
STORM_FVT_API const char* storm_fvt_last_error(void);

/*
 * Build the prepared mesh from a raw problem: the C++ restatement of read_data's
 * topology builders and of dataprepFVT (find_edges.f90, edge_normals.f90,
 * t_areas.f90, walls.f90, ibc_arrays.f90, node_db.f90:60-68, elemnt_db.f90:50-233,
 * cde_t2t.f90, dataprepFVT.f90:69-306, c2v_setup.f90:98-119, lsq_setup.f90:92-145).
 * The result is owned by the library and freed by storm_fvt_mesh_free().
 */
STORM_FVT_API int storm_fvt_mesh_build(const StormFvtProblem* prob, StormFvtMesh** out);
STORM_FVT_API void storm_fvt_mesh_free(StormFvtMesh* mesh);

/*
 * Create a solver on the device: copies the prepared mesh to HBM in the library's
 * reordered structure-of-arrays layout.  Replaces the state set-up part of
 * solverFVT.f90:53-126.  The mesh arrays are not retained.
 */
STORM_FVT_API int storm_fvt_create(const StormFvtMesh* mesh, const StormFvtOptions* opt,
                     StormFvtHandle** out);

/*
 * Batched solver: `n` independent scenarios (meshes of any sizes, same options,
 * each with its own boundary values) advance together, one launch per kernel for
 * all of them (the step graph covers every scenario).  Each scenario keeps its own
 * dt, clocks, stop test and statistics; a converged scenario is skipped by every
 * kernel.  No counterpart in the reference (it runs one mesh per process).
 */
STORM_FVT_API int storm_fvt_create_batch(const StormFvtMesh* const* meshes, int32_t n,
                                         const StormFvtOptions* opt, StormFvtHandle** out);
STORM_FVT_API int32_t storm_fvt_num_scenarios(const StormFvtHandle* hd);
STORM_FVT_API int storm_fvt_set_scenario_state(StormFvtHandle* hd, int32_t scenario, const double* h,
                                               const double* u, const double* v);
STORM_FVT_API int storm_fvt_get_scenario_state(StormFvtHandle* hd, int32_t scenario, double* h, double* u,
                                               double* v, double* rkh, double* rku, double* rkv,
                                               double* hvtx);
/* Statistics of one scenario after the last storm_fvt_step call. */
STORM_FVT_API int storm_fvt_scenario_stats(const StormFvtHandle* hd, int32_t scenario,
                                           StormFvtStepStats* stats);

/* Set the cell state h, u, v [n_elems] (dep_vars.f90 arrays, element order) and
 * reset the iteration counters; rk*(:,rkorder) = h, h*u, h*v (solverFVT.f90:122-126). */
STORM_FVT_API int storm_fvt_set_state(StormFvtHandle* hd, const double* h, const double* u,
                        const double* v);

/*
 * Advance up to `nsteps` iterations of the main loop (solverFVT.f90:129-478).  In
 * steady mode the loop stops early once rmax < rstop, like the EXIT at :431 (for a
 * batch: once every scenario has stopped).  `stats` (may be NULL) receives the
 * scalars after the last iteration done (scenario 0 of a batch).
 * storm_fvt_set_state / get_state / get_drycell address single-scenario handles.
 */
STORM_FVT_API int storm_fvt_step(StormFvtHandle* hd, int32_t nsteps, StormFvtStepStats* stats);

/* Copy the state back to host arrays in element/node order.  Any pointer may be
 * NULL.  rk* receive level rkorder; hvtx the vertex depth of the last stage. */
STORM_FVT_API int storm_fvt_get_state(StormFvtHandle* hd, double* h, double* u, double* v,
                        double* rkh, double* rku, double* rkv, double* hvtx);

/* Dry-cell flags of the first RK stage of the next iteration, as find_dry_cells
 * (find_dry_cells.f90:25-42) sets them, element order, int32 0/1. */
STORM_FVT_API int storm_fvt_get_drycell(StormFvtHandle* hd, int32_t* drycell);

/* Number of this library's kernel launches since create (launch accounting). */
STORM_FVT_API int64_t storm_fvt_kernel_launches(const StormFvtHandle* hd);

/* Kernel timing mode (off by default).  When on, storm_fvt_step launches the
 * kernels of each iteration one by one (no CUDA graph) with a CUDA event pair
 * around every flux-kernel launch, for per-kernel roofline figures. */
STORM_FVT_API int storm_fvt_set_kernel_timing(StormFvtHandle* hd, int32_t on);

/* Device time (ms, CUDA events on the handle's stream) of the last storm_fvt_step
 * call; in kernel timing mode also the summed time of its flux-kernel launches. */
STORM_FVT_API int storm_fvt_last_timing(const StormFvtHandle* hd, double* step_ms,
                          double* flux_kernel_ms, int64_t* flux_kernel_launches);

/* Per-kernel device time (ms) and launch counts of the last storm_fvt_step call in
 * kernel timing mode, indexed 0 node (vertex depth), 1 grad (gradients/limiter),
 * 2 bc (open boundaries), 3 flux (per-cell gather of the face fluxes + sources + RK
 * update), 4 fric (friction and reduction partials), 5 final (iteration scalars),
 * 6 eflux (interior-edge fluxes), 7 tile (the fused stage kernel).  On the fused path
 * 1 and 3 time the boundary cells' gradient and update kernels only. */
STORM_FVT_API int storm_fvt_kernel_times(const StormFvtHandle* hd, double* ms, int64_t* launches);

/* Project autotuner: first times `iters` whole iterations of each stage path
 * (storm_fvt_set_stage_path) and keeps the fastest, then times `iters` iterations per
 * candidate block size of the node, gradient, edge-flux and cell kernels on this
 * handle's meshes (per-kernel CUDA events) and keeps the fastest of each;
 * re-captures the iteration graph and restores the state it started from.  `chosen`
 * (may be NULL) receives the four sizes; storm_fvt_stage_path reports the path. */
STORM_FVT_API int storm_fvt_autotune(StormFvtHandle* hd, int32_t iters, int32_t* chosen);

/* Stage kernels of the captured iteration.  No counterpart in the reference (it
 * selects how this library schedules the same arithmetic; FP64 results are bitwise
 * the same either way, mixed-precision ones agree to within that path's own error,
 * its FP32 kernels being compiled with FMA contraction):
 *   STORM_STAGE_PHASES  k_node, k_grad, k_eflux, k_flux per stage (gradients and edge
 *                       fluxes pass through device memory between the kernels);
 *                       the default;
 *   STORM_STAGE_FUSED   one fused kernel per stage over Morton tiles of 256 cells
 *                       (vertex depths, gradients, edge fluxes and the RK update of a
 *                       tile in shared memory);
 *   STORM_STAGE_FUSED_NODE_KERNEL  the same with the vertex depths computed by k_node
 *                       before it (for measurement).
 * The fused path does not apply to culverts, residual smoothing or linked partitions
 * (those run the phase kernels whatever is set), nor to a mesh whose tiles do not fit
 * in shared memory.  Setting re-captures the iteration graph. */
enum { STORM_STAGE_PHASES = 0, STORM_STAGE_FUSED = 1, STORM_STAGE_FUSED_NODE_KERNEL = 2 };
STORM_FVT_API int storm_fvt_set_stage_path(StormFvtHandle* hd, int32_t path);
/* The path the captured iteration runs (one of the STORM_STAGE_* values). */
STORM_FVT_API int32_t storm_fvt_stage_path(const StormFvtHandle* hd);

/*
 * One part of a mesh per process (one GPU each).  No counterpart in the reference,
 * which runs one mesh in one process: these cut storm_fvt_step's iteration at the
 * points where the parts exchange halo values and agree on dt and on the stop test,
 * and the caller (storm_b200/partition.py, DistributedPart) does the exchanges
 * between the calls.  Single-mesh handles whose mesh is an extended part:
 *   storm_fvt_set_exchange   the part's elements (1-based) it sends to other parts and
 *                            the halo elements it receives (left out of its sums);
 *   storm_fvt_iter_begin     this part's CFL dt (unsteady: the global dt is the
 *                            minimum over the parts) or the carried steady dt;
 *   storm_fvt_iter_set_dt    the iteration's dt (unsteady);
 *   storm_fvt_iter_stage     RK stage s; *delt_last: steady, the local dt of the part's
 *                            last element (element n_elems of the mesh in its owner);
 *   storm_fvt_iter_fric      friction with dt `delt` (steady: element n_elems's), then
 *                            sums[4] = this part's sum (h-h0)^2, sum h0^2, mass, max|phi|;
 *   storm_fvt_iter_finish    the iteration's scalars and stop test from the sums of all
 *                            parts (SUM, SUM, SUM, MAX);
 *   storm_fvt_pack_halo      h, u, v, rkh, rku, rkv ([6][n_send], device memory) of the
 *                            sent elements after stage `level`, or after the friction
 *                            step (after_fric = 1, level 0);
 *   storm_fvt_unpack_halo    the received [6][n_recv] values into the halo elements,
 *                            with their dry flags derived from them.
 * pack/unpack synchronise the handle's stream before they return.
 */
STORM_FVT_API int storm_fvt_set_exchange(StormFvtHandle* hd, int32_t n_send, const int32_t* send_elems,
                                         int32_t n_recv, const int32_t* recv_elems);
STORM_FVT_API int storm_fvt_iter_begin(StormFvtHandle* hd, double* dt_local);
STORM_FVT_API int storm_fvt_iter_set_dt(StormFvtHandle* hd, double dt);
STORM_FVT_API int storm_fvt_iter_stage(StormFvtHandle* hd, int32_t s, double* delt_last);
STORM_FVT_API int storm_fvt_iter_fric(StormFvtHandle* hd, double delt, double* sums);
STORM_FVT_API int storm_fvt_iter_finish(StormFvtHandle* hd, const double* sums, StormFvtStepStats* stats);
STORM_FVT_API int storm_fvt_pack_halo(StormFvtHandle* hd, int32_t level, int32_t after_fric, double* dev_out);
STORM_FVT_API int storm_fvt_unpack_halo(StormFvtHandle* hd, int32_t level, int32_t after_fric,
                                        const double* dev_in);

/* Host-only check of the fused kernel's tile plan for a batch of prepared meshes
 * (no device needed; no counterpart in the reference).  stats[8] receives: tiles,
 * largest local cell count, largest gradient count, largest edge count, H1 cells,
 * H2 cells, back edges, and 0 if every local index maps back to the cell or edge the
 * layout names (else the number of the first failed check). */
STORM_FVT_API int storm_fvt_tile_check(const StormFvtMesh* const* meshes, int32_t n, int32_t tile_cells,
                                       int64_t* stats);

/*
 * Partitions of one mesh (domain decomposition, single-device form):
 * the scenarios of a batch handle are the parts of one mesh, each extended by two
 * rings of vertex-adjacent halo cells taken from its neighbours.  After this call:
 *  - after every RK stage but the last, and after the friction step, each halo cell
 *    (scenario dst_scen[i], 1-based element dst_elem[i]) takes the state of its owner
 *    (src_scen[i], src_elem[i]): depth, discharges and velocities of that level and
 *    the dry flags the next stage reads;
 *  - halo cells are left out of the mass, residual and CFL reductions, and the
 *    scenarios share one dt (the minimum over all of them), one stop test (on the
 *    combined residual) and, steady, the friction dt of the local dt of element
 *    n_elems of the whole mesh, taken from scenario fric_scen.
 * With two halo rings every owned cell's update reads exactly the values it reads in
 * the undivided mesh, so the parts evolve bit for bit as the whole (the combined mass
 * and residual sums round in another order).  Requires nscen >= 2, no residual
 * smoothing, no culverts; the graph is re-captured.  Calling it twice is an error.
 */
STORM_FVT_API int storm_fvt_link_partitions(StormFvtHandle* hd, int32_t n_halo, const int32_t* dst_scen,
                                            const int32_t* dst_elem, const int32_t* src_scen,
                                            const int32_t* src_elem, int32_t fric_scen);

/*
 * Boundary data of the output-time vertex pass (Fortran module arrays the host holds
 * after read_data: walls.f90:170-195 and ibc_arrays.f90:56-135, 181-252, 266-345).
 * Vectors (TYPE(vector) arrays) are x,y interleaved, 2-D arrays column-major.
 */
typedef struct StormFvtOutputBoundary {
  int32_t n_wall;            /* nodes on solid walls, not on a boundary string        */
  const int32_t* wall_pts;   /* [n_wall] 1-based                                      */
  const double* wtangs;      /* [n_wall] unit wall tangents                           */
  int32_t qin_ld;            /* SIZE(qin_nodes,1)                                     */
  const int32_t* n_qin;      /* [n_inflowbdr] nodes per inflow string                 */
  const int32_t* qin_nodes;  /* (qin_ld, n_inflowbdr) 1-based                         */
  const double* pnormals;    /* (qin_ld, n_inflowbdr) inward unit normals at the nodes */
  const double* l_inflow;    /* (qin_ld, n_inflowbdr) length of inflow edge i         */
  const double* qin2;        /* [n_inflowbdr] second velocity component (vtype 3), or NULL */
  int32_t hbc_ld;            /* SIZE(hbc_nodes,1)                                     */
  const double* hnormals;    /* (hbc_ld, n_outflowbdr) unit normals at the outflow nodes */
} StormFvtOutputBoundary;

/*
 * The output step of the loop (solverFVT.f90:389-405, and :483-487 at exit) on the
 * device: to_vertices.f90:26-65 (ctr2vtxWSE type 3, the cap, positivity_vtx, the u,v
 * zeroing of wet cells with a dry vertex, ctr2vtx type 3 of u and v, wetdryvfix,
 * the dry-vertex zeroing, enforce_bcs.f90:37-171 with vbc_by_h.f90), ctr2vtx of cd
 * and error_est(2) (error_est.f90).  As in the reference, the zeroing of u,v in the
 * partially wet cells is applied to the solution, so a run that writes output
 * continues exactly as the reference's does.  in_loop = 1 for the output at the
 * select_out iterations inside the loop, which sees the boundary values the last
 * iteration ran with (get_time_bcs follows it, solverFVT.f90:462); 0 for the output
 * after the loop, which sees them after the last get_time_bcs.  Outputs (node /
 * element order, any may be NULL): hvtx, uvtx, vvtx, cdvtx [n_pts], e_est [n_elems].
 * Single-scenario handles with rkorder >= 2 (the pass reads the last stage's input
 * depth).
 */
STORM_FVT_API int storm_fvt_output_vertices(StormFvtHandle* h, const StormFvtOutputBoundary* ob, int32_t in_loop,
                                            double* hvtx, double* uvtx, double* vvtx, double* cdvtx, double* e_est);

STORM_FVT_API int storm_fvt_destroy(StormFvtHandle* hd);

/*
 * CFL time step without any device allocation.  No counterpart in the reference:
 * it exists for callers that cannot call cudaMalloc -- a host whose device memory
 * is owned by an external pool, or a loop that cannot take the synchronisation an
 * allocation may bring.  It computes,
 * from device arrays in any cell order, the value storm_fvt_step reports as the next
 * dt for dt_op = 1:  *d_dt = MIN over cells of cfl*area/((|u|+c+small)*perim) with
 * |u| and c = sqrt(g h) of the find_dry_cells classification (deltatFVT.f90:32-38,
 * with the cell area and perimeter).  Its scratch is a 32 KiB static device array,
 * so at most 1,048,576 cells per call (larger n: STORM_ERR_ARG, nothing launched).
 * Asynchronous on `stream` (a cudaStream_t, NULL = legacy default stream).  The
 * array's address belongs to a CUDA context: a call outside stream capture resolves
 * it in the current context and records it; a call during capture uses the recorded
 * address of the current context (STORM_ERR_ARG if there is none).  The first call
 * in a context also loads the library's device module (lazy loading), which
 * allocates device memory and may synchronise: make it while allocation is still
 * allowed and outside capture, and again after cudaDeviceReset or a context change.
 * Calls share the array, so calls that overlap on the GPU race.
 */
STORM_FVT_API int storm_fvt_cfl_dt_noalloc(const double* d_h, const double* d_u, const double* d_v,
                                           const double* d_area, const double* d_perim, int32_t n,
                                           double cfl, double h_dry, double h_wet, double* d_dt,
                                           void* stream);

#ifdef __cplusplus
}
#endif
#endif /* STORM_FVT_H */
