/*
 * storm_oracle.c -- CPU FP64 oracle for the SToRM FVT time step.
 *
 * TEST INFRASTRUCTURE ONLY (see storm_oracle.h).  A plain-C restatement of the
 * reference Fortran, routine by routine; every function names the reference
 * file:line it follows (paths relative to the reference project root, all under
 * Source_xsy-64bit/).  Arrays use the Fortran 1-based ids and column-major
 * layouts of the reference so the code reads like the original.
 *
 * Build with -O2 -ffp-contract=off (no FMA contraction): every expression is
 * evaluated in the reference's left-to-right order, in IEEE double.
 *
 * Only deliberate departures from the reference (each documented where made):
 *   - topology searches that are O(n^2) in the reference (edge_in_array, the
 *     grid%edge search, is_edge) use a hash on the node pair; they return the
 *     same first match on any mesh with one edge per node pair;
 *   - flux_HLL: the two defects at flux_HLL.f90:103-109 are fixed (see flux_hll);
 *   - deltatFVT (dt_op=1): uses the cell area/perimeter, the evident intent of
 *     deltatFVT.f90:36 which reads node arrays with cell indices;
 *   - interior-edge fluxes are computed into a per-edge buffer (in parallel when
 *     threads > 1) and then scattered in flowedg1 order, which performs exactly the
 *     arithmetic of invisc_fluxes.f90:39-186 in the same order.
 */
#include "storm_oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* constants.f90:17-30 */
static const double zero = 0.0;
static const double half = 0.5;
static const double one = 1.0;
#define ONE_THIRD (1.0 / 3.0)   /* one_third = one/3.0_mp */
static const double g = 9.81;
#define FMACHP 2.220446049250313e-16 /* EPSILON(zero) */
#define VSMALL 2.2250738585072014e-308 /* TINY(zero) */
#define VLARGE 1.7976931348623157e+308 /* HUGE(zero) */
/* REAL(KIND=mp), PARAMETER :: small = 1.0E-9 -- a default-REAL literal
 * (solverFVT.f90:43, deltatFVT.f90:30, flux_ac.f90:46) */
#define SMALL_F ((double)1.0e-9f)

/* MIN/MAX written as the compare-select the Fortran intrinsics compile to. */
static inline double fmin2(double a, double b) { return (b < a) ? b : a; }
static inline double fmax2(double a, double b) { return (b > a) ? b : a; }

static __thread char g_err[512];
static int set_err(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return code;
}
const char* orc_last_error(void) { return g_err; }

/* equals.f90:1-27 */
static inline int equals(double a, double b) {
  double eps = fabs(a) * FMACHP;
  if (eps == zero) eps = VSMALL;
  return !(fabs(a - b) > eps);
}

struct orc {
  StormFvtOptions opt;
  int nthreads;
  int32_t n_pts, n_elems, n_edges;
  /* geometry (StormFvtMesh layout) */
  double *node_x, *node_y;
  int32_t *tri_vertex, *tri_edge;
  double *tri_area, *tri_perim, *tri_xc, *tri_yc;
  int32_t *edge_p, *edge_e;
  double *edge_normal, *edge_tang, *edge_length;
  double *rc_x, *rc_y;
  int32_t t2t_ncol;
  int32_t* t2t;
  double *lsq_dx, *lsq_dy, *lsq_w, *lsq_a, *lsq_b, *lsq_c, *lsq_det;
  int32_t* t2t3;
  int32_t n2t_ncol;
  int32_t* n2t;
  int32_t c2v_ncol;
  double* c2v_w;   /* c2v_weights_id */
  double* c2v_wn;  /* c2v_weights (normalised), used by dataprep's ctr2vtx */
  int32_t* csortedz;
  int32_t flow_edges1, wall_edges1, n_bcedges;
  int32_t *flowedg1, *walledg1, *bcedges, *hbar, *qbar;
  double *z, *zvtx, *cd;
  double *wcoef1, *wcoef2; /* dep_vars.f90:33, NULL: no wind terms */
  /* culverts, dep_vars.f90:68-82 */
  int32_t ncv, cv_ld;
  int32_t *cvtrigin, *cvtrigout, *ncvtable;
  double *cvptoin, *cvrin, *cvhead, *cvq, *cvsrc;
  /* boundaries */
  int32_t n_in, qin_ld, bcin_ld, tsq_ld;
  int32_t *vtype, *n_qin, *qin_nodes, *bcedgesinflow, *n_timeserq;
  double *qin, *timelocq, *timeserq;
  int32_t n_out, hbc_ld, bcout_ld, tsh_ld;
  int32_t *htype, *n_hbc, *hbc_nodes, *bcedgesoutflow, *n_timeserh;
  double *hbc, *timeloch, *timeserh;
  double bch_max;
  /* solution (dep_vars.f90, RKparams.f90) */
  double *h, *u, *v, *zeta, *u_mag, *wavec, *hvtx, *zetavtx, *rough;
  double *delh_x, *delh_y, *delu_x, *delu_y, *delv_x, *delv_y, *delz_x, *delz_y;
  double* phi;    /* phi(n_elems,3) */
  int32_t* drycell;
  double rkalpha[4][4], rkbeta[4];
  double *rkh, *rku, *rkv; /* (n_elems, 0:rkorder) */
  double* fedge;           /* interior-edge flux buffer (3, flow_edges1) */
  int32_t* fedge_set;      /* flux computed for this interior edge */
  double cqin3[STORM_MAX_BDR], cqout3[STORM_MAX_BDR];
  double qin_it[STORM_MAX_BDR], hbc_it[STORM_MAX_BDR]; /* the values the last iteration ran with */
  /* residual smoothing: phi0 copy, and the cells ordered by colour (rsavg_order 1) */
  double* phi0;
  int32_t* rs_seq;
  /* loop state (solverFVT.f90:53-62) */
  int32_t iter, converged, have_state;
  double ttime, stime, delt, rmax, rms, tmass;
};

/* ---- index helpers (Fortran layout, 1-based) ----------------------------- */
#define NX(p) o->node_x[(p)-1]
#define NY(p) o->node_y[(p)-1]
#define GV(i, j) o->tri_vertex[3 * ((i)-1) + (j)-1]
#define GE(i, j) o->tri_edge[3 * ((i)-1) + (j)-1]
#define AREA(i) o->tri_area[(i)-1]
#define PERIM(i) o->tri_perim[(i)-1]
#define XC(i) o->tri_xc[(i)-1]
#define YC(i) o->tri_yc[(i)-1]
#define EP(k, j) o->edge_p[2 * ((k)-1) + (j)-1]
#define EE(k, j) o->edge_e[2 * ((k)-1) + (j)-1]
#define ENRM(k, j) o->edge_normal[2 * ((k)-1) + (j)-1]
#define ETAN(k, j) o->edge_tang[2 * ((k)-1) + (j)-1]
#define ELEN(k) o->edge_length[(k)-1]
#define RCX(i, j) o->rc_x[((j)-1) * (size_t)o->n_elems + (i)-1]
#define RCY(i, j) o->rc_y[((j)-1) * (size_t)o->n_elems + (i)-1]
#define T2T(i, j) o->t2t[((j)-1) * (size_t)o->n_elems + (i)-1]
#define LDX(i, k) o->lsq_dx[((k)-1) * (size_t)o->n_elems + (i)-1]
#define LDY(i, k) o->lsq_dy[((k)-1) * (size_t)o->n_elems + (i)-1]
#define LW(i, k) o->lsq_w[((k)-1) * (size_t)o->n_elems + (i)-1]
#define T2T3(j, i) o->t2t3[3 * ((i)-1) + (j)-1]
#define N2T(p, j) o->n2t[((j)-1) * (size_t)o->n_pts + (p)-1]
#define C2VW(p, j) o->c2v_w[((j)-1) * (size_t)o->n_pts + (p)-1]
#define C2VWN(p, j) o->c2v_wn[((j)-1) * (size_t)o->n_pts + (p)-1]
#define CSZ(i, j) o->csortedz[3 * ((i)-1) + (j)-1]
#define QIN_NODES(i, b) o->qin_nodes[((b)-1) * (size_t)o->qin_ld + (i)-1]
#define HBC_NODES(i, b) o->hbc_nodes[((b)-1) * (size_t)o->hbc_ld + (i)-1]
#define BCIN(i, b) o->bcedgesinflow[((b)-1) * (size_t)o->bcin_ld + (i)]
#define BCOUT(i, b) o->bcedgesoutflow[((b)-1) * (size_t)o->bcout_ld + (i)]
#define H(i) o->h[(i)-1]
#define U(i) o->u[(i)-1]
#define V(i) o->v[(i)-1]
#define Z(i) o->z[(i)-1]
#define ZVTX(p) o->zvtx[(p)-1]
#define ZETA(i) o->zeta[(i)-1]
#define HVTX(p) o->hvtx[(p)-1]
#define DRY(i) o->drycell[(i)-1]
#define PHI(i, n) o->phi[((n)-1) * (size_t)o->n_elems + (i)-1]
#define RKH(i, l) o->rkh[(size_t)(l) * o->n_elems + (i)-1]
#define RKU(i, l) o->rku[(size_t)(l) * o->n_elems + (i)-1]
#define RKV(i, l) o->rkv[(size_t)(l) * o->n_elems + (i)-1]

static void* xcalloc(size_t n, size_t sz) { return calloc(n ? n : 1, sz); }

/* ========================================================================== */
/*                           T O P O L O G Y                                  */
/* ========================================================================== */

/* Open-addressing hash from an unordered node pair to the first edge id. */
typedef struct { int64_t* key; int32_t* val; size_t cap; } pairmap;
static uint64_t mix64(uint64_t x) {
  x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33; return x;
}
static int pm_init(pairmap* m, size_t n) {
  m->cap = 16;
  while (m->cap < 2 * n + 16) m->cap <<= 1;
  m->key = (int64_t*)malloc(m->cap * sizeof(int64_t));
  m->val = (int32_t*)malloc(m->cap * sizeof(int32_t));
  if (!m->key || !m->val) return -1;
  for (size_t i = 0; i < m->cap; i++) m->key[i] = -1;
  return 0;
}
static void pm_free(pairmap* m) { free(m->key); free(m->val); }
static int64_t pm_key(int32_t a, int32_t b) {
  int32_t lo = a < b ? a : b, hi = a < b ? b : a;
  return ((int64_t)lo << 32) | (uint32_t)hi;
}
/* returns existing value or inserts `v` and returns 0 */
static int32_t pm_get_or_put(pairmap* m, int32_t a, int32_t b, int32_t v) {
  int64_t k = pm_key(a, b);
  size_t i = mix64((uint64_t)k) & (m->cap - 1);
  while (m->key[i] != -1) {
    if (m->key[i] == k) return m->val[i];
    i = (i + 1) & (m->cap - 1);
  }
  m->key[i] = k;
  m->val[i] = v;
  return 0;
}
static int32_t pm_get(const pairmap* m, int32_t a, int32_t b) {
  int64_t k = pm_key(a, b);
  size_t i = mix64((uint64_t)k) & (m->cap - 1);
  while (m->key[i] != -1) {
    if (m->key[i] == k) return m->val[i];
    i = (i + 1) & (m->cap - 1);
  }
  return 0;
}

/* vertex(MAX(1,MOD(j+1,4))): the next vertex around the triangle */
static inline int jnext(int j) { int t = (j + 1) % 4; return t < 1 ? 1 : t; }

/* find_edges.f90:27-197 (edge_normals.f90:30-39 and the length loop :159-163). */
static int find_edges(orc_t* o, const StormFvtProblem* p) {
  const int32_t T = o->n_elems;
  pairmap pm;
  if (pm_init(&pm, (size_t)3 * T)) return set_err(STORM_ERR_NOMEM, "find_edges: out of memory");
  int tdata = p->n_edges > 0;
  if (!tdata) {
    /* :46-54  edges in order of first appearance, oriented as first seen */
    o->edge_p = (int32_t*)xcalloc((size_t)6 * T + 2, sizeof(int32_t));
    int32_t ne = 0;
    for (int32_t i = 1; i <= T; i++)
      for (int j = 1; j <= 3; j++) {
        int32_t a = GV(i, j), b = GV(i, jnext(j));
        if (pm_get_or_put(&pm, a, b, ne + 1) == 0) {
          ne++;
          o->edge_p[2 * (ne - 1)] = a;
          o->edge_p[2 * (ne - 1) + 1] = b;
        }
      }
    o->n_edges = ne;
  } else {
    o->n_edges = p->n_edges;
    o->edge_p = (int32_t*)xcalloc((size_t)2 * p->n_edges, sizeof(int32_t));
    o->edge_e = (int32_t*)xcalloc((size_t)2 * p->n_edges, sizeof(int32_t));
    memcpy(o->edge_p, p->edge_p, sizeof(int32_t) * 2 * p->n_edges);
    /* tecplot_read.f90:146-153 / read_cgns.f90:276-283: ray => e(1)=e(2), e(2)=-1 */
    for (int32_t k = 1; k <= o->n_edges; k++) {
      int32_t e1 = p->edge_e[2 * (k - 1)], e2 = p->edge_e[2 * (k - 1) + 1];
      if (e1 < 0) { e1 = e2; e2 = -1; }
      EE(k, 1) = e1; EE(k, 2) = e2;
    }
    for (int32_t k = 1; k <= o->n_edges; k++) {
      int32_t a = EP(k, 1), b = EP(k, 2);
      if (a < 1 || a > o->n_pts || b < 1 || b > o->n_pts) {
        pm_free(&pm);
        return set_err(STORM_ERR_MESH, "edge %d has a node out of range", k);
      }
      pm_get_or_put(&pm, a, b, k);
    }
  }
  const int32_t E = o->n_edges;
  if (tdata) {
    /* :74-114  grid%edge from the element ids stored with each edge */
    for (int32_t j = 1; j <= E; j++)
      for (int k = 1; k <= 2; k++) {
        int32_t i = EE(j, k);
        if (i < 0) continue;
        if (i == 0 || i > T) { pm_free(&pm); return set_err(STORM_ERR_MESH, "edge %d: element %d out of range", j, i); }
        for (int l = 1; l <= 3; l++) {
          int32_t a = GV(i, l), b = GV(i, jnext(l));
          if (a == EP(j, 1) && b == EP(j, 2)) { GE(i, l) = j; break; }
          else if (a == EP(j, 2) && b == EP(j, 1)) { GE(i, l) = -j; break; }
        }
      }
    for (int32_t i = 1; i <= T; i++)
      for (int j = 1; j <= 3; j++)
        if (GE(i, j) == 0) { pm_free(&pm); return set_err(STORM_ERR_MESH, "edge data structure incomplete (element %d)", i); }
  } else {
    /* :122-152  first edge matching either orientation */
    for (int32_t i = 1; i <= T; i++)
      for (int j = 1; j <= 3; j++) {
        int32_t a = GV(i, j), b = GV(i, jnext(j));
        int32_t k = pm_get(&pm, a, b);
        if (k == 0) { pm_free(&pm); return set_err(STORM_ERR_MESH, "edge data structure incomplete (element %d)", i); }
        GE(i, j) = (EP(k, 1) == a && EP(k, 2) == b) ? k : -k;
      }
  }
  pm_free(&pm);
  /* edge_normals.f90:30-39 */
  o->edge_normal = (double*)xcalloc((size_t)2 * E, sizeof(double));
  o->edge_tang = (double*)xcalloc((size_t)2 * E, sizeof(double));
  o->edge_length = (double*)xcalloc((size_t)E, sizeof(double));
  for (int32_t i = 1; i <= E; i++) {
    double x1 = NX(EP(i, 1)), y1 = NY(EP(i, 1));
    double x2 = NX(EP(i, 2)), y2 = NY(EP(i, 2));
    ENRM(i, 1) = y2 - y1;
    ENRM(i, 2) = x1 - x2;
    ETAN(i, 1) = x2 - x1;
    ETAN(i, 2) = y2 - y1;
  }
  /* :159-163 */
  for (int32_t k = 1; k <= E; k++) {
    double delx = NX(EP(k, 1)) - NX(EP(k, 2));
    double dely = NY(EP(k, 1)) - NY(EP(k, 2));
    ELEN(k) = sqrt(delx * delx + dely * dely);
  }
  if (!tdata) {
    /* :165-193  e(1) is the first element to reference the edge */
    o->edge_e = (int32_t*)xcalloc((size_t)2 * E, sizeof(int32_t));
    int32_t* counter = (int32_t*)xcalloc((size_t)E + 1, sizeof(int32_t));
    for (int32_t k = 1; k <= E; k++) { EE(k, 1) = -1; EE(k, 2) = -1; counter[k] = 1; }
    for (int32_t i = 1; i <= T; i++)
      for (int j = 1; j <= 3; j++) {
        int32_t k = abs(GE(i, j));
        if (counter[k] > 2) { free(counter); return set_err(STORM_ERR_MESH, "edge data structure incorrect (edge %d)", k); }
        EE(k, counter[k]) = i;
        counter[k]++;
      }
    free(counter);
  }
  return 0;
}

/* t_areas.f90:33-52 */
static void t_areas(orc_t* o) {
  for (int32_t i = 1; i <= o->n_elems; i++) {
    double x1 = NX(GV(i, 1)), y1 = NY(GV(i, 1));
    double x2 = NX(GV(i, 2)), y2 = NY(GV(i, 2));
    double x3 = NX(GV(i, 3)), y3 = NY(GV(i, 3));
    double area = half * fabs((x1 - x2) * (y1 + y2) + (x2 - x3) * (y2 + y3) + (x3 - x1) * (y3 + y1));
    AREA(i) = area;
    XC(i) = ONE_THIRD * (x1 + x2 + x3);
    YC(i) = ONE_THIRD * (y1 + y2 + y3);
    PERIM(i) = ELEN(abs(GE(i, 1))) + ELEN(abs(GE(i, 2))) + ELEN(abs(GE(i, 3)));
  }
}

/* in_array2(p,qin_nodes) .OR. in_array2(p,hbc_nodes) via a node mark */
static int walls(orc_t* o, const unsigned char* bcnode) {
  /* walls.f90:40-148 */
  const int32_t E = o->n_edges;
  int32_t* edge_count = (int32_t*)xcalloc((size_t)E + 1, sizeof(int32_t));
  for (int32_t n = 1; n <= o->n_elems; n++)
    for (int j = 1; j <= 3; j++) edge_count[abs(GE(n, j))]++;
  int32_t nw1 = 0, nf1 = 0;
  for (int32_t i = 1; i <= E; i++) {
    if (edge_count[i] == 1) {
      int bc1 = bcnode[EP(i, 1)], bc2 = bcnode[EP(i, 2)];
      if (!(bc1 && bc2)) nw1++;
    } else if (edge_count[i] == 2) {
      nf1++;
    } else {
      free(edge_count);
      return set_err(STORM_ERR_MESH, "grid construction error in edge %d (wall or inner edge)", i);
    }
  }
  o->walledg1 = (int32_t*)xcalloc((size_t)nw1 + 1, sizeof(int32_t));
  o->flowedg1 = (int32_t*)xcalloc((size_t)nf1 + 1, sizeof(int32_t));
  int32_t nb = 0;
  for (int32_t i = 1; i <= E; i++) nb += edge_count[i] == 1;
  int32_t* bpolygon = (int32_t*)xcalloc((size_t)nb + 1, sizeof(int32_t));
  int32_t l = 0, m = 0, n = 0;
  for (int32_t i = 1; i <= E; i++) {
    if (edge_count[i] == 1) {
      bpolygon[l++] = i;
      int bc1 = bcnode[EP(i, 1)], bc2 = bcnode[EP(i, 2)];
      if (!(bc1 && bc2)) o->walledg1[m++] = i;
    } else {
      o->flowedg1[n++] = i;
    }
  }
  o->wall_edges1 = m;
  o->flow_edges1 = n;
  free(edge_count);
  /* ibc_arrays.f90:377-413  bcedges = bounding polygon minus walledg1 */
  int32_t nbc = nb - m;
  int32_t k = 0;
  for (int32_t b = 1; b <= o->n_in; b++) k += o->n_qin[b - 1] - 1;
  for (int32_t b = 1; b <= o->n_out; b++) k += o->n_hbc[b - 1] - 1;
  if (k != nbc) {
    free(bpolygon);
    return set_err(STORM_ERR_MESH,
                   "number of boundary condition edges (%d) does not match the boundary chains (%d)", nbc, k);
  }
  o->n_bcedges = nbc;
  o->bcedges = (int32_t*)xcalloc((size_t)nbc + 1, sizeof(int32_t));
  o->hbar = (int32_t*)xcalloc((size_t)nbc + 1, sizeof(int32_t));
  o->qbar = (int32_t*)xcalloc((size_t)nbc + 1, sizeof(int32_t));
  /* walledg1 is increasing, so membership is a merge */
  int32_t c = 0, w = 0;
  for (int32_t i = 0; i < nb; i++) {
    int32_t j = bpolygon[i];
    while (w < m && o->walledg1[w] < j) w++;
    if (!(w < m && o->walledg1[w] == j)) o->bcedges[c++] = j;
  }
  free(bpolygon);
  if (c != nbc) return set_err(STORM_ERR_MESH, "wall edges and inflow/outflow edges do not add up");
  return 0;
}

/* is_edge.f90:26-49 through the pair hash (unique node pair per edge). */
static int32_t is_edge(const orc_t* o, const pairmap* pm, int32_t p1, int32_t p2) {
  if (p1 > o->n_pts || p1 < 1 || p2 > o->n_pts || p2 < 1) return -1;
  return pm_get(pm, p1, p2);
}

/* ibc_arrays.f90:42-137, 148-181, 416-466 (the parts the FVT step reads). */
static int ibc_arrays(orc_t* o) {
  pairmap pm;
  if (pm_init(&pm, (size_t)o->n_edges)) return set_err(STORM_ERR_NOMEM, "ibc_arrays: out of memory");
  for (int32_t k = 1; k <= o->n_edges; k++) pm_get_or_put(&pm, EP(k, 1), EP(k, 2), k);
  /* first bcedges position of each edge, for the qbar/hbar search (:433-438) */
  int32_t* first_pos = (int32_t*)xcalloc((size_t)o->n_edges + 1, sizeof(int32_t));
  for (int32_t j = o->n_bcedges; j >= 1; j--) first_pos[o->bcedges[j - 1]] = j;
  o->bcin_ld = o->qin_ld + 1;
  o->bcedgesinflow = (int32_t*)xcalloc((size_t)o->bcin_ld * (o->n_in ? o->n_in : 1), sizeof(int32_t));
  int rc = 0;
  for (int32_t b = 1; b <= o->n_in && !rc; b++) {
    BCIN(0, b) = o->n_qin[b - 1] - 1;
    for (int32_t i = 1; i <= o->n_qin[b - 1] - 1; i++) {
      int32_t e = is_edge(o, &pm, QIN_NODES(i, b), QIN_NODES(i + 1, b));
      if (e == 0) { rc = set_err(STORM_ERR_MESH, "inflow nodes %d %d are not connected by an edge", QIN_NODES(i, b), QIN_NODES(i + 1, b)); break; }
      if (e < 0) { rc = set_err(STORM_ERR_MESH, "inflow boundary node out of range"); break; }
      BCIN(i, b) = e;
      int32_t t = EE(e, 1) < 1 ? EE(e, 2) : EE(e, 1);
      if (t < 1) { rc = set_err(STORM_ERR_MESH, "inflow edge %d has no element", e); break; }
      if (first_pos[e]) o->qbar[first_pos[e] - 1] = 1;
    }
  }
  o->bcout_ld = o->hbc_ld + 1;
  o->bcedgesoutflow = (int32_t*)xcalloc((size_t)o->bcout_ld * (o->n_out ? o->n_out : 1), sizeof(int32_t));
  for (int32_t b = 1; b <= o->n_out && !rc; b++) {
    BCOUT(0, b) = o->n_hbc[b - 1] - 1;
    for (int32_t i = 1; i <= o->n_hbc[b - 1] - 1; i++) {
      int32_t e = is_edge(o, &pm, HBC_NODES(i, b), HBC_NODES(i + 1, b));
      if (e == 0) { rc = set_err(STORM_ERR_MESH, "outflow nodes %d %d are not connected by an edge", HBC_NODES(i, b), HBC_NODES(i + 1, b)); break; }
      if (e < 0) { rc = set_err(STORM_ERR_MESH, "outflow boundary node out of range"); break; }
      BCOUT(i, b) = e;
      if (first_pos[e]) o->hbar[first_pos[e] - 1] = 1;
    }
  }
  free(first_pos);
  pm_free(&pm);
  return rc;
}

/* node_db.f90:32-68 (n2t only; n2t2, cv_area/cv_perim and n2n serve other paths) */
static int node_db(orc_t* o) {
  const int32_t N = o->n_pts;
  int32_t* counter = (int32_t*)xcalloc((size_t)N + 1, sizeof(int32_t));
  for (int32_t i = 1; i <= o->n_elems; i++)
    for (int j = 1; j <= 3; j++) counter[GV(i, j)]++;
  int32_t k = 0;
  for (int32_t p = 1; p <= N; p++) k = counter[p] > k ? counter[p] : k;
  free(counter);
  o->n2t_ncol = k + 1;
  o->n2t = (int32_t*)xcalloc((size_t)N * o->n2t_ncol, sizeof(int32_t));
  for (int32_t i = 1; i <= o->n_elems; i++)
    for (int j = 1; j <= 3; j++) {
      int32_t p1 = GV(i, j);
      int32_t kk = N2T(p1, 1) + 1;
      N2T(p1, kk + 1) = i;
      N2T(p1, 1) = kk;
    }
  /* m = MAX(k,4); n2t2 is (n_pts, m+1); c2v_weights(_id) are (n_pts, m) */
  o->c2v_ncol = (k > 4 ? k : 4);
  return 0;
}

/* cde_t2t.f90:23-49, literally: the DO bound is fixed at loop entry while n
 * shrinks, and the shift reads one entry past the new end. */
static void cde_t2t(int32_t* t2tw, int32_t i, int32_t dim1, int32_t dim2) {
#define TW(ii, jj) t2tw[((jj)-1) * (size_t)dim1 + (ii)-1]
  (void)dim2;
  int32_t n = TW(i, 1);
  int32_t l = 1;
  for (;;) {
    int32_t j = TW(i, l + 1);
    int32_t mlast = n; /* DO m = l+1,n : trip count fixed here */
    for (int32_t m = l + 1; m <= mlast; m++) {
      int32_t k = TW(i, m + 1);
      if (j == k) {
        n = n - 1;
        for (int32_t nn = m; nn <= n; nn++) TW(i, nn + 1) = TW(i, nn + 2);
        TW(i, 1) = n;
      }
    }
    l = l + 1;
    if (l > n) break;
  }
#undef TW
}

/* elemnt_db.f90:32-128 (t2t) and :216-233 (t2t3).  t2tHD serves HDLS only. */
static int elemnt_db(orc_t* o) {
  const int32_t T = o->n_elems;
  if (T < 4) return set_err(STORM_ERR_MESH, "too few triangles (must be >= 4)");
  const int32_t maxdim = 20;
  int32_t* t2tw = (int32_t*)xcalloc((size_t)T * maxdim, sizeof(int32_t));
#define TW(ii, jj) t2tw[((jj)-1) * (size_t)T + (ii)-1]
  for (int32_t i = 1; i <= o->n_edges; i++) {
    int32_t e1 = EE(i, 1), e2 = EE(i, 2);
    if (e1 < 1 || e2 < 1) continue;
    int32_t k = TW(e1, 1) + 1; TW(e1, k + 1) = e2; TW(e1, 1) = k;
    k = TW(e2, 1) + 1; TW(e2, k + 1) = e1; TW(e2, 1) = k;
  }
  int rc = 0;
  for (int32_t i = 1; i <= T && !rc; i++) {
    int32_t n = TW(i, 1);
    if (n == 3) continue;
    if (n < 1 || n > 3) { rc = set_err(STORM_ERR_MESH, "triangle connectivity table incorrect (element %d)", i); break; }
    for (int32_t l = 1; l <= n; l++) {
      int32_t j = TW(i, l + 1);
      int32_t mm = TW(j, 1) < 3 ? TW(j, 1) : 3;
      for (int32_t m = 1; m <= mm; m++) {
        int32_t k = TW(j, m + 1);
        if (k == i) continue;
        int32_t nn = TW(i, 1) + 1;
        if (nn + 1 > maxdim) { rc = set_err(STORM_ERR_MESH, "t2t stencil of element %d exceeds %d entries", i, maxdim - 1); break; }
        TW(i, nn + 1) = k; TW(i, 1) = nn;
      }
      if (rc) break;
    }
    if (!rc) cde_t2t(t2tw, i, T, maxdim);
  }
  for (int32_t i = 1; i <= T && !rc; i++) {
    int32_t n = TW(i, 1);
    if (n >= 3) continue;
    int32_t j = TW(i, n + 1);
    int32_t mm = TW(j, 1);
    for (int32_t m = 1; m <= mm; m++) {
      int32_t k = TW(j, m + 1);
      if (k == i) continue;
      int32_t nn = TW(i, 1) + 1;
      if (nn + 1 > maxdim) { rc = set_err(STORM_ERR_MESH, "t2t stencil of element %d exceeds %d entries", i, maxdim - 1); break; }
      TW(i, nn + 1) = k; TW(i, 1) = nn;
    }
    if (!rc) cde_t2t(t2tw, i, T, maxdim);
  }
  if (rc) { free(t2tw); return rc; }
  int32_t md = 0;
  for (int32_t i = 1; i <= T; i++) md = TW(i, 1) > md ? TW(i, 1) : md;
  md = md + 1;
  o->t2t_ncol = md;
  o->t2t = (int32_t*)xcalloc((size_t)T * md, sizeof(int32_t));
  for (int32_t i = 1; i <= T; i++)
    for (int32_t j = 1; j <= md; j++) T2T(i, j) = TW(i, j);
#undef TW
  free(t2tw);
  o->t2t3 = (int32_t*)xcalloc((size_t)3 * T, sizeof(int32_t));
  for (int32_t i = 1; i <= T; i++)
    for (int j = 1; j <= 3; j++) {
      int32_t k = abs(GE(i, j));
      int32_t e1 = EE(k, 1);
      if (e1 == i) e1 = EE(k, 2);
      T2T3(j, i) = e1;
    }
  return 0;
}

/* c2v_setup.f90:98-119 (type 3, inverse distance) */
static void c2v_setup(orc_t* o) {
  const int32_t N = o->n_pts;
  o->c2v_w = (double*)xcalloc((size_t)N * o->c2v_ncol, sizeof(double));
  o->c2v_wn = (double*)xcalloc((size_t)N * o->c2v_ncol, sizeof(double));
  for (int32_t i = 1; i <= N; i++) {
    double tdist = zero;
    for (int32_t j = 2; j <= N2T(i, 1) + 1; j++) {
      int32_t k = N2T(i, j);
      double xk = XC(k) - NX(i);
      double yk = YC(k) - NY(i);
      C2VWN(i, j - 1) = one / sqrt(xk * xk + yk * yk);
      C2VW(i, j - 1) = C2VWN(i, j - 1);
      tdist = tdist + C2VWN(i, j - 1);
    }
    for (int32_t j = 2; j <= N2T(i, 1) + 1; j++) C2VWN(i, j - 1) = C2VWN(i, j - 1) / tdist;
  }
}

/* lsq_setup.f90:92-145 (solver 2, type 2) */
static void lsq_setup(orc_t* o) {
  const int32_t T = o->n_elems;
  const int32_t kc = o->t2t_ncol - 1 > 0 ? o->t2t_ncol - 1 : 1;
  o->lsq_dx = (double*)xcalloc((size_t)T * kc, sizeof(double));
  o->lsq_dy = (double*)xcalloc((size_t)T * kc, sizeof(double));
  o->lsq_w = (double*)xcalloc((size_t)T * kc, sizeof(double));
  o->lsq_a = (double*)xcalloc(T, sizeof(double));
  o->lsq_b = (double*)xcalloc(T, sizeof(double));
  o->lsq_c = (double*)xcalloc(T, sizeof(double));
  o->lsq_det = (double*)xcalloc(T, sizeof(double));
  for (int32_t i = 1; i <= T; i++) {
    int32_t j = T2T(i, 1);
    for (int32_t k = 2; k <= j + 1; k++) {
      int32_t l = T2T(i, k);
      LDX(i, k - 1) = XC(l) - XC(i);
      LDY(i, k - 1) = YC(l) - YC(i);
    }
  }
  for (int32_t i = 1; i <= T; i++) {
    int32_t j = T2T(i, 1);
    for (int32_t k = 1; k <= j; k++) LW(i, k) = one / (LDX(i, k) * LDX(i, k) + LDY(i, k) * LDY(i, k));
  }
  for (int32_t i = 1; i <= T; i++) {
    double ai = zero, bi = zero, ci = zero;
    int32_t j = T2T(i, 1);
    for (int32_t k = 1; k <= j; k++) {
      ai = ai + LW(i, k) * LDX(i, k) * LDX(i, k);
      bi = bi + LW(i, k) * LDX(i, k) * LDY(i, k);
      ci = ci + LW(i, k) * LDY(i, k) * LDY(i, k);
    }
    o->lsq_a[i - 1] = ai;
    o->lsq_b[i - 1] = bi;
    o->lsq_c[i - 1] = ci;
    o->lsq_det[i - 1] = ai * ci - bi * bi;
  }
}

/* ctr2vtx.f90:69-80 (type 3, normalised inverse-distance weights) */
static void ctr2vtx3(const orc_t* o, const double* carray, double* varray) {
  for (int32_t i = 1; i <= o->n_pts; i++) {
    double a = zero;
    for (int32_t j = 2; j <= N2T(i, 1) + 1; j++) {
      int32_t k = N2T(i, j);
      a = a + C2VWN(i, j - 1) * carray[k - 1];
    }
    varray[i - 1] = a;
  }
}

/* vtx2ctr.f90:32-35 */
static void vtx2ctr(const orc_t* o, const double* varray, double* carray) {
  for (int32_t i = 1; i <= o->n_elems; i++)
    carray[i - 1] = (varray[GV(i, 1) - 1] + varray[GV(i, 2) - 1] + varray[GV(i, 3) - 1]) * ONE_THIRD;
}

static int copy_boundaries(orc_t* o, const StormFvtProblem* p) {
  if (p->n_inflow > STORM_MAX_BDR || p->n_outflow > STORM_MAX_BDR)
    return set_err(STORM_ERR_ARG, "at most %d inflow and %d outflow boundaries", STORM_MAX_BDR, STORM_MAX_BDR);
  o->n_in = p->n_inflow;
  o->n_out = p->n_outflow;
  int32_t d1 = 1, ts = 1;
  for (int b = 0; b < o->n_in; b++) {
    const StormFvtBoundary* B = &p->inflow[b];
    if (B->n_nodes < 1) return set_err(STORM_ERR_MESH, "inflow boundary has no nodes assigned");
    /* vtype 0 and 3 set vertex velocities only (enforce_bcs.f90:133-164): no edge flux;
     * vtype 2 stops the reference (enforce_bcs.f90:151-155) */
    if (B->type < 0 || B->type > 5 || B->type == 2) return set_err(STORM_ERR_UNSUPPORTED, "inflow vtype %d is not supported", B->type);
    d1 = B->n_nodes > d1 ? B->n_nodes : d1;
    ts = B->n_series > ts ? B->n_series : ts;
  }
  o->qin_ld = d1;
  o->tsq_ld = ts;
  int32_t nb = o->n_in ? o->n_in : 1;
  o->vtype = (int32_t*)xcalloc(nb, sizeof(int32_t));
  o->n_qin = (int32_t*)xcalloc(nb, sizeof(int32_t));
  o->qin = (double*)xcalloc(nb, sizeof(double));
  o->n_timeserq = (int32_t*)xcalloc(nb, sizeof(int32_t));
  o->qin_nodes = (int32_t*)xcalloc((size_t)d1 * nb, sizeof(int32_t));
  o->timelocq = (double*)xcalloc((size_t)ts * nb, sizeof(double));
  o->timeserq = (double*)xcalloc((size_t)ts * nb, sizeof(double));
  for (int b = 1; b <= o->n_in; b++) {
    const StormFvtBoundary* B = &p->inflow[b - 1];
    o->vtype[b - 1] = B->type;
    o->n_qin[b - 1] = B->n_nodes;
    o->qin[b - 1] = B->value;
    o->n_timeserq[b - 1] = B->n_series;
    for (int i = 1; i <= d1; i++) QIN_NODES(i, b) = i <= B->n_nodes ? B->nodes[i - 1] : -1;
    for (int i = 0; i < B->n_series; i++) {
      o->timelocq[(size_t)(b - 1) * ts + i] = B->series_t[i];
      o->timeserq[(size_t)(b - 1) * ts + i] = B->series_v[i];
    }
  }
  d1 = 1; ts = 1;
  for (int b = 0; b < o->n_out; b++) {
    const StormFvtBoundary* B = &p->outflow[b];
    if (B->n_nodes < 1) return set_err(STORM_ERR_MESH, "outflow boundary has no nodes assigned");
    if (B->type < 0 || B->type > 2) return set_err(STORM_ERR_MESH, "invalid value in htype (%d)", B->type);
    d1 = B->n_nodes > d1 ? B->n_nodes : d1;
    ts = B->n_series > ts ? B->n_series : ts;
  }
  o->hbc_ld = d1;
  o->tsh_ld = ts;
  nb = o->n_out ? o->n_out : 1;
  o->htype = (int32_t*)xcalloc(nb, sizeof(int32_t));
  o->n_hbc = (int32_t*)xcalloc(nb, sizeof(int32_t));
  o->hbc = (double*)xcalloc(nb, sizeof(double));
  o->n_timeserh = (int32_t*)xcalloc(nb, sizeof(int32_t));
  o->hbc_nodes = (int32_t*)xcalloc((size_t)d1 * nb, sizeof(int32_t));
  o->timeloch = (double*)xcalloc((size_t)ts * nb, sizeof(double));
  o->timeserh = (double*)xcalloc((size_t)ts * nb, sizeof(double));
  for (int b = 1; b <= o->n_out; b++) {
    const StormFvtBoundary* B = &p->outflow[b - 1];
    o->htype[b - 1] = B->type;
    o->n_hbc[b - 1] = B->n_nodes;
    o->hbc[b - 1] = B->value;
    o->n_timeserh[b - 1] = B->n_series;
    for (int i = 1; i <= d1; i++) HBC_NODES(i, b) = i <= B->n_nodes ? B->nodes[i - 1] : -1;
    for (int i = 0; i < B->n_series; i++) {
      o->timeloch[(size_t)(b - 1) * ts + i] = B->series_t[i];
      o->timeserh[(size_t)(b - 1) * ts + i] = B->series_v[i];
    }
  }
  return 0;
}

/* get_time_bcs.f90:31-77 */
static void get_time_bcs(orc_t* o, double time) {
  for (int32_t k = 1; k <= o->n_out; k++) {
    if (o->htype[k - 1] != 1) continue;
    int32_t n = o->n_timeserh[k - 1];
    if (n > 0) {
      const double* tl = o->timeloch + (size_t)(k - 1) * o->tsh_ld;
      const double* ts = o->timeserh + (size_t)(k - 1) * o->tsh_ld;
      if (time < tl[0]) o->hbc[k - 1] = ts[0];
      else if (time >= tl[n - 1]) o->hbc[k - 1] = ts[n - 1];
      else
        for (int32_t i = 1; i <= n - 1; i++)
          if (time >= tl[i - 1] && time < tl[i]) {
            double delta = time - tl[i - 1];
            double delta2 = tl[i] - tl[i - 1];
            o->hbc[k - 1] = ts[i - 1] + delta * (ts[i] - ts[i - 1]) / delta2;
            break;
          }
    }
  }
  for (int32_t k = 1; k <= o->n_in; k++) {
    int32_t n = o->n_timeserq[k - 1];
    if (n > 0) {
      const double* tl = o->timelocq + (size_t)(k - 1) * o->tsq_ld;
      const double* ts = o->timeserq + (size_t)(k - 1) * o->tsq_ld;
      if (time < tl[0]) o->qin[k - 1] = ts[0];
      else if (time >= tl[n - 1]) o->qin[k - 1] = ts[n - 1];
      else
        for (int32_t j = 1; j <= n - 1; j++)
          if (time >= tl[j - 1] && time < tl[j]) {
            double delta = time - tl[j - 1];
            double delta2 = tl[j] - tl[j - 1];
            o->qin[k - 1] = ts[j - 1] + delta * (ts[j] - ts[j - 1]) / delta2;
            break;
          }
    }
  }
}

static int check_options(const StormFvtOptions* op) {
  if (op->rkorder < 1 || op->rkorder > 3) return set_err(STORM_ERR_ARG, "Incorrect Runge-Kutta order");
  if (op->opt_limiter < 0 || op->opt_limiter > 2) return set_err(STORM_ERR_ARG, "invalid limiter option");
  if (op->btype != 0 && op->btype != 1) return set_err(STORM_ERR_ARG, "invalid btype");
  if (op->opt_friction < 0 || op->opt_friction > 4) return set_err(STORM_ERR_UNSUPPORTED, "opt_friction %d is not supported", op->opt_friction);
  if (op->flux < 0 || op->flux > 2) return set_err(STORM_ERR_ARG, "invalid flux option");
  if (op->stop_cr != 0 && op->stop_cr != 1) return set_err(STORM_ERR_ARG, "invalid stop_cr");
  if (op->rsavg_passes < 0 || op->rsavg_passes > 64) return set_err(STORM_ERR_ARG, "invalid rsavg_passes");
  if (op->rsavg_passes > 0 && !(op->rsavg_eps > 0.0 && op->rsavg_eps <= 1.0))
    return set_err(STORM_ERR_ARG, "invalid rsavg_eps");
  if (op->rsavg_order != 0 && op->rsavg_order != 1) return set_err(STORM_ERR_ARG, "invalid rsavg_order");
  return 0;
}

/* pto_in_triangle.f90:1-45: barycentric test of (x, y) against triangle e */
static int pto_in_triangle(const orc_t* o, int32_t e, double x, double y) {
  const double tarea = AREA(e);
  const double x1 = NX(GV(e, 1)), y1 = NY(GV(e, 1));
  const double x2 = NX(GV(e, 2)), y2 = NY(GV(e, 2));
  const double x3 = NX(GV(e, 3)), y3 = NY(GV(e, 3));
  const double s = half / tarea * (y1 * x3 - x1 * y3 + (y3 - y1) * x + (x1 - x3) * y);
  const double t = half / tarea * (x1 * y2 - y1 * x2 + (y1 - y2) * x + (x2 - x1) * y);
  if (s < zero) return 0;
  if (t < zero) return 0;
  if (one - s - t < zero) return 0;
  return 1;
}

/* ioculvert.f90 checks + cvprep.f90:20-54: copy the culvert data, find the inlet and
 * outlet triangles (first triangle in index order that holds the point) */
static int cvprep(orc_t* o, const StormFvtProblem* p) {
  const int32_t T = o->n_elems, n = p->n_culvert;
  if (n <= 0) return 0;
  if (!p->cvptoin || !p->cvptoout || !p->ncvtable || !p->cvhead || !p->cvq || p->cv_ld < 1)
    return set_err(STORM_ERR_ARG, "culverts: missing data");
  for (int32_t i = 0; i < n; i++)
    if (p->ncvtable[i] < 1 || p->ncvtable[i] > p->cv_ld)
      return set_err(STORM_ERR_ARG, "culvert %d: too few (or too many) entries in the performance curve", i + 1);
  o->ncv = n;
  o->cv_ld = p->cv_ld;
  o->cvptoin = (double*)xcalloc((size_t)3 * n, sizeof(double));
  o->cvrin = (double*)xcalloc((size_t)2 * n, sizeof(double));
  o->cvtrigin = (int32_t*)xcalloc((size_t)n, sizeof(int32_t));
  o->cvtrigout = (int32_t*)xcalloc((size_t)n, sizeof(int32_t));
  o->ncvtable = (int32_t*)xcalloc((size_t)n, sizeof(int32_t));
  o->cvhead = (double*)xcalloc((size_t)p->cv_ld * n, sizeof(double));
  o->cvq = (double*)xcalloc((size_t)p->cv_ld * n, sizeof(double));
  o->cvsrc = (double*)xcalloc((size_t)n, sizeof(double));
  memcpy(o->cvptoin, p->cvptoin, sizeof(double) * 3 * (size_t)n);
  memcpy(o->ncvtable, p->ncvtable, sizeof(int32_t) * (size_t)n);
  memcpy(o->cvhead, p->cvhead, sizeof(double) * (size_t)p->cv_ld * n);
  memcpy(o->cvq, p->cvq, sizeof(double) * (size_t)p->cv_ld * n);
  for (int32_t i = 1; i <= n; i++) {
    const double xi = p->cvptoin[3 * (i - 1)], yi = p->cvptoin[3 * (i - 1) + 1];
    const double xo = p->cvptoout[2 * (i - 1)], yo = p->cvptoout[2 * (i - 1) + 1];
    int32_t j;
    for (j = 1; j <= T; j++)
      if (pto_in_triangle(o, j, xi, yi)) break;
    if (j > T) return set_err(STORM_ERR_MESH, "inlet of culvert %d not in computational domain", i);
    o->cvtrigin[i - 1] = j;
    o->cvrin[2 * (i - 1)] = xi - XC(j);
    o->cvrin[2 * (i - 1) + 1] = yi - YC(j);
    for (j = 1; j <= T; j++)
      if (pto_in_triangle(o, j, xo, yo)) break;
    if (j > T) return set_err(STORM_ERR_MESH, "outlet of culvert %d not in computational domain", i);
    o->cvtrigout[i - 1] = j;
  }
  return 0;
}

/* cvdisch.f90:19-49: discharge of each culvert from the headwater at its inlet
 * (zeta + the reconstructed stage gradient, minus the invert), interpolated in the
 * performance curve */
static void cvdisch(orc_t* o) {
  const int32_t ld = o->cv_ld;
  for (int32_t i = 1; i <= o->ncv; i++) o->cvsrc[i - 1] = zero;
  for (int32_t i = 1; i <= o->ncv; i++) {
    const int32_t c = o->cvtrigin[i - 1];
    if (DRY(c)) continue;
    double head = ZETA(c) + (o->delh_x[c - 1] + o->delz_x[c - 1]) * o->cvrin[2 * (i - 1)] +
                  (o->delh_y[c - 1] + o->delz_y[c - 1]) * o->cvrin[2 * (i - 1) + 1];
    head = head - o->cvptoin[3 * (i - 1) + 2];
    if (head < o->opt.h_dry) continue;
    const double* hd = o->cvhead + (size_t)(i - 1) * ld;
    const double* q = o->cvq + (size_t)(i - 1) * ld;
    const int32_t nt = o->ncvtable[i - 1];
    if (head < hd[0]) {
      o->cvsrc[i - 1] = q[0];
    } else if (head >= hd[nt - 1]) {
      o->cvsrc[i - 1] = q[nt - 1];
    } else {
      for (int32_t j = 1; j <= nt - 1; j++)
        if (head < hd[j]) {
          const double t = (head - hd[j - 1]) / (hd[j] - hd[j - 1]);
          o->cvsrc[i - 1] = q[j] * t + q[j - 1] * (one - t);
          break;
        }
    }
  }
}

int orc_create(const StormFvtProblem* p, const StormFvtOptions* opt, orc_t** out) {
  g_err[0] = 0;
  if (!p || !opt || !out) return set_err(STORM_ERR_ARG, "null argument");
  int rc = check_options(opt);
  if (rc) return rc;
  if (p->n_pts < 3 || p->n_elems < 1 || !p->x || !p->y || !p->tri || !p->zb || !p->cd)
    return set_err(STORM_ERR_ARG, "incomplete problem description");
  orc_t* o = (orc_t*)calloc(1, sizeof(orc_t));
  if (!o) return set_err(STORM_ERR_NOMEM, "out of memory");
  o->opt = *opt;
  o->nthreads = 1;
  o->n_pts = p->n_pts;
  o->n_elems = p->n_elems;
  const int32_t N = o->n_pts, T = o->n_elems;
  o->node_x = (double*)xcalloc(N, sizeof(double));
  o->node_y = (double*)xcalloc(N, sizeof(double));
  memcpy(o->node_x, p->x, sizeof(double) * N);
  memcpy(o->node_y, p->y, sizeof(double) * N);
  o->tri_vertex = (int32_t*)xcalloc((size_t)3 * T, sizeof(int32_t));
  o->tri_edge = (int32_t*)xcalloc((size_t)3 * T, sizeof(int32_t));
  memcpy(o->tri_vertex, p->tri, sizeof(int32_t) * 3 * T);
  for (size_t i = 0; i < (size_t)3 * T; i++)
    if (o->tri_vertex[i] < 1 || o->tri_vertex[i] > N) { orc_destroy(o); return set_err(STORM_ERR_MESH, "triangle vertex out of range"); }
  o->tri_area = (double*)xcalloc(T, sizeof(double));
  o->tri_perim = (double*)xcalloc(T, sizeof(double));
  o->tri_xc = (double*)xcalloc(T, sizeof(double));
  o->tri_yc = (double*)xcalloc(T, sizeof(double));
  if ((rc = copy_boundaries(o, p))) { orc_destroy(o); return rc; }
  /* read_mfa.f90:95-173 order: find_edges, t_areas, bcs (walls, ibc_arrays), node_db, elemnt_db */
  if ((rc = find_edges(o, p))) { orc_destroy(o); return rc; }
  t_areas(o);
  unsigned char* bcnode = (unsigned char*)xcalloc((size_t)N + 1, 1);
  for (int b = 1; b <= o->n_in; b++)
    for (int i = 1; i <= o->n_qin[b - 1]; i++) {
      int32_t q = QIN_NODES(i, b);
      if (q < 1 || q > N) { free(bcnode); orc_destroy(o); return set_err(STORM_ERR_MESH, "inflow node out of range"); }
      bcnode[q] = 1;
    }
  for (int b = 1; b <= o->n_out; b++)
    for (int i = 1; i <= o->n_hbc[b - 1]; i++) {
      int32_t q = HBC_NODES(i, b);
      if (q < 1 || q > N) { free(bcnode); orc_destroy(o); return set_err(STORM_ERR_MESH, "outflow node out of range"); }
      bcnode[q] = 1;
    }
  rc = walls(o, bcnode);
  free(bcnode);
  if (rc || (rc = ibc_arrays(o)) || (rc = node_db(o)) || (rc = elemnt_db(o))) { orc_destroy(o); return rc; }

  /* ---- dataprepFVT.f90:31-306 ---- */
  c2v_setup(o); /* :69 */
  o->z = (double*)xcalloc(T, sizeof(double));
  o->zvtx = (double*)xcalloc(N, sizeof(double));
  o->cd = (double*)xcalloc(T, sizeof(double));
  if (p->zb_at_vertices) { /* :73-77 */
    memcpy(o->zvtx, p->zb, sizeof(double) * N);
    vtx2ctr(o, o->zvtx, o->z);
  } else { /* :79-87 */
    ctr2vtx3(o, p->zb, o->zvtx);
    vtx2ctr(o, o->zvtx, o->z);
  }
  if (p->cd_at_vertices) vtx2ctr(o, p->cd, o->cd); /* :132-134 */
  else memcpy(o->cd, p->cd, sizeof(double) * T);
  /* windforcing.f90:80-104 (text input, centred finite-volume solvers) */
  if (p->wind_c0 && p->wind_x && p->wind_y) {
    double* c0 = (double*)xcalloc((size_t)T, sizeof(double));
    double* wx = (double*)xcalloc((size_t)T, sizeof(double));
    double* wy = (double*)xcalloc((size_t)T, sizeof(double));
    if (p->wind_at_vertices) {
      vtx2ctr(o, p->wind_c0, c0);
      vtx2ctr(o, p->wind_x, wx);
      vtx2ctr(o, p->wind_y, wy);
    } else {
      memcpy(c0, p->wind_c0, sizeof(double) * T);
      memcpy(wx, p->wind_x, sizeof(double) * T);
      memcpy(wy, p->wind_y, sizeof(double) * T);
    }
    const double rho = 998.60; /* constants.f90:29 */
    o->wcoef1 = (double*)xcalloc((size_t)T, sizeof(double));
    o->wcoef2 = (double*)xcalloc((size_t)T, sizeof(double));
    for (int32_t i = 1; i <= T; i++) {
      double windmag = sqrt(wx[i - 1] * wx[i - 1] + wy[i - 1] * wy[i - 1]);
      o->wcoef1[i - 1] = c0[i - 1] * wx[i - 1] * windmag / rho;
      o->wcoef2[i - 1] = c0[i - 1] * wy[i - 1] * windmag / rho;
    }
    free(c0);
    free(wx);
    free(wy);
  }
  /* :161-173 rc (before the normals are normalised) */
  o->rc_x = (double*)xcalloc((size_t)3 * T, sizeof(double));
  o->rc_y = (double*)xcalloc((size_t)3 * T, sizeof(double));
  for (int32_t i = 1; i <= T; i++)
    for (int j = 1; j <= 3; j++) {
      int32_t k = abs(GE(i, j));
      double xc = half * (NX(EP(k, 1)) + NX(EP(k, 2)));
      double yc = half * (NY(EP(k, 1)) + NY(EP(k, 2)));
      RCX(i, j) = xc - XC(i);
      RCY(i, j) = yc - YC(i);
    }
  /* :176-181 */
  for (int32_t i = 1; i <= o->n_edges; i++) {
    ENRM(i, 1) = ENRM(i, 1) / ELEN(i);
    ENRM(i, 2) = ENRM(i, 2) / ELEN(i);
    ETAN(i, 1) = ETAN(i, 1) / ELEN(i);
    ETAN(i, 2) = ETAN(i, 2) / ELEN(i);
  }
  lsq_setup(o); /* :221 */
  /* :256-273 RK tables */
  memset(o->rkalpha, 0, sizeof o->rkalpha);
  memset(o->rkbeta, 0, sizeof o->rkbeta);
  switch (o->opt.rkorder) {
    case 1: o->rkalpha[1][0] = one; o->rkbeta[1] = one; break;
    case 2:
      o->rkalpha[1][0] = one; o->rkbeta[1] = one;
      o->rkalpha[2][0] = half; o->rkalpha[2][1] = half; o->rkbeta[2] = half;
      break;
    case 3:
      o->rkalpha[1][0] = one;
      o->rkalpha[2][0] = 0.750; o->rkalpha[2][1] = 0.250;
      o->rkalpha[3][0] = ONE_THIRD; o->rkalpha[3][1] = zero; o->rkalpha[3][2] = 2.0 / 3.0;
      o->rkbeta[1] = one; o->rkbeta[2] = 0.250; o->rkbeta[3] = 2.0 / 3.0;
      break;
  }
  /* :278-286 */
  o->bch_max = zero;
  for (int32_t l = 1; l <= o->n_bcedges; l++) {
    if (!o->qbar[l - 1]) continue;
    int32_t k = o->bcedges[l - 1];
    o->bch_max = fmax2(o->bch_max, ZVTX(EP(k, 1)));
    o->bch_max = fmax2(o->bch_max, ZVTX(EP(k, 2)));
  }
  /* :290-306 csortedz: bubble sort on zvtx */
  o->csortedz = (int32_t*)xcalloc((size_t)3 * T, sizeof(int32_t));
  for (int32_t i = 1; i <= T; i++) {
    CSZ(i, 1) = GV(i, 1); CSZ(i, 2) = GV(i, 2); CSZ(i, 3) = GV(i, 3);
    for (int j = 1; j <= 2; j++)
      for (int k = 1; k <= 2; k++)
        if (ZVTX(CSZ(i, k)) > ZVTX(CSZ(i, k + 1))) {
          int32_t aux = CSZ(i, k); CSZ(i, k) = CSZ(i, k + 1); CSZ(i, k + 1) = aux;
        }
  }
  /* solution arrays */
  size_t L = (size_t)o->opt.rkorder + 1;
  o->h = (double*)xcalloc(T, sizeof(double));
  o->u = (double*)xcalloc(T, sizeof(double));
  o->v = (double*)xcalloc(T, sizeof(double));
  o->zeta = (double*)xcalloc(T, sizeof(double));
  o->u_mag = (double*)xcalloc(T, sizeof(double));
  o->wavec = (double*)xcalloc(T, sizeof(double));
  o->rough = (double*)xcalloc(T, sizeof(double));
  o->hvtx = (double*)xcalloc(N, sizeof(double));
  o->zetavtx = (double*)xcalloc(N, sizeof(double));
  o->delh_x = (double*)xcalloc(T, sizeof(double)); o->delh_y = (double*)xcalloc(T, sizeof(double));
  o->delu_x = (double*)xcalloc(T, sizeof(double)); o->delu_y = (double*)xcalloc(T, sizeof(double));
  o->delv_x = (double*)xcalloc(T, sizeof(double)); o->delv_y = (double*)xcalloc(T, sizeof(double));
  o->delz_x = (double*)xcalloc(T, sizeof(double)); o->delz_y = (double*)xcalloc(T, sizeof(double));
  o->phi = (double*)xcalloc((size_t)3 * T, sizeof(double));
  o->drycell = (int32_t*)xcalloc(T, sizeof(int32_t));
  o->rkh = (double*)xcalloc(L * T, sizeof(double));
  o->rku = (double*)xcalloc(L * T, sizeof(double));
  o->rkv = (double*)xcalloc(L * T, sizeof(double));
  o->fedge = (double*)xcalloc((size_t)3 * (o->flow_edges1 + 1), sizeof(double));
  o->fedge_set = (int32_t*)xcalloc((size_t)o->flow_edges1 + 1, sizeof(int32_t));
  if ((rc = cvprep(o, p))) { orc_destroy(o); return rc; } /* dataprepFVT.f90:308-309 */
  *out = o;
  return 0;
}

void orc_destroy(orc_t* o) {
  if (!o) return;
  void* ptrs[] = {o->node_x, o->node_y, o->tri_vertex, o->tri_edge, o->tri_area, o->tri_perim, o->tri_xc,
                  o->tri_yc, o->edge_p, o->edge_e, o->edge_normal, o->edge_tang, o->edge_length, o->rc_x,
                  o->rc_y, o->t2t, o->lsq_dx, o->lsq_dy, o->lsq_w, o->lsq_a, o->lsq_b, o->lsq_c, o->lsq_det,
                  o->t2t3, o->n2t, o->c2v_w, o->c2v_wn, o->csortedz, o->flowedg1, o->walledg1, o->bcedges,
                  o->hbar, o->qbar, o->z, o->zvtx, o->cd, o->vtype, o->n_qin, o->qin_nodes, o->bcedgesinflow,
                  o->n_timeserq, o->qin, o->timelocq, o->timeserq, o->htype, o->n_hbc, o->hbc_nodes,
                  o->bcedgesoutflow, o->n_timeserh, o->hbc, o->timeloch, o->timeserh, o->h, o->u, o->v,
                  o->zeta, o->u_mag, o->wavec, o->hvtx, o->zetavtx, o->rough, o->delh_x, o->delh_y, o->delu_x,
                  o->delu_y, o->delv_x, o->delv_y, o->delz_x, o->delz_y, o->phi, o->drycell, o->rkh, o->rku,
                  o->rkv, o->fedge, o->fedge_set, o->phi0, o->rs_seq, o->wcoef1, o->wcoef2,
                  o->cvtrigin, o->cvtrigout, o->ncvtable, o->cvptoin, o->cvrin, o->cvhead, o->cvq, o->cvsrc};
  for (size_t i = 0; i < sizeof ptrs / sizeof ptrs[0]; i++) free(ptrs[i]);
  free(o);
}

int orc_export_mesh(const orc_t* o, StormFvtMesh* m) {
  memset(m, 0, sizeof *m);
  m->n_pts = o->n_pts; m->n_elems = o->n_elems; m->n_edges = o->n_edges;
  m->node_x = o->node_x; m->node_y = o->node_y;
  m->tri_vertex = o->tri_vertex; m->tri_edge = o->tri_edge;
  m->tri_area = o->tri_area; m->tri_perim = o->tri_perim; m->tri_xc = o->tri_xc; m->tri_yc = o->tri_yc;
  m->edge_p = o->edge_p; m->edge_e = o->edge_e; m->edge_normal = o->edge_normal; m->edge_tang = o->edge_tang;
  m->edge_length = o->edge_length;
  m->rc_x = o->rc_x; m->rc_y = o->rc_y;
  m->t2t_ncol = o->t2t_ncol; m->t2t = o->t2t;
  m->lsq_dx = o->lsq_dx; m->lsq_dy = o->lsq_dy; m->lsq_w = o->lsq_w;
  m->lsq_a = o->lsq_a; m->lsq_b = o->lsq_b; m->lsq_c = o->lsq_c; m->lsq_det = o->lsq_det;
  m->t2t3 = o->t2t3;
  m->n2t_ncol = o->n2t_ncol; m->n2t = o->n2t;
  m->c2v_ncol = o->c2v_ncol; m->c2v_w = o->c2v_w;
  m->csortedz = o->csortedz;
  m->flow_edges1 = o->flow_edges1; m->flowedg1 = o->flowedg1;
  m->wall_edges1 = o->wall_edges1; m->walledg1 = o->walledg1;
  m->n_bcedges = o->n_bcedges; m->bcedges = o->bcedges; m->hbar = o->hbar;
  m->z = o->z; m->zvtx = o->zvtx; m->cd = o->cd;
  m->n_inflowbdr = o->n_in; m->vtype = o->vtype; m->qin = o->qin;
  m->bcin_ld = o->bcin_ld; m->bcedgesinflow = o->bcedgesinflow;
  m->tsq_ld = o->tsq_ld; m->n_timeserq = o->n_timeserq; m->timelocq = o->timelocq; m->timeserq = o->timeserq;
  m->n_outflowbdr = o->n_out; m->htype = o->htype; m->hbc = o->hbc;
  m->bcout_ld = o->bcout_ld; m->bcedgesoutflow = o->bcedgesoutflow;
  m->hbc_ld = o->hbc_ld; m->n_hbc = o->n_hbc; m->hbc_nodes = o->hbc_nodes;
  m->tsh_ld = o->tsh_ld; m->n_timeserh = o->n_timeserh; m->timeloch = o->timeloch; m->timeserh = o->timeserh;
  m->bch_max = o->bch_max;
  m->wcoef1 = o->wcoef1;
  m->wcoef2 = o->wcoef2;
  m->n_culvert = o->ncv; m->cv_ld = o->cv_ld;
  m->cvtrigin = o->cvtrigin; m->cvtrigout = o->cvtrigout; m->cvptoin = o->cvptoin; m->cvrin = o->cvrin;
  m->ncvtable = o->ncvtable; m->cvhead = o->cvhead; m->cvq = o->cvq;
  return 0;
}

void orc_set_threads(orc_t* o, int n) { o->nthreads = n < 1 ? 1 : n; }

/* ========================================================================== */
/*                     S O L V E R   (solverFVT.f90)                          */
/* ========================================================================== */

/* bed_slope_VTX.f90:22-38 */
static void bed_slope_vtx(orc_t* o) {
  for (int32_t i = 1; i <= o->n_elems; i++) {
    double x1 = NX(GV(i, 1)), y1 = NY(GV(i, 1));
    double x2 = NX(GV(i, 2)), y2 = NY(GV(i, 2));
    double x3 = NX(GV(i, 3)), y3 = NY(GV(i, 3));
    double zz1 = ZVTX(GV(i, 1)), zz2 = ZVTX(GV(i, 2)), zz3 = ZVTX(GV(i, 3));
    o->delz_x[i - 1] = half * (zz1 * (y2 - y3) + zz2 * (y3 - y1) + zz3 * (y1 - y2)) / AREA(i);
    o->delz_y[i - 1] = half * (zz1 * (x3 - x2) + zz2 * (x1 - x3) + zz3 * (x2 - x1)) / AREA(i);
  }
}

int orc_set_state(orc_t* o, const double* h, const double* u, const double* v) {
  const int32_t T = o->n_elems;
  memcpy(o->h, h, sizeof(double) * T);
  memcpy(o->u, u, sizeof(double) * T);
  memcpy(o->v, v, sizeof(double) * T);
  /* solverFVT.f90:53-62 */
  o->iter = 0; o->rmax = zero; o->stime = zero; o->ttime = zero; o->delt = zero; o->converged = 0;
  memset(o->delh_x, 0, sizeof(double) * T); memset(o->delh_y, 0, sizeof(double) * T);
  memset(o->delu_x, 0, sizeof(double) * T); memset(o->delu_y, 0, sizeof(double) * T);
  memset(o->delv_x, 0, sizeof(double) * T); memset(o->delv_y, 0, sizeof(double) * T);
  bed_slope_vtx(o);   /* :93 */
  get_time_bcs(o, o->stime); /* :103 */
  for (int32_t b = 0; b < o->n_in; b++) o->qin_it[b] = o->qin[b];
  for (int32_t b = 0; b < o->n_out; b++) o->hbc_it[b] = o->hbc[b];
  /* :122-126 */
  int K = o->opt.rkorder;
  for (int32_t i = 1; i <= T; i++) {
    RKU(i, K) = H(i) * U(i);
    RKV(i, K) = H(i) * V(i);
    RKH(i, K) = H(i);
  }
  o->have_state = 1;
  return 0;
}

/* find_dry_cells.f90:25-42 */
static void find_dry_cells(orc_t* o) {
  const int32_t T = o->n_elems;
  const double h_dry = o->opt.h_dry, h_wet = o->opt.h_wet;
#pragma omp parallel for num_threads(o->nthreads) schedule(static)
  for (int32_t i = 1; i <= T; i++) {
    int dry = H(i) < h_dry;
    double um = zero;
    if (!dry) um = sqrt(U(i) * U(i) + V(i) * V(i));
    o->u_mag[i - 1] = um;
    if (!dry && (H(i) < h_wet) && equals(um, zero)) dry = 1;
    DRY(i) = dry;
  }
}

/* lsq_grad_array.f90:60-73 */
static inline void lsq_grad(const orc_t* o, const double* phi, int32_t i, double* gx, double* gy) {
  double di = zero, ei = zero;
  int32_t n = T2T(i, 1);
  for (int32_t k = 1; k <= n; k++) {
    double dphi = phi[T2T(i, k + 1) - 1] - phi[i - 1];
    di = di + LW(i, k) * dphi * LDX(i, k);
    ei = ei + LW(i, k) * dphi * LDY(i, k);
  }
  *gx = (o->lsq_c[i - 1] * di - o->lsq_b[i - 1] * ei) / o->lsq_det[i - 1];
  *gy = (o->lsq_a[i - 1] * ei - di * o->lsq_b[i - 1]) / o->lsq_det[i - 1];
}

/* limiterBJ.f90:42-81 with beta = one (cell_grads.f90:59) */
static inline void limiter_bj(const orc_t* o, const double* q, int32_t i, double* gx, double* gy) {
  const double beta = one;
  double q0 = q[i - 1], r[3];
  for (int j = 1; j <= 3; j++) {
    int32_t k = T2T3(j, i);
    double qneighb = (k < 1) ? q0 : q[k - 1];
    double qmin = fmin2(q0, qneighb);
    double qmax = fmax2(q0, qneighb);
    double qj = q0 + *gx * RCX(i, j) + *gy * RCY(i, j);
    double delq = qj - q0;
    double rj;
    if (equals(delq, zero)) rj = one;
    else if (delq < 0) rj = (qmin - q0) / delq;
    else rj = (qmax - q0) / delq;
    double a = fmin2(beta * rj, one);
    double b = fmin2(rj, beta);
    r[j - 1] = fmax2(a, b);
  }
  double phi = fmin2(fmin2(r[0], r[1]), r[2]);
  *gx = phi * *gx;
  *gy = phi * *gy;
}

/* cell_grads.f90:24-75 followed by hgradfix2.f90:48-98 (solver 2) */
static void cell_grads_and_fix(orc_t* o, int rkstep) {
  const int32_t T = o->n_elems;
  const int lim = o->opt.opt_limiter;
#pragma omp parallel for num_threads(o->nthreads) schedule(static)
  for (int32_t i = 1; i <= T; i++) {
    double hx = zero, hy = zero, ux = zero, uy = zero, vx = zero, vy = zero;
    if (lim == 1 || lim == 2) {
      lsq_grad(o, o->zeta, i, &hx, &hy);
      lsq_grad(o, o->u, i, &ux, &uy);
      lsq_grad(o, o->v, i, &vx, &vy);
    }
    if (lim == 2) {
      limiter_bj(o, o->zeta, i, &hx, &hy);
      limiter_bj(o, o->u, i, &ux, &uy);
      limiter_bj(o, o->v, i, &vx, &vy);
    }
    o->delh_x[i - 1] = hx - o->delz_x[i - 1];
    o->delh_y[i - 1] = hy - o->delz_y[i - 1];
    o->delu_x[i - 1] = ux; o->delu_y[i - 1] = uy;
    o->delv_x[i - 1] = vx; o->delv_y[i - 1] = vy;
  }
  /* hgradfix2: the tests read zeta/z/drycell only, so the loop is order-free;
   * u and v are zeroed after every gradient above was taken. */
#pragma omp parallel for num_threads(o->nthreads) schedule(static)
  for (int32_t i = 1; i <= T; i++) {
    if (DRY(i)) continue;
    int setgrad = ZETA(i) < ZVTX(CSZ(i, 3));
    for (int k = 1; k <= 3; k++) {
      int32_t l = T2T3(k, i);
      if (l < 1) continue;
      if (DRY(l) && Z(l) < ZETA(i)) setgrad = 0;
    }
    if (setgrad) {
      o->delh_x[i - 1] = -o->delz_x[i - 1];
      o->delh_y[i - 1] = -o->delz_y[i - 1];
      U(i) = zero;
      V(i) = zero;
      RKU(i, rkstep - 1) = zero;
      RKV(i, rkstep - 1) = zero;
      o->delu_x[i - 1] = zero; o->delu_y[i - 1] = zero;
      o->delv_x[i - 1] = zero; o->delv_y[i - 1] = zero;
    }
  }
}

/* to_vertices.f90:26-57 (hvtx path: ctr2vtxWSE type 3, the cap, positivity_vtx,
 * the u/v zeroing of cells with a dry vertex) and enforce_bcs.f90:37-56 (the
 * stage-boundary vertex depth).  Vertex velocities are output-only. */
static void to_vertices(orc_t* o) {
  const int32_t N = o->n_pts, T = o->n_elems;
  const double h_dry = o->opt.h_dry;
#pragma omp parallel for num_threads(o->nthreads) schedule(static)
  for (int32_t i = 1; i <= N; i++) {
    /* ctr2vtxWSE.f90:89-105 */
    double id = zero, a = zero;
    int counter = 0;
    for (int32_t j = 2; j <= N2T(i, 1) + 1; j++) {
      int32_t k = N2T(i, j);
      if (DRY(k)) continue;
      counter++;
      id = id + C2VW(i, j - 1);
      a = a + C2VW(i, j - 1) * ZETA(k);
    }
    double zv = counter > 0 ? a / id : ZVTX(i);
    o->zetavtx[i - 1] = zv;
    HVTX(i) = zv - ZVTX(i);
    /* to_vertices.f90:31-40 */
    double zetaref = ZVTX(i);
    for (int32_t j = 2; j <= N2T(i, 1) + 1; j++) {
      int32_t k = N2T(i, j);
      if (DRY(k)) continue;
      zetaref = fmax2(ZETA(k), zetaref);
    }
    zv = fmin2(zv, zetaref);
    o->zetavtx[i - 1] = zv;
    HVTX(i) = zv - ZVTX(i);
    /* positivity_vtx.f90:22-27 */
    if (HVTX(i) < zero) { HVTX(i) = zero; o->zetavtx[i - 1] = ZVTX(i); }
  }
  /* to_vertices.f90:44-55 */
#pragma omp parallel for num_threads(o->nthreads) schedule(static)
  for (int32_t i = 1; i <= T; i++) {
    if (DRY(i)) continue;
    int flag = 1;
    for (int j = 1; j <= 3; j++) flag = flag && (HVTX(GV(i, j)) > h_dry);
    if (!flag) { U(i) = zero; V(i) = zero; }
  }
  /* enforce_bcs.f90:37-56, htype 1: the relaxed update is overwritten by the
   * instantaneous one, leaving h0(j) = MAX(zero,hbc(i0) - z0(j)) */
  for (int32_t b = 1; b <= o->n_out; b++) {
    if (o->htype[b - 1] != 1) continue;
    for (int32_t i = 1; i <= o->n_hbc[b - 1]; i++) {
      int32_t j = HBC_NODES(i, b);
      double hnot = fmax2(zero, o->hbc[b - 1] - ZVTX(j));
      double incr = 0.100 * (hnot - HVTX(j)); /* alpha = 0.1 (initialize_options.f90:86) */
      if (fabs(incr) < 0.0100) incr = hnot - HVTX(j); /* kappa = 0.01 */
      HVTX(j) = HVTX(j) - incr;
      HVTX(j) = fmax2(zero, o->hbc[b - 1] - ZVTX(j));
    }
  }
}

/* flux_ac.f90:48-126 (Roe with the Alcrudo entropy fix) */
static void flux_ac(double nx, double ny, double hlefty, double uleft, double vleft, double hrighty,
                    double uright, double vright, double* flux) {
  const double delta = 0.10;
  double hleft = hlefty, hright = hrighty;
  double fileft[3], gileft[3], firight[3], giright[3];
  fileft[0] = hleft * uleft;
  fileft[1] = hleft * uleft * uleft + half * g * hleft * hleft;
  fileft[2] = hleft * uleft * vleft;
  gileft[0] = hleft * vleft;
  gileft[1] = hleft * uleft * vleft;
  gileft[2] = hleft * vleft * vleft + half * g * hleft * hleft;
  firight[0] = hright * uright;
  firight[1] = hright * uright * uright + half * g * hright * hright;
  firight[2] = hright * uright * vright;
  giright[0] = hright * vright;
  giright[1] = hright * uright * vright;
  giright[2] = hright * vright * vright + half * g * hright * hright;
  hleft = fmax2(hleft, SMALL_F);
  double hleftsqr = sqrt(hleft);
  hright = fmax2(hright, SMALL_F);
  double hrightsqr = sqrt(hright);
  double denom = hrightsqr + hleftsqr;
  double uavg = (uright * hrightsqr + uleft * hleftsqr) / denom;
  double vavg = (vright * hrightsqr + vleft * hleftsqr) / denom;
  double cavg = sqrt(half * g * (hleft + hright));
  double qdiff[3];
  qdiff[0] = hright - hleft;
  qdiff[1] = hright * uright - hleft * uleft;
  qdiff[2] = hright * vright - hleft * vleft;
  double rev[3][3], lev[3][3], a[3][3], temp1[3][3], temp2[3][3], aq[3];
  rev[0][0] = zero; rev[0][1] = one; rev[0][2] = one;
  rev[1][0] = ny; rev[1][1] = uavg - cavg * nx; rev[1][2] = uavg + cavg * nx;
  rev[2][0] = -nx; rev[2][1] = vavg - cavg * ny; rev[2][2] = vavg + cavg * ny;
  lev[0][0] = -(uavg * ny - vavg * nx);
  lev[0][1] = ny;
  lev[0][2] = -nx;
  lev[1][0] = half * (uavg * nx + vavg * ny) / cavg + half;
  lev[1][1] = -(half * nx / cavg);
  lev[1][2] = -(half * ny / cavg);
  lev[2][0] = -(half * (uavg * nx + vavg * ny) / cavg) + half;
  lev[2][1] = half * nx / cavg;
  lev[2][2] = half * ny / cavg;
  double eigv[3];
  eigv[0] = fmax2(fabs(uavg * nx + vavg * ny), delta);
  eigv[1] = fmax2(fabs(uavg * nx + vavg * ny - cavg), delta);
  eigv[2] = fmax2(fabs(uavg * nx + vavg * ny + cavg), delta);
  memset(a, 0, sizeof a);
  a[0][0] = eigv[0]; a[1][1] = eigv[1]; a[2][2] = eigv[2];
  /* MATMUL: dest(i,j) = 0, then dest += x(i,k)*y(k,j) for k = 1..3 */
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double s = zero;
      for (int k = 0; k < 3; k++) s = s + rev[i][k] * a[k][j];
      temp1[i][j] = s;
    }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double s = zero;
      for (int k = 0; k < 3; k++) s = s + temp1[i][k] * lev[k][j];
      temp2[i][j] = s;
    }
  for (int i = 0; i < 3; i++) {
    double s = zero;
    for (int k = 0; k < 3; k++) s = s + temp2[i][k] * qdiff[k];
    aq[i] = s;
  }
  for (int i = 0; i < 3; i++)
    flux[i] = half * (firight[i] * nx + giright[i] * ny + fileft[i] * nx + gileft[i] * ny - aq[i]);
}

/*
 * flux_HLL.f90:41-110 (Yoon & Kang wave speeds).  Two defects of the reference
 * are fixed here: (1) flux(3) is never assigned in the subsonic branch because
 * :108 writes flux(2) a second time -- flux(3) takes that expression; (2) the
 * subsonic branch divides only the last term by (sright - sleft) (:104-109), so
 * F(q,q) = (sright-sleft)*F(q) -- the whole HLL numerator is divided, as in the
 * standard HLL formula.  The debug stop at :88-91 (sleft > 0 .AND. sright < 0)
 * is reported through *bad instead of stopping.
 */
static void flux_hll(double nx, double ny, double hleft, double uleft, double vleft, double hright,
                     double uright, double vright, double h0, double* flux, int* bad) {
  double cleft = sqrt(g * hleft);
  double cright = sqrt(g * hright);
  double ustar = half * ((uleft + uright) * nx + (vleft + vright) * ny) + cleft - cright;
  double cstar = half * (cleft + cright) + ((uleft - uright) * nx + (vleft - vright) * ny) / 4.0;
  double sleft, sright, aux1, aux2;
  if (hleft < h0) sleft = uright * nx + vright * ny - 2.0 * cright;
  else if (hright < h0) sleft = uleft * nx + vleft * ny - cleft;
  else { aux1 = uleft * nx + vleft * ny - cleft; aux2 = ustar - cstar; sleft = fmin2(aux1, aux2); }
  if (hleft < h0) sright = uright * nx + vright * ny + cright;
  else if (hright < h0) sright = uleft * nx + vleft * ny + 2.0 * cleft;
  else { aux1 = uright * nx + vright * ny - cright; aux2 = ustar + cstar; sright = fmax2(aux1, aux2); }
  double fleft[3], gleft[3], fright[3], gright[3];
  fleft[0] = hleft * uleft * nx;
  fleft[1] = (hleft * uleft * uleft + half * g * hleft * hleft) * nx;
  fleft[2] = hleft * uleft * vleft * nx;
  gleft[0] = hleft * vleft * ny;
  gleft[1] = hleft * uleft * vleft * ny;
  gleft[2] = (hleft * vleft * vleft + half * g * hleft * hleft) * ny;
  fright[0] = hright * uright * nx;
  fright[1] = (hright * uright * uright + half * g * hright * hright) * nx;
  fright[2] = hright * uright * vright * nx;
  gright[0] = hright * vright * ny;
  gright[1] = hright * uright * vright * ny;
  gright[2] = (hright * vright * vright + half * g * hright * hright) * ny;
  if (sleft > zero && sright < zero) *bad = 1;
  if (sleft > zero) {
    for (int i = 0; i < 3; i++) flux[i] = fleft[i] + gleft[i];
  } else if (sright < zero) {
    for (int i = 0; i < 3; i++) flux[i] = fright[i] + gright[i];
  } else {
    aux1 = sright - sleft;
    flux[0] = (sright * (fleft[0] + gleft[0]) - sleft * (fright[0] + gright[0]) + sleft * sright * (hright - hleft)) / aux1;
    flux[1] = (sright * (fleft[1] + gleft[1]) - sleft * (fright[1] + gright[1]) +
               sleft * sright * (hright * uright - hleft * uleft)) / aux1;
    flux[2] = (sright * (fleft[2] + gleft[2]) - sleft * (fright[2] + gright[2]) +
               sleft * sright * (hright * vright - hleft * vleft)) / aux1;
  }
}

/* flux_rusanov.f90:47-80 */
static void flux_rusanov(double nx, double ny, double hleft, double uleft, double vleft, double sqrtghleft,
                         double hright, double uright, double vright, double sqrtghright, double* flux) {
  double fileft[3], gileft[3], firight[3], giright[3], qdiff[3];
  fileft[0] = hleft * uleft;
  fileft[1] = hleft * uleft * uleft + half * g * hleft * hleft;
  fileft[2] = hleft * uleft * vleft;
  gileft[0] = hleft * vleft;
  gileft[1] = hleft * uleft * vleft;
  gileft[2] = hleft * vleft * vleft + half * g * hleft * hleft;
  firight[0] = hright * uright;
  firight[1] = hright * uright * uright + half * g * hright * hright;
  firight[2] = hright * uright * vright;
  giright[0] = hright * vright;
  giright[1] = hright * uright * vright;
  giright[2] = hright * vright * vright + half * g * hright * hright;
  double ul = uleft * nx + vleft * ny;
  double ur = uright * nx + vright * ny;
  double splus = fmax2(fabs(ul) + sqrtghleft, fabs(ur) + sqrtghright);
  qdiff[0] = hright - hleft;
  qdiff[1] = hright * uright - hleft * uleft;
  qdiff[2] = hright * vright - hleft * vleft;
  for (int i = 0; i < 3; i++)
    flux[i] = half * (firight[i] * nx + giright[i] * ny + fileft[i] * nx + gileft[i] * ny - splus * qdiff[i]);
}

/* local_edge.f90:26-39 */
static inline int local_edge(const orc_t* o, int32_t i, int32_t k) {
  for (int j = 1; j <= 3; j++)
    if (abs(GE(i, j)) == k) return j;
  return -1;
}

/* invisc_fluxes.f90:39-147: the flux of interior edge k (no accumulation). */
static int interior_flux(const orc_t* o, int32_t k, double* f, int* bad) {
  int32_t i = EE(k, 1), j = EE(k, 2);
  int set_wall = 0;
  const double h_dry = o->opt.h_dry, h_wet = o->opt.h_wet;
  if (DRY(i) && DRY(j)) return 0;
  double nx = ENRM(k, 1), ny = ENRM(k, 2);
  int m = local_edge(o, i, k);
  if (GE(i, m) < 0) { nx = -nx; ny = -ny; } /* invert_edge_dirs.f90:20-25 */
  double hleft, uleft, vleft, hright, uright, vright;
  if (DRY(i)) { uleft = zero; vleft = zero; hleft = zero; }
  else {
    hleft = H(i) + o->delh_x[i - 1] * RCX(i, m) + o->delh_y[i - 1] * RCY(i, m);
    if (hleft < zero) hleft = zero;
    uleft = U(i) + o->delu_x[i - 1] * RCX(i, m) + o->delu_y[i - 1] * RCY(i, m);
    vleft = V(i) + o->delv_x[i - 1] * RCX(i, m) + o->delv_y[i - 1] * RCY(i, m);
  }
  int n = local_edge(o, j, k);
  if (DRY(j)) { uright = zero; vright = zero; hright = zero; }
  else {
    hright = H(j) + o->delh_x[j - 1] * RCX(j, n) + o->delh_y[j - 1] * RCY(j, n);
    if (hright < zero) hright = zero;
    uright = U(j) + o->delu_x[j - 1] * RCX(j, n) + o->delu_y[j - 1] * RCY(j, n);
    vright = V(j) + o->delv_x[j - 1] * RCX(j, n) + o->delv_y[j - 1] * RCY(j, n);
  }
  if (hleft < h_dry && hright < h_dry) return 0;
  /* ALGORITHM I1 (:87-119) */
  if (DRY(i) || DRY(j)) {
    double h0 = fmax2(hright, hleft);
    double z0 = half * (ZVTX(EP(k, 1)) + ZVTX(EP(k, 2)));
    h0 = h0 + z0;
    if (DRY(i))
      if (Z(i) + h_wet > h0) { set_wall = 1; hleft = hright; }
    if (DRY(j))
      if (Z(j) + h_wet > h0) { set_wall = 1; hright = hleft; }
  }
  if (set_wall) {
    f[0] = zero;
    hleft = fmax2(hleft, hright);
    f[1] = half * g * hleft * hleft * nx;
    f[2] = half * g * hleft * hleft * ny;
  } else if (o->opt.flux == STORM_FLUX_HLL) {
    flux_hll(nx, ny, hleft, uleft, vleft, hright, uright, vright, h_dry, f, bad);
  } else if (o->opt.flux == STORM_FLUX_RUSANOV) {
    flux_rusanov(nx, ny, hleft, uleft, vleft, o->wavec[i - 1], hright, uright, vright, o->wavec[j - 1], f);
  } else {
    flux_ac(nx, ny, hleft, uleft, vleft, hright, uright, vright, f);
  }
  return 1;
}

/* wenslp3_fluxes.f90:34-67 (btype 0) */
static void wenslp3_fluxes(orc_t* o) {
  const double hdry = o->opt.h_dry;
  for (int32_t l = 1; l <= o->wall_edges1; l++) {
    int32_t k = o->walledg1[l - 1];
    int32_t i = EE(k, 1) < 1 ? EE(k, 2) : EE(k, 1);
    if (DRY(i)) continue;
    double h1 = HVTX(EP(k, 1)), h2 = HVTX(EP(k, 2));
    double hedge = sqrt((h1 * h1 + h1 * h2 + h2 * h2) * ONE_THIRD);
    if (hedge < zero) hedge = zero;
    if (hedge < hdry) continue;
    int m = local_edge(o, i, k);
    double nx = ENRM(k, 1), ny = ENRM(k, 2);
    if (GE(i, m) < 0) { nx = -nx; ny = -ny; }
    PHI(i, 2) = PHI(i, 2) - half * g * hedge * hedge * nx * ELEN(k);
    PHI(i, 3) = PHI(i, 3) - half * g * hedge * hedge * ny * ELEN(k);
  }
}

/* weslp2_fluxes.f90:34-76 (btype 1) */
static void weslp2_fluxes(orc_t* o) {
  const double hdry = o->opt.h_dry;
  for (int32_t l = 1; l <= o->wall_edges1; l++) {
    int32_t k = o->walledg1[l - 1];
    int32_t i = EE(k, 1) < 1 ? EE(k, 2) : EE(k, 1);
    if (DRY(i)) continue;
    int m = local_edge(o, i, k);
    double hleft = H(i) + o->delh_x[i - 1] * RCX(i, m) + o->delh_y[i - 1] * RCY(i, m);
    if (hleft < hdry) continue;
    double uleft = U(i) + o->delu_x[i - 1] * RCX(i, m) + o->delu_y[i - 1] * RCY(i, m);
    double vleft = V(i) + o->delv_x[i - 1] * RCX(i, m) + o->delv_y[i - 1] * RCY(i, m);
    double nx = ENRM(k, 1), ny = ENRM(k, 2), tx = ETAN(k, 1), ty = ETAN(k, 2);
    if (GE(i, m) < 0) { nx = -nx; ny = -ny; tx = -tx; ty = -ty; }
    double uright = uleft * tx + vleft * ty;
    uright = uright + 2.0 * sqrt(g * hleft);
    double hright = uright * uright / 4.0 / g;
    double f2 = half * g * hright * hright * nx;
    double f3 = half * g * hright * hright * ny;
    double dh = zero; /* :69-71 computes dh, then sets it to zero */
    PHI(i, 2) = PHI(i, 2) - (f2 + dh * nx) * ELEN(k);
    PHI(i, 3) = PHI(i, 3) - (f3 + dh * ny) * ELEN(k);
  }
}

/* reconstructed edge state of cell i at its slot m (shared by the BC routines) */
#define EDGE_H(i, m) (H(i) + o->delh_x[(i)-1] * RCX(i, m) + o->delh_y[(i)-1] * RCY(i, m))
#define EDGE_U(i, m) (U(i) + o->delu_x[(i)-1] * RCX(i, m) + o->delu_y[(i)-1] * RCY(i, m))
#define EDGE_V(i, m) (V(i) + o->delv_x[(i)-1] * RCX(i, m) + o->delv_y[(i)-1] * RCY(i, m))

/* inflowQbyH.f90:31-212 (vtype 1) and :221-402 (vtype 5, wet cells only). */
static void inflow_q_by_h(orc_t* o, int vt) {
  const double h_dry = o->opt.h_dry;
  for (int32_t ic = 1; ic <= o->n_in; ic++) {
    if (o->vtype[ic - 1] != vt) continue;
    double qin = o->qin[ic - 1];
    if (qin < VSMALL) continue;
    int32_t ne = BCIN(0, ic);
    double atotal = zero;
    for (int32_t l = 1; l <= ne; l++) {
      int32_t k = BCIN(l, ic);
      int32_t i = EE(k, 1) < 1 ? EE(k, 2) : EE(k, 1);
      int m = local_edge(o, i, k);
      if (vt == 5 && DRY(i)) continue;
      double hleft;
      if (DRY(i)) hleft = zero;
      else { hleft = EDGE_H(i, m); hleft = fmax2(hleft, zero); }
      atotal = atotal + hleft * ELEN(k);
    }
    int null_area = equals(atotal, zero);
    int counter = 0;
    double newatotal = zero;
    for (;;) {
      newatotal = zero;
      double qtotal = zero;
      for (int32_t l = 1; l <= ne; l++) {
        int32_t k = BCIN(l, ic);
        int32_t i = EE(k, 1) < 1 ? EE(k, 2) : EE(k, 1);
        if (vt == 5 && DRY(i)) continue;
        int m = local_edge(o, i, k);
        double hleft = EDGE_H(i, m), uedg, vedg;
        if (null_area) hleft = o->bch_max;
        if (hleft < h_dry) { hleft = fmax2(hleft, zero); uedg = zero; vedg = zero; }
        else { uedg = EDGE_U(i, m); vedg = EDGE_V(i, m); }
        double nx = ENRM(k, 1), ny = ENRM(k, 2);
        if (GE(i, m) < 0) { nx = -nx; ny = -ny; }
        double qfrac = qin / atotal;
        double uright = -qfrac;
        double uleft = uedg * nx + vedg * ny;
        double sqrtghleft = sqrt(g * hleft);
        double hright = 2.0 * sqrtghleft + uleft - uright;
        hright = hright * hright / 4.0 / g;
        uright = -qfrac * nx;
        double vright = -qfrac * ny;
        if (hright < h_dry) continue;
        newatotal = newatotal + hright * ELEN(k);
        qtotal = qtotal + (uright * nx + vright * ny) * hright * ELEN(k);
      }
      qtotal = fabs(qtotal);
      if (fabs(qtotal - qin) / qin < 0.005 || counter > 50) break;
      counter++;
      atotal = newatotal;
    }
    atotal = newatotal;
    for (int32_t l = 1; l <= ne; l++) {
      int32_t k = BCIN(l, ic);
      int32_t i = EE(k, 1) < 1 ? EE(k, 2) : EE(k, 1);
      if (vt == 5 && DRY(i)) continue;
      int m = local_edge(o, i, k);
      double hleft = EDGE_H(i, m), uedg, vedg;
      if (null_area) hleft = o->bch_max;
      if (hleft < h_dry) { hleft = fmax2(hleft, zero); uedg = zero; vedg = zero; }
      else { uedg = EDGE_U(i, m); vedg = EDGE_V(i, m); }
      double nx = ENRM(k, 1), ny = ENRM(k, 2);
      if (GE(i, m) < 0) { nx = -nx; ny = -ny; }
      double qfrac = qin / atotal;
      double uright = -qfrac;
      double uleft = uedg * nx + vedg * ny;
      double sqrtghleft = sqrt(g * hleft);
      double hright = 2.0 * sqrtghleft + uleft - uright;
      hright = hright * hright / 4.0 / g;
      uright = -qfrac * nx;
      double vright = -qfrac * ny;
      if (hright < h_dry) continue;
      double f[3];
      f[0] = hright * (uright * nx + vright * ny);
      f[1] = hright * uright * (uright * nx + vright * ny) + half * g * hright * hright * nx;
      f[2] = hright * vright * (uright * nx + vright * ny) + half * g * hright * hright * ny;
      o->cqin3[ic - 1] = o->cqin3[ic - 1] + f[0] * ELEN(k);
      PHI(i, 1) = PHI(i, 1) - f[0] * ELEN(k);
      PHI(i, 2) = PHI(i, 2) - f[1] * ELEN(k);
      PHI(i, 3) = PHI(i, 3) - f[2] * ELEN(k);
    }
  }
}

/* inflowH.f90:28-93 (vtype 4) */
static void inflow_h(orc_t* o) {
  const double h_dry = o->opt.h_dry;
  for (int32_t ic = 1; ic <= o->n_in; ic++) {
    if (o->vtype[ic - 1] != 4) continue;
    for (int32_t l = 1; l <= BCIN(0, ic); l++) {
      int32_t k = BCIN(l, ic);
      int32_t i = EE(k, 1) < 1 ? EE(k, 2) : EE(k, 1);
      int m = local_edge(o, i, k);
      double hleft = EDGE_H(i, m), uedg, vedg;
      hleft = fmax2(hleft, zero);
      if (H(i) < h_dry) { uedg = zero; vedg = zero; }
      else { uedg = EDGE_U(i, m); vedg = EDGE_V(i, m); }
      double nx = ENRM(k, 1), ny = ENRM(k, 2);
      if (GE(i, m) < 0) { nx = -nx; ny = -ny; }
      double zmiddle = half * (ZVTX(EP(k, 1)) + ZVTX(EP(k, 2)));
      double hright = fmax2(zero, o->qin[ic - 1] - zmiddle);
      double uleft = uedg * nx + vedg * ny;
      double sqrtghleft = sqrt(g * hleft);
      double sqrtghright = sqrt(g * hright);
      double uright = uleft + (sqrtghleft - sqrtghright);
      double vright = uright * ny;
      uright = uright * nx;
      uleft = uedg;
      double vleft = vedg;
      if (hleft < h_dry && hright < h_dry) continue;
      double f[3];
      flux_ac(nx, ny, hleft, uleft, vleft, hright, uright, vright, f);
      o->cqin3[ic - 1] = o->cqin3[ic - 1] + f[0] * ELEN(k);
      for (int n = 1; n <= 3; n++) PHI(i, n) = PHI(i, n) - f[n - 1] * ELEN(k);
    }
  }
}

/* outflowbyH.f90:30-137 (htype 1) */
static void outflow_by_h(orc_t* o) {
  const double h_dry = o->opt.h_dry;
  for (int32_t ic = 1; ic <= o->n_out; ic++) {
    if (o->htype[ic - 1] != 1) continue;
    for (int32_t l = 1; l <= BCOUT(0, ic); l++) {
      int32_t k = BCOUT(l, ic);
      int32_t i = EE(k, 1) < 1 ? EE(k, 2) : EE(k, 1);
      int m = local_edge(o, i, k);
      double hleft = EDGE_H(i, m), uedg, vedg;
      if (DRY(i) || hleft < h_dry) { uedg = zero; vedg = zero; hleft = fmax2(hleft, zero); }
      else { uedg = EDGE_U(i, m); vedg = EDGE_V(i, m); }
      double nx = ENRM(k, 1), ny = ENRM(k, 2), tx = ETAN(k, 1), ty = ETAN(k, 2);
      if (GE(i, m) < 0) { nx = -nx; ny = -ny; tx = -tx; ty = -ty; }
      double zmiddle = half * (ZVTX(EP(k, 1)) + ZVTX(EP(k, 2)));
      double hright = fmax2(zero, o->hbc[ic - 1] - zmiddle);
      if (hleft < h_dry && hright < h_dry) continue;
      double uleft, vleft, uright, vright;
      if (hright < h_dry) { uright = zero; uleft = uedg; vright = zero; vleft = vedg; }
      else {
        uleft = uedg * nx + vedg * ny;
        vleft = uedg * tx + vedg * ty;
        double sqrtghleft = sqrt(g * hleft);
        double sqrtghright = sqrt(g * hright);
        uright = uleft + (sqrtghleft - sqrtghright);
        vright = vleft;
        uleft = uedg;
        vleft = vedg;
        uedg = uright;
        vedg = vright;
        uright = uedg * nx + vedg * tx;
        vright = uedg * ny + vedg * ty;
      }
      int set_wall = 0;
      if (o->opt.hvalve) {
        double dotprod = uright * nx + vright * ny;
        if (dotprod < zero) { set_wall = 1; hright = hleft; uright = zero; vright = zero; }
      }
      double f[3];
      flux_ac(nx, ny, hleft, uleft, vleft, hright, uright, vright, f);
      if (set_wall) f[0] = zero;
      o->cqout3[ic - 1] = o->cqout3[ic - 1] + f[0] * ELEN(k);
      PHI(i, 1) = PHI(i, 1) - f[0] * ELEN(k);
      PHI(i, 2) = PHI(i, 2) - f[1] * ELEN(k);
      PHI(i, 3) = PHI(i, 3) - f[2] * ELEN(k);
    }
  }
}

/* crit_outflow.f90:29-107 (htype 2) */
static void crit_outflow(orc_t* o) {
  const double h_dry = o->opt.h_dry;
  for (int32_t ic = 1; ic <= o->n_out; ic++) {
    if (o->htype[ic - 1] != 2) continue;
    for (int32_t l = 1; l <= BCOUT(0, ic); l++) {
      int32_t k = BCOUT(l, ic);
      int32_t i = EE(k, 1) < 1 ? EE(k, 2) : EE(k, 1);
      int m = local_edge(o, i, k);
      double hleft = EDGE_H(i, m), uedg, vedg;
      if (DRY(i) || hleft < h_dry) { uedg = zero; vedg = zero; hleft = fmax2(hleft, zero); }
      else { uedg = EDGE_U(i, m); vedg = EDGE_V(i, m); }
      double nx = ENRM(k, 1), ny = ENRM(k, 2), tx = ETAN(k, 1), ty = ETAN(k, 2);
      if (GE(i, m) < 0) { nx = -nx; ny = -ny; tx = -tx; ty = -ty; }
      if (hleft < h_dry) continue;
      double uleft = uedg * nx + vedg * ny;
      double vleft = uedg * tx + vedg * ty;
      double uright = uleft, vright = vleft;
      double hright = uright * uright / g;
      uedg = uright;
      vedg = vright;
      uright = uedg * nx + vedg * tx;
      vright = uedg * ny + vedg * ty;
      if (o->opt.hvalve) {
        double dotprod = uright * nx + vright * ny;
        if (dotprod < zero) { hright = hleft; uright = zero; vright = zero; }
      }
      double f[3];
      f[0] = hright * (uright * nx + vright * ny);
      f[1] = hright * uright * (uright * nx + vright * ny) + half * g * hright * hright * nx;
      f[2] = hright * vright * (uright * nx + vright * ny) + half * g * hright * hright * ny;
      o->cqout3[ic - 1] = o->cqout3[ic - 1] + f[0] * ELEN(k);
      double dh = zero; /* :97-99 computes dh, then sets it to zero */
      PHI(i, 1) = PHI(i, 1) - f[0] * ELEN(k);
      PHI(i, 2) = PHI(i, 2) - (f[1] + dh * nx) * ELEN(k);
      PHI(i, 3) = PHI(i, 3) - (f[2] + dh * ny) * ELEN(k);
    }
  }
}

/* free_flow.f90:30-93 (htype 0) */
static void free_flow(orc_t* o) {
  const double h_dry = o->opt.h_dry;
  for (int32_t ic = 1; ic <= o->n_out; ic++) {
    if (o->htype[ic - 1] != 0) continue;
    for (int32_t l = 1; l <= BCOUT(0, ic); l++) {
      int32_t k = BCOUT(l, ic);
      int32_t i = EE(k, 1) < 1 ? EE(k, 2) : EE(k, 1);
      int m = local_edge(o, i, k);
      double hleft = EDGE_H(i, m), uedg, vedg;
      hleft = fmax2(hleft, zero);
      if (hleft < h_dry) continue;
      if (H(i) < h_dry) { uedg = zero; vedg = zero; }
      else { uedg = EDGE_U(i, m); vedg = EDGE_V(i, m); }
      double nx = ENRM(k, 1), ny = ENRM(k, 2);
      if (GE(i, m) < 0) { nx = -nx; ny = -ny; }
      double uleft = uedg, vleft = vedg;
      double hright = hleft, uright = uleft, vright = vleft;
      int set_wall = 0;
      if (o->opt.hvalve) {
        double dotprod = uright * nx + vright * ny;
        if (dotprod < 0) { set_wall = 1; uright = zero; vright = zero; }
      }
      double f[3];
      flux_ac(nx, ny, hleft, uleft, vleft, hright, uright, vright, f);
      if (set_wall) f[0] = zero;
      for (int n = 1; n <= 3; n++) PHI(i, n) = PHI(i, n) - f[n - 1] * ELEN(k);
    }
  }
}

/* invisc_fluxes.f90:39-238 */
static int invisc_fluxes(orc_t* o) {
  const int32_t nf = o->flow_edges1;
  int bad = 0;
#pragma omp parallel for num_threads(o->nthreads) schedule(static) reduction(| : bad)
  for (int32_t l = 1; l <= nf; l++) {
    int b = 0;
    o->fedge_set[l] = interior_flux(o, o->flowedg1[l - 1], &o->fedge[3 * l], &b);
    bad |= b;
  }
  /* :153-166, in flowedg1 order */
  for (int32_t l = 1; l <= nf; l++) {
    if (!o->fedge_set[l]) continue;
    int32_t k = o->flowedg1[l - 1];
    int32_t i = EE(k, 1), j = EE(k, 2);
    const double* f = &o->fedge[3 * l];
    PHI(i, 1) = PHI(i, 1) - f[0] * ELEN(k);
    PHI(i, 2) = PHI(i, 2) - f[1] * ELEN(k);
    PHI(i, 3) = PHI(i, 3) - f[2] * ELEN(k);
    PHI(j, 1) = PHI(j, 1) + f[0] * ELEN(k);
    PHI(j, 2) = PHI(j, 2) + f[1] * ELEN(k);
    PHI(j, 3) = PHI(j, 3) + f[2] * ELEN(k);
  }
  if (o->opt.btype == 0) wenslp3_fluxes(o);
  else weslp2_fluxes(o);
  inflow_q_by_h(o, 1);
  inflow_q_by_h(o, 5);
  inflow_h(o);
  outflow_by_h(o);
  crit_outflow(o);
  free_flow(o);
  return bad;
}

/* bed_slope_STD.f90:23-70 with adjustZb.f90:41-70 (flag = .FALSE.) */
static void bed_slope_std(orc_t* o) {
  const int32_t T = o->n_elems;
#pragma omp parallel for num_threads(o->nthreads) schedule(static)
  for (int32_t e = 1; e <= T; e++) {
    if (DRY(e)) continue;
    int adjust = 0;
    double hp[3], zp[3], x[3], y[3], gx, gy;
    for (int i = 1; i <= 3; i++) {
      int32_t j = GV(e, i);
      hp[i - 1] = H(e) + o->delh_x[e - 1] * (NX(j) - XC(e)) + o->delh_y[e - 1] * (NY(j) - YC(e));
      if (hp[i - 1] < zero) adjust = 1;
    }
    if (adjust) {
      for (int i = 1; i <= 3; i++) {
        int32_t j = GV(e, i);
        hp[i - 1] = fmin2(zero, hp[i - 1]);
        zp[i - 1] = ZVTX(j) + hp[i - 1];
        x[i - 1] = NX(j);
        y[i - 1] = NY(j);
      }
      double b1 = y[1] - y[2], c1 = x[2] - x[1];
      double b2 = y[2] - y[0], c2 = x[0] - x[2];
      double b3 = y[0] - y[1], c3 = x[1] - x[0];
      double a = half / AREA(e);
      gx = a * (b1 * zp[0] + b2 * zp[1] + b3 * zp[2]);
      gy = a * (c1 * zp[0] + c2 * zp[1] + c3 * zp[2]);
    } else {
      gx = o->delz_x[e - 1];
      gy = o->delz_y[e - 1];
    }
    PHI(e, 2) = PHI(e, 2) - g * H(e) * gx * AREA(e);
    PHI(e, 3) = PHI(e, 3) - g * H(e) * gy * AREA(e);
  }
}

/* deltatFVT.f90:32-38, with the cell area/perimeter (see the file header) */
static double deltat_fvt(const orc_t* o, double cfl) {
  double dt = VLARGE;
  for (int32_t i = 1; i <= o->n_elems; i++) {
    double delt = o->u_mag[i - 1] + o->wavec[i - 1] + SMALL_F;
    delt = cfl * AREA(i) / (delt * PERIM(i));
    dt = fmin2(delt, dt);
  }
  return dt;
}

/* wavec at the current state, solverFVT.f90:180-181 */
static void wave_celerity(orc_t* o) {
  for (int32_t i = 1; i <= o->n_elems; i++) o->wavec[i - 1] = DRY(i) ? zero : sqrt(g * H(i));
}

/* fric_terms_impl.f90:32-99 */
static void fric_terms_impl(orc_t* o, double delta_t) {
  const int32_t T = o->n_elems;
  const int K = o->opt.rkorder;
  for (int32_t i = 1; i <= T; i++) {
    double rough = zero, cd = o->cd[i - 1], h = H(i);
    switch (o->opt.opt_friction) {
      case 0:
        if (!DRY(i)) rough = g * cd * cd / pow(h, ONE_THIRD);
        break;
      case 1:
        rough = (cd < FMACHP) ? VLARGE : g / (cd * cd);
        break;
      case 2:
        rough = cd;
        break;
      case 3:
        if (!DRY(i)) {
          double re = o->u_mag[i - 1] * h / o->opt.visc;
          re = fmax2(re, 1000.0);
          re = fmin2(re, (double)2.5e7f);
          rough = cd;
          if (cd / h > 0.20) rough = 0.20 * h;
          /* `**1.11` is a default-REAL literal, widened to double */
          double ln = log(1.725 / re + pow(rough / (14.8 * h), (double)1.11f));
          rough = 0.204 / (ln * ln);
        }
        break;
      case 4:
        if (!DRY(i)) {
          rough = pow(100.0 * cd, 0.16666666666666667) / 51.79;
          rough = g * rough * rough / pow(h, ONE_THIRD);
        }
        break;
    }
    if (!DRY(i)) rough = h / (h + delta_t * rough * o->u_mag[i - 1]);
    o->rough[i - 1] = rough;
    U(i) = U(i) * rough;
    V(i) = V(i) * rough;
    if (!DRY(i)) {
      RKU(i, K) = H(i) * U(i);
      RKV(i, K) = H(i) * V(i);
    }
  }
}

/* Greedy colouring of the smoothing stencil t2t (made symmetric), cells visited in
 * index order, each taking the smallest colour none of its already coloured
 * neighbours has; rs_seq lists the cells by colour, in index order within a colour.
 * The CUDA library builds the same colouring from the same t2t. */
static void rsavg_colour(orc_t* o) {
  const int32_t T = o->n_elems;
  int32_t* deg = (int32_t*)xcalloc((size_t)T + 1, sizeof(int32_t));
  for (int32_t i = 1; i <= T; i++)
    for (int32_t m = 2; m <= T2T(i, 1) + 1; m++) {
      deg[i - 1]++;
      deg[T2T(i, m) - 1]++;
    }
  int32_t* off = (int32_t*)xcalloc((size_t)T + 1, sizeof(int32_t));
  for (int32_t i = 0; i < T; i++) off[i + 1] = off[i] + deg[i];
  int32_t* adj = (int32_t*)xcalloc((size_t)off[T] + 1, sizeof(int32_t));
  int32_t* fill = (int32_t*)xcalloc((size_t)T + 1, sizeof(int32_t));
  for (int32_t i = 1; i <= T; i++)
    for (int32_t m = 2; m <= T2T(i, 1) + 1; m++) {
      int32_t j = T2T(i, m);
      adj[off[i - 1] + fill[i - 1]++] = j;
      adj[off[j - 1] + fill[j - 1]++] = i;
    }
  int32_t* col = (int32_t*)xcalloc((size_t)T + 1, sizeof(int32_t));
  int32_t ncol = 0;
  unsigned char used[256];
  for (int32_t i = 1; i <= T; i++) {
    memset(used, 0, sizeof used);
    for (int32_t q = off[i - 1]; q < off[i]; q++) {
      int32_t j = adj[q];
      if (j < i && col[j - 1] < 256) used[col[j - 1]] = 1;
    }
    int32_t c = 0;
    while (c < 255 && used[c]) c++;
    col[i - 1] = c;
    if (c + 1 > ncol) ncol = c + 1;
  }
  o->rs_seq = (int32_t*)xcalloc((size_t)T + 1, sizeof(int32_t));
  int32_t k = 0;
  for (int32_t c = 0; c < ncol; c++)
    for (int32_t i = 1; i <= T; i++)
      if (col[i - 1] == c) o->rs_seq[k++] = i;
  free(deg); free(off); free(adj); free(fill); free(col);
}

/* solverFVT.f90:238-256: residual smoothing (Jameson and Mavriplis), Gauss-Seidel
 * passes over t2t; rsavg_order 0 visits the cells in index order as the reference,
 * 1 by colour (the order of the CUDA library) */
static void rsavg(orc_t* o) {
  const StormFvtOptions* op = &o->opt;
  const int32_t T = o->n_elems;
  const double fac1 = one / (one + op->rsavg_eps * 3.0);
  const double fac2 = op->rsavg_eps / (one + op->rsavg_eps * 3.0);
  if (!o->phi0) o->phi0 = (double*)xcalloc((size_t)3 * T, sizeof(double));
  if (op->rsavg_order == 1 && !o->rs_seq) rsavg_colour(o);
  memcpy(o->phi0, o->phi, sizeof(double) * 3 * (size_t)T);
  for (int k = 1; k <= op->rsavg_passes; k++)
    for (int32_t q = 0; q < T; q++) {
      const int32_t i = op->rsavg_order == 1 ? o->rs_seq[q] : q + 1;
      for (int n = 1; n <= 3; n++) {
        PHI(i, n) = fac1 * o->phi0[(size_t)(n - 1) * T + i - 1];
        for (int32_t m = 2; m <= T2T(i, 1) + 1; m++) PHI(i, n) = PHI(i, n) + fac2 * PHI(T2T(i, m), n);
      }
    }
}

/* One RK stage, solverFVT.f90:161-325.  `upto` < 5 stops after a phase (probe). */
static int rk_stage(orc_t* o, int rkstep, int upto, double* delt_io) {
  const int32_t T = o->n_elems;
  const StormFvtOptions* op = &o->opt;
  for (int b = 0; b < STORM_MAX_BDR; b++) { o->cqin3[b] = zero; o->cqout3[b] = zero; }
  for (int32_t i = 1; i <= T; i++) ZETA(i) = H(i) + Z(i);
  find_dry_cells(o);
  wave_celerity(o);
  if (upto <= 1) return 0;
  cell_grads_and_fix(o, rkstep);
  if (upto <= 2) return 0;
  to_vertices(o);
  if (upto <= 3) return 0;
  memset(o->phi, 0, sizeof(double) * 3 * T);
  int bad = invisc_fluxes(o);
  bed_slope_std(o);
  if (o->wcoef1) /* solverFVT.f90:218-224 */
    for (int32_t i = 1; i <= T; i++) {
      if (DRY(i)) continue;
      PHI(i, 2) = PHI(i, 2) + o->wcoef1[i - 1];
      PHI(i, 3) = PHI(i, 3) + o->wcoef2[i - 1];
    }
  if (o->ncv > 0) { /* solverFVT.f90:227-233 */
    cvdisch(o);
    for (int32_t i = 1; i <= o->ncv; i++) {
      PHI(o->cvtrigin[i - 1], 1) = PHI(o->cvtrigin[i - 1], 1) - o->cvsrc[i - 1];
      PHI(o->cvtrigout[i - 1], 1) = PHI(o->cvtrigout[i - 1], 1) + o->cvsrc[i - 1];
    }
  }
  if (op->rsavg_passes > 0) rsavg(o);
  if (upto <= 4) return bad;
  /* :259-283 */
  double delt = *delt_io;
  const int32_t K = rkstep;
  for (int32_t i = 1; i <= T; i++) {
    if (op->steady) {
      delt = o->u_mag[i - 1] + o->wavec[i - 1];
      if (delt < SMALL_F) delt = 1.044;
      delt = op->cfl * AREA(i) / (delt * PERIM(i));
    }
    double aeff = AREA(i);
    double dt = delt / aeff;
    RKH(i, K) = zero; RKU(i, K) = zero; RKV(i, K) = zero;
    for (int j = 0; j <= K - 1; j++) {
      RKH(i, K) = RKH(i, K) + o->rkalpha[K][j] * RKH(i, j);
      RKU(i, K) = RKU(i, K) + o->rkalpha[K][j] * RKU(i, j);
      RKV(i, K) = RKV(i, K) + o->rkalpha[K][j] * RKV(i, j);
    }
    RKH(i, K) = RKH(i, K) + o->rkbeta[K] * dt * PHI(i, 1);
    RKU(i, K) = (RKU(i, K) + o->rkbeta[K] * dt * PHI(i, 2));
    RKV(i, K) = (RKV(i, K) + o->rkbeta[K] * dt * PHI(i, 3));
  }
  *delt_io = delt;
  /* :286-296 */
  if (op->vclip)
    for (int32_t i = 1; i <= T; i++) {
      double heff = fmax2(op->h_dry, RKH(i, K));
      double umag = sqrt(RKU(i, K) * RKU(i, K) + RKV(i, K) * RKV(i, K)) / heff;
      if (umag > op->vceiling) {
        RKU(i, K) = op->vceiling * RKU(i, K) / umag;
        RKV(i, K) = op->vceiling * RKV(i, K) / umag;
      }
    }
  /* :300-325 */
  for (int32_t i = 1; i <= T; i++) {
    RKH(i, K) = fmax2(RKH(i, K), zero);
    H(i) = RKH(i, K);
    double h_delta = DRY(i) ? op->h_wet : op->h_dry;
    if (H(i) > h_delta) {
      double heff = H(i);
      U(i) = RKU(i, K) / heff;
      V(i) = RKV(i, K) / heff;
    } else {
      RKU(i, K) = zero; RKV(i, K) = zero; U(i) = zero; V(i) = zero;
    }
  }
  return bad;
}

/* ---- output step (solverFVT.f90:389-405, :483-487) ----------------------------- */

/* vbc_by_h.f90:1-98; v_inflow is written to `v_in` [n_qin] */
static double vbc_by_h(const orc_t* o, const StormFvtOutputBoundary* ob, int32_t ib, const double* wdepth,
                       double* v_in) {
  const int32_t n = ob->n_qin[ib - 1];
  const int32_t ld = ob->qin_ld;
  double* h_in = (double*)xcalloc((size_t)n + 1, sizeof(double));
  double* a_in = (double*)xcalloc((size_t)n + 1, sizeof(double));
  double* u_in = (double*)xcalloc((size_t)n + 1, sizeof(double));
  for (int32_t i = 1; i <= n; i++) h_in[i - 1] = wdepth[ob->qin_nodes[(ib - 1) * ld + i - 1] - 1];
  double ht = zero, at = zero;
  for (int32_t i = 1; i <= n - 1; i++) {
    a_in[i - 1] = ob->l_inflow[(ib - 1) * ld + i - 1] * (h_in[i - 1] + h_in[i]) * half;
    ht = ht + (h_in[i - 1] + h_in[i]) * half;
    at = at + a_in[i - 1];
  }
  const double qin = o->qin[ib - 1];
  for (int32_t i = 1; i <= n - 1; i++) u_in[i - 1] = half * (h_in[i - 1] + h_in[i]) * qin / ht / at;
  for (int32_t i = 1; i <= n; i++) v_in[i - 1] = zero;
  for (int32_t i = 2; i <= n - 1; i++)
    if (h_in[i - 1] > o->opt.h_dry) v_in[i - 1] = half * (u_in[i - 2] + u_in[i - 1]);
  for (int32_t i = 1; i <= n - 1; i++) u_in[i - 1] = half * (v_in[i - 1] + v_in[i]);
  double q = zero;
  for (int32_t i = 1; i <= n - 1; i++) q = q + u_in[i - 1] * a_in[i - 1];
  for (int32_t i = 2; i <= n - 1; i++)
    if (h_in[i - 1] > o->opt.h_dry) v_in[i - 1] = v_in[i - 1] * qin / q;
  for (int32_t i = 1; i <= n - 1; i++) u_in[i - 1] = half * (v_in[i - 1] + v_in[i]);
  q = zero;
  for (int32_t i = 1; i <= n - 1; i++) q = q + u_in[i - 1] * a_in[i - 1];
  free(h_in);
  free(a_in);
  free(u_in);
  return q;
}

int orc_output_vertices(orc_t* o, const StormFvtOutputBoundary* ob, int in_loop, double* hvtx_out,
                        double* uvtx_out, double* vvtx_out, double* cdvtx_out, double* e_est_out) {
  if (!o->have_state) return set_err(STORM_ERR_ARG, "state not set");
  const int32_t N = o->n_pts, T = o->n_elems;
  const double h_dry = o->opt.h_dry;
  double* hv = (double*)xcalloc((size_t)N, sizeof(double));
  double* uv = (double*)xcalloc((size_t)N, sizeof(double));
  double* vv = (double*)xcalloc((size_t)N, sizeof(double));
  /* to_vertices.f90:26-41 with ctr2vtxWSE.f90:89-105 and positivity_vtx.f90:22-27 */
  for (int32_t i = 1; i <= N; i++) {
    double id = zero, a = zero;
    int counter = 0;
    for (int32_t j = 2; j <= N2T(i, 1) + 1; j++) {
      int32_t k = N2T(i, j);
      if (DRY(k)) continue;
      counter++;
      id = id + C2VW(i, j - 1);
      a = a + C2VW(i, j - 1) * ZETA(k);
    }
    double zv = counter > 0 ? a / id : ZVTX(i);
    double zetaref = ZVTX(i);
    for (int32_t j = 2; j <= N2T(i, 1) + 1; j++) {
      int32_t k = N2T(i, j);
      if (DRY(k)) continue;
      zetaref = fmax2(ZETA(k), zetaref);
    }
    zv = fmin2(zv, zetaref);
    hv[i - 1] = zv - ZVTX(i);
    if (hv[i - 1] < zero) hv[i - 1] = zero;
  }
  /* to_vertices.f90:44-55: applied to the solution */
  for (int32_t i = 1; i <= T; i++) {
    if (DRY(i)) continue;
    int flag = 1;
    for (int j = 1; j <= 3; j++) flag = flag && (hv[GV(i, j) - 1] > h_dry);
    if (!flag) { U(i) = zero; V(i) = zero; }
  }
  /* :56-62 */
  ctr2vtx3(o, o->u, uv);
  ctr2vtx3(o, o->v, vv);
  if (o->opt.btype == 0) /* wetdryvfix.f90:26-46 */
    for (int32_t i = 1; i <= N; i++) {
      int wett = 0, dryt = 0;
      for (int32_t j = 2; j <= N2T(i, 1) + 1; j++) {
        if (DRY(N2T(i, j))) dryt = 1;
        else wett = 1;
      }
      if (wett && dryt) { uv[i - 1] = zero; vv[i - 1] = zero; }
    }
  for (int32_t i = 1; i <= N; i++)
    if (hv[i - 1] < h_dry) { uv[i - 1] = zero; vv[i - 1] = zero; }
  /* enforce_bcs.f90:37-171 */
  for (int32_t b = 1; b <= o->n_out; b++) {
    const int32_t ht = o->htype[b - 1];
    const double* hn = ob->hnormals + 2 * (size_t)(b - 1) * ob->hbc_ld;
    if (ht == 1) {
      for (int32_t i = 1; i <= o->n_hbc[b - 1]; i++) {
        int32_t j = HBC_NODES(i, b);
        const double hbc = in_loop ? o->hbc_it[b - 1] : o->hbc[b - 1];
        double hnot = fmax2(zero, hbc - ZVTX(j));
        double incr = 0.100 * (hnot - hv[j - 1]);
        if (fabs(incr) < 0.0100) incr = hnot - hv[j - 1];
        hv[j - 1] = hv[j - 1] - incr;
        hv[j - 1] = fmax2(zero, hbc - ZVTX(j));
      }
      if (o->opt.hvalve)
        for (int32_t i = 1; i <= o->n_hbc[b - 1]; i++) {
          int32_t j = HBC_NODES(i, b);
          double dot = uv[j - 1] * hn[2 * (i - 1)] + vv[j - 1] * hn[2 * (i - 1) + 1];
          if (dot < zero) { uv[j - 1] = zero; vv[j - 1] = zero; }
        }
    } else if (ht == 0) {
      for (int32_t i = 1; i <= o->n_hbc[b - 1]; i++) {
        int32_t j = HBC_NODES(i, b);
        double dot = uv[j - 1] * hn[2 * (i - 1)] + vv[j - 1] * hn[2 * (i - 1) + 1];
        if (dot < zero) { uv[j - 1] = zero; vv[j - 1] = zero; }
      }
    }
  }
  if (o->opt.btype == 0) {
    for (int32_t i = 1; i <= ob->n_wall; i++) {
      int32_t p = ob->wall_pts[i - 1];
      uv[p - 1] = zero;
      vv[p - 1] = zero;
    }
  } else {
    for (int32_t i = 1; i <= ob->n_wall; i++) {
      int32_t p = ob->wall_pts[i - 1];
      double tx = ob->wtangs[2 * (i - 1)], ty = ob->wtangs[2 * (i - 1) + 1];
      double dot = uv[p - 1] * tx + vv[p - 1] * ty;
      uv[p - 1] = dot * tx;
      vv[p - 1] = dot * ty;
    }
  }
  for (int32_t i = 1; i <= N; i++)
    if (hv[i - 1] < h_dry) { uv[i - 1] = zero; vv[i - 1] = zero; }
  double qin_save[STORM_MAX_BDR];
  for (int32_t b = 0; b < o->n_in; b++) {
    qin_save[b] = o->qin[b];
    if (in_loop) o->qin[b] = o->qin_it[b];
  }
  for (int32_t b = 1; b <= o->n_in; b++) {
    const int32_t vt = o->vtype[b - 1], n = ob->n_qin[b - 1];
    const int32_t* qn = ob->qin_nodes + (size_t)(b - 1) * ob->qin_ld;
    const double* pn = ob->pnormals + 2 * (size_t)(b - 1) * ob->qin_ld;
    if (vt == 0) {
      for (int32_t i = 1; i <= n; i++)
        if (hv[qn[i - 1] - 1] > h_dry) {
          uv[qn[i - 1] - 1] = o->qin[b - 1] * pn[2 * (i - 1)];
          vv[qn[i - 1] - 1] = o->qin[b - 1] * pn[2 * (i - 1) + 1];
        }
    } else if (vt == 1 || vt == 5) {
      double* v_in = (double*)xcalloc((size_t)n + 1, sizeof(double));
      (void)vbc_by_h(o, ob, b, hv, v_in);
      for (int32_t i = 1; i <= n; i++)
        if (hv[qn[i - 1] - 1] > h_dry) {
          uv[qn[i - 1] - 1] = v_in[i - 1] * pn[2 * (i - 1)];
          vv[qn[i - 1] - 1] = v_in[i - 1] * pn[2 * (i - 1) + 1];
        }
      free(v_in);
    } else if (vt == 3) {
      for (int32_t i = 1; i <= n; i++)
        if (hv[qn[i - 1] - 1] > h_dry) {
          uv[qn[i - 1] - 1] = o->qin[b - 1];
          vv[qn[i - 1] - 1] = ob->qin2 ? ob->qin2[b - 1] : zero;
        }
    }
  }
  for (int32_t b = 0; b < o->n_in; b++) o->qin[b] = qin_save[b];
  if (hvtx_out) memcpy(hvtx_out, hv, sizeof(double) * N);
  if (uvtx_out) memcpy(uvtx_out, uv, sizeof(double) * N);
  if (vvtx_out) memcpy(vvtx_out, vv, sizeof(double) * N);
  if (cdvtx_out) ctr2vtx3(o, o->cd, cdvtx_out);
  if (e_est_out) /* error_est.f90, etype 2 */
    for (int32_t i = 1; i <= T; i++) {
      e_est_out[i - 1] = zero;
      if (H(i) < h_dry) continue;
      int32_t n1 = GV(i, 1), n2 = GV(i, 2), n3 = GV(i, 3);
      double gzx = (ZVTX(n1) * (NY(n2) - NY(n3)) + ZVTX(n2) * (NY(n3) - NY(n1)) + ZVTX(n3) * (NY(n1) - NY(n2))) *
                   half / AREA(i);
      double gzy = (ZVTX(n1) * (NX(n3) - NX(n2)) + ZVTX(n2) * (NX(n1) - NX(n3)) + ZVTX(n3) * (NX(n2) - NX(n1))) *
                   half / AREA(i);
      double l = PERIM(i) * ONE_THIRD;
      double gx = gzx + o->delh_x[i - 1], gy = gzy + o->delh_y[i - 1];
      e_est_out[i - 1] = sqrt(gx * gx + gy * gy) * l / (Z(i) + H(i));
    }
  free(hv);
  free(uv);
  free(vv);
  return 0;
}

/* The main loop body, solverFVT.f90:129-476, `nsteps` times. */
int orc_step(orc_t* o, int nsteps, StormFvtStepStats* st) {
  if (!o->have_state) return set_err(STORM_ERR_ARG, "state not set");
  const int32_t T = o->n_elems;
  const StormFvtOptions* op = &o->opt;
  const int K = op->rkorder;
  int bad = 0;
  for (int s = 0; s < nsteps && !o->converged; s++) {
    o->iter++;
    for (int32_t i = 1; i <= T; i++) { RKU(i, 0) = RKU(i, K); RKV(i, 0) = RKV(i, K); RKH(i, 0) = RKH(i, K); }
    if (!op->steady) {
      if (op->dt_op == 0) o->delt = op->cfl;
      else {
        /* u_mag and wavec of the current state (see the file header) */
        for (int32_t i = 1; i <= T; i++) ZETA(i) = H(i) + Z(i);
        find_dry_cells(o);
        wave_celerity(o);
        o->delt = deltat_fvt(o, op->cfl);
      }
    }
    o->ttime = o->ttime + o->delt;
    for (int rkstep = 1; rkstep <= K; rkstep++) bad |= rk_stage(o, rkstep, 5, &o->delt);
    /* :335-346 */
    find_dry_cells(o);
    fric_terms_impl(o, o->delt);
    double sumtop = zero, sumbot = zero;
    for (int32_t i = 1; i <= T; i++) {
      sumtop = sumtop + (H(i) - RKH(i, 0)) * (H(i) - RKH(i, 0));
      sumbot = sumbot + RKH(i, 0) * RKH(i, 0);
    }
    /* :357-370 */
    if (op->hvalve)
      for (int32_t j = 1; j <= o->n_bcedges; j++) {
        if (!o->hbar[j - 1]) continue;
        int32_t k = o->bcedges[j - 1];
        int32_t i = EE(k, 1) < 1 ? EE(k, 2) : EE(k, 1);
        int m = local_edge(o, i, k);
        double ksign = GE(i, m) >= 0 ? one : -one;
        double dotprod = ksign * (U(i) * ENRM(k, 1) + V(i) * ENRM(k, 2));
        if (dotprod < 0) { U(i) = zero; V(i) = zero; }
      }
    /* :376-386 */
    for (int32_t i = 1; i <= T; i++)
      if (DRY(i)) { PHI(i, 1) = zero; PHI(i, 2) = zero; PHI(i, 3) = zero; }
    double rmax_phi = zero;
    for (int32_t i = 1; i <= T; i++)
      rmax_phi = fmax2(fmax2(fmax2(rmax_phi, fabs(PHI(i, 1))), fabs(PHI(i, 2))), fabs(PHI(i, 3)));
    double tmass = zero;
    for (int32_t i = 1; i <= T; i++) tmass = tmass + H(i) * AREA(i);
    double sb = sumbot;
    if (equals(sb, zero)) sb = one;
    o->rms = sqrt(sumtop / sb);
    o->tmass = tmass;
    if (op->steady) {
      o->rmax = (op->stop_cr == 0) ? rmax_phi : o->rms;
      o->stime = (double)o->iter;
      if (o->rmax < op->rstop) o->converged = 1;
    } else {
      o->stime = o->stime + o->delt;
      o->rmax = rmax_phi;
      for (int32_t b = 0; b < o->n_in; b++) o->qin_it[b] = o->qin[b];
      for (int32_t b = 0; b < o->n_out; b++) o->hbc_it[b] = o->hbc[b];
      get_time_bcs(o, o->stime);
    }
  }
  if (st) {
    memset(st, 0, sizeof *st);
    st->iter = o->iter; st->converged = o->converged; st->ttime = o->ttime; st->stime = o->stime;
    st->delt = o->delt; st->rmax = o->rmax; st->rms_dh = o->rms; st->tmass = o->tmass;
    for (int b = 0; b < STORM_MAX_BDR; b++) { st->cqin3[b] = o->cqin3[b]; st->cqout3[b] = o->cqout3[b]; }
    st->device_status = bad ? 1 : 0;
  }
  return 0;
}

/* ---- one iteration in steps, for one part of a mesh split over processes ----------
 * orc_step's iteration cut where a part's halo takes its owners' values and where the
 * parts agree on dt and on the stop test; the caller does the exchanges between the
 * calls.  orc_iter_begin returns this part's CFL minimum (unsteady, dt_op = 1: the
 * global dt is the minimum over the parts) or the dt the part would use. */
int orc_iter_begin(orc_t* o, double* dt_local) {
  if (!o->have_state) return set_err(STORM_ERR_ARG, "state not set");
  const int32_t T = o->n_elems;
  const StormFvtOptions* op = &o->opt;
  const int K = op->rkorder;
  o->iter++;
  for (int32_t i = 1; i <= T; i++) { RKU(i, 0) = RKU(i, K); RKV(i, 0) = RKV(i, K); RKH(i, 0) = RKH(i, K); }
  if (!op->steady) {
    if (op->dt_op == 0) o->delt = op->cfl;
    else {
      for (int32_t i = 1; i <= T; i++) ZETA(i) = H(i) + Z(i);
      find_dry_cells(o);
      wave_celerity(o);
      o->delt = deltat_fvt(o, op->cfl);
    }
  }
  *dt_local = o->delt;
  return 0;
}

/* The iteration's dt (unsteady: the minimum over the parts); advances ttime as
 * orc_step does before its stages. */
void orc_iter_set_dt(orc_t* o, double delt) {
  if (!o->opt.steady) o->delt = delt;
  o->ttime = o->ttime + o->delt;
}

/* RK stage `rkstep`; *delt_out: steady, the local dt of this part's last element (the
 * friction dt when that element is element n_elems of the whole mesh). */
int orc_iter_stage(orc_t* o, int rkstep, double* delt_out, int* bad) {
  if (rkstep < 1 || rkstep > o->opt.rkorder) return set_err(STORM_ERR_ARG, "bad rkstep");
  *bad |= rk_stage(o, rkstep, 5, &o->delt);
  *delt_out = o->delt;
  return 0;
}

/* Friction with dt `delt` (steady: the whole mesh's element n_elems dt), the valve,
 * and this part's sums over its owned cells: sums[0..3] = sum (h - h0)^2, sum h0^2,
 * sum h*area, max |phi| (owned[i] != 0: element i+1 is owned). */
int orc_iter_fric(orc_t* o, double delt, const uint8_t* owned, double* sums) {
  const int32_t T = o->n_elems;
  const StormFvtOptions* op = &o->opt;
  o->delt = delt;
  find_dry_cells(o);
  fric_terms_impl(o, o->delt);
  double sumtop = zero, sumbot = zero;
  for (int32_t i = 1; i <= T; i++) {
    if (!owned[i - 1]) continue;
    sumtop = sumtop + (H(i) - RKH(i, 0)) * (H(i) - RKH(i, 0));
    sumbot = sumbot + RKH(i, 0) * RKH(i, 0);
  }
  if (op->hvalve)
    for (int32_t j = 1; j <= o->n_bcedges; j++) {
      if (!o->hbar[j - 1]) continue;
      int32_t k = o->bcedges[j - 1];
      int32_t i = EE(k, 1) < 1 ? EE(k, 2) : EE(k, 1);
      int m = local_edge(o, i, k);
      double ksign = GE(i, m) >= 0 ? one : -one;
      double dotprod = ksign * (U(i) * ENRM(k, 1) + V(i) * ENRM(k, 2));
      if (dotprod < 0) { U(i) = zero; V(i) = zero; }
    }
  for (int32_t i = 1; i <= T; i++)
    if (DRY(i)) { PHI(i, 1) = zero; PHI(i, 2) = zero; PHI(i, 3) = zero; }
  double rmax_phi = zero, tmass = zero;
  for (int32_t i = 1; i <= T; i++) {
    if (!owned[i - 1]) continue;
    rmax_phi = fmax2(fmax2(fmax2(rmax_phi, fabs(PHI(i, 1))), fabs(PHI(i, 2))), fabs(PHI(i, 3)));
    tmass = tmass + H(i) * AREA(i);
  }
  sums[0] = sumtop;
  sums[1] = sumbot;
  sums[2] = tmass;
  sums[3] = rmax_phi;
  return 0;
}

/* The iteration's scalars from the sums over all parts (as orc_iter_fric's), the
 * stop test and the boundary time series, as the end of orc_step's iteration. */
int orc_iter_finish(orc_t* o, const double* sums, StormFvtStepStats* st) {
  const StormFvtOptions* op = &o->opt;
  double sb = sums[1];
  if (equals(sb, zero)) sb = one;
  o->rms = sqrt(sums[0] / sb);
  o->tmass = sums[2];
  if (op->steady) {
    o->rmax = (op->stop_cr == 0) ? sums[3] : o->rms;
    o->stime = (double)o->iter;
    if (o->rmax < op->rstop) o->converged = 1;
  } else {
    o->stime = o->stime + o->delt;
    o->rmax = sums[3];
    for (int32_t b = 0; b < o->n_in; b++) o->qin_it[b] = o->qin[b];
    for (int32_t b = 0; b < o->n_out; b++) o->hbc_it[b] = o->hbc[b];
    get_time_bcs(o, o->stime);
  }
  if (st) {
    memset(st, 0, sizeof *st);
    st->iter = o->iter; st->converged = o->converged; st->ttime = o->ttime; st->stime = o->stime;
    st->delt = o->delt; st->rmax = o->rmax; st->rms_dh = o->rms; st->tmass = o->tmass;
    for (int b = 0; b < STORM_MAX_BDR; b++) { st->cqin3[b] = o->cqin3[b]; st->cqout3[b] = o->cqout3[b]; }
  }
  return 0;
}

/* h, u, v and RK level `level` of every element (get) or of the listed elements
 * (put: n entries, 1-based element ids, values in list order). */
int orc_get_level(const orc_t* o, int level, double* out6) {
  const int32_t T = o->n_elems;
  if (level < 0 || level > o->opt.rkorder) return set_err(STORM_ERR_ARG, "bad level");
  memcpy(out6, o->h, sizeof(double) * T);
  memcpy(out6 + T, o->u, sizeof(double) * T);
  memcpy(out6 + 2 * (size_t)T, o->v, sizeof(double) * T);
  memcpy(out6 + 3 * (size_t)T, o->rkh + (size_t)level * T, sizeof(double) * T);
  memcpy(out6 + 4 * (size_t)T, o->rku + (size_t)level * T, sizeof(double) * T);
  memcpy(out6 + 5 * (size_t)T, o->rkv + (size_t)level * T, sizeof(double) * T);
  return 0;
}
int orc_put_level(orc_t* o, int level, int32_t n, const int32_t* elems, const double* in6) {
  const int32_t T = o->n_elems;
  if (level < 0 || level > o->opt.rkorder) return set_err(STORM_ERR_ARG, "bad level");
  for (int32_t k = 0; k < n; k++) {
    const int32_t i = elems[k];
    if (i < 1 || i > T) return set_err(STORM_ERR_ARG, "element out of range");
    H(i) = in6[k];
    U(i) = in6[n + k];
    V(i) = in6[2 * (size_t)n + k];
    RKH(i, level) = in6[3 * (size_t)n + k];
    RKU(i, level) = in6[4 * (size_t)n + k];
    RKV(i, level) = in6[5 * (size_t)n + k];
  }
  return 0;
}

/* The inflow safety-net elevation (dataprepFVT.f90:278-286) of the whole mesh, for a
 * part that holds only some of its boundary. */
void orc_set_bch_max(orc_t* o, double v) { o->bch_max = v; }
double orc_get_bch_max(const orc_t* o) { return o->bch_max; }

int orc_get_state(const orc_t* o, double* h, double* u, double* v, double* rkh, double* rku, double* rkv,
                  double* hvtx) {
  const int32_t T = o->n_elems, K = o->opt.rkorder;
  if (h) memcpy(h, o->h, sizeof(double) * T);
  if (u) memcpy(u, o->u, sizeof(double) * T);
  if (v) memcpy(v, o->v, sizeof(double) * T);
  if (rkh) memcpy(rkh, o->rkh + (size_t)K * T, sizeof(double) * T);
  if (rku) memcpy(rku, o->rku + (size_t)K * T, sizeof(double) * T);
  if (rkv) memcpy(rkv, o->rkv + (size_t)K * T, sizeof(double) * T);
  if (hvtx) memcpy(hvtx, o->hvtx, sizeof(double) * o->n_pts);
  return 0;
}

int orc_get_drycell(orc_t* o, int32_t* dry) {
  find_dry_cells(o);
  memcpy(dry, o->drycell, sizeof(int32_t) * o->n_elems);
  return 0;
}

int orc_stage_probe(orc_t* o, int rkstep, int upto, int32_t* dry, double* grads6, double* uv2, double* hvtx,
                    double* phi3) {
  if (!o->have_state) return set_err(STORM_ERR_ARG, "state not set");
  if (rkstep < 1 || rkstep > o->opt.rkorder) return set_err(STORM_ERR_ARG, "bad rkstep");
  const int32_t T = o->n_elems;
  const size_t L = (size_t)o->opt.rkorder + 1;
  double* sv = (double*)malloc(sizeof(double) * (3 * T + 3 * L * T));
  memcpy(sv, o->h, sizeof(double) * T);
  memcpy(sv + T, o->u, sizeof(double) * T);
  memcpy(sv + 2 * T, o->v, sizeof(double) * T);
  memcpy(sv + 3 * T, o->rkh, sizeof(double) * L * T);
  memcpy(sv + 3 * T + L * T, o->rku, sizeof(double) * L * T);
  memcpy(sv + 3 * T + 2 * L * T, o->rkv, sizeof(double) * L * T);
  double delt = o->delt;
  rk_stage(o, rkstep, upto, &delt);
  if (dry) memcpy(dry, o->drycell, sizeof(int32_t) * T);
  if (grads6)
    for (int32_t i = 0; i < T; i++) {
      grads6[6 * i] = o->delh_x[i]; grads6[6 * i + 1] = o->delh_y[i];
      grads6[6 * i + 2] = o->delu_x[i]; grads6[6 * i + 3] = o->delu_y[i];
      grads6[6 * i + 4] = o->delv_x[i]; grads6[6 * i + 5] = o->delv_y[i];
    }
  if (uv2)
    for (int32_t i = 0; i < T; i++) { uv2[2 * i] = o->u[i]; uv2[2 * i + 1] = o->v[i]; }
  if (hvtx) memcpy(hvtx, o->hvtx, sizeof(double) * o->n_pts);
  if (phi3)
    for (int32_t i = 1; i <= T; i++) { phi3[3 * (i - 1)] = PHI(i, 1); phi3[3 * (i - 1) + 1] = PHI(i, 2); phi3[3 * (i - 1) + 2] = PHI(i, 3); }
  memcpy(o->h, sv, sizeof(double) * T);
  memcpy(o->u, sv + T, sizeof(double) * T);
  memcpy(o->v, sv + 2 * T, sizeof(double) * T);
  memcpy(o->rkh, sv + 3 * T, sizeof(double) * L * T);
  memcpy(o->rku, sv + 3 * T + L * T, sizeof(double) * L * T);
  memcpy(o->rkv, sv + 3 * T + 2 * L * T, sizeof(double) * L * T);
  free(sv);
  return 0;
}
