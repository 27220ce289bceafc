// fvt_device.cuh -- device-side data of the FVT step and the per-edge physics shared
// by the kernels (flux functions, the reference's compare helpers).
//
// Every formula below is the reference's expression evaluated in the reference's
// order (the library is compiled with --fmad=false, so no product is fused into a
// sum): with the oracle's own inputs the kernels reproduce its results bit for bit
// except where CUDA's pow() (friction) differs from the host libm.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace storm {

constexpr int kMaxBdrDev = 16;

// Per-scenario scalars that live on the device (one struct per scenario of the
// handle, written by the kernels), followed by the scenario's static description.
struct Scalars {
  int32_t iter;       // iterations completed
  int32_t converged;  // steady: rmax < rstop reached (solverFVT.f90:431)
  int32_t status;     // bit 0: non-finite state; bit 1: HLL wave-speed inversion
  int32_t pad;
  double delt;        // dt of the current iteration (unsteady), or the steady
                      // last-element local dt carried into ttime (solverFVT.f90:155)
  double delt_fric;   // steady: local dt of element n_elems in the last stage (N3)
  double ttime, stime, rmax, rms, tmass;
  double qin[kMaxBdrDev], hbc[kMaxBdrDev];
  double cqin3[kMaxBdrDev], cqout3[kMaxBdrDev];
  double qin_it[kMaxBdrDev], hbc_it[kMaxBdrDev];  // values the last iteration ran with
  double bch_max;               // dataprepFVT.f90:278-286
  double sumtop, sumbot, rmax_phi;  // this iteration's residual sums (linked partitions)
  // static: boundary series and the scenario's ranges in the merged arrays
  int32_t n_in, n_out;
  int32_t last_cell;            // merged id of element n_elems (steady friction dt)
  int32_t blk_off, blk_cnt;     // reduction blocks of the scenario's cell range
  int32_t pad2;
  int32_t out_type[kMaxBdrDev];
  int32_t ts_off[2 * kMaxBdrDev], ts_cnt[2 * kMaxBdrDev];  // inflows, then outflows
};

// Kernel parameters: options, the device layout and the state buffers.
struct Dev {
  int32_t T, N, K, kst, nbdr, nbce;  // T counts the padded cell slots of all scenarios
  int32_t steady, dt_op, lim, btype, hvalve, vclip, fric, stop_cr, flux;
  int32_t nscen;
  int32_t t_real;  // one-scenario handles: its cells are the slots below t_real
  int32_t lsq_derived;  // FP64 gradients form lsq_a/b/c/det from the stencil (bit-equal)
  // scenario of each cell slot (-1: padding), node, interior edge and open boundary
  const int32_t *cell_sid, *node_sid, *edge_sid, *bdr_sid;
  double h_dry, h_wet, cfl, vceiling, visc, rstop;
  double alpha[4][4], beta[4];
  // cells
  const double *area, *perim, *xc, *yc, *z, *delz_x, *delz_y, *zmax, *cd;
  const double *vox, *voy;  // [3][T] vertex minus centroid of each cell vertex (bed_slope_STD)
  const double *wcoef1, *wcoef2;  // wind stress terms per cell (null: no wind)
  // linked partitions of one mesh: halo cell slots and their owners' slots, the halo
  // mask (null: no halo), the scenario holding element n_elems of the whole mesh
  int32_t nhalo, linked, fric_scen;
  const int32_t *halo_dst, *halo_src;
  const uint8_t* halo_mask;
  // culverts: inlet cell, table rows, inlet offset from the centroid, invert elevation,
  // performance curves [ncv][cv_ld]; per-cell term list (cvc_*); discharges cvsrc
  int32_t ncv, cv_ld, ncvc;
  const int32_t *cv_in, *cv_n, *cvc_cell, *cvc_code;
  const double *cv_rx, *cv_ry, *cv_zinv, *cv_head, *cv_q;
  double* cvsrc;
  const double *lsq_a, *lsq_b, *lsq_c, *lsq_det;
  const uint8_t *nst, *forder, *hvmask, *fkind;
  const int32_t *vert, *t2t3, *fref, *st_id;
  // the faces of each cell in the order their terms are added (forder): kinds, 3 bits
  // each, and references ([3][T]) of the t-th face added
  const uint16_t* fko;
  const int32_t* frefo;
  const double *rc_x, *rc_y, *fnx, *fny, *flen, *fz0, *st_w, *st_dx, *st_dy;
  const int32_t *wall_p1, *wall_p2;
  // interior edges
  int32_t ne;
  const int32_t *eL, *eR;
  const uint8_t* eslot;
  const double *enx, *eny, *elen, *ez0;
  double* efx;              // [3][ne] flux * length of the last k_eflux
  uint8_t* eok;             // [ne] the edge produced a flux (not skipped)
  // nodes
  const double *zvtx, *node_x, *node_y, *n2t_w;
  const int32_t *n2t_off, *n2t_cell;
  const int16_t* node_hbc;
  // open boundaries
  const int32_t *bdr_kind, *bdr_slot, *bdr_off, *bdr_cnt, *bce_cell, *bce_slot;
  const double *bce_nx, *bce_ny, *bce_tx, *bce_ty, *bce_len, *bce_zmid;
  const double *ts_t, *ts_v;
  // state
  double *rkh, *rku, *rkv;  // [K+1][T]
  double *u_a, *v_a;        // stage-input velocities (find_dry_cells, LSQ)
  // the velocities this stage's fluxes use (after hgradfix2 / to_vertices zeroing):
  // FP64 path, a flag per cell (1: zero, else the stage-input u, v); mixed path, the
  // values themselves (read by the lighter FP32 edge kernel while still in L2)
  uint8_t* vzero;
  double *u_b, *v_b;
  double *delh_x, *delh_y, *delu_x, *delu_y, *delv_x, *delv_y;
  uint8_t *dry_a, *dry_b;   // stage dry flags (ping-pong)
  uint8_t* dry_out;         // find_dry_cells before the friction step (the output pass)
  double* hvtx;             // vertex depth after enforce_bcs (wall fluxes, output)
  uint8_t* vwet;            // hvtx > h_dry before enforce_bcs (to_vertices.f90:44-55)
  double* phimax;           // MAX(|phi|) of the last stage (stop criterion)
  // residual smoothing: phi and its copy [3][T], cells by colour of the t2t stencil
  double *phi, *phi0;
  const int32_t* rs_cells;
  double rs_fac1, rs_fac2;
  int32_t bc_cache;         // k_bc keeps the inflow fixed point's invariants in shared memory
  double* bc_c;             // [3][nbce] boundary contributions to phi
  double* bc_rec;           // [3][nbce] reconstructed boundary-edge h, u, v
  double* part;             // [5][nblk] reduction partials, field-major (blocks never span scenarios)
  int32_t nbc_cells;        // cells with an open-boundary face (finished after k_bc)
  const int32_t* bc_cells;
  int32_t nblk_red;
  Scalars* sc;              // [nscen]
};

// Geometry and per-stage arrays read or written in the flux/gradient arithmetic type R:
// double views of the FP64 arrays, or float copies for the mixed-precision path.
template <class R>
struct Geo {
  const R *rc_x, *rc_y, *st_w, *st_dx, *st_dy, *lsq_a, *lsq_b, *lsq_c, *lsq_det, *delz_x, *delz_y;
  const R *enx, *eny, *elen;
  const R *vox, *voy;  // [3][T] vertex minus centroid (bed_slope_STD), in R
  R *delh_x, *delh_y, *delu_x, *delu_y, *delv_x, *delv_y;
  R* efx;  // [3][ne]
};

// Device view of the tile plan of the fused stage kernel (TilePlan in storm_internal.h).
struct TileDev {
  int32_t tc, ntiles, kst, ns_max, ng_max, ne_max, nn_max;
  int32_t nodes;                       // the tile computes its vertex depths (else k_node does)
  const int32_t* info;                 // [ntiles][TI_N]
  const int32_t* halo;                 // H1 then H2 slots per tile
  const uint16_t *h1_t3, *h1_st;       // local topology of the H1 cells
  const uint16_t *lt3, *lst, *lfe;     // local topology of every cell in its own tile
  const uint32_t* eloc;                // [ne] local L | R << 16 (range edges)
  const int32_t* be;                   // back edges
  const uint32_t* beloc;               // their local L | R << 16
  const int32_t *tnode, *tn_start;     // nodes per tile; start of their incident cells in tn_cells
  const uint8_t* tn_own;               // the tile writes the node's depth out
  const uint16_t* tn_cells;            // local incident cells (n2t order)
  const uint16_t *lvt, *h1_vt;         // local vertex ids of owned / H1 cells
  const uint32_t* lwall;               // [3][T] local ends of wall faces
};

// One launch of a templated stage kernel (see launch_stage in fvt_kernels.cu).
enum StageKernel { STAGE_GRAD, STAGE_BC, STAGE_EFLUX, STAGE_FLUX, STAGE_FLUX_BC, STAGE_PHI, STAGE_PHI_BC,
                   STAGE_UPDATE, STAGE_CULVERT, STAGE_GRAD_BC, STAGE_TILE };
struct StageLaunch {
  int which;
  dim3 grid, block;
  size_t smem;
  cudaStream_t stream;
  int s;
  const double* hs;
  const uint8_t* dry;
  uint8_t* dry_next;
  double *rku_prev, *rkv_prev;
  // stage-input velocities and where the stage writes its new ones (the same arrays
  // for the phase kernels; ping-pong buffers for the fused tile kernel)
  const double *u_in, *v_in;
  double *u_out, *v_out;
  const TileDev* tiles;  // STAGE_TILE only
};
size_t tile_smem_bytes(const TileDev& t, bool mixed);
int tile_blocks_per_sm(bool mixed, size_t smem);  // resident CTAs of k_tile per SM
void set_tile_smem_limit(int bytes);
void launch_stage(const StageLaunch& L, const Dev& d, const Geo<double>& Gd, const Geo<float>& Gf, bool mixed);
void set_bc_smem_limit(int bytes);
// Linked partitions: halo exchange of one level (+ up to two flag arrays), the shared
// friction dt before k_fric, the shared dt / stop test after k_final.
void launch_halo(const Dev& d, int level, uint8_t* f1, uint8_t* f2, cudaStream_t st);
void launch_link_fric(const Dev& d, cudaStream_t st);
void launch_link(const Dev& d, cudaStream_t st);
void launch_link_dt(const Dev& d, cudaStream_t st);
// Friction, hvalve and the iteration partials (halo cells left out when linked).
void launch_fric(const Dev& d, const double* u_src, const double* v_src, cudaStream_t st);
void launch_rsavg(const Dev& d, int off, int cnt, cudaStream_t st);
// One part of a mesh per process: set dt (which 0) or the friction dt (1), pack /
// unpack [6][n] halo values of the listed slots, finish the iteration with the sums
// of all parts {sumtop, sumbot, tmass, max |phi|}.
void launch_part_scalar(const Dev& d, int which, double v, cudaStream_t st);
void launch_pack(const Dev& d, int level, int n, const int32_t* slots, const double* u, const double* v,
                 double* out, cudaStream_t st);
void launch_unpack(const Dev& d, int level, int n, const int32_t* slots, const double* in, double* u, double* v,
                   uint8_t* dry, cudaStream_t st);
void launch_part_finish(const Dev& d, const double* sums, cudaStream_t st);
// k_node over every node (list == nullptr) or the n listed nodes
void launch_node(const Dev& d, const double* hs, const uint8_t* dry, const int32_t* list, int n, int block,
                 cudaStream_t st);

// The output pass (to_vertices, ctr2vtx of cd, error_est(2)) after an iteration.
struct OutputArgs {
  // outflow strings: nodes [out_off[b], out_off[b+1]) of out_node, unit normals hn[2*i]
  int32_t n_out;
  const int32_t *out_node, *out_off, *out_type;
  const double *hn, *hbc;
  int32_t n_wall;
  const int32_t* wall_node;
  const double* wtang;
  // inflow strings: nodes [in_off[b], in_off[b+1]) of in_node, normals pn, lengths lin
  int32_t n_in;
  const int32_t *in_node, *in_off, *in_type;
  const double *pn, *lin, *qin, *qin2;
  double *hv, *uv, *vv, *cdv, *e_est;  // outputs (device, new numbering)
};
void launch_output(const Dev& d, const Geo<double>& Gd, const Geo<float>& Gf, bool mixed, const OutputArgs& a,
                   cudaStream_t st);

}  // namespace storm
