// storm_internal.h -- shared declarations of the FVT step library (not part of the ABI).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/storm_fvt.h"

namespace storm {

// ---- error reporting (thread-local last error, storm_fvt_last_error) -------
int set_error(int code, const std::string& msg);
void clear_error();

// ---- face kinds of the per-cell face table ---------------------------------
enum FaceKind : uint8_t {
  FACE_NONE = 0,   // boundary edge with no flux routine (e.g. between two BC strings)
  FACE_LEFT = 1,   // interior edge, this cell is edges(k)%e(1)
  FACE_RIGHT = 2,  // interior edge, this cell is edges(k)%e(2)
  FACE_WALL = 3,   // walledg1 edge
  FACE_BC = 4      // open-boundary edge; contribution computed by the boundary kernel
};

// Open-boundary routine kinds, in the order invisc_fluxes.f90:218-238 calls them.
enum BcKind : int32_t {
  BC_QBYH = 0,      // inflowQbyH vtype 1
  BC_QBYH_WET = 1,  // inflowQbyH vtype 5
  BC_HIN = 2,       // inflowH vtype 4
  BC_HOUT = 3,      // outflowbyH htype 1
  BC_CRIT = 4,      // crit_outflow htype 2
  BC_FREE = 5       // free_flow htype 0
};

constexpr uint8_t kOrderHasBc = 0x40;  // forder flag: the cell has an open-boundary face
constexpr uint8_t kOrderHasCulvert = 0x80;  // forder flag: a culvert end lies in the cell
constexpr int kMaxStencil = 19;   // elemnt_db.f90:42 maxdim = 20 (count + 19 ids)
constexpr int kMaxBcEdges = 8192; // edges per open boundary handled by one CTA

// Host-side image of the device layout: cells and nodes renumbered along a Morton
// curve, structure-of-arrays, per-cell face table in local-slot order.
struct HostLayout {
  int32_t T = 0, N = 0, kst = 0, nwall = 0, nbce = 0, nbdr = 0, n2t_nnz = 0;
  std::vector<int32_t> cell_old;  // new -> old (0-based)
  std::vector<int32_t> node_old;
  std::vector<int32_t> cell_new;  // old -> new
  std::vector<int32_t> node_new;
  // cells [T]
  std::vector<double> area, perim, xc, yc, z, delz_x, delz_y, zmax, cd;
  std::vector<double> wcoef1, wcoef2;  // wind terms (empty: none)
  std::vector<double> lsq_a, lsq_b, lsq_c, lsq_det;
  // every cell's lsq_a/b/c/det equal, bit for bit, the sums lsq_setup forms from its
  // stencil weights and offsets (a = sum w dx dx, b = sum w dx dy, c = sum w dy dy in
  // stencil order, det = a c - b b), so the FP64 gradient kernel forms them again from
  // the stencil values it loads instead of reading four more arrays
  bool lsq_derived = false;
  std::vector<uint8_t> nst, forder, hvmask;
  std::vector<int32_t> bc_cells;  // cells with an open-boundary face, increasing
  std::vector<int32_t> rs_cells, rs_off;  // cells by colour of the t2t stencil (new ids), CSR
  // [3][T]
  std::vector<int32_t> vert, t2t3, fref;
  std::vector<double> rc_x, rc_y, fnx, fny, flen, fz0;
  std::vector<uint8_t> fkind;
  // stencil [kst][T]
  std::vector<int32_t> st_id;
  std::vector<double> st_w, st_dx, st_dy;
  // interior edges [ne], ordered by (min, max) of their two cells' new ids
  int32_t ne = 0;
  std::vector<int32_t> eL, eR;       // edges(k)%e(1), e(2)
  std::vector<uint8_t> eslot;        // local slot of the edge in L | (in R) << 2
  std::vector<double> enx, eny, elen, ez0;  // normal out of e(1), length, midpoint bed
  // walls [nwall]
  std::vector<int32_t> wall_p1, wall_p2;
  // nodes [N]
  std::vector<double> zvtx, node_x, node_y;
  std::vector<int32_t> n2t_off, n2t_cell;  // CSR [N+1], [nnz]
  std::vector<double> n2t_w;               // c2v_weights_id [nnz]
  std::vector<int16_t> node_hbc;           // htype-1 boundary (slot in hbc[]) or -1
  std::vector<int32_t> out_node, out_off;  // nodes of every outflow string (new ids), CSR [n_out+1]
  // open boundaries [nbdr], in call order; edges [nbce]
  std::vector<int32_t> bdr_kind, bdr_slot, bdr_off, bdr_cnt;
  std::vector<int32_t> bce_cell, bce_slot;
  std::vector<double> bce_nx, bce_ny, bce_tx, bce_ty, bce_len, bce_zmid;
  // boundary values and time series (vbc_arrays / dep_vars)
  int32_t n_in = 0, n_out = 0;
  std::vector<int32_t> in_type, out_type;
  std::vector<double> qin, hbc;
  std::vector<int32_t> ts_off, ts_cnt;  // [n_in + n_out] into ts_t/ts_v (inflows first)
  std::vector<double> ts_t, ts_v;
  double bch_max = 0.0;
  int32_t last_cell_new = 0;  // new id of element n_elems (steady friction dt)
  // culverts [ncv] (cells in new ids); performance curves [ncv][cv_ld]
  int32_t ncv = 0, cv_ld = 0;
  std::vector<int32_t> cv_in, cv_n;
  std::vector<double> cv_rx, cv_ry, cv_zinv, cv_head, cv_q;
  // culvert terms of phi(:,1), sorted by cell and, within a cell, in the order the
  // reference adds them: code = culvert << 1 | (1: outlet, adds; 0: inlet, subtracts)
  std::vector<int32_t> cvc_cell, cvc_code;
  // merged layouts only
  std::vector<int32_t> cell_sid, node_sid, edge_sid, bdr_sid;
};

// Placement of one scenario inside a merged (batched) layout.
struct ScenarioInfo {
  int32_t cell_off = 0, cell_cnt = 0;  // cell slots [cell_off, cell_off + cell_cnt)
  int32_t node_off = 0, node_cnt = 0;
  int32_t blk_off = 0, blk_cnt = 0;    // reduction blocks covering the padded range
  int32_t last_cell = 0;               // merged id of element n_elems
};

// Build the device layout of one prepared (Fortran-layout) mesh.
int build_layout(const StormFvtMesh& m, const StormFvtOptions& opt, HostLayout& L);

// Tiles of the fused stage kernel: tile t owns the cell slots [t*tc, (t+1)*tc).  Its
// local cells are the owned ones (local id = slot - t*tc), then H1 (face neighbours
// of owned cells in other tiles: their gradients and face states are recomputed in
// the tile), then H2 (stencil and face neighbours of H1 cells outside owned and H1:
// state only), then H3 (the other cells around the tile's nodes: state only).  Its
// nodes are the vertices of its owned and H1 cells; each node's vertex depth is
// computed in the tile from its incident cells, and the tile owning the node's
// smallest incident cell slot writes it out.  Its edges are the interior edges whose
// smaller cell slot is owned (a contiguous range of the edge arrays, sorted by that
// slot) followed by the "back" edges whose larger slot is owned.  Local ids are
// 16-bit; kNoLocal marks none.
constexpr uint16_t kNoLocal = 0xFFFF;
constexpr uint8_t kEdgeExport = 0x10;  // eslot flag: the edge has a cell with an open-boundary face
enum TileInfo { TI_NOWN = 0, TI_N1, TI_N2, TI_HOFF, TI_H1OFF, TI_ER0, TI_NR, TI_NB, TI_BOFF, TI_SID,
                TI_N3, TI_NOFF, TI_NN, TI_N };
struct TilePlan {
  int32_t tc = 0, ntiles = 0, kst = 0;
  int32_t ns_max = 0, ng_max = 0, ne_max = 0;  // largest local cell, gradient and edge counts
  int32_t nn_max = 0;                           // largest node count
  std::vector<int32_t> info;    // [ntiles][TI_N]; TI_SID: the tile's one scenario, or -1 if several
  std::vector<int32_t> halo;    // global slots of H1, H2 then H3, per tile from info[TI_HOFF]
  std::vector<uint16_t> h1_t3;  // [sum n1][3]   local t2t3 of the H1 cells
  std::vector<uint16_t> h1_st;  // [sum n1][kst] local stencil of the H1 cells
  std::vector<uint16_t> lt3;    // [3][T]   local t2t3 of every cell in its own tile
  std::vector<uint16_t> lst;    // [kst][T] local stencil of every cell in its own tile
  std::vector<uint16_t> lfe;    // [3][T]   local edge of each interior face in its own tile
  std::vector<uint32_t> eloc;   // [ne]     local L | R << 16 of each edge in the tile of its smaller slot
  std::vector<int32_t> be;      // back edges (global edge ids), per tile from info[TI_BOFF]
  std::vector<uint32_t> beloc;  // local L | R << 16 of each back edge
  // nodes, per tile from info[TI_NOFF]: global id, whether this tile writes its depth
  // out, and where its incident cells (local ids, in the n2t order) start in tn_cells
  std::vector<int32_t> tnode, tn_start;
  std::vector<uint8_t> tn_own;
  std::vector<uint16_t> tn_cells;
  std::vector<uint16_t> lvt;    // [3][T]   local vertex ids of every cell in its own tile
  std::vector<uint16_t> h1_vt;  // [sum n1][3] local vertex ids of the H1 cells
  std::vector<uint32_t> lwall;  // [3][T]   local p1 | p2 << 16 of each wall face in its own tile
  std::vector<int32_t> bc_nodes;  // vertices of the cells with an open-boundary face
};
// Returns 0, or -1 when a tile needs more than 65,534 local cells or edges.
int build_tiles(const HostLayout& L, int tc, TilePlan& P);
// Host-side consistency check of a plan against its layout: 0, or the failed check.
int check_tiles(const HostLayout& L, const TilePlan& P);

// Concatenate per-scenario layouts into one: every scenario's cell range starts on
// a multiple of `block` (reduction blocks never span two scenarios); ids are shifted
// by the scenario's offsets; cell_sid/node_sid/edge_sid/bdr_sid name the scenario
// of every cell slot (-1 for padding), node, interior edge and open boundary.
void merge_layouts(const std::vector<HostLayout>& parts, int block, HostLayout& M,
                   std::vector<ScenarioInfo>& info);

}  // namespace storm
