// layout.cpp -- prepared Fortran-layout mesh -> the library's device layout.
//
// Cells and nodes are renumbered along a Morton (Z-order) curve of their
// coordinates so that the stencil, face and node-to-cell gathers of one warp hit
// the same L2 lines; every per-cell quantity is a structure-of-arrays column.
// What is precomputed here is exactly what the reference precomputes or computes
// once before its time loop, with the same expressions:
//   delz      bed_slope_VTX.f90:22-38 (called at solverFVT.f90:93)
//   zmax      zvtx(csortedz(i)%p(3)) read by hgradfix2.f90:50
//   fz0       half*(zvtx(p1)+zvtx(p2)) of invisc_fluxes.f90:89, inflowH.f90:53,
//             outflowbyH.f90:67
//   fnx/fny   edges(k)%normal flipped by invert_edge_dirs when grid(i)%edge(m) < 0
// The per-cell visiting order of faces reproduces the order in which
// invisc_fluxes.f90 adds edge contributions to phi(i,:) (interior edges in
// flowedg1 order, then walledg1, then inflowQbyH vtype 1, vtype 5, inflowH,
// outflowbyH, crit_outflow, free_flow), so the per-cell gather performs the
// reference's scatter additions in the reference's order.
// Compiled with -ffp-contract=off.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <unordered_map>

#include "storm_internal.h"

namespace storm {
namespace {

constexpr double kHalf = 0.5;

uint32_t spread16(uint32_t x) {
  x &= 0xffff;
  x = (x | (x << 8)) & 0x00ff00ff;
  x = (x | (x << 4)) & 0x0f0f0f0f;
  x = (x | (x << 2)) & 0x33333333;
  x = (x | (x << 1)) & 0x55555555;
  return x;
}

// Permutation (new -> old) sorting points by their 32-bit Morton key.
std::vector<int32_t> morton_order(const std::vector<double>& x, const std::vector<double>& y) {
  size_t n = x.size();
  double x0 = *std::min_element(x.begin(), x.end()), x1 = *std::max_element(x.begin(), x.end());
  double y0 = *std::min_element(y.begin(), y.end()), y1 = *std::max_element(y.begin(), y.end());
  double s = std::max(x1 - x0, y1 - y0);
  if (!(s > 0)) s = 1.0;
  std::vector<uint32_t> key(n);
  for (size_t i = 0; i < n; i++) {
    uint32_t qx = (uint32_t)std::min(65535.0, std::floor((x[i] - x0) / s * 65535.0));
    uint32_t qy = (uint32_t)std::min(65535.0, std::floor((y[i] - y0) / s * 65535.0));
    key[i] = spread16(qx) | (spread16(qy) << 1);
  }
  std::vector<int32_t> perm(n);
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.end(), [&](int32_t a, int32_t b) { return key[a] < key[b]; });
  return perm;
}

bool same_bits(double a, double b) {
  uint64_t x, y;
  std::memcpy(&x, &a, 8);
  std::memcpy(&y, &b, 8);
  return x == y;
}

}  // namespace

int build_layout(const StormFvtMesh& m, const StormFvtOptions& opt, HostLayout& L) {
  const int32_t T = m.n_elems, N = m.n_pts, E = m.n_edges;
  L.T = T;
  L.N = N;
  auto GV = [&](int32_t i, int j) { return m.tri_vertex[3 * (size_t)(i - 1) + (j - 1)]; };
  auto GE = [&](int32_t i, int j) { return m.tri_edge[3 * (size_t)(i - 1) + (j - 1)]; };
  auto EP = [&](int32_t k, int j) { return m.edge_p[2 * (size_t)(k - 1) + (j - 1)]; };
  auto EE = [&](int32_t k, int j) { return m.edge_e[2 * (size_t)(k - 1) + (j - 1)]; };
  auto local_edge = [&](int32_t i, int32_t k) {  // local_edge.f90:32-39
    for (int j = 1; j <= 3; j++)
      if (std::abs(GE(i, j)) == k) return j;
    return -1;
  };
  auto in_elem = [&](int32_t k) { return EE(k, 1) < 1 ? EE(k, 2) : EE(k, 1); };  // edge_in_element.f90

  // ---- argument checks -----------------------------------------------------
  if (T < 1 || N < 3 || E < 1) return set_error(STORM_ERR_ARG, "storm_fvt_create: empty mesh");
  if (m.t2t_ncol < 2 || m.t2t_ncol - 1 > kMaxStencil)
    return set_error(STORM_ERR_MESH, "storm_fvt_create: t2t width out of range");
  if (m.n_inflowbdr > STORM_MAX_BDR || m.n_outflowbdr > STORM_MAX_BDR)
    return set_error(STORM_ERR_ARG, "storm_fvt_create: too many boundaries");
  for (size_t q = 0; q < 3 * (size_t)T; q++) {
    if (m.tri_vertex[q] < 1 || m.tri_vertex[q] > N) return set_error(STORM_ERR_MESH, "storm_fvt_create: vertex id out of range");
    int32_t k = std::abs(m.tri_edge[q]);
    if (k < 1 || k > E) return set_error(STORM_ERR_MESH, "storm_fvt_create: edge id out of range");
  }

  // ---- renumbering ---------------------------------------------------------
  {
    std::vector<double> cx(m.tri_xc, m.tri_xc + T), cy(m.tri_yc, m.tri_yc + T);
    L.cell_old = morton_order(cx, cy);
    std::vector<double> nxv(m.node_x, m.node_x + N), nyv(m.node_y, m.node_y + N);
    L.node_old = morton_order(nxv, nyv);
  }
  L.cell_new.assign(T, 0);
  L.node_new.assign(N, 0);
  for (int32_t i = 0; i < T; i++) L.cell_new[L.cell_old[i]] = i;
  for (int32_t i = 0; i < N; i++) L.node_new[L.node_old[i]] = i;
  auto CN = [&](int32_t old1) { return L.cell_new[old1 - 1]; };  // 1-based old -> new
  auto NN = [&](int32_t old1) { return L.node_new[old1 - 1]; };
  L.last_cell_new = L.cell_new[T - 1];

  // ---- nodes ---------------------------------------------------------------
  L.zvtx.resize(N);
  L.node_x.resize(N);
  L.node_y.resize(N);
  for (int32_t n = 0; n < N; n++) {
    int32_t o = L.node_old[n];
    L.zvtx[n] = m.zvtx[o];
    L.node_x[n] = m.node_x[o];
    L.node_y[n] = m.node_y[o];
  }
  L.n2t_off.assign(N + 1, 0);
  for (int32_t n = 0; n < N; n++) {
    int32_t o = L.node_old[n];
    int32_t cnt = m.n2t[o];  // n2t(o+1,1)
    if (cnt < 0 || cnt > m.n2t_ncol - 1 || cnt > m.c2v_ncol)
      return set_error(STORM_ERR_MESH, "storm_fvt_create: n2t count out of range");
    L.n2t_off[n + 1] = L.n2t_off[n] + cnt;
  }
  L.n2t_nnz = L.n2t_off[N];
  L.n2t_cell.resize(L.n2t_nnz);
  L.n2t_w.resize(L.n2t_nnz);
  for (int32_t n = 0; n < N; n++) {
    int32_t o = L.node_old[n];
    int32_t cnt = m.n2t[o];
    for (int32_t j = 0; j < cnt; j++) {
      int32_t c = m.n2t[(size_t)(j + 1) * N + o];
      if (c < 1 || c > T) return set_error(STORM_ERR_MESH, "storm_fvt_create: n2t entry out of range");
      L.n2t_cell[L.n2t_off[n] + j] = CN(c);
      L.n2t_w[L.n2t_off[n] + j] = m.c2v_w[(size_t)j * N + o];
    }
  }
  L.out_node.clear();
  L.out_off.assign(1, 0);
  for (int32_t b = 0; b < m.n_outflowbdr; b++) {
    for (int32_t i = 0; i < m.n_hbc[b]; i++) {
      int32_t p = m.hbc_nodes[(size_t)b * m.hbc_ld + i];
      if (p < 1 || p > N) return set_error(STORM_ERR_MESH, "storm_fvt_create: hbc node out of range");
      L.out_node.push_back(NN(p));
    }
    L.out_off.push_back((int32_t)L.out_node.size());
  }
  L.node_hbc.assign(N, -1);
  for (int32_t b = 0; b < m.n_outflowbdr; b++) {
    if (m.htype[b] != 1) continue;
    for (int32_t i = 0; i < m.n_hbc[b]; i++) {
      int32_t p = m.hbc_nodes[(size_t)b * m.hbc_ld + i];
      if (p < 1 || p > N) return set_error(STORM_ERR_MESH, "storm_fvt_create: hbc node out of range");
      L.node_hbc[NN(p)] = (int16_t)b;  // enforce_bcs loops boundaries in order: last wins
    }
  }

  // ---- open boundaries -----------------------------------------------------
  // bc edge occurrence per (edge) -> position in the flat bc edge list
  std::unordered_map<int32_t, int32_t> bce_of_edge;
  std::unordered_map<int32_t, int32_t> bce_rank;  // edge -> visiting-order key
  auto add_bdr = [&](int kind, int32_t slot, const int32_t* col) -> int {
    int32_t cnt = col[0];
    if (cnt < 0) return set_error(STORM_ERR_MESH, "storm_fvt_create: negative boundary edge count");
    if (cnt > kMaxBcEdges) return set_error(STORM_ERR_UNSUPPORTED, "storm_fvt_create: boundary with more than 8192 edges");
    L.bdr_kind.push_back(kind);
    L.bdr_slot.push_back(slot);
    L.bdr_off.push_back((int32_t)L.bce_cell.size());
    L.bdr_cnt.push_back(cnt);
    for (int32_t l = 1; l <= cnt; l++) {
      int32_t k = col[l];
      if (k < 1 || k > E) return set_error(STORM_ERR_MESH, "storm_fvt_create: boundary edge out of range");
      int32_t i = in_elem(k);
      if (i < 1 || i > T) return set_error(STORM_ERR_MESH, "storm_fvt_create: boundary edge without element");
      int mm = local_edge(i, k);
      if (mm < 1) return set_error(STORM_ERR_MESH, "storm_fvt_create: boundary edge not in its element");
      double nx = m.edge_normal[2 * (size_t)(k - 1)], ny = m.edge_normal[2 * (size_t)(k - 1) + 1];
      double tx = m.edge_tang[2 * (size_t)(k - 1)], ty = m.edge_tang[2 * (size_t)(k - 1) + 1];
      if (GE(i, mm) < 0) {
        nx = -nx;
        ny = -ny;
        tx = -tx;
        ty = -ty;
      }
      if (bce_of_edge.count(k))
        return set_error(STORM_ERR_MESH, "storm_fvt_create: edge " + std::to_string(k) + " is in two boundary strings");
      int32_t pos = (int32_t)L.bce_cell.size();
      bce_of_edge[k] = pos;
      L.bce_cell.push_back(CN(i));
      L.bce_slot.push_back(mm - 1);
      L.bce_nx.push_back(nx);
      L.bce_ny.push_back(ny);
      L.bce_tx.push_back(tx);
      L.bce_ty.push_back(ty);
      L.bce_len.push_back(m.edge_length[k - 1]);
      L.bce_zmid.push_back(kHalf * (m.zvtx[EP(k, 1) - 1] + m.zvtx[EP(k, 2) - 1]));
    }
    return 0;
  };
  const int in_kinds[3] = {1, 5, 4};
  const int in_bc[3] = {BC_QBYH, BC_QBYH_WET, BC_HIN};
  for (int pass = 0; pass < 3; pass++)
    for (int32_t b = 0; b < m.n_inflowbdr; b++)
      if (m.vtype[b] == in_kinds[pass]) {
        int rc = add_bdr(in_bc[pass], b, m.bcedgesinflow + (size_t)b * m.bcin_ld);
        if (rc) return rc;
      }
  const int out_kinds[3] = {1, 2, 0};
  const int out_bc[3] = {BC_HOUT, BC_CRIT, BC_FREE};
  for (int pass = 0; pass < 3; pass++)
    for (int32_t b = 0; b < m.n_outflowbdr; b++)
      if (m.htype[b] == out_kinds[pass]) {
        int rc = add_bdr(out_bc[pass], b, m.bcedgesoutflow + (size_t)b * m.bcout_ld);
        if (rc) return rc;
      }
  L.nbdr = (int32_t)L.bdr_kind.size();
  L.nbce = (int32_t)L.bce_cell.size();

  // boundary values / series
  L.n_in = m.n_inflowbdr;
  L.n_out = m.n_outflowbdr;
  L.in_type.assign(m.vtype, m.vtype + m.n_inflowbdr);
  L.out_type.assign(m.htype, m.htype + m.n_outflowbdr);
  L.qin.assign(m.qin, m.qin + m.n_inflowbdr);
  L.hbc.assign(m.hbc, m.hbc + m.n_outflowbdr);
  L.ts_off.clear();
  L.ts_cnt.clear();
  for (int32_t b = 0; b < m.n_inflowbdr; b++) {
    L.ts_off.push_back((int32_t)L.ts_t.size());
    L.ts_cnt.push_back(m.n_timeserq[b]);
    for (int32_t i = 0; i < m.n_timeserq[b]; i++) {
      L.ts_t.push_back(m.timelocq[(size_t)b * m.tsq_ld + i]);
      L.ts_v.push_back(m.timeserq[(size_t)b * m.tsq_ld + i]);
    }
  }
  for (int32_t b = 0; b < m.n_outflowbdr; b++) {
    L.ts_off.push_back((int32_t)L.ts_t.size());
    L.ts_cnt.push_back(m.n_timeserh[b]);
    for (int32_t i = 0; i < m.n_timeserh[b]; i++) {
      L.ts_t.push_back(m.timeloch[(size_t)b * m.tsh_ld + i]);
      L.ts_v.push_back(m.timeserh[(size_t)b * m.tsh_ld + i]);
    }
  }
  L.bch_max = m.bch_max;

  // ---- edge classification -------------------------------------------------
  std::vector<uint8_t> ekind((size_t)E + 1, FACE_NONE);
  std::vector<int32_t> wall_pos((size_t)E + 1, -1);
  for (int32_t l = 0; l < m.flow_edges1; l++) {
    int32_t k = m.flowedg1[l];
    if (k < 1 || k > E || EE(k, 1) < 1 || EE(k, 2) < 1 || EE(k, 1) > T || EE(k, 2) > T)
      return set_error(STORM_ERR_MESH, "storm_fvt_create: interior edge without two elements");
    ekind[k] = FACE_LEFT;
  }
  L.nwall = m.wall_edges1;
  for (int32_t l = 0; l < m.wall_edges1; l++) {
    int32_t k = m.walledg1[l];
    if (k < 1 || k > E) return set_error(STORM_ERR_MESH, "storm_fvt_create: wall edge out of range");
    if (ekind[k] != FACE_NONE) return set_error(STORM_ERR_MESH, "storm_fvt_create: wall edge listed as interior");
    ekind[k] = FACE_WALL;
    wall_pos[k] = l;
    L.wall_p1.push_back(NN(EP(k, 1)));
    L.wall_p2.push_back(NN(EP(k, 2)));
  }
  // ---- interior edges (one flux evaluation each) ----------------------------
  std::vector<int32_t> ie_of((size_t)E + 1, -1);
  {
    std::vector<int32_t> ks(m.flowedg1, m.flowedg1 + m.flow_edges1);
    auto key = [&](int32_t k) {
      int32_t a = CN(EE(k, 1)), b = CN(EE(k, 2));
      return ((int64_t)std::min(a, b) << 32) | (uint32_t)std::max(a, b);
    };
    std::stable_sort(ks.begin(), ks.end(), [&](int32_t x, int32_t y) { return key(x) < key(y); });
    L.ne = (int32_t)ks.size();
    L.eL.resize(L.ne); L.eR.resize(L.ne); L.eslot.resize(L.ne);
    L.enx.resize(L.ne); L.eny.resize(L.ne); L.elen.resize(L.ne); L.ez0.resize(L.ne);
    for (int32_t e = 0; e < L.ne; e++) {
      const int32_t k = ks[e], e1 = EE(k, 1), e2 = EE(k, 2);
      const int m1 = local_edge(e1, k), m2 = local_edge(e2, k);
      if (m1 < 1 || m2 < 1) return set_error(STORM_ERR_MESH, "storm_fvt_create: edge not in its element");
      double nx = m.edge_normal[2 * (size_t)(k - 1)], ny = m.edge_normal[2 * (size_t)(k - 1) + 1];
      if (GE(e1, m1) < 0) {  // invert_edge_dirs: the normal points out of e(1)
        nx = -nx;
        ny = -ny;
      }
      ie_of[k] = e;
      L.eL[e] = CN(e1);
      L.eR[e] = CN(e2);
      L.eslot[e] = (uint8_t)((m1 - 1) | ((m2 - 1) << 2));
      L.enx[e] = nx;
      L.eny[e] = ny;
      L.elen[e] = m.edge_length[k - 1];
      L.ez0[e] = kHalf * (m.zvtx[EP(k, 1) - 1] + m.zvtx[EP(k, 2) - 1]);
    }
  }

  // ---- cells ---------------------------------------------------------------
  L.area.resize(T); L.perim.resize(T); L.xc.resize(T); L.yc.resize(T); L.z.resize(T);
  L.delz_x.resize(T); L.delz_y.resize(T); L.zmax.resize(T); L.cd.resize(T);
  if (m.wcoef1 && m.wcoef2) { L.wcoef1.resize(T); L.wcoef2.resize(T); }
  L.lsq_a.resize(T); L.lsq_b.resize(T); L.lsq_c.resize(T); L.lsq_det.resize(T);
  L.nst.resize(T); L.forder.resize(T); L.hvmask.assign(T, 0);
  L.vert.resize(3 * (size_t)T); L.t2t3.resize(3 * (size_t)T); L.fref.assign(3 * (size_t)T, 0);
  L.rc_x.resize(3 * (size_t)T); L.rc_y.resize(3 * (size_t)T);
  L.fnx.assign(3 * (size_t)T, 0.0); L.fny.assign(3 * (size_t)T, 0.0);
  L.flen.assign(3 * (size_t)T, 0.0); L.fz0.assign(3 * (size_t)T, 0.0);
  L.fkind.assign(3 * (size_t)T, FACE_NONE);
  int32_t kst = 0;
  for (int32_t i = 0; i < T; i++) kst = std::max(kst, m.t2t[i]);
  L.kst = std::max(kst, 1);
  L.st_id.assign((size_t)L.kst * T, 0);
  L.st_w.assign((size_t)L.kst * T, 0.0);
  L.st_dx.assign((size_t)L.kst * T, 0.0);
  L.st_dy.assign((size_t)L.kst * T, 0.0);
  const size_t lsq_ld = (size_t)T;
  bool lsq_all = true;
  for (int32_t c = 0; c < T; c++) {
    const int32_t o = L.cell_old[c];  // 0-based old id
    const int32_t i1 = o + 1;         // 1-based old id
    L.area[c] = m.tri_area[o];
    L.perim[c] = m.tri_perim[o];
    L.xc[c] = m.tri_xc[o];
    L.yc[c] = m.tri_yc[o];
    L.z[c] = m.z[o];
    L.cd[c] = m.cd[o];
    if (m.wcoef1 && m.wcoef2) {
      L.wcoef1[c] = m.wcoef1[o];
      L.wcoef2[c] = m.wcoef2[o];
    }
    L.lsq_a[c] = m.lsq_a[o];
    L.lsq_b[c] = m.lsq_b[o];
    L.lsq_c[c] = m.lsq_c[o];
    L.lsq_det[c] = m.lsq_det[o];
    int32_t p3 = m.csortedz[3 * (size_t)o + 2];
    if (p3 < 1 || p3 > N) return set_error(STORM_ERR_MESH, "storm_fvt_create: csortedz out of range");
    L.zmax[c] = m.zvtx[p3 - 1];
    // bed_slope_VTX.f90:24-33
    {
      double x1 = m.node_x[GV(i1, 1) - 1], y1 = m.node_y[GV(i1, 1) - 1];
      double x2 = m.node_x[GV(i1, 2) - 1], y2 = m.node_y[GV(i1, 2) - 1];
      double x3 = m.node_x[GV(i1, 3) - 1], y3 = m.node_y[GV(i1, 3) - 1];
      double zz1 = m.zvtx[GV(i1, 1) - 1], zz2 = m.zvtx[GV(i1, 2) - 1], zz3 = m.zvtx[GV(i1, 3) - 1];
      L.delz_x[c] = kHalf * (zz1 * (y2 - y3) + zz2 * (y3 - y1) + zz3 * (y1 - y2)) / m.tri_area[o];
      L.delz_y[c] = kHalf * (zz1 * (x3 - x2) + zz2 * (x1 - x3) + zz3 * (x2 - x1)) / m.tri_area[o];
    }
    // LSQ stencil, reference order (t2t(i,2:n+1))
    int32_t n = m.t2t[o];
    if (n < 0 || n > m.t2t_ncol - 1) return set_error(STORM_ERR_MESH, "storm_fvt_create: t2t count out of range");
    L.nst[c] = (uint8_t)n;
    double sa = 0.0, sb = 0.0, sc = 0.0;
    for (int32_t k = 0; k < n; k++) {
      int32_t nb = m.t2t[(size_t)(k + 1) * T + o];
      if (nb < 1 || nb > T) return set_error(STORM_ERR_MESH, "storm_fvt_create: t2t entry out of range");
      L.st_id[(size_t)k * T + c] = CN(nb);
      const double w = m.lsq_w[(size_t)k * lsq_ld + o];
      const double dx = m.lsq_dx[(size_t)k * lsq_ld + o];
      const double dy = m.lsq_dy[(size_t)k * lsq_ld + o];
      L.st_w[(size_t)k * T + c] = w;
      L.st_dx[(size_t)k * T + c] = dx;
      L.st_dy[(size_t)k * T + c] = dy;
      sa = sa + w * dx * dx;  // lsq_setup.f90:92-145, in its order
      sb = sb + w * dx * dy;
      sc = sc + w * dy * dy;
    }
    const double sd = sa * sc - sb * sb;
    if (!same_bits(sa, L.lsq_a[c]) || !same_bits(sb, L.lsq_b[c]) || !same_bits(sc, L.lsq_c[c]) ||
        !same_bits(sd, L.lsq_det[c]))
      lsq_all = false;
    // per-slot data
    int64_t key[3];
    for (int j = 1; j <= 3; j++) {
      size_t q = (size_t)(j - 1) * T + c;
      L.vert[q] = NN(GV(i1, j));
      int32_t nb = m.t2t3[3 * (size_t)o + (j - 1)];
      L.t2t3[q] = (nb >= 1 && nb <= T) ? CN(nb) : -1;
      L.rc_x[q] = m.rc_x[(size_t)(j - 1) * T + o];
      L.rc_y[q] = m.rc_y[(size_t)(j - 1) * T + o];
      int32_t k = std::abs(GE(i1, j));
      uint8_t kind = ekind[k];
      L.flen[q] = m.edge_length[k - 1];
      double nx = m.edge_normal[2 * (size_t)(k - 1)], ny = m.edge_normal[2 * (size_t)(k - 1) + 1];
      if (kind == FACE_LEFT) {
        int32_t e1 = EE(k, 1), e2 = EE(k, 2);
        int m1 = local_edge(e1, k);
        if (m1 < 1) return set_error(STORM_ERR_MESH, "storm_fvt_create: edge not in its element");
        if (GE(e1, m1) < 0) {
          nx = -nx;
          ny = -ny;
        }
        int32_t other = (e1 == i1) ? e2 : e1;
        if (e1 != i1 && e2 != i1) return set_error(STORM_ERR_MESH, "storm_fvt_create: edge/element tables disagree");
        int mo = local_edge(other, k);
        if (mo < 1) return set_error(STORM_ERR_MESH, "storm_fvt_create: edge not in its element");
        L.fkind[q] = (uint8_t)((e1 == i1 ? FACE_LEFT : FACE_RIGHT) | ((mo - 1) << 4));
        L.fref[q] = ie_of[k];  // the interior-edge record holding this face's flux
        L.fz0[q] = kHalf * (m.zvtx[EP(k, 1) - 1] + m.zvtx[EP(k, 2) - 1]);
        key[j - 1] = (int64_t)k;
      } else {
        if (GE(i1, j) < 0) {
          nx = -nx;
          ny = -ny;
        }
        if (kind == FACE_WALL) {
          if (in_elem(k) != i1) return set_error(STORM_ERR_MESH, "storm_fvt_create: wall edge element mismatch");
          L.fkind[q] = FACE_WALL;
          L.fref[q] = wall_pos[k];
          key[j - 1] = ((int64_t)1 << 40) + k;
        } else {
          auto it = bce_of_edge.find(k);
          if (it != bce_of_edge.end() && in_elem(k) == i1) {
            L.fkind[q] = FACE_BC;
            L.fref[q] = it->second;
            key[j - 1] = ((int64_t)2 << 40) + it->second;
          } else {
            L.fkind[q] = FACE_NONE;
            key[j - 1] = ((int64_t)3 << 40) + j;
          }
        }
      }
      L.fnx[q] = nx;
      L.fny[q] = ny;
    }
    int ord[3] = {0, 1, 2};
    std::sort(ord, ord + 3, [&](int a, int b) { return key[a] < key[b]; });
    L.forder[c] = (uint8_t)(ord[0] | (ord[1] << 2) | (ord[2] << 4));
    for (int j = 0; j < 3; j++)
      if (L.fkind[(size_t)j * T + c] == FACE_BC) L.forder[c] |= kOrderHasBc;
    if (L.forder[c] & kOrderHasBc) L.bc_cells.push_back(c);
  }
  L.lsq_derived = lsq_all;
  // culverts (cvprep.f90 placed them; solverFVT.f90:227-233 adds their terms)
  if (m.n_culvert > 0) {
    const int32_t n = m.n_culvert, ld = m.cv_ld;
    if (!m.cvtrigin || !m.cvtrigout || !m.cvptoin || !m.cvrin || !m.ncvtable || !m.cvhead || !m.cvq || ld < 1)
      return set_error(STORM_ERR_MESH, "storm_fvt_create: culvert arrays missing");
    L.ncv = n;
    L.cv_ld = ld;
    L.cv_in.resize(n); L.cv_n.resize(n); L.cv_rx.resize(n); L.cv_ry.resize(n); L.cv_zinv.resize(n);
    L.cv_head.assign(m.cvhead, m.cvhead + (size_t)ld * n);
    L.cv_q.assign(m.cvq, m.cvq + (size_t)ld * n);
    std::vector<std::pair<int32_t, int32_t>> terms;  // (cell, code), in the reference's order
    for (int32_t i = 0; i < n; i++) {
      const int32_t a = m.cvtrigin[i], b = m.cvtrigout[i];
      if (a < 1 || a > T || b < 1 || b > T) return set_error(STORM_ERR_MESH, "storm_fvt_create: culvert triangle out of range");
      if (m.ncvtable[i] < 1 || m.ncvtable[i] > ld)
        return set_error(STORM_ERR_MESH, "storm_fvt_create: culvert performance curve size out of range");
      L.cv_in[i] = CN(a);
      L.cv_n[i] = m.ncvtable[i];
      L.cv_rx[i] = m.cvrin[2 * (size_t)i];
      L.cv_ry[i] = m.cvrin[2 * (size_t)i + 1];
      L.cv_zinv[i] = m.cvptoin[3 * (size_t)i + 2];
      terms.push_back({CN(a), i << 1});
      terms.push_back({CN(b), (i << 1) | 1});
    }
    std::stable_sort(terms.begin(), terms.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
    for (const auto& t : terms) {
      L.cvc_cell.push_back(t.first);
      L.cvc_code.push_back(t.second);
      L.forder[t.first] |= kOrderHasCulvert;
    }
  }
  // Greedy colouring of the t2t stencil made symmetric, cells in reference index order,
  // each taking the smallest colour none of its already coloured neighbours has (the
  // order residual smoothing visits them; the oracle builds the same colouring).
  {
    std::vector<int32_t> deg((size_t)T + 1, 0);
    for (int32_t o = 0; o < T; o++) {
      const int32_t n = m.t2t[o];
      for (int32_t k = 0; k < n; k++) {
        deg[o]++;
        deg[m.t2t[(size_t)(k + 1) * T + o] - 1]++;
      }
    }
    std::vector<int32_t> off((size_t)T + 1, 0);
    for (int32_t o = 0; o < T; o++) off[o + 1] = off[o] + deg[o];
    std::vector<int32_t> adj(off[T]), fill(T, 0);
    for (int32_t o = 0; o < T; o++) {
      const int32_t n = m.t2t[o];
      for (int32_t k = 0; k < n; k++) {
        const int32_t j = m.t2t[(size_t)(k + 1) * T + o] - 1;
        adj[off[o] + fill[o]++] = j;
        adj[off[j] + fill[j]++] = o;
      }
    }
    std::vector<int32_t> col(T, 0);
    int32_t ncol = 0;
    for (int32_t o = 0; o < T; o++) {
      bool used[256] = {false};
      for (int32_t q = off[o]; q < off[o + 1]; q++)
        if (adj[q] < o && col[adj[q]] < 256) used[col[adj[q]]] = true;
      int32_t c = 0;
      while (c < 255 && used[c]) c++;
      col[o] = c;
      ncol = std::max(ncol, c + 1);
    }
    L.rs_off.assign(1, 0);
    L.rs_cells.clear();
    for (int32_t c = 0; c < ncol; c++) {
      for (int32_t o = 0; o < T; o++)
        if (col[o] == c) L.rs_cells.push_back(CN(o + 1));
      L.rs_off.push_back((int32_t)L.rs_cells.size());
    }
  }
  // numerical valve targets (solverFVT.f90:357-370)
  for (int32_t j = 0; j < m.n_bcedges; j++) {
    if (!m.hbar[j]) continue;
    int32_t k = m.bcedges[j];
    if (k < 1 || k > E) return set_error(STORM_ERR_MESH, "storm_fvt_create: bcedges entry out of range");
    int32_t i = in_elem(k);
    int mm = local_edge(i, k);
    if (i < 1 || mm < 1) return set_error(STORM_ERR_MESH, "storm_fvt_create: stage edge without element");
    L.hvmask[CN(i)] |= (uint8_t)(1u << (mm - 1));
  }
  (void)opt;
  return 0;
}

void merge_layouts(const std::vector<HostLayout>& parts, int block, HostLayout& M, std::vector<ScenarioInfo>& info) {
  const size_t S = parts.size();
  info.assign(S, ScenarioInfo{});
  int32_t T = 0, N = 0, ne = 0, nwall = 0, nbce = 0, nnz = 0, kst = 1;
  for (size_t s = 0; s < S; s++) {
    const HostLayout& P = parts[s];
    ScenarioInfo& I = info[s];
    I.cell_off = T;
    I.cell_cnt = P.T;
    I.node_off = N;
    I.node_cnt = P.N;
    I.blk_off = T / block;
    I.blk_cnt = (P.T + block - 1) / block;
    I.last_cell = T + P.last_cell_new;
    T += I.blk_cnt * block;
    N += P.N;
    ne += P.ne;
    nwall += P.nwall;
    nbce += P.nbce;
    nnz += P.n2t_nnz;
    kst = std::max(kst, P.kst);
  }
  M = HostLayout();
  M.T = T;
  M.N = N;
  M.kst = kst;
  M.ne = ne;
  M.nwall = nwall;
  M.nbce = nbce;
  M.n2t_nnz = nnz;
  const size_t T3 = 3 * (size_t)T;
  // per cell slot
  M.cell_sid.assign(T, -1);
  M.area.assign(T, 1.0); M.perim.assign(T, 1.0); M.xc.assign(T, 0.0); M.yc.assign(T, 0.0);
  M.z.assign(T, 0.0); M.delz_x.assign(T, 0.0); M.delz_y.assign(T, 0.0); M.zmax.assign(T, 0.0);
  M.cd.assign(T, 0.0); M.lsq_a.assign(T, 1.0); M.lsq_b.assign(T, 0.0); M.lsq_c.assign(T, 1.0);
  M.lsq_det.assign(T, 1.0); M.nst.assign(T, 0); M.forder.assign(T, 0); M.hvmask.assign(T, 0);
  // padding slots are never live, so only the scenarios' own cells decide
  M.lsq_derived = true;
  for (const HostLayout& P : parts) M.lsq_derived = M.lsq_derived && P.lsq_derived;
  M.vert.assign(T3, 0); M.t2t3.assign(T3, -1); M.fref.assign(T3, 0); M.fkind.assign(T3, FACE_NONE);
  M.rc_x.assign(T3, 0.0); M.rc_y.assign(T3, 0.0); M.fnx.assign(T3, 0.0); M.fny.assign(T3, 0.0);
  M.flen.assign(T3, 0.0); M.fz0.assign(T3, 0.0);
  M.st_id.assign((size_t)kst * T, 0); M.st_w.assign((size_t)kst * T, 0.0);
  M.st_dx.assign((size_t)kst * T, 0.0); M.st_dy.assign((size_t)kst * T, 0.0);
  bool any_wind = false;
  for (size_t s = 0; s < S; s++) any_wind = any_wind || !parts[s].wcoef1.empty();
  if (any_wind) { M.wcoef1.assign(T, 0.0); M.wcoef2.assign(T, 0.0); }
  M.node_sid.reserve(N); M.edge_sid.reserve(ne);
  int32_t eoff = 0, woff = 0, boff = 0, noff_nnz = 0, tsoff = 0;
  M.n2t_off.assign(1, 0);
  for (size_t s = 0; s < S; s++) {
    const HostLayout& P = parts[s];
    const ScenarioInfo& I = info[s];
    const int32_t co = I.cell_off, no = I.node_off;
    for (int32_t c = 0; c < P.T; c++) {
      const int32_t g = co + c;
      M.cell_sid[g] = (int32_t)s;
      M.area[g] = P.area[c]; M.perim[g] = P.perim[c]; M.xc[g] = P.xc[c]; M.yc[g] = P.yc[c];
      M.z[g] = P.z[c]; M.delz_x[g] = P.delz_x[c]; M.delz_y[g] = P.delz_y[c]; M.zmax[g] = P.zmax[c];
      M.cd[g] = P.cd[c]; M.lsq_a[g] = P.lsq_a[c]; M.lsq_b[g] = P.lsq_b[c]; M.lsq_c[g] = P.lsq_c[c];
      M.lsq_det[g] = P.lsq_det[c]; M.nst[g] = P.nst[c]; M.forder[g] = P.forder[c]; M.hvmask[g] = P.hvmask[c];
      if (!P.wcoef1.empty()) { M.wcoef1[g] = P.wcoef1[c]; M.wcoef2[g] = P.wcoef2[c]; }
      for (int j = 0; j < 3; j++) {
        const size_t q = (size_t)j * P.T + c, qg = (size_t)j * T + g;
        M.vert[qg] = P.vert[q] + no;
        M.t2t3[qg] = P.t2t3[q] < 0 ? -1 : P.t2t3[q] + co;
        const uint8_t kind = P.fkind[q] & 7;
        int32_t r = P.fref[q];
        if (kind == FACE_LEFT || kind == FACE_RIGHT) r += eoff;
        else if (kind == FACE_WALL) r += woff;
        else if (kind == FACE_BC) r += boff;
        M.fref[qg] = r;
        M.fkind[qg] = P.fkind[q];
        M.rc_x[qg] = P.rc_x[q]; M.rc_y[qg] = P.rc_y[q]; M.fnx[qg] = P.fnx[q]; M.fny[qg] = P.fny[q];
        M.flen[qg] = P.flen[q]; M.fz0[qg] = P.fz0[q];
      }
      for (int k = 0; k < P.kst; k++) {
        const size_t q = (size_t)k * P.T + c, qg = (size_t)k * T + g;
        M.st_id[qg] = P.st_id[q] + co;
        M.st_w[qg] = P.st_w[q]; M.st_dx[qg] = P.st_dx[q]; M.st_dy[qg] = P.st_dy[q];
      }
    }
    for (int32_t n = 0; n < P.N; n++) {
      M.node_sid.push_back((int32_t)s);
      M.zvtx.push_back(P.zvtx[n]); M.node_x.push_back(P.node_x[n]); M.node_y.push_back(P.node_y[n]);
      M.node_hbc.push_back(P.node_hbc[n]);
      M.n2t_off.push_back(P.n2t_off[n + 1] + noff_nnz);
    }
    for (int32_t q = 0; q < P.n2t_nnz; q++) {
      M.n2t_cell.push_back(P.n2t_cell[q] + co);
      M.n2t_w.push_back(P.n2t_w[q]);
    }
    for (int32_t e = 0; e < P.ne; e++) {
      M.edge_sid.push_back((int32_t)s);
      M.eL.push_back(P.eL[e] + co); M.eR.push_back(P.eR[e] + co); M.eslot.push_back(P.eslot[e]);
      M.enx.push_back(P.enx[e]); M.eny.push_back(P.eny[e]); M.elen.push_back(P.elen[e]); M.ez0.push_back(P.ez0[e]);
    }
    for (int32_t w = 0; w < P.nwall; w++) {
      M.wall_p1.push_back(P.wall_p1[w] + no);
      M.wall_p2.push_back(P.wall_p2[w] + no);
    }
    for (int32_t b = 0; b < P.nbdr; b++) {
      M.bdr_sid.push_back((int32_t)s);
      M.bdr_kind.push_back(P.bdr_kind[b]); M.bdr_slot.push_back(P.bdr_slot[b]);
      M.bdr_off.push_back(P.bdr_off[b] + boff); M.bdr_cnt.push_back(P.bdr_cnt[b]);
    }
    for (int32_t e = 0; e < P.nbce; e++) {
      M.bce_cell.push_back(P.bce_cell[e] + co); M.bce_slot.push_back(P.bce_slot[e]);
      M.bce_nx.push_back(P.bce_nx[e]); M.bce_ny.push_back(P.bce_ny[e]);
      M.bce_tx.push_back(P.bce_tx[e]); M.bce_ty.push_back(P.bce_ty[e]);
      M.bce_len.push_back(P.bce_len[e]); M.bce_zmid.push_back(P.bce_zmid[e]);
    }
    for (int32_t c : P.bc_cells) M.bc_cells.push_back(c + co);
    for (size_t i = 0; i < P.ts_t.size(); i++) {
      M.ts_t.push_back(P.ts_t[i]);
      M.ts_v.push_back(P.ts_v[i]);
    }
    (void)tsoff;
    eoff += P.ne;
    woff += P.nwall;
    boff += P.nbce;
    noff_nnz += P.n2t_nnz;
  }
  M.nbdr = (int32_t)M.bdr_kind.size();
  // culverts: concatenated, performance curves padded to the widest table
  M.ncv = 0;
  M.cv_ld = 0;
  for (const HostLayout& P : parts) { M.ncv += P.ncv; M.cv_ld = std::max(M.cv_ld, P.cv_ld); }
  M.cv_head.assign((size_t)M.ncv * M.cv_ld, 0.0);
  M.cv_q.assign((size_t)M.ncv * M.cv_ld, 0.0);
  for (size_t s = 0, cvo = 0; s < S; s++) {
    const HostLayout& P = parts[s];
    const int32_t co = info[s].cell_off;
    for (int32_t i = 0; i < P.ncv; i++) {
      M.cv_in.push_back(P.cv_in[i] + co); M.cv_n.push_back(P.cv_n[i]);
      M.cv_rx.push_back(P.cv_rx[i]); M.cv_ry.push_back(P.cv_ry[i]); M.cv_zinv.push_back(P.cv_zinv[i]);
      for (int32_t j = 0; j < P.cv_n[i]; j++) {
        M.cv_head[(cvo + i) * M.cv_ld + j] = P.cv_head[(size_t)i * P.cv_ld + j];
        M.cv_q[(cvo + i) * M.cv_ld + j] = P.cv_q[(size_t)i * P.cv_ld + j];
      }
    }
    for (size_t k = 0; k < P.cvc_cell.size(); k++) {
      M.cvc_cell.push_back(P.cvc_cell[k] + co);
      M.cvc_code.push_back(P.cvc_code[k] + (int32_t)(cvo << 1));
    }
    cvo += P.ncv;
  }
  // residual-smoothing colours: colour c of every scenario together (scenarios share no cell)
  size_t ncol = 0;
  for (const HostLayout& P : parts) ncol = std::max(ncol, P.rs_off.empty() ? 0 : P.rs_off.size() - 1);
  M.rs_off.assign(1, 0);
  M.rs_cells.clear();
  for (size_t c = 0; c < ncol; c++) {
    for (size_t s = 0; s < S; s++) {
      const HostLayout& P = parts[s];
      if (c + 1 >= P.rs_off.size()) continue;
      for (int32_t q = P.rs_off[c]; q < P.rs_off[c + 1]; q++) M.rs_cells.push_back(P.rs_cells[q] + info[s].cell_off);
    }
    M.rs_off.push_back((int32_t)M.rs_cells.size());
  }
}

}  // namespace storm
