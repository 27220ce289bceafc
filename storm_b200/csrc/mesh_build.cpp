// mesh_build.cpp -- host-side builder of the prepared FVT mesh (storm_fvt_mesh_build).
//
// For callers that do not hold SToRM's Fortran module arrays, this reproduces what
// read_data and dataprepFVT leave in MODULE geometry/dep_vars/vbc_arrays before
// `CALL solverFVT` (Source_xsy-64bit/solver.f90:50-57):
//   find_edges.f90:27-197, edge_normals.f90:30-39, t_areas.f90:33-52,
//   walls.f90:40-148, ibc_arrays.f90:42-137/377-466, node_db.f90:32-68,
//   elemnt_db.f90:32-128/216-233, cde_t2t.f90:23-49, c2v_setup.f90:98-119,
//   lsq_setup.f90:92-145, dataprepFVT.f90:69-306.
// Numbering conventions are the reference's (edge order of first appearance,
// orientation as first seen, e(1) = first element to reference the edge, Triangle
// .edge/.v.edge order when edges are supplied), so ids match the Fortran host's.
// Arithmetic follows the reference's expressions in order; the file is compiled with
// -ffp-contract=off so every product and sum rounds as written.  Node-pair searches
// that are linear scans in the reference (edge_in_array, is_edge) use a hash map,
// which returns the same edge on meshes with one edge per node pair.
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <type_traits>
#include <utility>
#include <unordered_map>
#include <vector>

#include "../../include/storm_fvt.h"
#include "storm_internal.h"

namespace storm {
namespace {

constexpr double kHalf = 0.5;
constexpr double kOneThird = 1.0 / 3.0;

inline double max2(double a, double b) { return (b > a) ? b : a; }

struct MeshError {
  int code;
  std::string msg;
};

[[noreturn]] void fail(int code, const std::string& m) { throw MeshError{code, m}; }

inline uint64_t pair_key(int32_t a, int32_t b) {
  uint32_t lo = (uint32_t)(a < b ? a : b), hi = (uint32_t)(a < b ? b : a);
  return ((uint64_t)lo << 32) | hi;
}

// Owning storage behind a StormFvtMesh.
struct MeshStorage {
  std::vector<double> node_x, node_y, tri_area, tri_perim, tri_xc, tri_yc, edge_normal, edge_tang,
      edge_length, rc_x, rc_y, lsq_dx, lsq_dy, lsq_w, lsq_a, lsq_b, lsq_c, lsq_det, c2v_w, z, zvtx, cd,
      qin, timelocq, timeserq, hbc, timeloch, timeserh, wcoef1, wcoef2, cvptoin, cvrin, cvhead, cvq;
  std::vector<int32_t> tri_vertex, tri_edge, edge_p, edge_e, t2t, t2t3, n2t, csortedz, flowedg1, walledg1,
      bcedges, hbar, qbar, vtype, bcedgesinflow, n_timeserq, htype, bcedgesoutflow, n_hbc, hbc_nodes,
      n_timeserh, n_qin, qin_nodes, cvtrigin, cvtrigout, ncvtable;
  int32_t t2t_ncol = 0, n2t_ncol = 0, c2v_ncol = 0, qin_ld = 1, hbc_ld = 1, tsq_ld = 1, tsh_ld = 1;
  double bch_max = 0.0;
  StormFvtMesh view{};
};

// Standard-layout handle: the public StormFvtMesh first, then the storage behind it.
struct OwnedMesh {
  StormFvtMesh view;
  MeshStorage* store;
};

class Builder {
 public:
  Builder(const StormFvtProblem& p, MeshStorage& m) : p_(p), m_(m), N_(p.n_pts), T_(p.n_elems) {}

  void run() {
    copy_input();
    find_edges();
    t_areas();
    walls_and_bcedges();
    ibc_arrays();
    node_db();
    elemnt_db();
    dataprep();
    culverts();
    fill_view();
  }

 private:
  const StormFvtProblem& p_;
  MeshStorage& m_;
  int32_t N_, T_, E_ = 0;
  std::vector<uint8_t> bcnode_;

  // 1-based accessors over the Fortran layouts
  int32_t& gv(int32_t i, int j) { return m_.tri_vertex[3 * (size_t)(i - 1) + (j - 1)]; }
  int32_t& ge(int32_t i, int j) { return m_.tri_edge[3 * (size_t)(i - 1) + (j - 1)]; }
  int32_t& ep(int32_t k, int j) { return m_.edge_p[2 * (size_t)(k - 1) + (j - 1)]; }
  int32_t& ee(int32_t k, int j) { return m_.edge_e[2 * (size_t)(k - 1) + (j - 1)]; }
  double nx(int32_t p) const { return m_.node_x[p - 1]; }
  double ny(int32_t p) const { return m_.node_y[p - 1]; }
  static int jnext(int j) { return j == 3 ? 1 : j + 1; }  // MAX(1,MOD(j+1,4))

  void copy_input() {
    if (N_ < 3 || T_ < 1 || !p_.x || !p_.y || !p_.tri || !p_.zb || !p_.cd)
      fail(STORM_ERR_ARG, "incomplete problem description");
    m_.node_x.assign(p_.x, p_.x + N_);
    m_.node_y.assign(p_.y, p_.y + N_);
    m_.tri_vertex.assign(p_.tri, p_.tri + 3 * (size_t)T_);
    for (int32_t v : m_.tri_vertex)
      if (v < 1 || v > N_) fail(STORM_ERR_MESH, "triangle vertex out of range");
    m_.tri_edge.assign(3 * (size_t)T_, 0);
    if (p_.n_inflow > STORM_MAX_BDR || p_.n_outflow > STORM_MAX_BDR)
      fail(STORM_ERR_ARG, "too many boundaries");
    bcnode_.assign((size_t)N_ + 1, 0);
    // inflow strings (read_cgns.f90:433-490 layout: qin_nodes(maxnin,n), -1 padded)
    int32_t d1 = 1, ts = 1;
    for (int b = 0; b < p_.n_inflow; b++) {
      const StormFvtBoundary& B = p_.inflow[b];
      if (B.n_nodes < 1) fail(STORM_ERR_MESH, "inflow boundary has no nodes assigned");
      if (B.type < 0 || B.type > 5 || B.type == 2)
        fail(STORM_ERR_UNSUPPORTED, "inflow vtype " + std::to_string(B.type) + " is not supported");
      d1 = B.n_nodes > d1 ? B.n_nodes : d1;
      ts = B.n_series > ts ? B.n_series : ts;
    }
    int32_t nb = p_.n_inflow > 0 ? p_.n_inflow : 1;
    m_.qin_ld = d1;
    m_.tsq_ld = ts;
    m_.vtype.assign(nb, 0);
    m_.n_qin.assign(nb, 0);
    m_.qin.assign(nb, 0.0);
    m_.n_timeserq.assign(nb, 0);
    m_.qin_nodes.assign((size_t)d1 * nb, -1);
    m_.timelocq.assign((size_t)ts * nb, 0.0);
    m_.timeserq.assign((size_t)ts * nb, 0.0);
    for (int b = 0; b < p_.n_inflow; b++) {
      const StormFvtBoundary& B = p_.inflow[b];
      m_.vtype[b] = B.type;
      m_.n_qin[b] = B.n_nodes;
      m_.qin[b] = B.value;
      m_.n_timeserq[b] = B.n_series;
      for (int i = 0; i < B.n_nodes; i++) {
        int32_t q = B.nodes[i];
        if (q < 1 || q > N_) fail(STORM_ERR_MESH, "inflow node out of range");
        m_.qin_nodes[(size_t)b * d1 + i] = q;
        bcnode_[q] = 1;
      }
      for (int i = 0; i < B.n_series; i++) {
        m_.timelocq[(size_t)b * ts + i] = B.series_t[i];
        m_.timeserq[(size_t)b * ts + i] = B.series_v[i];
      }
    }
    d1 = 1;
    ts = 1;
    for (int b = 0; b < p_.n_outflow; b++) {
      const StormFvtBoundary& B = p_.outflow[b];
      if (B.n_nodes < 1) fail(STORM_ERR_MESH, "outflow boundary has no nodes assigned");
      if (B.type < 0 || B.type > 2) fail(STORM_ERR_MESH, "invalid value in htype");
      d1 = B.n_nodes > d1 ? B.n_nodes : d1;
      ts = B.n_series > ts ? B.n_series : ts;
    }
    nb = p_.n_outflow > 0 ? p_.n_outflow : 1;
    m_.hbc_ld = d1;
    m_.tsh_ld = ts;
    m_.htype.assign(nb, 0);
    m_.n_hbc.assign(nb, 0);
    m_.hbc.assign(nb, 0.0);
    m_.n_timeserh.assign(nb, 0);
    m_.hbc_nodes.assign((size_t)d1 * nb, -1);
    m_.timeloch.assign((size_t)ts * nb, 0.0);
    m_.timeserh.assign((size_t)ts * nb, 0.0);
    for (int b = 0; b < p_.n_outflow; b++) {
      const StormFvtBoundary& B = p_.outflow[b];
      m_.htype[b] = B.type;
      m_.n_hbc[b] = B.n_nodes;
      m_.hbc[b] = B.value;
      m_.n_timeserh[b] = B.n_series;
      for (int i = 0; i < B.n_nodes; i++) {
        int32_t q = B.nodes[i];
        if (q < 1 || q > N_) fail(STORM_ERR_MESH, "outflow node out of range");
        m_.hbc_nodes[(size_t)b * d1 + i] = q;
        bcnode_[q] = 1;
      }
      for (int i = 0; i < B.n_series; i++) {
        m_.timeloch[(size_t)b * ts + i] = B.series_t[i];
        m_.timeserh[(size_t)b * ts + i] = B.series_v[i];
      }
    }
  }

  // find_edges.f90:27-197
  void find_edges() {
    std::unordered_map<uint64_t, int32_t> first;  // node pair -> first edge id
    const bool tdata = p_.n_edges > 0;
    if (!tdata) {
      first.reserve((size_t)3 * T_);
      m_.edge_p.reserve((size_t)3 * T_);
      for (int32_t i = 1; i <= T_; i++)
        for (int j = 1; j <= 3; j++) {
          int32_t a = gv(i, j), b = gv(i, jnext(j));
          auto ins = first.emplace(pair_key(a, b), (int32_t)(m_.edge_p.size() / 2 + 1));
          if (ins.second) {
            m_.edge_p.push_back(a);
            m_.edge_p.push_back(b);
          }
        }
      E_ = (int32_t)(m_.edge_p.size() / 2);
    } else {
      E_ = p_.n_edges;
      m_.edge_p.assign(p_.edge_p, p_.edge_p + 2 * (size_t)E_);
      m_.edge_e.assign(2 * (size_t)E_, 0);
      for (int32_t k = 1; k <= E_; k++) {
        int32_t e1 = p_.edge_e[2 * (k - 1)], e2 = p_.edge_e[2 * (k - 1) + 1];
        if (e1 < 0) {  // tecplot_read.f90:146-153: a Voronoi ray
          e1 = e2;
          e2 = -1;
        }
        ee(k, 1) = e1;
        ee(k, 2) = e2;
        if (ep(k, 1) < 1 || ep(k, 1) > N_ || ep(k, 2) < 1 || ep(k, 2) > N_)
          fail(STORM_ERR_MESH, "edge node out of range");
      }
      first.reserve((size_t)E_);
      for (int32_t k = 1; k <= E_; k++) first.emplace(pair_key(ep(k, 1), ep(k, 2)), k);
    }
    if (tdata) {
      for (int32_t j = 1; j <= E_; j++)
        for (int k = 1; k <= 2; k++) {
          int32_t i = ee(j, k);
          if (i < 0) continue;
          if (i == 0 || i > T_) fail(STORM_ERR_MESH, "edge element out of range");
          for (int l = 1; l <= 3; l++) {
            int32_t a = gv(i, l), b = gv(i, jnext(l));
            if (a == ep(j, 1) && b == ep(j, 2)) {
              ge(i, l) = j;
              break;
            } else if (a == ep(j, 2) && b == ep(j, 1)) {
              ge(i, l) = -j;
              break;
            }
          }
        }
      for (int32_t v : m_.tri_edge)
        if (v == 0) fail(STORM_ERR_MESH, "edge data structure incomplete");
    } else {
      for (int32_t i = 1; i <= T_; i++)
        for (int j = 1; j <= 3; j++) {
          int32_t a = gv(i, j), b = gv(i, jnext(j));
          int32_t k = first.at(pair_key(a, b));
          ge(i, j) = (ep(k, 1) == a && ep(k, 2) == b) ? k : -k;
        }
    }
    // edge_normals.f90:30-39 and the lengths (find_edges.f90:159-163)
    m_.edge_normal.resize(2 * (size_t)E_);
    m_.edge_tang.resize(2 * (size_t)E_);
    m_.edge_length.resize(E_);
    for (int32_t k = 1; k <= E_; k++) {
      double x1 = nx(ep(k, 1)), y1 = ny(ep(k, 1)), x2 = nx(ep(k, 2)), y2 = ny(ep(k, 2));
      m_.edge_normal[2 * (k - 1)] = y2 - y1;
      m_.edge_normal[2 * (k - 1) + 1] = x1 - x2;
      m_.edge_tang[2 * (k - 1)] = x2 - x1;
      m_.edge_tang[2 * (k - 1) + 1] = y2 - y1;
      double delx = nx(ep(k, 1)) - nx(ep(k, 2));
      double dely = ny(ep(k, 1)) - ny(ep(k, 2));
      m_.edge_length[k - 1] = std::sqrt(delx * delx + dely * dely);
    }
    if (!tdata) {  // find_edges.f90:165-193
      m_.edge_e.assign(2 * (size_t)E_, -1);
      std::vector<int32_t> counter((size_t)E_ + 1, 1);
      for (int32_t i = 1; i <= T_; i++)
        for (int j = 1; j <= 3; j++) {
          int32_t k = std::abs(ge(i, j));
          if (counter[k] > 2) fail(STORM_ERR_MESH, "edge data structure incorrect");
          ee(k, counter[k]) = i;
          counter[k]++;
        }
    }
  }

  // t_areas.f90:33-52
  void t_areas() {
    m_.tri_area.resize(T_);
    m_.tri_perim.resize(T_);
    m_.tri_xc.resize(T_);
    m_.tri_yc.resize(T_);
    for (int32_t i = 1; i <= T_; i++) {
      double x1 = nx(gv(i, 1)), y1 = ny(gv(i, 1));
      double x2 = nx(gv(i, 2)), y2 = ny(gv(i, 2));
      double x3 = nx(gv(i, 3)), y3 = ny(gv(i, 3));
      m_.tri_area[i - 1] = kHalf * std::fabs((x1 - x2) * (y1 + y2) + (x2 - x3) * (y2 + y3) + (x3 - x1) * (y3 + y1));
      m_.tri_xc[i - 1] = kOneThird * (x1 + x2 + x3);
      m_.tri_yc[i - 1] = kOneThird * (y1 + y2 + y3);
      m_.tri_perim[i - 1] = m_.edge_length[std::abs(ge(i, 1)) - 1] + m_.edge_length[std::abs(ge(i, 2)) - 1] +
                            m_.edge_length[std::abs(ge(i, 3)) - 1];
    }
  }

  // walls.f90:40-148 and ibc_arrays.f90:377-413 (bcedges)
  void walls_and_bcedges() {
    std::vector<int32_t> count((size_t)E_ + 1, 0);
    for (int32_t v : m_.tri_edge) count[std::abs(v)]++;
    std::vector<int32_t> bpolygon;
    for (int32_t i = 1; i <= E_; i++) {
      if (count[i] == 1) {
        bpolygon.push_back(i);
        if (!(bcnode_[ep(i, 1)] && bcnode_[ep(i, 2)])) m_.walledg1.push_back(i);
      } else if (count[i] == 2) {
        m_.flowedg1.push_back(i);
      } else {
        fail(STORM_ERR_MESH, "grid construction error in edge " + std::to_string(i));
      }
    }
    int32_t nbc = (int32_t)(bpolygon.size() - m_.walledg1.size());
    int32_t k = 0;
    for (int b = 0; b < p_.n_inflow; b++) k += m_.n_qin[b] - 1;
    for (int b = 0; b < p_.n_outflow; b++) k += m_.n_hbc[b] - 1;
    if (k != nbc) fail(STORM_ERR_MESH, "number of boundary condition edges does not match the boundary chains");
    std::vector<uint8_t> is_wall((size_t)E_ + 1, 0);
    for (int32_t w : m_.walledg1) is_wall[w] = 1;
    for (int32_t e : bpolygon)
      if (!is_wall[e]) m_.bcedges.push_back(e);
    m_.hbar.assign(m_.bcedges.size(), 0);
    m_.qbar.assign(m_.bcedges.size(), 0);
  }

  // ibc_arrays.f90:59-137 (inflow chains), :161-181 (outflow chains), :416-466
  void ibc_arrays() {
    std::unordered_map<uint64_t, int32_t> first;
    first.reserve((size_t)E_);
    for (int32_t k = 1; k <= E_; k++) first.emplace(pair_key(ep(k, 1), ep(k, 2)), k);
    auto is_edge = [&](int32_t a, int32_t b) -> int32_t {
      if (a < 1 || a > N_ || b < 1 || b > N_) return -1;
      auto it = first.find(pair_key(a, b));
      return it == first.end() ? 0 : it->second;
    };
    std::unordered_map<int32_t, int32_t> pos;  // edge -> first bcedges position (1-based)
    for (size_t j = 0; j < m_.bcedges.size(); j++) pos.emplace(m_.bcedges[j], (int32_t)j + 1);
    const int32_t nin = p_.n_inflow > 0 ? p_.n_inflow : 1;
    m_.bcedgesinflow.assign((size_t)(m_.qin_ld + 1) * nin, 0);
    for (int b = 0; b < p_.n_inflow; b++) {
      int32_t* col = &m_.bcedgesinflow[(size_t)b * (m_.qin_ld + 1)];
      col[0] = m_.n_qin[b] - 1;
      for (int i = 1; i <= m_.n_qin[b] - 1; i++) {
        int32_t a = m_.qin_nodes[(size_t)b * m_.qin_ld + i - 1], c = m_.qin_nodes[(size_t)b * m_.qin_ld + i];
        int32_t e = is_edge(a, c);
        if (e == 0) fail(STORM_ERR_MESH, "inflow boundary nodes are not connected by an edge");
        if (e < 0) fail(STORM_ERR_MESH, "inflow boundary node out of range");
        col[i] = e;
        int32_t t = ee(e, 1) < 1 ? ee(e, 2) : ee(e, 1);
        if (t < 1) fail(STORM_ERR_MESH, "inflow edge has no element");
        auto it = pos.find(e);
        if (it != pos.end()) m_.qbar[it->second - 1] = 1;
      }
    }
    const int32_t nout = p_.n_outflow > 0 ? p_.n_outflow : 1;
    m_.bcedgesoutflow.assign((size_t)(m_.hbc_ld + 1) * nout, 0);
    for (int b = 0; b < p_.n_outflow; b++) {
      int32_t* col = &m_.bcedgesoutflow[(size_t)b * (m_.hbc_ld + 1)];
      col[0] = m_.n_hbc[b] - 1;
      for (int i = 1; i <= m_.n_hbc[b] - 1; i++) {
        int32_t a = m_.hbc_nodes[(size_t)b * m_.hbc_ld + i - 1], c = m_.hbc_nodes[(size_t)b * m_.hbc_ld + i];
        int32_t e = is_edge(a, c);
        if (e == 0) fail(STORM_ERR_MESH, "outflow boundary nodes are not connected by an edge");
        if (e < 0) fail(STORM_ERR_MESH, "outflow boundary node out of range");
        col[i] = e;
        auto it = pos.find(e);
        if (it != pos.end()) m_.hbar[it->second - 1] = 1;
      }
    }
  }

  // node_db.f90:32-68
  void node_db() {
    std::vector<int32_t> counter((size_t)N_ + 1, 0);
    for (int32_t v : m_.tri_vertex) counter[v]++;
    int32_t k = 0;
    for (int32_t p = 1; p <= N_; p++) k = counter[p] > k ? counter[p] : k;
    m_.n2t_ncol = k + 1;
    m_.c2v_ncol = k > 4 ? k : 4;  // c2v_setup.f90:33-34 with n2t2 of width MAX(k,4)+1
    m_.n2t.assign((size_t)N_ * m_.n2t_ncol, 0);
    auto n2t = [&](int32_t p, int32_t j) -> int32_t& { return m_.n2t[(size_t)(j - 1) * N_ + (p - 1)]; };
    for (int32_t i = 1; i <= T_; i++)
      for (int j = 1; j <= 3; j++) {
        int32_t p1 = gv(i, j);
        int32_t kk = n2t(p1, 1) + 1;
        n2t(p1, kk + 1) = i;
        n2t(p1, 1) = kk;
      }
  }

  // cde_t2t.f90:23-49: duplicate removal as the Fortran executes it (the inner DO
  // keeps the trip count fixed at entry while n shrinks; shifts read one past the end)
  static void cde_t2t(std::vector<int32_t>& w, int32_t T, int32_t i) {
    auto tw = [&](int32_t r, int32_t c) -> int32_t& { return w[(size_t)(c - 1) * T + (r - 1)]; };
    int32_t n = tw(i, 1), l = 1;
    for (;;) {
      int32_t j = tw(i, l + 1), trips_end = n;
      for (int32_t m = l + 1; m <= trips_end; m++) {
        if (j == tw(i, m + 1)) {
          n -= 1;
          for (int32_t nn = m; nn <= n; nn++) tw(i, nn + 1) = tw(i, nn + 2);
          tw(i, 1) = n;
        }
      }
      l += 1;
      if (l > n) break;
    }
  }

  // elemnt_db.f90:32-128, 216-233
  void elemnt_db() {
    if (T_ < 4) fail(STORM_ERR_MESH, "too few triangles in computational domain (must be >= 4)");
    const int32_t maxdim = 20;
    std::vector<int32_t> w((size_t)T_ * maxdim, 0);
    auto tw = [&](int32_t r, int32_t c) -> int32_t& { return w[(size_t)(c - 1) * T_ + (r - 1)]; };
    auto append = [&](int32_t i, int32_t k) {
      int32_t nn = tw(i, 1) + 1;
      if (nn + 1 > maxdim) fail(STORM_ERR_MESH, "t2t stencil exceeds its working width");
      tw(i, nn + 1) = k;
      tw(i, 1) = nn;
    };
    for (int32_t k = 1; k <= E_; k++) {
      int32_t e1 = ee(k, 1), e2 = ee(k, 2);
      if (e1 < 1 || e2 < 1) continue;
      append(e1, e2);
      append(e2, e1);
    }
    for (int32_t i = 1; i <= T_; i++) {
      int32_t n = tw(i, 1);
      if (n == 3) continue;
      if (n < 1 || n > 3) fail(STORM_ERR_MESH, "triangle connectivity table incorrect");
      for (int32_t l = 1; l <= n; l++) {
        int32_t j = tw(i, l + 1);
        int32_t trips = tw(j, 1) < 3 ? tw(j, 1) : 3;
        for (int32_t m = 1; m <= trips; m++) {
          int32_t k = tw(j, m + 1);
          if (k != i) append(i, k);
        }
      }
      cde_t2t(w, T_, i);
    }
    for (int32_t i = 1; i <= T_; i++) {
      int32_t n = tw(i, 1);
      if (n >= 3) continue;
      int32_t j = tw(i, n + 1), trips = tw(j, 1);
      for (int32_t m = 1; m <= trips; m++) {
        int32_t k = tw(j, m + 1);
        if (k != i) append(i, k);
      }
      cde_t2t(w, T_, i);
    }
    int32_t md = 0;
    for (int32_t i = 1; i <= T_; i++) md = tw(i, 1) > md ? tw(i, 1) : md;
    md += 1;
    m_.t2t_ncol = md;
    m_.t2t.assign(w.begin(), w.begin() + (size_t)T_ * md);
    m_.t2t3.assign(3 * (size_t)T_, 0);
    for (int32_t i = 1; i <= T_; i++)
      for (int j = 1; j <= 3; j++) {
        int32_t k = std::abs(ge(i, j));
        int32_t e1 = ee(k, 1);
        if (e1 == i) e1 = ee(k, 2);
        m_.t2t3[3 * (size_t)(i - 1) + (j - 1)] = e1;
      }
  }

  // dataprepFVT.f90:69-306 (with c2v_setup type 3 and lsq_setup solver 2 type 2)
  void dataprep() {
    const int32_t kc = m_.c2v_ncol;
    auto n2t = [&](int32_t p, int32_t j) { return m_.n2t[(size_t)(j - 1) * N_ + (p - 1)]; };
    std::vector<double> wn((size_t)N_ * kc, 0.0);  // c2v_weights (normalised)
    m_.c2v_w.assign((size_t)N_ * kc, 0.0);         // c2v_weights_id
    for (int32_t i = 1; i <= N_; i++) {
      double tdist = 0.0;
      for (int32_t j = 2; j <= n2t(i, 1) + 1; j++) {
        int32_t k = n2t(i, j);
        double xk = m_.tri_xc[k - 1] - nx(i);
        double yk = m_.tri_yc[k - 1] - ny(i);
        double wgt = 1.0 / std::sqrt(xk * xk + yk * yk);
        wn[(size_t)(j - 2) * N_ + (i - 1)] = wgt;
        m_.c2v_w[(size_t)(j - 2) * N_ + (i - 1)] = wgt;
        tdist = tdist + wgt;
      }
      for (int32_t j = 2; j <= n2t(i, 1) + 1; j++) {
        double& wref = wn[(size_t)(j - 2) * N_ + (i - 1)];
        wref = wref / tdist;
      }
    }
    auto vtx2ctr = [&](const double* va, double* ca) {
      for (int32_t i = 1; i <= T_; i++)
        ca[i - 1] = (va[gv(i, 1) - 1] + va[gv(i, 2) - 1] + va[gv(i, 3) - 1]) * kOneThird;
    };
    m_.z.resize(T_);
    m_.zvtx.resize(N_);
    m_.cd.resize(T_);
    if (p_.zb_at_vertices) {
      m_.zvtx.assign(p_.zb, p_.zb + N_);
    } else {  // ctr2vtx type 3 (ctr2vtx.f90:69-80)
      for (int32_t i = 1; i <= N_; i++) {
        double a = 0.0;
        for (int32_t j = 2; j <= n2t(i, 1) + 1; j++) a = a + wn[(size_t)(j - 2) * N_ + (i - 1)] * p_.zb[n2t(i, j) - 1];
        m_.zvtx[i - 1] = a;
      }
    }
    vtx2ctr(m_.zvtx.data(), m_.z.data());
    if (p_.cd_at_vertices) vtx2ctr(p_.cd, m_.cd.data());
    else m_.cd.assign(p_.cd, p_.cd + T_);
    // windforcing.f90 (text input, centred finite-volume solvers): per cell
    // wcoef = c0 * w * |w| / rho, the inputs moved to the cells by vtx2ctr when they
    // are given at the nodes
    if (p_.wind_c0 && p_.wind_x && p_.wind_y) {
      std::vector<double> c0(T_), wx(T_), wy(T_);
      if (p_.wind_at_vertices) {
        vtx2ctr(p_.wind_c0, c0.data());
        vtx2ctr(p_.wind_x, wx.data());
        vtx2ctr(p_.wind_y, wy.data());
      } else {
        c0.assign(p_.wind_c0, p_.wind_c0 + T_);
        wx.assign(p_.wind_x, p_.wind_x + T_);
        wy.assign(p_.wind_y, p_.wind_y + T_);
      }
      const double rho = 998.60;  // constants.f90:29
      m_.wcoef1.resize(T_);
      m_.wcoef2.resize(T_);
      for (int32_t i = 0; i < T_; i++) {
        const double windmag = std::sqrt(wx[i] * wx[i] + wy[i] * wy[i]);
        m_.wcoef1[i] = c0[i] * wx[i] * windmag / rho;
        m_.wcoef2[i] = c0[i] * wy[i] * windmag / rho;
      }
    }
    // rc (dataprepFVT.f90:161-173), before the normals are normalised
    m_.rc_x.resize(3 * (size_t)T_);
    m_.rc_y.resize(3 * (size_t)T_);
    for (int32_t i = 1; i <= T_; i++)
      for (int j = 1; j <= 3; j++) {
        int32_t k = std::abs(ge(i, j));
        double xc = kHalf * (nx(ep(k, 1)) + nx(ep(k, 2)));
        double yc = kHalf * (ny(ep(k, 1)) + ny(ep(k, 2)));
        m_.rc_x[(size_t)(j - 1) * T_ + (i - 1)] = xc - m_.tri_xc[i - 1];
        m_.rc_y[(size_t)(j - 1) * T_ + (i - 1)] = yc - m_.tri_yc[i - 1];
      }
    for (int32_t k = 0; k < E_; k++) {  // :176-181
      double L = m_.edge_length[k];
      m_.edge_normal[2 * k] = m_.edge_normal[2 * k] / L;
      m_.edge_normal[2 * k + 1] = m_.edge_normal[2 * k + 1] / L;
      m_.edge_tang[2 * k] = m_.edge_tang[2 * k] / L;
      m_.edge_tang[2 * k + 1] = m_.edge_tang[2 * k + 1] / L;
    }
    // lsq_setup.f90:92-145
    const int32_t kl = m_.t2t_ncol - 1 > 0 ? m_.t2t_ncol - 1 : 1;
    m_.lsq_dx.assign((size_t)T_ * kl, 0.0);
    m_.lsq_dy.assign((size_t)T_ * kl, 0.0);
    m_.lsq_w.assign((size_t)T_ * kl, 0.0);
    m_.lsq_a.assign(T_, 0.0);
    m_.lsq_b.assign(T_, 0.0);
    m_.lsq_c.assign(T_, 0.0);
    m_.lsq_det.assign(T_, 0.0);
    auto t2t = [&](int32_t i, int32_t j) { return m_.t2t[(size_t)(j - 1) * T_ + (i - 1)]; };
    for (int32_t i = 1; i <= T_; i++) {
      int32_t n = t2t(i, 1);
      double ai = 0.0, bi = 0.0, ci = 0.0;
      for (int32_t k = 1; k <= n; k++) {
        int32_t l = t2t(i, k + 1);
        size_t o = (size_t)(k - 1) * T_ + (i - 1);
        double dx = m_.tri_xc[l - 1] - m_.tri_xc[i - 1];
        double dy = m_.tri_yc[l - 1] - m_.tri_yc[i - 1];
        double wgt = 1.0 / (dx * dx + dy * dy);
        m_.lsq_dx[o] = dx;
        m_.lsq_dy[o] = dy;
        m_.lsq_w[o] = wgt;
        ai = ai + wgt * dx * dx;
        bi = bi + wgt * dx * dy;
        ci = ci + wgt * dy * dy;
      }
      m_.lsq_a[i - 1] = ai;
      m_.lsq_b[i - 1] = bi;
      m_.lsq_c[i - 1] = ci;
      m_.lsq_det[i - 1] = ai * ci - bi * bi;
    }
    // bch_max (:278-286)
    m_.bch_max = 0.0;
    for (size_t l = 0; l < m_.bcedges.size(); l++) {
      if (!m_.qbar[l]) continue;
      int32_t k = m_.bcedges[l];
      m_.bch_max = max2(m_.bch_max, m_.zvtx[ep(k, 1) - 1]);
      m_.bch_max = max2(m_.bch_max, m_.zvtx[ep(k, 2) - 1]);
    }
    // csortedz (:290-306): two bubble passes on zvtx
    m_.csortedz.assign(3 * (size_t)T_, 0);
    for (int32_t i = 1; i <= T_; i++) {
      int32_t* c = &m_.csortedz[3 * (size_t)(i - 1)];
      c[0] = gv(i, 1);
      c[1] = gv(i, 2);
      c[2] = gv(i, 3);
      for (int pass = 0; pass < 2; pass++)
        for (int k = 0; k < 2; k++)
          if (m_.zvtx[c[k] - 1] > m_.zvtx[c[k + 1] - 1]) std::swap(c[k], c[k + 1]);
    }
  }

  // pto_in_triangle.f90: barycentric test of (x, y) against triangle e
  bool pto_in_triangle(int32_t e, double x, double y) {
    const double tarea = m_.tri_area[e - 1];
    const double x1 = nx(gv(e, 1)), y1 = ny(gv(e, 1));
    const double x2 = nx(gv(e, 2)), y2 = ny(gv(e, 2));
    const double x3 = nx(gv(e, 3)), y3 = ny(gv(e, 3));
    const double s = kHalf / tarea * (y1 * x3 - x1 * y3 + (y3 - y1) * x + (x1 - x3) * y);
    const double t = kHalf / tarea * (x1 * y2 - y1 * x2 + (y1 - y2) * x + (x2 - x1) * y);
    if (s < 0.0) return false;
    if (t < 0.0) return false;
    if (1.0 - s - t < 0.0) return false;
    return true;
  }

  // The first triangle in index order that holds (x, y), 0 if none.
  int32_t locate(double x, double y) {
    for (int32_t j = 1; j <= T_; j++)
      if (pto_in_triangle(j, x, y)) return j;
    return 0;
  }

  // ioculvert.f90 checks + cvprep.f90:20-54 (run at dataprepFVT.f90:308-309)
  void culverts() {
    const int32_t n = p_.n_culvert;
    if (n <= 0) return;
    if (!p_.cvptoin || !p_.cvptoout || !p_.ncvtable || !p_.cvhead || !p_.cvq || p_.cv_ld < 1)
      fail(STORM_ERR_ARG, "culverts: missing data");
    const size_t ld = (size_t)p_.cv_ld;
    for (int32_t i = 0; i < n; i++)
      if (p_.ncvtable[i] < 1 || p_.ncvtable[i] > p_.cv_ld)
        fail(STORM_ERR_ARG, "culvert " + std::to_string(i + 1) +
                                ": too few (or too many) entries in the performance curve");
    m_.cvptoin.assign(p_.cvptoin, p_.cvptoin + 3 * (size_t)n);
    m_.ncvtable.assign(p_.ncvtable, p_.ncvtable + n);
    m_.cvhead.assign(p_.cvhead, p_.cvhead + ld * n);
    m_.cvq.assign(p_.cvq, p_.cvq + ld * n);
    m_.cvtrigin.resize(n);
    m_.cvtrigout.resize(n);
    m_.cvrin.resize(2 * (size_t)n);
    for (int32_t i = 0; i < n; i++) {
      const double xi = p_.cvptoin[3 * (size_t)i], yi = p_.cvptoin[3 * (size_t)i + 1];
      const int32_t a = locate(xi, yi);
      if (a == 0) fail(STORM_ERR_MESH, "inlet of culvert " + std::to_string(i + 1) + " not in computational domain");
      m_.cvtrigin[i] = a;
      m_.cvrin[2 * (size_t)i] = xi - m_.tri_xc[a - 1];
      m_.cvrin[2 * (size_t)i + 1] = yi - m_.tri_yc[a - 1];
      const int32_t b = locate(p_.cvptoout[2 * (size_t)i], p_.cvptoout[2 * (size_t)i + 1]);
      if (b == 0) fail(STORM_ERR_MESH, "outlet of culvert " + std::to_string(i + 1) + " not in computational domain");
      m_.cvtrigout[i] = b;
    }
  }

  void fill_view() {
    StormFvtMesh& v = m_.view;
    std::memset(&v, 0, sizeof v);
    v.n_pts = N_;
    v.n_elems = T_;
    v.n_edges = E_;
    v.node_x = m_.node_x.data();
    v.node_y = m_.node_y.data();
    v.tri_vertex = m_.tri_vertex.data();
    v.tri_edge = m_.tri_edge.data();
    v.tri_area = m_.tri_area.data();
    v.tri_perim = m_.tri_perim.data();
    v.tri_xc = m_.tri_xc.data();
    v.tri_yc = m_.tri_yc.data();
    v.edge_p = m_.edge_p.data();
    v.edge_e = m_.edge_e.data();
    v.edge_normal = m_.edge_normal.data();
    v.edge_tang = m_.edge_tang.data();
    v.edge_length = m_.edge_length.data();
    v.rc_x = m_.rc_x.data();
    v.rc_y = m_.rc_y.data();
    v.t2t_ncol = m_.t2t_ncol;
    v.t2t = m_.t2t.data();
    v.lsq_dx = m_.lsq_dx.data();
    v.lsq_dy = m_.lsq_dy.data();
    v.lsq_w = m_.lsq_w.data();
    v.lsq_a = m_.lsq_a.data();
    v.lsq_b = m_.lsq_b.data();
    v.lsq_c = m_.lsq_c.data();
    v.lsq_det = m_.lsq_det.data();
    v.t2t3 = m_.t2t3.data();
    v.n2t_ncol = m_.n2t_ncol;
    v.n2t = m_.n2t.data();
    v.c2v_ncol = m_.c2v_ncol;
    v.c2v_w = m_.c2v_w.data();
    v.csortedz = m_.csortedz.data();
    v.flow_edges1 = (int32_t)m_.flowedg1.size();
    v.flowedg1 = m_.flowedg1.data();
    v.wall_edges1 = (int32_t)m_.walledg1.size();
    v.walledg1 = m_.walledg1.data();
    v.n_bcedges = (int32_t)m_.bcedges.size();
    v.bcedges = m_.bcedges.data();
    v.hbar = m_.hbar.data();
    v.z = m_.z.data();
    v.zvtx = m_.zvtx.data();
    v.cd = m_.cd.data();
    v.n_inflowbdr = p_.n_inflow;
    v.vtype = m_.vtype.data();
    v.qin = m_.qin.data();
    v.bcin_ld = m_.qin_ld + 1;
    v.bcedgesinflow = m_.bcedgesinflow.data();
    v.tsq_ld = m_.tsq_ld;
    v.n_timeserq = m_.n_timeserq.data();
    v.timelocq = m_.timelocq.data();
    v.timeserq = m_.timeserq.data();
    v.n_outflowbdr = p_.n_outflow;
    v.htype = m_.htype.data();
    v.hbc = m_.hbc.data();
    v.bcout_ld = m_.hbc_ld + 1;
    v.bcedgesoutflow = m_.bcedgesoutflow.data();
    v.hbc_ld = m_.hbc_ld;
    v.n_hbc = m_.n_hbc.data();
    v.hbc_nodes = m_.hbc_nodes.data();
    v.tsh_ld = m_.tsh_ld;
    v.n_timeserh = m_.n_timeserh.data();
    v.timeloch = m_.timeloch.data();
    v.timeserh = m_.timeserh.data();
    v.bch_max = m_.bch_max;
    v.wcoef1 = m_.wcoef1.empty() ? nullptr : m_.wcoef1.data();
    v.wcoef2 = m_.wcoef2.empty() ? nullptr : m_.wcoef2.data();
    if (!m_.cvtrigin.empty()) {
      v.n_culvert = p_.n_culvert;
      v.cv_ld = p_.cv_ld;
      v.cvtrigin = m_.cvtrigin.data();
      v.cvtrigout = m_.cvtrigout.data();
      v.cvptoin = m_.cvptoin.data();
      v.cvrin = m_.cvrin.data();
      v.ncvtable = m_.ncvtable.data();
      v.cvhead = m_.cvhead.data();
      v.cvq = m_.cvq.data();
    }
  }
};

}  // namespace
}  // namespace storm

extern "C" int storm_fvt_mesh_build(const StormFvtProblem* prob, StormFvtMesh** out) {
  storm::clear_error();
  if (!prob || !out) return storm::set_error(STORM_ERR_ARG, "storm_fvt_mesh_build: null argument");
  *out = nullptr;
  storm::MeshStorage* st = new (std::nothrow) storm::MeshStorage();
  storm::OwnedMesh* m = new (std::nothrow) storm::OwnedMesh();
  if (!st || !m) {
    delete st;
    delete m;
    return storm::set_error(STORM_ERR_NOMEM, "storm_fvt_mesh_build: out of memory");
  }
  try {
    storm::Builder(*prob, *st).run();
  } catch (const storm::MeshError& e) {
    delete st;
    delete m;
    return storm::set_error(e.code, "storm_fvt_mesh_build: " + e.msg);
  } catch (const std::bad_alloc&) {
    delete st;
    delete m;
    return storm::set_error(STORM_ERR_NOMEM, "storm_fvt_mesh_build: out of memory");
  } catch (const std::exception& e) {
    delete st;
    delete m;
    return storm::set_error(STORM_ERR_MESH, std::string("storm_fvt_mesh_build: ") + e.what());
  }
  m->view = st->view;
  m->store = st;
  static_assert(std::is_standard_layout<storm::OwnedMesh>::value, "OwnedMesh must be standard layout");
  *out = &m->view;
  return STORM_OK;
}

extern "C" void storm_fvt_mesh_free(StormFvtMesh* mesh) {
  if (!mesh) return;
  storm::OwnedMesh* m = reinterpret_cast<storm::OwnedMesh*>(mesh);
  delete m->store;
  delete m;
}
