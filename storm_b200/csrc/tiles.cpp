// tiles.cpp -- tiles of the fused stage kernel (k_tile) over the Morton-ordered layout.
//
// A tile owns `tc` consecutive cell slots.  Every interior edge whose smaller cell
// slot is owned belongs to the tile's contiguous edge range (the edge arrays are
// sorted by that slot); an edge whose larger slot is owned and smaller slot lies in an
// earlier tile is one of the tile's back edges, so every edge of every owned cell is
// evaluated in the tile.  The tile also recomputes the gradients of H1, the face
// neighbours of its cells that other tiles own, and reads the state of H2, the cells
// the H1 gradients need.  All indices the kernel follows are local (16-bit).
#include <algorithm>
#include <vector>

#include "storm_internal.h"

namespace storm {

int build_tiles(const HostLayout& L, int tc, TilePlan& P) {
  const int32_t T = L.T, N = L.N, kst = L.kst, ne = L.ne;
  P = TilePlan();
  P.tc = tc;
  P.kst = kst;
  P.ntiles = (T + tc - 1) / tc;
  P.info.assign((size_t)P.ntiles * TI_N, 0);
  P.lt3.assign(3 * (size_t)T, kNoLocal);
  P.lst.assign((size_t)kst * T, kNoLocal);
  P.lfe.assign(3 * (size_t)T, kNoLocal);
  P.eloc.assign(std::max(ne, 1), 0xFFFFFFFFu);
  P.lvt.assign(3 * (size_t)T, kNoLocal);
  P.lwall.assign(3 * (size_t)T, 0xFFFFFFFFu);
  // the tile that writes each node's depth: the tile of its smallest incident cell slot
  std::vector<int32_t> node_owner(N, -1);
  for (int32_t n = 0; n < N; n++) {
    int32_t m = T;
    for (int32_t q = L.n2t_off[n]; q < L.n2t_off[n + 1]; q++) m = std::min(m, L.n2t_cell[q]);
    if (m < T) node_owner[n] = m / tc;
  }
  // local id of a slot (node) in the tile being built (stamp = tile id + 1)
  std::vector<int32_t> stamp(T, 0), loc(T, 0), nstamp(N, 0), nloc(N, 0);
  std::vector<int32_t> list, nodes;
  auto real = [&](int32_t c) { return L.cell_sid.empty() || L.cell_sid[c] >= 0; };
  auto smaller = [&](int32_t e) { return std::min(L.eL[e], L.eR[e]); };
  int32_t er = 0;  // first edge of the current tile's range
  for (int32_t t = 0; t < P.ntiles; t++) {
    const int32_t c0 = t * tc, c1 = std::min(c0 + tc, T), nown = c1 - c0;
    const int32_t tag = t + 1;
    list.clear();
    auto local = [&](int32_t g) -> int32_t { return stamp[g] == tag ? loc[g] : -1; };
    auto add = [&](int32_t g) {
      if (stamp[g] != tag) {
        stamp[g] = tag;
        loc[g] = nown + (int32_t)list.size();
        list.push_back(g);
      }
    };
    int32_t sid = -2;
    for (int32_t c = c0; c < c1; c++) {
      stamp[c] = tag;
      loc[c] = c - c0;
      const int32_t s = L.cell_sid.empty() ? 0 : L.cell_sid[c];
      if (s >= 0) sid = (sid == -2 || sid == s) ? s : -1;
    }
    // H1: face neighbours of owned cells
    for (int32_t c = c0; c < c1; c++)
      for (int j = 0; j < 3; j++) {
        const int32_t n = L.t2t3[(size_t)j * T + c];
        if (n >= 0) add(n);
      }
    const int32_t n1 = (int32_t)list.size();
    // H2: stencil and face neighbours of owned and H1 cells
    auto add_nb = [&](int32_t c) {
      for (int k = 0; k < L.nst[c]; k++) add(L.st_id[(size_t)k * T + c]);
      for (int j = 0; j < 3; j++) {
        const int32_t n = L.t2t3[(size_t)j * T + c];
        if (n >= 0) add(n);
      }
    };
    for (int32_t c = c0; c < c1; c++) add_nb(c);
    for (int32_t i = 0; i < n1; i++) add_nb(list[i]);
    const int32_t n2 = (int32_t)list.size() - n1;
    // nodes: vertices of the owned and H1 cells; H3: their other incident cells
    nodes.clear();
    auto add_node = [&](int32_t n) {
      if (nstamp[n] != tag) {
        nstamp[n] = tag;
        nloc[n] = (int32_t)nodes.size();
        nodes.push_back(n);
      }
    };
    for (int32_t c = c0; c < c1; c++)
      if (real(c))
        for (int j = 0; j < 3; j++) add_node(L.vert[(size_t)j * T + c]);
    for (int32_t i = 0; i < n1; i++)
      for (int j = 0; j < 3; j++) add_node(L.vert[(size_t)j * T + list[i]]);
    for (int32_t n : nodes)
      for (int32_t q = L.n2t_off[n]; q < L.n2t_off[n + 1]; q++) add(L.n2t_cell[q]);
    const int32_t n3 = (int32_t)list.size() - n1 - n2;
    if (nown + n1 + n2 + n3 >= kNoLocal || (int32_t)nodes.size() >= kNoLocal) return -1;
    const int32_t noff = (int32_t)P.tnode.size();
    for (int32_t n : nodes) {
      P.tnode.push_back(n);
      P.tn_own.push_back(node_owner[n] == t);
      P.tn_start.push_back((int32_t)P.tn_cells.size());
      for (int32_t q = L.n2t_off[n]; q < L.n2t_off[n + 1]; q++) P.tn_cells.push_back((uint16_t)local(L.n2t_cell[q]));
    }
    for (int32_t c = c0; c < c1; c++) {
      if (!real(c)) continue;
      for (int j = 0; j < 3; j++) {
        const size_t q = (size_t)j * T + c;
        P.lvt[q] = (uint16_t)nloc[L.vert[q]];
        if ((L.fkind[q] & 7) == FACE_WALL) {
          const int32_t w = L.fref[q];
          if (nstamp[L.wall_p1[w]] != tag || nstamp[L.wall_p2[w]] != tag) return -1;
          P.lwall[q] = (uint32_t)nloc[L.wall_p1[w]] | ((uint32_t)nloc[L.wall_p2[w]] << 16);
        }
      }
    }
    // local topology of owned cells and of H1
    auto t3_of = [&](int32_t c, int j) -> uint16_t {
      const int32_t n = L.t2t3[(size_t)j * T + c];
      return n < 0 ? kNoLocal : (uint16_t)local(n);
    };
    for (int32_t c = c0; c < c1; c++) {
      for (int j = 0; j < 3; j++) P.lt3[(size_t)j * T + c] = t3_of(c, j);
      for (int k = 0; k < L.nst[c]; k++) P.lst[(size_t)k * T + c] = (uint16_t)local(L.st_id[(size_t)k * T + c]);
    }
    const size_t h1o = P.h1_t3.size() / 3;
    P.h1_t3.resize(3 * (h1o + n1), kNoLocal);
    P.h1_vt.resize(3 * (h1o + n1), kNoLocal);
    P.h1_st.resize((size_t)kst * (h1o + n1), kNoLocal);
    for (int32_t i = 0; i < n1; i++) {
      const int32_t c = list[i];
      for (int j = 0; j < 3; j++) P.h1_t3[3 * (h1o + i) + j] = t3_of(c, j);
      for (int j = 0; j < 3; j++) P.h1_vt[3 * (h1o + i) + j] = (uint16_t)nloc[L.vert[(size_t)j * T + c]];
      for (int k = 0; k < L.nst[c]; k++)
        P.h1_st[(size_t)kst * (h1o + i) + k] = (uint16_t)local(L.st_id[(size_t)k * T + c]);
    }
    // edges: the range [er, er_end) whose smaller slot is owned, then back edges
    while (er < ne && smaller(er) < c0) er++;
    int32_t er_end = er;
    while (er_end < ne && smaller(er_end) < c1) er_end++;
    const int32_t nr = er_end - er;
    for (int32_t e = er; e < er_end; e++) {
      const int32_t a = local(L.eL[e]), b = local(L.eR[e]);
      if (a < 0 || b < 0) return -1;  // an edge cell outside the tile's H1: inconsistent tables
      P.eloc[e] = (uint32_t)a | ((uint32_t)b << 16);
    }
    const int32_t boff = (int32_t)P.be.size();
    for (int32_t c = c0; c < c1; c++)
      for (int j = 0; j < 3; j++) {
        const size_t q = (size_t)j * T + c;
        const int kind = L.fkind[q] & 7;
        if (kind != FACE_LEFT && kind != FACE_RIGHT) continue;
        const int32_t e = L.fref[q];
        if (smaller(e) >= c0) {
          P.lfe[q] = (uint16_t)(e - er);
        } else {
          P.lfe[q] = (uint16_t)(nr + (int32_t)P.be.size() - boff);
          P.be.push_back(e);
          const int32_t a = local(L.eL[e]), b = local(L.eR[e]);
          if (a < 0 || b < 0) return -1;
          P.beloc.push_back((uint32_t)a | ((uint32_t)b << 16));
        }
      }
    const int32_t nb = (int32_t)P.be.size() - boff;
    if (nr + nb >= kNoLocal) return -1;
    int32_t* I = &P.info[(size_t)t * TI_N];
    I[TI_NOWN] = nown;
    I[TI_N1] = n1;
    I[TI_N2] = n2;
    I[TI_HOFF] = (int32_t)P.halo.size();
    I[TI_H1OFF] = (int32_t)h1o;
    I[TI_ER0] = er;
    I[TI_NR] = nr;
    I[TI_NB] = nb;
    I[TI_BOFF] = boff;
    I[TI_SID] = sid < 0 ? -1 : sid;
    I[TI_N3] = n3;
    I[TI_NOFF] = noff;
    I[TI_NN] = (int32_t)nodes.size();
    P.halo.insert(P.halo.end(), list.begin(), list.end());
    P.ns_max = std::max(P.ns_max, nown + n1 + n2 + n3);
    P.nn_max = std::max(P.nn_max, (int32_t)nodes.size());
    P.ng_max = std::max(P.ng_max, nown + n1);
    P.ne_max = std::max(P.ne_max, nr + nb);
    er = er_end;
  }
  if (P.h1_t3.empty()) {
    P.h1_t3.assign(3, kNoLocal);
    P.h1_vt.assign(3, kNoLocal);
    P.h1_st.assign(std::max(kst, 1), kNoLocal);
  }
  if (P.tnode.empty()) {
    P.tnode.push_back(0);
    P.tn_own.push_back(0);
    P.tn_start.push_back(0);
  }
  if (P.tn_cells.empty()) P.tn_cells.push_back(0);
  // vertices of the cells with an open-boundary face (their depths are needed by the
  // boundary cells' gradients and walls on the side stream, before the tiles finish)
  {
    std::vector<uint8_t> mark(N, 0);
    for (int32_t c : L.bc_cells)
      for (int j = 0; j < 3; j++) mark[L.vert[(size_t)j * T + c]] = 1;
    for (int32_t n = 0; n < N; n++)
      if (mark[n]) P.bc_nodes.push_back(n);
    if (P.bc_nodes.empty()) P.bc_nodes.push_back(0);
  }
  if (P.be.empty()) {
    P.be.push_back(0);
    P.beloc.push_back(0);
  }
  if (P.halo.empty()) P.halo.push_back(0);
  return 0;
}

}  // namespace storm

namespace storm {

// Consistency of a tile plan against the layout it was built from (host only): every
// local id of every tile maps back to the cell or edge the layout names, stays below
// the tile's counts, and every interior edge is the range edge of exactly one tile.
// Returns 0 or the number of the first failed check.
int check_tiles(const HostLayout& L, const TilePlan& P) {
  const int32_t T = L.T;
  std::vector<int32_t> range_count(std::max(L.ne, 1), 0), node_owner_count(L.N, 0);
  for (int32_t t = 0; t < P.ntiles; t++) {
    const int32_t* I = &P.info[(size_t)t * TI_N];
    const int32_t nown = I[TI_NOWN], n1 = I[TI_N1], n2 = I[TI_N2], hoff = I[TI_HOFF], h1off = I[TI_H1OFF];
    const int32_t er0 = I[TI_ER0], nr = I[TI_NR], nb = I[TI_NB], boff = I[TI_BOFF];
    const int32_t n3 = I[TI_N3], noff = I[TI_NOFF], nn = I[TI_NN];
    const int32_t c0 = t * P.tc, nS = nown + n1 + n2 + n3, nG = nown + n1;
    if (nS > P.ns_max || nG > P.ng_max || nr + nb > P.ne_max) return 1;
    auto glob = [&](int32_t l) -> int32_t { return l < nown ? c0 + l : P.halo[hoff + l - nown]; };
    auto same_cell = [&](uint16_t l, int32_t g) {
      if (g < 0) return l == kNoLocal;
      return l != kNoLocal && (int32_t)l < nS && glob(l) == g;
    };
    for (int32_t l = nG; l < nS; l++) {
      const int32_t g = glob(l);
      if (g < 0 || g >= T || (L.cell_sid.size() && L.cell_sid[g] < 0)) return 2;
    }
    for (int32_t l = 0; l < nG; l++) {
      const int32_t g = glob(l);
      if (g < 0 || g >= T) return 2;
      if (L.cell_sid.size() && L.cell_sid[g] < 0) {
        if (l >= nown) return 3;  // a halo cell is never padding
        continue;
      }
      for (int j = 0; j < 3; j++) {
        const uint16_t x = l < nown ? P.lt3[(size_t)j * T + g] : P.h1_t3[3 * (size_t)(h1off + l - nown) + j];
        if (!same_cell(x, L.t2t3[(size_t)j * T + g])) return 4;
      }
      for (int k = 0; k < L.nst[g]; k++) {
        const uint16_t x = l < nown ? P.lst[(size_t)k * T + g] : P.h1_st[(size_t)P.kst * (h1off + l - nown) + k];
        if (!same_cell(x, L.st_id[(size_t)k * T + g])) return 5;
      }
    }
    for (int32_t i = 0; i < nr + nb; i++) {
      const int32_t e = i < nr ? er0 + i : P.be[boff + i - nr];
      const uint32_t lo = i < nr ? P.eloc[e] : P.beloc[boff + i - nr];
      const int32_t a = lo & 0xFFFF, b = lo >> 16;
      if (e < 0 || e >= L.ne || a >= nG || b >= nG) return 6;
      if (glob(a) != L.eL[e] || glob(b) != L.eR[e]) return 7;
      if (a >= nown && b >= nown) return 8;  // every tile edge has an owned cell
      if (i < nr) range_count[e]++;
    }
    // nodes: incident cells in n2t order, vertices and wall ends of the cells
    if (nn > P.nn_max) return 12;
    for (int32_t i = 0; i < nn; i++) {
      const int32_t n = P.tnode[noff + i];
      if (n < 0 || n >= L.N) return 13;
      if (P.tn_own[noff + i]) node_owner_count[n]++;
      for (int32_t q = L.n2t_off[n]; q < L.n2t_off[n + 1]; q++) {
        const uint16_t x = P.tn_cells[P.tn_start[noff + i] + (q - L.n2t_off[n])];
        if (!same_cell(x, L.n2t_cell[q])) return 14;
      }
    }
    for (int32_t l = 0; l < nG; l++) {
      const int32_t g = glob(l);
      if (L.cell_sid.size() && L.cell_sid[g] < 0) continue;
      for (int j = 0; j < 3; j++) {
        const uint16_t x = l < nown ? P.lvt[(size_t)j * T + g] : P.h1_vt[3 * (size_t)(h1off + l - nown) + j];
        if (x >= nn || P.tnode[noff + x] != L.vert[(size_t)j * T + g]) return 15;
      }
    }
    for (int32_t c = c0; c < c0 + nown; c++)
      for (int j = 0; j < 3; j++) {
        const size_t q = (size_t)j * T + c;
        if ((L.fkind[q] & 7) != FACE_WALL || (L.cell_sid.size() && L.cell_sid[c] < 0)) continue;
        const uint32_t lw = P.lwall[q];
        const int32_t a = lw & 0xFFFF, b = lw >> 16, w = L.fref[q];
        if (a >= nn || b >= nn || P.tnode[noff + a] != L.wall_p1[w] || P.tnode[noff + b] != L.wall_p2[w]) return 16;
      }
    for (int32_t c = c0; c < c0 + nown; c++)
      for (int j = 0; j < 3; j++) {
        const size_t q = (size_t)j * T + c;
        const int kind = L.fkind[q] & 7;
        if (kind != FACE_LEFT && kind != FACE_RIGHT) continue;
        const uint16_t le = P.lfe[q];
        if (le == kNoLocal || le >= nr + nb) return 9;
        const int32_t e = le < nr ? er0 + le : P.be[boff + le - nr];
        if (e != L.fref[q]) return 10;
      }
  }
  for (int32_t e = 0; e < L.ne; e++)
    if (range_count[e] != 1) return 11;
  for (int32_t n = 0; n < L.N; n++)  // every node with incident cells is written by one tile
    if (node_owner_count[n] != (L.n2t_off[n + 1] > L.n2t_off[n] ? 1 : 0)) return 17;
  return 0;
}

}  // namespace storm
