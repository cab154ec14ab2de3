// structure.cpp -- host side of g2oc_upload: the active set and Hessian index
// mapping of SparseOptimizer::initializeOptimization / buildIndexMapping
// (g2o/core/sparse_optimizer.cpp:175-287) and the block patterns of
// BlockSolver::buildStructure (g2o/core/block_solver.hpp:110-269), laid out
// as device orderings, ranges and gather lists. Runs once per upload; all
// sorts are stable counting / radix sorts, so every list is deterministic.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <numeric>

#include "g2oc_internal.h"

namespace g2oc {

namespace {

int edge_dim(int et) { return et == G2OC_EDGE_SE2 ? 3 : et == G2OC_EDGE_SE3 ? 6 : 2; }
int meas_dim(int et) { return et == G2OC_EDGE_SE2 ? 3 : et == G2OC_EDGE_SE3 ? 12 : 2; }
int pose_dim(int pt) { return pt == G2OC_POSE_SE2 ? 3 : 6; }
int pose_est_dim(int pt) { return pt == G2OC_POSE_SE2 ? 3 : pt == G2OC_POSE_SE3 ? 12 : 7; }

// stable counting sort of items by key in [0, nkeys): returns the order and
// the CSR pointer over keys
void counting_sort(const std::vector<int>& key, int nkeys, std::vector<int>& order, std::vector<int>& ptr) {
  ptr.assign(nkeys + 1, 0);
  for (int k : key) ptr[k + 1]++;
  for (int i = 0; i < nkeys; ++i) ptr[i + 1] += ptr[i];
  order.resize(key.size());
  std::vector<int> pos(ptr.begin(), ptr.end() - 1);
  for (size_t i = 0; i < key.size(); ++i) order[pos[key[i]]++] = (int)i;
}

// stable LSD radix sort of 64-bit keys, returns the permutation
void radix_sort(std::vector<uint64_t>& keys, std::vector<uint32_t>& perm) {
  const size_t n = keys.size();
  perm.resize(n);
  std::iota(perm.begin(), perm.end(), 0u);
  uint64_t maxk = 0;
  for (uint64_t k : keys) maxk = std::max(maxk, k);
  std::vector<uint64_t> k2(n);
  std::vector<uint32_t> p2(n);
  std::vector<size_t> cnt(1 << 16);
  for (int shift = 0; shift < 64 && (maxk >> shift) != 0; shift += 16) {
    std::fill(cnt.begin(), cnt.end(), 0);
    for (size_t i = 0; i < n; ++i) cnt[(keys[i] >> shift) & 0xFFFF]++;
    size_t s = 0;
    for (auto& c : cnt) {
      size_t t = c;
      c = s;
      s += t;
    }
    for (size_t i = 0; i < n; ++i) {
      size_t d = cnt[(keys[i] >> shift) & 0xFFFF]++;
      k2[d] = keys[i];
      p2[d] = perm[i];
    }
    keys.swap(k2);
    perm.swap(p2);
  }
}

}  // namespace

void build_sym_lists(int nb, const std::vector<int32_t>& rc, Structure& s) {
  const int nnzb = (int)(rc.size() / 2);
  s.sys_nb = nb;
  s.sys_nnzb = nnzb;
  // internal order: by (row, col); the column-major pattern lists (col, row)
  std::vector<uint64_t> keys(nnzb);
  for (int k = 0; k < nnzb; ++k) keys[k] = (uint64_t)rc[2 * k] * (uint64_t)nb + (uint64_t)rc[2 * k + 1];
  std::vector<uint32_t> perm;
  radix_sort(keys, perm);
  s.sys_perm.assign(perm.begin(), perm.end());
  s.sys_rptr.assign(nb + 1, 0);
  s.sys_rcol.resize(nnzb);
  s.sys_brow.resize(nnzb);
  s.sys_diag.assign(nb, -1);
  std::vector<int> ckey;
  std::vector<int> cidx;
  for (int k = 0; k < nnzb; ++k) {
    const int p = (int)perm[k];
    const int r = rc[2 * p], c = rc[2 * p + 1];
    s.sys_rptr[r + 1]++;
    s.sys_rcol[k] = c;
    s.sys_brow[k] = r;
    if (r == c) s.sys_diag[r] = k;
    else {
      ckey.push_back(c);
      cidx.push_back(k);
    }
  }
  for (int i = 0; i < nb; ++i) s.sys_rptr[i + 1] += s.sys_rptr[i];
  std::vector<int> order;
  counting_sort(ckey, nb, order, s.sys_cptr);
  s.sys_cblk.resize(order.size());
  for (size_t i = 0; i < order.size(); ++i) s.sys_cblk[i] = cidx[order[i]];
}

static int build_ba(const g2oc_graph* g, Structure& s) {
  const int C = s.C, P = s.P, E = s.E;
  const uint8_t* pf = g->pose_fixed;
  const uint8_t* qf = g->point_fixed;
  std::vector<char> pa(C, 0), qa(P, 0);
  s.act.clear();
  s.act.reserve(E);
  for (int e = 0; e < E; ++e) {
    const int v0 = g->edge_vertex[2 * e], v1 = g->edge_vertex[2 * e + 1];
    const bool f0 = qf && qf[v0], f1 = pf && pf[v1];
    if (f0 && f1) continue;  // allVerticesFixed: not active
    s.act.push_back(e);
    qa[v0] = 1;
    pa[v1] = 1;
  }
  if (s.act.empty()) {
    set_error("graph has no active edge");
    return G2OC_ERR_BAD_GRAPH;
  }
  s.pose_h.assign(C, -1);
  s.point_l.assign(P, -1);
  s.free_pose_of_h.clear();
  s.free_point_of_l.clear();
  for (int i = 0; i < C; ++i)
    if (pa[i] && !(pf && pf[i])) {
      s.pose_h[i] = (int)s.free_pose_of_h.size();
      s.free_pose_of_h.push_back(i);
    }
  for (int i = 0; i < P; ++i)
    if (qa[i] && !(qf && qf[i])) {
      s.point_l[i] = (int)s.free_point_of_l.size();
      s.free_point_of_l.push_back(i);
    }
  s.Cf = (int)s.free_pose_of_h.size();
  s.Pf = (int)s.free_point_of_l.size();
  s.schur = s.Pf > 0;
  const int na = (int)s.act.size();
  // device order: (point fixed?, point, camera, insertion)
  std::vector<int> key(na), ord1, ord2, ptr;
  for (int k = 0; k < na; ++k) key[k] = g->edge_vertex[2 * s.act[k] + 1];
  counting_sort(key, C, ord1, ptr);
  std::vector<int> key2(na);
  for (int k = 0; k < na; ++k) {
    const int v0 = g->edge_vertex[2 * s.act[ord1[k]]];
    const int l = s.point_l[v0];
    key2[k] = l >= 0 ? l : s.Pf + v0;
  }
  counting_sort(key2, s.Pf + P, ord2, ptr);
  s.dev_edge.resize(na);
  s.dev_of_act.resize(na);
  for (int k = 0; k < na; ++k) {
    const int a = ord1[ord2[k]];
    s.dev_edge[k] = s.act[a];
    s.dev_of_act[a] = k;
  }
  s.l_ptr.assign(ptr.begin(), ptr.begin() + s.Pf + 1);
  // Hpl blocks (column-major over (landmark, camera)); duplicates share a block
  s.e_hpl.assign(na, -1);
  s.hb_ptr.assign(s.Pf + 1, 0);
  s.hpl_rc.clear();
  for (int l = 0; l < s.Pf; ++l) {
    int last_cam = -1;
    for (int k = s.l_ptr[l]; k < s.l_ptr[l + 1]; ++k) {
      const int h = s.pose_h[g->edge_vertex[2 * s.dev_edge[k] + 1]];
      if (h < 0) continue;
      if (h != last_cam) {
        s.hpl_rc.push_back(h);
        s.hpl_rc.push_back(l);
        last_cam = h;
      }
      s.e_hpl[k] = (int)(s.hpl_rc.size() / 2) - 1;
    }
    s.hb_ptr[l + 1] = (int)(s.hpl_rc.size() / 2);
  }
  const int nhpl = (int)(s.hpl_rc.size() / 2);
  // camera-major edge list over free cameras
  {
    std::vector<int> ck, idx;
    ck.reserve(na);
    idx.reserve(na);
    for (int k = 0; k < na; ++k) {
      const int h = s.pose_h[g->edge_vertex[2 * s.dev_edge[k] + 1]];
      if (h >= 0) {
        ck.push_back(h);
        idx.push_back(k);
      }
    }
    std::vector<int> ord;
    counting_sort(ck, s.Cf, ord, s.c_ptr);
    s.c_edge.resize(ord.size());
    for (size_t i = 0; i < ord.size(); ++i) s.c_edge[i] = idx[ord[i]];
  }
  {
    std::vector<int> rk(nhpl), ord;
    for (int b = 0; b < nhpl; ++b) rk[b] = s.hpl_rc[2 * b];
    counting_sort(rk, s.Cf, ord, s.hc_ptr);
    s.hc_blk = ord;
  }
  // Hpp: the diagonal blocks only (projection edges join a pose and a point)
  s.hpp_rc.resize(2 * (size_t)s.Cf);
  s.hpp_diag.resize(s.Cf);
  for (int h = 0; h < s.Cf; ++h) {
    s.hpp_rc[2 * h] = h;
    s.hpp_rc[2 * h + 1] = h;
    s.hpp_diag[h] = h;
  }
  // position of each Hpl block in its camera's list
  s.hc_pos.assign(nhpl, 0);
  s.max_blocks_per_cam = 0;
  for (int h = 0; h < s.Cf; ++h) {
    s.max_blocks_per_cam = std::max(s.max_blocks_per_cam, s.hc_ptr[h + 1] - s.hc_ptr[h]);
    for (int p = s.hc_ptr[h]; p < s.hc_ptr[h + 1]; ++p) s.hc_pos[s.hc_blk[p]] = p - s.hc_ptr[h];
  }
  // Schur pattern: Hpp pattern + co-observing pose pairs (block_solver.hpp:229-266),
  // with the pair list of each block in landmark order
  s.schur_rc.clear();
  s.s_pair_ptr.clear();
  s.s_pairs.clear();
  s.s_hpp.clear();
  if (s.schur) {
    int64_t np = 0;
    for (int l = 0; l < s.Pf; ++l) {
      const int64_t m = s.hb_ptr[l + 1] - s.hb_ptr[l];
      np += m * (m + 1) / 2;
    }
    s.num_pairs = np;
    const uint64_t Cf = (uint64_t)s.Cf;
    std::vector<uint64_t> keys;  // row-major: r * Cf + c
    keys.reserve(np + s.Cf);
    std::vector<int32_t> pa2;
    pa2.reserve(2 * np);
    for (int l = 0; l < s.Pf; ++l)
      for (int a = s.hb_ptr[l]; a < s.hb_ptr[l + 1]; ++a)
        for (int b = a; b < s.hb_ptr[l + 1]; ++b) {
          const uint64_t r = (uint64_t)s.hpl_rc[2 * a], c = (uint64_t)s.hpl_rc[2 * b];
          keys.push_back(r * Cf + c);
          pa2.push_back(s.hc_pos[a]);
          pa2.push_back(b);
        }
    for (int h = 0; h < s.Cf; ++h) keys.push_back((uint64_t)h * Cf + h);  // diagonal markers (no pair)
    std::vector<uint32_t> perm;
    radix_sort(keys, perm);
    s.s_pairs.reserve(2 * np);
    std::vector<int32_t> rm_rc;  // internal (row-major) blocks
    s.s_pair_ptr.push_back(0);
    uint64_t prev = ~0ull;
    for (size_t i = 0; i < keys.size(); ++i) {
      if (keys[i] != prev) {
        if (prev != ~0ull) s.s_pair_ptr.push_back((int)(s.s_pairs.size() / 2));
        prev = keys[i];
        const int r = (int)(keys[i] / Cf), c = (int)(keys[i] % Cf);
        rm_rc.push_back(r);
        rm_rc.push_back(c);
        s.s_hpp.push_back(r == c ? s.hpp_diag[r] : -1);
      }
      const uint32_t p = perm[i];
      if (p < (uint32_t)np) {
        s.s_pairs.push_back(pa2[2 * (size_t)p]);
        s.s_pairs.push_back(pa2[2 * (size_t)p + 1]);
      }
    }
    s.s_pair_ptr.push_back((int)(s.s_pairs.size() / 2));
    // column-major pattern (the order of SparseBlockMatrix::blockCols)
    const size_t nS = rm_rc.size() / 2;
    std::vector<uint64_t> ck(nS);
    for (size_t k = 0; k < nS; ++k) ck[k] = (uint64_t)rm_rc[2 * k + 1] * Cf + (uint64_t)rm_rc[2 * k];
    std::vector<uint32_t> cperm;
    radix_sort(ck, cperm);
    s.schur_rc.resize(2 * nS);
    for (size_t i = 0; i < nS; ++i) {
      s.schur_rc[2 * i] = rm_rc[2 * (size_t)cperm[i]];
      s.schur_rc[2 * i + 1] = rm_rc[2 * (size_t)cperm[i] + 1];
    }
    build_sym_lists(s.Cf, s.schur_rc, s);  // internal order = row-major = the order above
  } else {
    build_sym_lists(s.Cf, s.hpp_rc, s);
  }
  return G2OC_OK;
}

static int build_pg(const g2oc_graph* g, Structure& s) {
  const int C = s.C, E = s.E;
  const uint8_t* pf = g->pose_fixed;
  std::vector<char> pa(C, 0);
  s.act.clear();
  for (int e = 0; e < E; ++e) {
    const int v0 = g->edge_vertex[2 * e], v1 = g->edge_vertex[2 * e + 1];
    if (pf && pf[v0] && pf[v1]) continue;
    s.act.push_back(e);
    pa[v0] = 1;
    pa[v1] = 1;
  }
  if (s.act.empty()) {
    set_error("graph has no active edge");
    return G2OC_ERR_BAD_GRAPH;
  }
  s.pose_h.assign(C, -1);
  s.point_l.clear();
  s.free_pose_of_h.clear();
  for (int i = 0; i < C; ++i)
    if (pa[i] && !(pf && pf[i])) {
      s.pose_h[i] = (int)s.free_pose_of_h.size();
      s.free_pose_of_h.push_back(i);
    }
  s.Cf = (int)s.free_pose_of_h.size();
  s.Pf = 0;
  s.schur = false;
  if (s.Cf == 0) {
    set_error("graph has no free vertex");
    return G2OC_ERR_BAD_GRAPH;
  }
  const int na = (int)s.act.size();
  s.dev_edge = s.act;
  s.dev_of_act.resize(na);
  std::iota(s.dev_of_act.begin(), s.dev_of_act.end(), 0);
  const uint64_t Cf = (uint64_t)s.Cf;
  std::vector<uint64_t> keys;
  keys.reserve(s.Cf + na);
  for (int h = 0; h < s.Cf; ++h) keys.push_back((uint64_t)h * Cf + h);
  for (int k = 0; k < na; ++k) {
    int a = s.pose_h[g->edge_vertex[2 * s.act[k]]], b = s.pose_h[g->edge_vertex[2 * s.act[k] + 1]];
    if (a < 0 || b < 0) continue;
    if (a > b) std::swap(a, b);
    keys.push_back((uint64_t)b * Cf + a);
  }
  std::vector<uint32_t> perm;
  radix_sort(keys, perm);
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  s.hpp_rc.resize(2 * keys.size());
  s.hpp_diag.assign(s.Cf, -1);
  for (size_t i = 0; i < keys.size(); ++i) {
    const int c = (int)(keys[i] / Cf), r = (int)(keys[i] % Cf);
    s.hpp_rc[2 * i] = r;
    s.hpp_rc[2 * i + 1] = c;
    if (r == c) s.hpp_diag[r] = (int)i;
  }
  auto find_block = [&](int r, int c) -> int {
    const uint64_t k = (uint64_t)c * Cf + r;
    auto it = std::lower_bound(keys.begin(), keys.end(), k);
    return (int)(it - keys.begin());
  };
  s.pe_blk.assign(3 * (size_t)na, -1);
  s.pe_trans.assign(na, 0);
  std::vector<int> src_key, src_val, bv_key, bv_val;
  for (int k = 0; k < na; ++k) {
    const int a = s.pose_h[g->edge_vertex[2 * s.act[k]]], b = s.pose_h[g->edge_vertex[2 * s.act[k] + 1]];
    if (a >= 0) {
      s.pe_blk[3 * k] = s.hpp_diag[a];
      src_key.push_back(s.hpp_diag[a]);
      src_val.push_back(3 * k + 0);
      bv_key.push_back(a);
      bv_val.push_back(2 * k + 0);
    }
    if (b >= 0) {
      s.pe_blk[3 * k + 1] = s.hpp_diag[b];
      src_key.push_back(s.hpp_diag[b]);
      src_val.push_back(3 * k + 1);
      bv_key.push_back(b);
      bv_val.push_back(2 * k + 1);
    }
    if (a >= 0 && b >= 0) {
      s.pe_trans[k] = a > b;
      const int blk = find_block(std::min(a, b), std::max(a, b));
      s.pe_blk[3 * k + 2] = blk;
      src_key.push_back(blk);
      src_val.push_back(3 * k + 2);
    }
  }
  std::vector<int> ord;
  counting_sort(src_key, (int)keys.size(), ord, s.hb_src_ptr);
  s.hb_src.resize(ord.size());
  for (size_t i = 0; i < ord.size(); ++i) s.hb_src[i] = src_val[ord[i]];
  counting_sort(bv_key, s.Cf, ord, s.bv_src_ptr);
  s.bv_src.resize(ord.size());
  for (size_t i = 0; i < ord.size(); ++i) s.bv_src[i] = bv_val[ord[i]];
  build_sym_lists(s.Cf, s.hpp_rc, s);
  return G2OC_OK;
}

int build_structure(const g2oc_graph* g, Structure& s) {
  if (!g) {
    set_error("graph is NULL");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  const bool ba = g->edge_type == G2OC_EDGE_PROJECT_XYZ2UV;
  if (g->pose_type < 1 || g->pose_type > 3 || g->edge_type < 1 || g->edge_type > 3 ||
      (g->edge_type == G2OC_EDGE_SE2) != (g->pose_type == G2OC_POSE_SE2) ||
      (g->edge_type == G2OC_EDGE_SE3) != (g->pose_type == G2OC_POSE_SE3) ||
      ba != (g->pose_type == G2OC_POSE_SE3EXPMAP)) {
    set_error("unsupported vertex/edge type combination (pose %d, edge %d)", g->pose_type, g->edge_type);
    return G2OC_ERR_BAD_GRAPH;
  }
  if (g->num_poses <= 0 || g->num_points < 0 || g->num_edges <= 0) {
    set_error("empty graph (poses %d, points %d, edges %d)", g->num_poses, g->num_points, g->num_edges);
    return G2OC_ERR_BAD_GRAPH;
  }
  if (!g->pose_estimate || !g->edge_vertex || !g->measurement || !g->information ||
      (ba && g->num_points > 0 && !g->point_estimate)) {
    set_error("graph array is NULL");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  s.pose_type = g->pose_type;
  s.edge_type = g->edge_type;
  s.ba = ba;
  s.C = g->num_poses;
  s.P = ba ? g->num_points : 0;
  s.E = g->num_edges;
  s.pd = pose_dim(s.pose_type);
  s.ped = pose_est_dim(s.pose_type);
  s.D = edge_dim(s.edge_type);
  s.md = meas_dim(s.edge_type);
  const int n0 = ba ? s.P : s.C;
  for (int e = 0; e < s.E; ++e) {
    const int v0 = g->edge_vertex[2 * e], v1 = g->edge_vertex[2 * e + 1];
    if (v0 < 0 || v0 >= n0 || v1 < 0 || v1 >= s.C || (!ba && v0 == v1)) {
      set_error("edge %d has vertex indices (%d, %d) out of range", e, v0, v1);
      return G2OC_ERR_BAD_GRAPH;
    }
  }
  return ba ? build_ba(g, s) : build_pg(g, s);
}

}  // namespace g2oc
