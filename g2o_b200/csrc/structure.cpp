// structure.cpp -- host side of g2oc_upload: the active set and Hessian index
// mapping of SparseOptimizer::initializeOptimization / buildIndexMapping
// (g2o/core/sparse_optimizer.cpp:175-287) and the block patterns of
// BlockSolver::buildStructure (g2o/core/block_solver.hpp:110-269), laid out
// as device orderings, ranges and gather lists. Runs once per upload; all
// sorts are stable counting / radix sorts, so every list is deterministic.
#include <algorithm>
#include <array>
#include <cstdarg>
#include <cstdio>
#include <numeric>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "g2oc_internal.h"

namespace g2oc {

namespace {

int edge_dim(int et) {
  return (et == G2OC_EDGE_SE2 || et == G2OC_EDGE_STEREO_SE3_PROJECT_XYZ) ? 3
         : (et == G2OC_EDGE_SE3 || et == G2OC_EDGE_SE3_EXPMAP)          ? 6
                                                                          : 2;
}
int meas_dim(int et) {
  return (et == G2OC_EDGE_SE2 || et == G2OC_EDGE_STEREO_SE3_PROJECT_XYZ) ? 3
         : et == G2OC_EDGE_SE3                                           ? 12
         : et == G2OC_EDGE_SE3_EXPMAP                                    ? 7
                                                                         : 2;
}
int pose_dim(int pt) { return pt == G2OC_POSE_SE2 ? 3 : pt == G2OC_POSE_BAL_CAMERA ? 9 : 6; }
int pose_est_dim(int pt) {
  return pt == G2OC_POSE_SE2 ? 3 : pt == G2OC_POSE_SE3 ? 12 : pt == G2OC_POSE_BAL_CAMERA ? 9 : 7;
}

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

// Dense tiles of kTileBlocks x kTileBlocks blocks for a nearly full matrix:
// the upper tiles (I <= J) holding at least one block, diagonal tiles stored
// with both triangles. Chosen when the tiles hold at most 1.25x the blocks of
// the pattern (plus the lower halves of the diagonal tiles).
static void build_tiles(int nb, Structure& s) {
  s.tile_ok = false;
  s.tile_ij.clear();
  s.tile_off.clear();
  const int nnzb = s.sys_nnzb;
  if (nb < 2 * kTileBlocks || s.pd != 6) return;  // the tiles hold 6 x 6 blocks
  const int nbt = (nb + kTileBlocks - 1) / kTileBlocks;
  std::vector<int> id((size_t)nbt * nbt, -1);
  for (int k = 0; k < nnzb; ++k) {
    const int I = s.sys_brow[k] / kTileBlocks, J = s.sys_rcol[k] / kTileBlocks;
    id[(size_t)I * nbt + J] = 0;
  }
  if (s.shard_world > 1)  // every rank: the whole upper triangle
    for (int I = 0; I < nbt; ++I)
      for (int J = I; J < nbt; ++J) id[(size_t)I * nbt + J] = 0;
  int nt = 0;
  for (size_t q = 0; q < id.size(); ++q)
    if (id[q] == 0) id[q] = nt++;
  const double stored = (double)nt * kTileBlocks * kTileBlocks;
  const double allowed = 1.25 * nnzb + (double)nbt * kTileBlocks * kTileBlocks / 2;
  if ((long long)nt * kTileBlocks * kTileBlocks * 36 >= (1LL << 31)) return;
  if (stored > allowed && s.shard_world <= 1) return;
  s.tile_ok = true;
  s.tile_ij.resize(2 * (size_t)nt);
  for (int I = 0; I < nbt; ++I)
    for (int J = I; J < nbt; ++J) {
      const int t = id[(size_t)I * nbt + J];
      if (t < 0) continue;
      s.tile_ij[2 * (size_t)t] = I;
      s.tile_ij[2 * (size_t)t + 1] = J;
    }
  constexpr int TS = kTileBlocks * 6;  // scalar rows of a tile (6x6 blocks)
  s.tile_off.resize(nnzb);
  for (int k = 0; k < nnzb; ++k) {
    const int r = s.sys_brow[k], c = s.sys_rcol[k];
    const int t = id[(size_t)(r / kTileBlocks) * nbt + c / kTileBlocks];
    s.tile_off[k] = t * TS * TS + (r % kTileBlocks) * 6 * TS + (c % kTileBlocks) * 6;
  }
}

void build_sym_lists(int nb, const std::vector<int32_t>& rc, Structure& s) {
  const int nnzb = (int)(rc.size() / 2);
  s.sys_nb = nb;
  s.sys_nnzb = nnzb;
  // internal order = (row, col): a stable counting sort of the column-major
  // list by row keeps the columns ascending inside each row
  std::vector<int> rkey(nnzb), order;
  for (int k = 0; k < nnzb; ++k) rkey[k] = rc[2 * k];
  counting_sort(rkey, nb, order, s.sys_rptr);
  s.sys_perm.assign(order.begin(), order.end());
  s.sys_rcol.resize(nnzb);
  s.sys_brow.resize(nnzb);
  s.sys_diag.assign(nb, -1);
  std::vector<int> ckey;
  std::vector<int> cidx;
  ckey.reserve(nnzb);
  cidx.reserve(nnzb);
  for (int k = 0; k < nnzb; ++k) {
    const int p = order[k];
    const int r = rc[2 * p], c = rc[2 * p + 1];
    s.sys_rcol[k] = c;
    s.sys_brow[k] = r;
    if (r == c) s.sys_diag[r] = k;
    else {
      ckey.push_back(c);
      cidx.push_back(k);
    }
  }
  std::vector<int> corder;
  counting_sort(ckey, nb, corder, s.sys_cptr);
  s.sys_cblk.resize(corder.size());
  for (size_t i = 0; i < corder.size(); ++i) s.sys_cblk[i] = cidx[corder[i]];
  // row chunks of at most kSysChunk blocks (one warp each in the persistent PCG)
  s.sys_chunk_ptr.assign(nb + 1, 0);
  for (int r = 0; r < nb; ++r)
    s.sys_chunk_ptr[r + 1] = s.sys_chunk_ptr[r] + (s.sys_rptr[r + 1] - s.sys_rptr[r] + kSysChunk - 1) / kSysChunk;
  s.sys_chunk_row.resize(s.sys_chunk_ptr[nb]);
  for (int r = 0; r < nb; ++r)
    for (int ch = s.sys_chunk_ptr[r]; ch < s.sys_chunk_ptr[r + 1]; ++ch) s.sys_chunk_row[ch] = r;
  build_tiles(nb, s);
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
  // the pose edge set (EdgeSE3Expmap between cameras): active unless both fixed
  s.pact.clear();
  for (int e = 0; e < g->num_pose_edges; ++e) {
    const int v0 = g->pose_edge_vertex[2 * e], v1 = g->pose_edge_vertex[2 * e + 1];
    if (pf && pf[v0] && pf[v1]) continue;
    s.pact.push_back(e);
    pa[v0] = 1;
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
  if (s.shard_world > 1) std::fill(pa.begin(), pa.end(), (char)1);
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
  // device order: (point fixed?, point, camera, insertion). Graphs built
  // point by point with ascending cameras (as g2o's ba_demo does) are already
  // in that order; detect it and skip the sorts.
  std::vector<int> key2(na), ptr;
  for (int k = 0; k < na; ++k) {
    const int v0 = g->edge_vertex[2 * s.act[k]];
    const int l = s.point_l[v0];
    key2[k] = l >= 0 ? l : s.Pf + v0;
  }
  bool sorted = true;
  for (int k = 1; k < na && sorted; ++k) {
    if (key2[k] < key2[k - 1]) sorted = false;
    else if (key2[k] == key2[k - 1] && g->edge_vertex[2 * s.act[k] + 1] < g->edge_vertex[2 * s.act[k - 1] + 1])
      sorted = false;
  }
  s.dev_edge.resize(na);
  s.dev_of_act.resize(na);
  if (sorted) {
    ptr.assign(s.Pf + P + 1, 0);
    for (int k = 0; k < na; ++k) ptr[key2[k] + 1]++;
    for (int i = 0; i < s.Pf + P; ++i) ptr[i + 1] += ptr[i];
    for (int k = 0; k < na; ++k) {
      s.dev_edge[k] = s.act[k];
      s.dev_of_act[k] = k;
    }
  } else {
    std::vector<int> key(na), ord1, ord2;
    for (int k = 0; k < na; ++k) key[k] = g->edge_vertex[2 * s.act[k] + 1];
    counting_sort(key, C, ord1, ptr);
    for (int k = 0; k < na; ++k) {
      const int v0 = g->edge_vertex[2 * s.act[ord1[k]]];
      const int l = s.point_l[v0];
      key2[k] = l >= 0 ? l : s.Pf + v0;
    }
    counting_sort(key2, s.Pf + P, ord2, ptr);
    for (int k = 0; k < na; ++k) {
      const int a = ord1[ord2[k]];
      s.dev_edge[k] = s.act[a];
      s.dev_of_act[a] = k;
    }
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
  // warp chunks for the edge-parallel landmark pass
  {
    bool ok = true;
    for (int l = 0; l < s.Pf && ok; ++l) {
      if (s.l_ptr[l + 1] - s.l_ptr[l] > 32) ok = false;
      for (int k = s.l_ptr[l] + 1; k < s.l_ptr[l + 1] && ok; ++k)
        if (s.e_hpl[k] >= 0 && s.e_hpl[k] == s.e_hpl[k - 1]) ok = false;
    }
    // (the edge-parallel passes are written for the two-row projection
    // edges, BAL's included; the stereo edge's landmarks take the
    // thread-per-landmark ones)
    s.lm_warp_ok = ok && s.Pf > 0 && s.D == 2;
    s.lm_chunk_ptr.clear();
    s.e_lm.clear();
    if (s.lm_warp_ok) {
      s.e_lm.resize(s.l_ptr[s.Pf]);
      s.lm_chunk_ptr.push_back(0);
      int start = 0;
      for (int l = 0; l < s.Pf; ++l) {
        for (int k = s.l_ptr[l]; k < s.l_ptr[l + 1]; ++k) s.e_lm[k] = l;
        if (s.l_ptr[l + 1] - start > 32) {
          s.lm_chunk_ptr.push_back(s.l_ptr[l]);
          start = s.l_ptr[l];
        }
      }
      s.lm_chunk_ptr.push_back(s.l_ptr[s.Pf]);
    }
  }
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
  // Hpp: the diagonal blocks (projection edges join a pose and a point),
  // stored at index h, and the pose edges' pose-pose blocks (row < column),
  // stored after them at Cf + p in (row, column) order; hpp_rc lists all of
  // them column-major (the order of SparseBlockMatrix::blockCols) and
  // hpp_store maps that order to storage
  std::vector<std::pair<int, int>> pp;  // (row, column) of the pose-pose blocks
  for (int e : s.pact) {
    int a = s.pose_h[g->pose_edge_vertex[2 * e]], b = s.pose_h[g->pose_edge_vertex[2 * e + 1]];
    if (a < 0 || b < 0) continue;
    if (a > b) std::swap(a, b);
    pp.push_back({a, b});
  }
  std::sort(pp.begin(), pp.end());
  pp.erase(std::unique(pp.begin(), pp.end()), pp.end());
  s.npp = (int)pp.size();
  s.hpp_diag.resize(s.Cf);
  for (int h = 0; h < s.Cf; ++h) s.hpp_diag[h] = h;
  {
    std::vector<std::array<int, 3>> cm;  // (column, row, storage)
    cm.reserve(s.Cf + pp.size());
    for (int h = 0; h < s.Cf; ++h) cm.push_back({h, h, h});
    for (size_t q = 0; q < pp.size(); ++q) cm.push_back({pp[q].second, pp[q].first, s.Cf + (int)q});
    std::sort(cm.begin(), cm.end());
    s.hpp_rc.resize(2 * cm.size());
    s.hpp_store.resize(cm.size());
    for (size_t i = 0; i < cm.size(); ++i) {
      s.hpp_rc[2 * i] = cm[i][1];
      s.hpp_rc[2 * i + 1] = cm[i][0];
      s.hpp_store[i] = cm[i][2];
    }
  }
  {  // per camera its pose-pose blocks (the Hpp product of Dogleg / g2oc_multiply_hessian)
    std::vector<std::vector<std::array<int, 3>>> per(s.Cf);
    for (size_t q = 0; q < pp.size(); ++q) {
      per[pp[q].first].push_back({s.Cf + (int)q, pp[q].second, 0});
      per[pp[q].second].push_back({s.Cf + (int)q, pp[q].first, 1});
    }
    s.pp_ptr.assign(s.Cf + 1, 0);
    s.pp_ent.clear();
    for (int h = 0; h < s.Cf; ++h) {
      for (const auto& en : per[h]) s.pp_ent.insert(s.pp_ent.end(), {en[0], en[1], en[2], 0});
      s.pp_ptr[h + 1] = (int)(s.pp_ent.size() / 4);
    }
  }
  auto pair_store = [&](int r, int c) -> int {  // storage index of pose-pose block (r < c), or -1
    auto it = std::lower_bound(pp.begin(), pp.end(), std::make_pair(r, c));
    return (it != pp.end() && *it == std::make_pair(r, c)) ? s.Cf + (int)(it - pp.begin()) : -1;
  };
  // the pose edges' contributions (pg_linearize slots: edge * 3 + {0: (v0,v0),
  // 1: (v1,v1), 2: (v0,v1)}; gradient edge * 2 + {0, 1}) routed to the
  // storage blocks and the cameras, in edge order
  {
    const int npa = (int)s.pact.size();
    s.pe_trans.assign(npa, 0);
    std::vector<int> src_key, src_val, bv_key, bv_val;
    for (int k = 0; k < npa; ++k) {
      const int e = s.pact[k];
      const int a = s.pose_h[g->pose_edge_vertex[2 * e]], b = s.pose_h[g->pose_edge_vertex[2 * e + 1]];
      if (a >= 0) {
        src_key.push_back(a);
        src_val.push_back(3 * k + 0);
        bv_key.push_back(a);
        bv_val.push_back(2 * k + 0);
      }
      if (b >= 0) {
        src_key.push_back(b);
        src_val.push_back(3 * k + 1);
        bv_key.push_back(b);
        bv_val.push_back(2 * k + 1);
      }
      if (a >= 0 && b >= 0) {
        s.pe_trans[k] = a > b;
        src_key.push_back(pair_store(std::min(a, b), std::max(a, b)));
        src_val.push_back(3 * k + 2);
      }
    }
    std::vector<int> ord;
    counting_sort(src_key, s.Cf + s.npp, ord, s.hb_src_ptr);
    s.hb_src.resize(ord.size());
    for (size_t i = 0; i < ord.size(); ++i) s.hb_src[i] = src_val[ord[i]];
    counting_sort(bv_key, s.Cf, ord, s.bv_src_ptr);
    s.bv_src.resize(ord.size());
    for (size_t i = 0; i < ord.size(); ++i) s.bv_src[i] = bv_val[ord[i]];
  }
  // position of each Hpl block in its camera's list
  s.hc_pos.assign(nhpl, 0);
  s.max_blocks_per_cam = 0;
  for (int h = 0; h < s.Cf; ++h) {
    s.max_blocks_per_cam = std::max(s.max_blocks_per_cam, s.hc_ptr[h + 1] - s.hc_ptr[h]);
    for (int p = s.hc_ptr[h]; p < s.hc_ptr[h + 1]; ++p) s.hc_pos[s.hc_blk[p]] = p - s.hc_ptr[h];
  }
  // Schur pattern: Hpp pattern + co-observing pose pairs (block_solver.hpp:229-266),
  // with the pair list of each off-diagonal block in landmark order. The
  // diagonal block of each camera is formed from the camera's own Hpl blocks
  // (no pair list). Rows are bucketed by a counting sort (landmark order kept),
  // then each row is sorted by column with a stable counting sort.
  s.schur_rc.clear();
  s.s_pair_ptr.clear();
  s.s_pairs.clear();
  s.s_hpp.clear();
  s.num_pairs = 0;
  if (s.schur) {
    const int Cf = s.Cf;
    std::vector<int64_t> rcount(Cf + 1, 0);
    for (int l = 0; l < s.Pf; ++l)
      for (int a = s.hb_ptr[l]; a < s.hb_ptr[l + 1]; ++a) rcount[s.hpl_rc[2 * a] + 1] += s.hb_ptr[l + 1] - a - 1;
    for (int h = 0; h < Cf; ++h) rcount[h + 1] += rcount[h];
    const int64_t np = rcount[Cf];
    s.num_pairs = np;
    std::vector<int32_t> pc(np), pa(np), pb(np);  // column, a (position in row camera list), b
    {
      // parallel bucketing: landmark chunks in order, each chunk writes its
      // own slice of every row, so each row stays in landmark order
#ifdef _OPENMP
      const int nt = std::max(1, std::min(omp_get_max_threads(), 32));
#else
      const int nt = 1;
#endif
      std::vector<int64_t> cnt((size_t)nt * Cf, 0);
      auto chunk = [&](int t, int& l0, int& l1) {
        l0 = (int)((int64_t)s.Pf * t / nt);
        l1 = (int)((int64_t)s.Pf * (t + 1) / nt);
      };
#pragma omp parallel for num_threads(nt)
      for (int t = 0; t < nt; ++t) {
        int l0, l1;
        chunk(t, l0, l1);
        int64_t* ct = cnt.data() + (size_t)t * Cf;
        for (int l = l0; l < l1; ++l)
          for (int a = s.hb_ptr[l]; a < s.hb_ptr[l + 1]; ++a) ct[s.hpl_rc[2 * a]] += s.hb_ptr[l + 1] - a - 1;
      }
      std::vector<int64_t> start((size_t)nt * Cf);
      for (int r = 0; r < Cf; ++r) {
        int64_t o = rcount[r];
        for (int t = 0; t < nt; ++t) {
          start[(size_t)t * Cf + r] = o;
          o += cnt[(size_t)t * Cf + r];
        }
      }
#pragma omp parallel for num_threads(nt)
      for (int t = 0; t < nt; ++t) {
        int l0, l1;
        chunk(t, l0, l1);
        int64_t* pos = start.data() + (size_t)t * Cf;
        for (int l = l0; l < l1; ++l)
          for (int a = s.hb_ptr[l]; a < s.hb_ptr[l + 1]; ++a) {
            const int r = s.hpl_rc[2 * a];
            for (int b = a + 1; b < s.hb_ptr[l + 1]; ++b) {
              const int64_t q = pos[r]++;
              pc[q] = s.hpl_rc[2 * b];
              pa[q] = s.hc_pos[a];
              pb[q] = b;
            }
          }
      }
    }
    // per row: stable counting sort by column; blocks = diagonal + distinct columns
    std::vector<std::vector<int32_t>> row_cols(Cf);
    std::vector<std::vector<int32_t>> row_cnt(Cf);
    std::vector<int32_t> sp(2 * np);
#pragma omp parallel for schedule(dynamic, 8)
    for (int r = 0; r < Cf; ++r) {
      const int64_t q0 = rcount[r], q1 = rcount[r + 1];
      std::vector<int32_t> cnt(Cf - r + 1, 0);
      for (int64_t q = q0; q < q1; ++q) cnt[pc[q] - r + 1]++;
      std::vector<int32_t>& cols = row_cols[r];
      std::vector<int32_t>& cc = row_cnt[r];
      for (int c = r + 1; c < Cf; ++c)
        if (cnt[c - r + 1]) {
          cols.push_back(c);
          cc.push_back(cnt[c - r + 1]);
        }
      for (int c = 1; c <= Cf - r; ++c) cnt[c] += cnt[c - 1];
      for (int64_t q = q0; q < q1; ++q) {
        const int64_t d = q0 + cnt[pc[q] - r]++;
        sp[2 * d] = pa[q];
        sp[2 * d + 1] = pb[q];
      }
    }
    s.s_pairs.swap(sp);
    // the pose-pose blocks join the pattern (no co-observation pair of their own)
    for (const auto& q : pp) {
      std::vector<int32_t>& cols = row_cols[q.first];
      std::vector<int32_t>& cc = row_cnt[q.first];
      auto it = std::lower_bound(cols.begin(), cols.end(), q.second);
      if (it == cols.end() || *it != q.second) {
        const size_t at = (size_t)(it - cols.begin());
        cols.insert(it, q.second);
        cc.insert(cc.begin() + at, 0);
      }
    }
    // internal (row-major) blocks: per row the diagonal, then the columns
    std::vector<int32_t> rm;
    std::vector<int> ptr;
    ptr.push_back(0);
    int64_t acc = 0;
    for (int r = 0; r < Cf; ++r) {
      rm.push_back(r);
      rm.push_back(r);
      s.s_hpp.push_back(s.hpp_diag[r]);
      ptr.push_back((int)acc);  // the diagonal has no pair list
      for (size_t i = 0; i < row_cols[r].size(); ++i) {
        rm.push_back(r);
        rm.push_back(row_cols[r][i]);
        s.s_hpp.push_back(pp.empty() ? -1 : pair_store(r, row_cols[r][i]));
        acc += row_cnt[r][i];
        ptr.push_back((int)acc);
      }
    }
    s.s_pair_ptr.swap(ptr);
    // column-major pattern (the order of SparseBlockMatrix::blockCols):
    // stable counting sort of the row-major list by column
    const int nS = (int)(rm.size() / 2);
    std::vector<int> ckey(nS), corder, cptr;
    for (int k = 0; k < nS; ++k) ckey[k] = rm[2 * k + 1];
    counting_sort(ckey, Cf, corder, cptr);
    s.schur_rc.resize(2 * (size_t)nS);
    for (int i = 0; i < nS; ++i) {
      s.schur_rc[2 * i] = rm[2 * (size_t)corder[i]];
      s.schur_rc[2 * i + 1] = rm[2 * (size_t)corder[i] + 1];
    }
    build_sym_lists(Cf, s.schur_rc, s);  // internal order = the row-major order above
  } else {
    if (s.npp > 0) {
      set_error("a pose edge set needs free landmarks (the Schur complement carries the pose-pose blocks)");
      return G2OC_ERR_NOT_SUPPORTED;
    }
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
  const bool bal = g->edge_type == G2OC_EDGE_BAL_OBSERVATION;
  const bool ba = g->edge_type == G2OC_EDGE_PROJECT_XYZ2UV || g->edge_type == G2OC_EDGE_SE3_PROJECT_XYZ ||
                  g->edge_type == G2OC_EDGE_STEREO_SE3_PROJECT_XYZ || bal;
  if (g->pose_type < 1 || g->pose_type > 4 || g->edge_type < 1 || g->edge_type > 7 ||
      (g->edge_type == G2OC_EDGE_SE2) != (g->pose_type == G2OC_POSE_SE2) ||
      (g->edge_type == G2OC_EDGE_SE3) != (g->pose_type == G2OC_POSE_SE3) ||
      bal != (g->pose_type == G2OC_POSE_BAL_CAMERA) ||
      ((ba && !bal) || g->edge_type == G2OC_EDGE_SE3_EXPMAP) != (g->pose_type == G2OC_POSE_SE3EXPMAP)) {
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
  s.bal = bal;
  s.C = g->num_poses;
  s.P = ba ? g->num_points : 0;
  s.E = g->num_edges;
  s.pd = pose_dim(s.pose_type);
  s.ped = pose_est_dim(s.pose_type);
  s.D = edge_dim(s.edge_type);
  s.md = meas_dim(s.edge_type);
  if (g->num_pose_edges < 0) {
    set_error("num_pose_edges is negative");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  if (g->num_pose_edges > 0) {
    if (!ba || bal || g->pose_type != G2OC_POSE_SE3EXPMAP) {
      set_error("a pose edge set (EdgeSE3Expmap) joins the VertexSE3Expmap cameras of a projection-edge graph");
      return G2OC_ERR_BAD_GRAPH;
    }
    if (!g->pose_edge_vertex || !g->pose_edge_measurement || !g->pose_edge_information) {
      set_error("pose edge array is NULL");
      return G2OC_ERR_INVALID_ARGUMENT;
    }
    for (int e = 0; e < g->num_pose_edges; ++e) {
      const int v0 = g->pose_edge_vertex[2 * e], v1 = g->pose_edge_vertex[2 * e + 1];
      if (v0 < 0 || v0 >= s.C || v1 < 0 || v1 >= s.C || v0 == v1) {
        set_error("pose edge %d has vertex indices (%d, %d) out of range", e, v0, v1);
        return G2OC_ERR_BAD_GRAPH;
      }
    }
  }
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
