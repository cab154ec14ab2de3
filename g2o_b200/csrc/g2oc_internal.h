// g2oc_internal.h -- shared declarations of the backend: host-side structure
// (index mapping and block patterns, computed once per upload), device
// buffers, and the context behind the C-ABI handle.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/g2o_cuda.h"

namespace g2oc {

void set_error(const char* fmt, ...);

#define G2OC_CUDA_TRY(expr)                                                         \
  do {                                                                              \
    cudaError_t _e = (expr);                                                        \
    if (_e != cudaSuccess) {                                                        \
      ::g2oc::set_error("%s:%d %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(_e)); \
      return G2OC_ERR_CUDA;                                                         \
    }                                                                               \
  } while (0)

#define G2OC_TRY(expr)            \
  do {                            \
    int _s = (expr);              \
    if (_s != G2OC_OK) return _s; \
  } while (0)

// Device allocation owned by the context (cudaMalloc at upload, cudaFree at
// re-upload or destroy).
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  int alloc(size_t count) {
    if (count == n && p) return G2OC_OK;
    release();
    if (count == 0) return G2OC_OK;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
      set_error("cudaMalloc of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
      p = nullptr;
      return G2OC_ERR_CUDA;
    }
    n = count;
    return G2OC_OK;
  }
  int upload(const std::vector<T>& v, cudaStream_t s) {
    G2OC_TRY(alloc(v.size()));
    if (!v.empty()) G2OC_CUDA_TRY(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    return G2OC_OK;
  }
  size_t bytes() const { return n * sizeof(T); }
};

// ------------------------------------------------------------------ structure
// Everything BlockSolver::buildStructure and SparseOptimizer::buildIndexMapping
// decide, laid out for the device (g2o/core/block_solver.hpp:110-269,
// g2o/core/sparse_optimizer.cpp:175-287).
struct Structure {
  int pose_type = 0, edge_type = 0;
  int C = 0, P = 0, E = 0;
  int pd = 0, ped = 0, D = 0, md = 0;
  bool ba = false, schur = false;
  bool bal = false;  // EdgeObservationBAL + VertexCameraBAL (9-parameter cameras, bal_kernels.cuh)
  // the pose edge set of a projection graph (EdgeSE3Expmap between cameras):
  // active edges; the pose-pose Hpp blocks are stored after the Cf diagonal
  // blocks (storage index Cf + p), hpp_store maps hpp_rc order to storage
  std::vector<int> pact;
  int npp = 0;
  std::vector<int> hpp_store;
  std::vector<int> pp_ptr;    // Cf + 1: per camera its pose-pose blocks in pp_ent
  std::vector<int> pp_ent;    // 4 per entry: storage block, other camera, transposed, 0
  std::vector<int> act;                 // active edge ids, insertion order
  std::vector<int> pose_h, point_l;     // Hessian index of each pose / landmark index of each point, -1 = none
  std::vector<int> free_pose_of_h;      // pose index of Hessian row h
  std::vector<int> free_point_of_l;     // point index of landmark l
  int Cf = 0, Pf = 0;
  // patterns, (row, col) in column-major order
  std::vector<int32_t> hpp_rc, hpl_rc, schur_rc;
  std::vector<int> hpp_diag;            // Hpp block index of the diagonal of row h

  // ---- BA (EdgeProjectXYZ2UV): device edge order = point-major
  // (free landmarks by landmark index, then edges of fixed points), cameras
  // ascending within a point.
  std::vector<int> dev_edge;            // device position -> edge id
  std::vector<int> dev_of_act;          // active position -> device position
  std::vector<int> l_ptr;               // Pf + 1, device edge range of landmark l
  std::vector<int> e_hpl;               // per device edge, Hpl block or -1
  std::vector<int> hb_ptr;              // Pf + 1, Hpl block range of landmark l
  std::vector<int> c_ptr;               // Cf + 1, camera-major range of free camera h
  std::vector<int> c_edge;              // camera-major -> device edge
  std::vector<int> hc_ptr, hc_blk;      // Cf + 1 / hpl_nnzb: Hpl blocks by camera row
  std::vector<int> hc_pos;              // per Hpl block: position in its camera's list
  bool lm_warp_ok = false;              // landmarks <= 32 edges, unique (camera, landmark) pairs
  std::vector<int> lm_chunk_ptr;        // chunks of whole landmarks, <= 32 edges each
  std::vector<int> e_lm;                // per device edge of a free landmark: the landmark
  int max_blocks_per_cam = 0;
  // Schur pairs per Schur block in the internal (row-major) order: the
  // co-observing (a, b) pairs of BD_a B_b^T, a as a position in row r's
  // camera list, b as an Hpl block, in landmark order
  std::vector<int> s_pair_ptr;          // nnzS + 1
  std::vector<int32_t> s_pairs;         // 2 per pair
  std::vector<int> s_hpp;               // per internal Schur block: Hpp block or -1
  int64_t num_pairs = 0;

  // ---- pose graphs (EdgeSE2 / EdgeSE3): device edge order = active order
  std::vector<int> pe_blk;              // 3 per active edge: Hpp block of (v0,v0), (v1,v1), (v0,v1) or -1
  std::vector<uint8_t> pe_trans;        // (v0,v1) stored transposed (hessian index of v0 > v1)
  std::vector<int> hb_src_ptr, hb_src;  // per Hpp block: contributions, encoded edge*3 + slot
  std::vector<int> bv_src_ptr, bv_src;  // per free pose: contributions, encoded edge*2 + which

  // ---- the linear system matrix (S for BA, Hpp for pose graphs): upper
  // blocks stored row by row (internal order, diagonal first in each row);
  // sys_perm maps an internal block to its index in the column-major pattern
  int sys_nb = 0, sys_nnzb = 0;
  std::vector<int> sys_perm;            // internal -> column-major pattern index
  std::vector<int> sys_rptr;            // nb + 1
  std::vector<int> sys_rcol;            // per internal block: column
  std::vector<int> sys_brow;            // per internal block: row
  std::vector<int> sys_diag;            // per row: internal index of the diagonal
  std::vector<int> sys_cptr, sys_cblk;  // strictly-upper blocks by column, rows ascending
  std::vector<int> sys_chunk_ptr;       // nb + 1: chunks of row r (kSysChunk blocks each, the last ragged)
  std::vector<int> sys_chunk_row;       // per chunk: its row
  // dense tiles (6x6 blocks only): kTileBlocks x kTileBlocks blocks each,
  // stored scalar-row-major (96 x 96), upper tiles only, diagonal tiles full
  bool tile_ok = false;
  // ranks of a sharded bundle adjustment (> 1: every non-fixed camera is
  // free whether or not this rank has edges on it, and the tiles cover the
  // whole upper triangle, so every rank has the same Hessian order and the
  // same tile layout)
  int shard_world = 1;
  std::vector<int> tile_ij;             // 2 per tile: tile row I, tile column J (I <= J)
  std::vector<int> tile_off;            // per internal block: offset of its (0,0) entry in the tile array
};

constexpr int kSysChunk = 32;  // blocks per row chunk = lanes of a warp
constexpr int kTileBlocks = 16;  // blocks per tile side of the dense path

int build_structure(const g2oc_graph* g, Structure& s);
// internal row-major order and column lists of a block-symmetric matrix from
// its column-major upper pattern
void build_sym_lists(int nb, const std::vector<int32_t>& rc, Structure& s);

// ------------------------------------------------------------ device scalars
// LM / PCG control state kept on the device so the trial loop needs one small
// read-back per trial.
struct DevScalars {
  double chi2_current;   // currentChi of the LM iteration
  double chi2_temp;      // tempChi after the trial update
  double chi2_plain;     // activeChi2
  double lambda;
  double ni;
  double scale;          // computeScale() + 1e-3
  double rho;
  double max_diag;
  double pcg_residual;   // LinearSolverPCG::_residual carried between solves
  double pcg_d0;
  double pcg_dn;
  double refine_rnorm;   // mixed precision: |r| / |b| of the last refinement
  double refine_bnorm;   // pose-graph refinement: |b|^2 beside |r|^2 in refine_rnorm
  double chi2_temp_plain;  // activeChi2 after the trial update
  int pcg_iterations;
  int pcg_done;
  int solve_ok;
  int accept;            // last trial accepted
  int nonfinite;         // a non-finite value was met
  int pad[3];
};

}  // namespace g2oc
