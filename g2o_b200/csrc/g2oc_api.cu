// g2oc_api.cu -- the C-ABI of include/g2o_cuda.h: context, upload, the
// Gauss-Newton / Levenberg-Marquardt drivers over the device block solver,
// and the parity hooks. Host code only orchestrates: every per-edge,
// per-vertex, per-block and per-vector loop of the iteration runs in the
// kernels of ba_kernels.cuh, pg_kernels.cuh, pcg_kernels.cuh,
// lm_kernels.cuh and cholesky.cuh.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "adjoint_kernels.cuh"
#include "ba_kernels.cuh"
#include "bal_kernels.cuh"
#include "batch_kernels.cuh"
#include "cholesky.cuh"
#include "g2oc_internal.h"
#include "io_kernels.cuh"
#include "lm_kernels.cuh"
#include "pcg_kernels.cuh"
#include "pcg_persistent.cuh"
#include "pcg_tiles.cuh"
#include "tc_chol.cuh"
#include "stereo_kernels.cuh"
#include "pg_kernels.cuh"

namespace g2oc {

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

// Raise a kernel's dynamic shared-memory limit to at least `bytes`, never
// lower it. The limit belongs to the function (per device, process-wide):
// contexts on several host threads sizing it for their own launches must not
// lower it between another thread's setting and that thread's launch, which
// then fails with "invalid argument".
static int raise_dyn_smem(const void* fn, size_t bytes) {
  static std::mutex m;
  static std::map<std::pair<int, const void*>, size_t> applied;
  int dev = 0;
  G2OC_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(m);
  size_t& cur = applied[std::make_pair(dev, fn)];
  if (bytes <= cur) return G2OC_OK;
  G2OC_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  cur = bytes;
  return G2OC_OK;
}

#define G2OC_LAUNCH_CHECK()                                                             \
  do {                                                                                  \
    cudaError_t _e = cudaGetLastError();                                                \
    if (_e != cudaSuccess) {                                                            \
      ::g2oc::set_error("%s:%d kernel launch: %s", __FILE__, __LINE__, cudaGetErrorString(_e)); \
      return G2OC_ERR_CUDA;                                                             \
    }                                                                                   \
  } while (0)

static inline int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

constexpr int kRedBlocks = 592;    // 4 x 148 SMs: fixed grid of the reductions
constexpr int kChi2Blocks = 2048;  // BA chi2: ~2 edges per thread for the 1M-edge graphs
constexpr int kPcgChunkMax = 64;
constexpr int kMixedInnerMaxIter = 256;
// adjoint: outer CG steps, the recurrence's stopping residual |g - H v| / |g|,
// and the true residual accepted at the end
constexpr int kAdjointMaxSteps = 100;
constexpr double kAdjointTolerance = 1e-12;
constexpr double kAdjointAcceptance = 1e-6;

// --------------------------------------------------------------- engine
struct EngineBase {
  virtual ~EngineBase() = default;
  virtual int alloc() = 0;
  virtual int build_system() = 0;
  virtual int max_diag() = 0;  // -> sc.max_diag
  // dst = Hpp src over the Hessian-order vector (landmark part of dst zero):
  // BlockSolver::multiplyHessian (g2o/core/block_solver.h:96)
  virtual int multiply_hessian(const double* src, double* dst) = 0;
  virtual int solve(double lambda) = 0;  // -> x, sc.solve_ok (PCG iterations: PcgState::total_iterations)
  virtual int get_hessian(double* hpp, double* hll, double* hpl) = 0;
  virtual int schur_export(double lambda, double* S, double* bs) = 0;
  // Gauss-Newton solve H x = rhs (lambda 0) with a given device right-hand
  // side in Hessian order, through the same Schur + PCG / Cholesky path (BA)
  // reuse_schur: the Schur complement of the last call still stands (same
  // linearization, lambda 0); only the reduced right-hand side is formed
  virtual int solve_rhs(const double* rhs, double* out, bool reuse_schur = false) = 0;
  // batched windows: per-window lambda initialisation, and the trial's solve
  // (Schur with per-vertex damping, dense Cholesky per window, back-substitution)
  virtual int batch_lambda_init(double user_lambda, double tau) = 0;
  virtual int batch_solve(bool autotune) = 0;
};

// kernel identifiers for the launch counters and the optional per-launch
// CUDA-event timing (g2oc_set_kernel_timing / g2oc_get_kernel_stats)
enum KernelId {
  K_CHI2, K_ERRORS, K_JACOBIANS, K_LANDMARK_PASS, K_CAMERA_PASS, K_SCHUR_LANDMARK, K_SCHUR_BLOCKS, K_SCHUR_RHS,
  K_BACKSUB, K_RESID_CAM, K_RESID_LM, K_OPLUS, K_MAX_DIAG, K_PCG_DIAG_INV, K_PCG_INIT, K_PCG_SPMV, K_PCG_UPDATE,
  K_PCG_CHECK, K_PG_LINEARIZE, K_PG_ASSEMBLE_H, K_PG_ASSEMBLE_B, K_DAMP, K_LM_CONTROL, K_REDUCE, K_AXPY,
  K_CHOLESKY, K_PCG_COLPASS, K_SCHUR_DB, K_IO, K_PCG_SOLVE, K_PCG_TILES, K_TILE_COPY, K_BACKWARD, K_PG_RESID,
  K_TC_EXPAND, K_TC_POTRF, K_TC_TILES, K_TC_SOLVE, K_COUNT
};
static const char* kKernelNames[K_COUNT] = {
  "chi2", "errors", "jacobians", "ba_landmark_pass", "ba_camera_pass", "schur_landmark", "schur_blocks",
  "schur_rhs", "ba_backsub", "ba_resid_cam", "ba_resid_lm", "oplus", "max_diag", "pcg_diag_inv", "pcg_init",
  "pcg_spmv", "pcg_update", "pcg_check_dn", "pg_linearize", "pg_assemble_h", "pg_assemble_b", "damp_diag",
  "lm_control", "reduce", "axpy", "cholesky", "pcg_colpass", "schur_db", "io_reorder", "pcg_solve", "pcg_solve_tiles",
  "sys_to_tiles", "ba_backward", "pg_resid64", "tc_expand", "tc_potrf", "tc_tiles", "tc_solve"};

struct PendingTiming {
  int kid;
  cudaEvent_t a, b;
};

}  // namespace g2oc

namespace g2oc {
// page-locked host array (grown, never shrunk): the windows are packed here so
// that their upload is one DMA copy per array
template <typename T>
struct PinnedVec {
  T* p = nullptr;
  size_t n = 0, cap = 0;
  PinnedVec() = default;
  PinnedVec(const PinnedVec&) = delete;
  PinnedVec& operator=(const PinnedVec&) = delete;
  ~PinnedVec() {
    if (p) cudaFreeHost(p);
  }
  int resize(size_t m) {
    if (m > cap) {
      if (p) cudaFreeHost(p);
      p = nullptr;
      cap = 0;
      cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&p), std::max<size_t>(m, 1) * sizeof(T),
                                    cudaHostAllocDefault);
      if (e != cudaSuccess) {
        p = nullptr;
        n = 0;
        set_error("cudaHostAlloc of %zu bytes failed: %s", m * sizeof(T), cudaGetErrorString(e));
        return G2OC_ERR_CUDA;
      }
      cap = m;
    }
    n = m;
    return G2OC_OK;
  }
  T* data() { return p; }
};
}  // namespace g2oc

struct g2oc_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  g2oc_params prm{};
  g2oc::Structure S;
  bool uploaded = false;
  bool last_upload_reused = false;  // the last g2oc_upload kept the structure (same topology)
  bool system_built = false;
  double fx = 1, fy = 1, cx = 0, cy = 0, bf = 0;
  // every edge has the same information and Huber delta (two-row edges): the
  // kernels take om_const and read no per-edge record
  bool om_uniform = false;
  double4 om_const = {0.0, 0.0, 0.0, 0.0};
  // vertex state
  g2oc::DBuf<double> pose, point, pose_bak, point_bak, pose_init, point_init;
  g2oc::DBuf<int> oplus_count, free_pose, free_point, pose_h, point_l;
  // BA edges
  g2oc::DBuf<int2> e_v, c_v;
  g2oc::DBuf<double2> e_z, c_z;
  g2oc::DBuf<double4> e_om, c_om;
  g2oc::DBuf<double4> e_z3, e_oa3, c_z3, c_oa3;  // stereo edges (stereo_kernels.cuh)
  g2oc::DBuf<double2> e_ob3, c_ob3;
  g2oc::DBuf<int> e_hpl, e_lm, lm_chunk_ptr, l_ptr, c_ptr, hb_ptr, hpl_row, hpl_col, hc_ptr, hc_blk, hc_col, hc_index, s_pair_ptr, s_hpp;
  g2oc::DBuf<int2> s_pairs;
  // pose-graph edges
  g2oc::DBuf<int2> pe_v;
  g2oc::DBuf<double> pe_zinv, pe_info, pe_delta;
  g2oc::DBuf<uint8_t> pe_trans;
  g2oc::DBuf<int> hb_src_ptr, hb_src, bv_src_ptr, bv_src;
  // linear system lists
  g2oc::DBuf<int> sys_perm, sys_rptr, sys_rcol, sys_brow, sys_diag, sys_cptr, sys_cblk, sys_chunk_ptr, sys_chunk_row,
      tile_ij, tile_off;
  int pcg_grid[6] = {0, 0, 0, 0, 0, 0};  // CTAs of the persistent PCG per (storage type, block size 3 / 6 / 9)
  int tile_grid[2] = {0, 0};       // CTAs of the dense-tile PCG per storage type
  // FP64 vectors
  g2oc::DBuf<double> b, x, xs, rhs, resid, dx, partials, errbuf, db;
  g2oc::DBuf<double> adj_g, adj_v, adj_r, adj_dv, adj_p, adj_q, adj_rold, adj_dmeas, adj_dlogw;  // adjoint
  bool adj_schur_ready = false;  // the preconditioner's H and Schur complement of this backward call are built
  // sharded bundle adjustment (g2oc_set_sharding)
  int shard_rank = 0, shard_world = 1;
  g2oc_allreduce_fn shard_fn = nullptr;
  void* shard_user = nullptr;
  g2oc::DBuf<double> shard_diag;  // the summed Hpp diagonal for the initial lambda
  // batched windows (g2oc_upload_windows): packed into one graph
  bool batch = false;
  int nw = 0;
  std::vector<int> win_cam_h, win_lm_h, win_pose_h, win_point_h;  // nw + 1 each
  // host packing buffers (page-locked), kept for re-uploads
  g2oc::PinnedVec<double> pk_pose, pk_point, pk_meas, pk_info, pk_delta;
  g2oc::PinnedVec<uint8_t> pk_pf, pk_qf;
  g2oc::PinnedVec<int32_t> pk_ev;
  // the LM / PCG state read once per trial: page-locked, so the copy is a DMA
  // the host can poll for
  g2oc::PinnedVec<g2oc::DevScalars> h_sc;
  g2oc::PinnedVec<g2oc::PcgState> h_pcg;
  cudaEvent_t ev_read = nullptr;
  cudaEvent_t coop_done = nullptr;  // completion of this context's last grid-barrier launch
  // Dogleg state (OptimizationAlgorithmDogleg's members) and its vectors
  // (steepest-descent step, Gauss-Newton step, scratch)
  double dl_delta = 0.0, dl_lambda = 0.0;
  bool dl_was_pd = true;
  g2oc::DBuf<double> dl_buf;
  g2oc::DBuf<int> win_cam, win_lm, win_edge, win_pose, win_point, win_of_cam, win_of_lm, win_of_pose, win_of_point;
  g2oc::DBuf<int> win_chunk_w, win_chunk_e0, win_chunk_ptr;  // chi2 edge chunks (kWinChi2Chunk)
  g2oc::DBuf<double> win_chunk_sum;
  int win_nchunks = 0;
  g2oc::DBuf<long long> win_mat;
  g2oc::DBuf<double> win_scratch, lam_c, lam_l;
  g2oc::DBuf<g2oc::WinState> win_state;
  g2oc::DBuf<int> win_active;
  g2oc::DBuf<int> win_list[3];       // windows factored with 128 / 256 / 512 threads
  int win_list_n[3] = {0, 0, 0};
  int win_list_nmax[3] = {0, 0, 0};  // largest window of each list (its shared memory)
  int win_threads_of_class[3] = {0, 0, 0};  // autotuned, per size class (n < 96, < 192, >= 192)
  std::vector<int> win_threads;      // per window, for the statistics
  int win_nmax = 0;
  int win_iterations = 0;
  int win_rounds = 0;
  bool win_tuned = false;
  bool win_sparse = false;  // some window's reduced system has blocks outside its pattern (zeroed each round)
  cudaGraphExec_t win_graph = nullptr;
  g2oc::WinDev windev() const {
    return g2oc::WinDev{nw, win_cam.p, win_lm.p, win_edge.p, win_pose.p, win_point.p, win_mat.p};
  }
  g2oc::DBuf<g2oc::DevScalars> sc;
  g2oc::DBuf<g2oc::PcgState> pcg;
  g2oc::DBuf<int> flag;  // nonfinite flag
  // the caller's arrays as copied (g2oc_graph layout), reordered on the device
  g2oc::DBuf<double> raw_meas, raw_info, raw_delta, raw_pose, raw_point;
  g2oc::DBuf<int> src_dev, src_cam;  // input edge of each point-major / camera-major row
  // topology of the uploaded graph: an upload with the same topology keeps
  // the structure, the device lists, the engine and the Cholesky plan
  struct Topology {
    bool valid = false;
    int32_t pose_type = 0, num_poses = 0, num_points = 0, edge_type = 0, num_edges = 0;
    std::vector<int32_t> edge_vertex;
    std::vector<uint8_t> pose_fixed, point_fixed;
    bool has_pose_fixed = false, has_point_fixed = false;
    std::vector<int32_t> pose_edge_vertex;  // the pose edge set's endpoints
  } topo;
  std::unique_ptr<g2oc::EngineBase> eng;
  std::unique_ptr<g2oc::CholPlan> chol;
  long long pcg_seen = 0;        // PcgState::total_iterations at the last read
  double lambda_host = 0.0;      // the device's LM lambda as of the last read
  bool chi2_carry = false;       // chi2_current / chi2_plain hold the current estimates' values
  g2oc_iteration_stats* cur_stats = nullptr;  // stats of the iteration in progress
  double last_refine_dn = 0.0;
  long long refine_steps = 0;
  // launch accounting
  bool timing = false;
  long long kcount[g2oc::K_COUNT] = {};
  // grid-barrier arrivals expected beyond the grid: 0, or 1 when the context
  // was created with G2OC_TEST_BARRIER_EXTRA set (every bounded barrier wait
  // of the persistent PCG then runs out: the test of that path)
  unsigned barrier_extra = 0;
  double ktime_ms[g2oc::K_COUNT] = {};
  long long chol_launches = 0;
  std::vector<cudaEvent_t> event_pool;
  std::vector<g2oc::PendingTiming> pending;
  cudaEvent_t event() {
    if (!event_pool.empty()) {
      cudaEvent_t e = event_pool.back();
      event_pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  // phase times without waiting: events recorded around a phase; the elapsed
  // time is added to *out (and subtracted from *out2) when the spans are
  // resolved, at a point where the host waits for the stream anyway
  struct Span {
    cudaEvent_t a, b;
    double* out;
    double* out2;
  };
  std::vector<Span> spans;
  cudaEvent_t mark() {
    cudaEvent_t e = event();
    cudaEventRecord(e, stream);
    return e;
  }
  void span(cudaEvent_t a, double* out, double* out2 = nullptr) { spans.push_back({a, mark(), out, out2}); }
  // forget the recorded spans without writing their times: after a call that
  // failed half-way their targets (the call's own stats) no longer exist
  void drop_spans() {
    for (auto& sp : spans) {
      event_pool.push_back(sp.a);
      event_pool.push_back(sp.b);
    }
    spans.clear();
    cur_stats = nullptr;
  }
  void resolve_spans() {
    if (spans.empty()) return;
    cudaEventSynchronize(spans.back().b);
    for (auto& sp : spans) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, sp.a, sp.b);
      if (sp.out) *sp.out += ms * 1e-3;
      if (sp.out2) *sp.out2 -= ms * 1e-3;
      event_pool.push_back(sp.a);
      event_pool.push_back(sp.b);
    }
    spans.clear();
  }
  void flush_timing() {
    if (pending.empty()) return;
    cudaEventSynchronize(pending.back().b);
    for (auto& p : pending) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, p.a, p.b);
      ktime_ms[p.kid] += ms;
      event_pool.push_back(p.a);
      event_pool.push_back(p.b);
    }
    pending.clear();
  }
  ~g2oc_ctx() {
    if (ev_read) cudaEventDestroy(ev_read);
    if (coop_done) cudaEventDestroy(coop_done);
    if (win_graph) cudaGraphExecDestroy(win_graph);
    eng.reset();
    chol.reset();
    flush_timing();
    drop_spans();
    for (cudaEvent_t e : event_pool) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
  }
  int vec_size() const { return S.Cf * S.pd + S.Pf * 3; }
  g2oc::BAVertices ba_vertices() {
    g2oc::BAVertices V;
    V.cam = pose.p;
    V.pt = point.p;
    V.free_pose = free_pose.p;
    V.free_point = free_point.p;
    V.fx = fx;
    V.fy = fy;
    V.cx = cx;
    V.cy = cy;
    V.bf = bf;
    return V;
  }
  g2oc::BAEdges ba_edges() {
    g2oc::BAEdges E;
    E.n = (int)S.act.size();
    E.v = e_v.p;
    E.z = e_z.p;
    E.om = om_uniform ? nullptr : e_om.p;
    E.om_const = om_const;
    E.hpl = e_hpl.p;
    E.z3 = e_z3.p;
    E.oa3 = e_oa3.p;
    E.ob3 = e_ob3.p;
    return E;
  }
  g2oc::BACamEdges ba_cam_edges() {
    g2oc::BACamEdges CE{c_ptr.p, c_v.p, c_z.p, om_uniform ? nullptr : c_om.p};
    CE.om_const = om_const;
    CE.z3 = c_z3.p;
    CE.oa3 = c_oa3.p;
    CE.ob3 = c_ob3.p;
    return CE;
  }
  // the pose edge set of a projection graph (EdgeSE3Expmap between cameras)
  // on the pose-graph kernels: the active pose edges, the cameras in the
  // SE3Quat::toVector layout those kernels read (pgpose, unpacked per use)
  g2oc::DBuf<double> pgpose;
  g2oc::DBuf<int> pp_ptr;    // per camera its pose-pose blocks (the Hpp product)
  g2oc::DBuf<int4> pp_ent;
  bool pose_edges() const { return !S.pact.empty(); }
  g2oc::PGEdges ba_pose_edges() {
    g2oc::PGEdges E;
    E.n = (int)S.pact.size();
    E.v = pe_v.p;
    E.zinv = pe_zinv.p;
    E.info = pe_info.p;
    E.delta = pe_delta.p;
    return E;
  }
  g2oc::PGEdges pg_edges() {
    g2oc::PGEdges E;
    E.n = (int)S.act.size();
    E.v = pe_v.p;
    E.zinv = pe_zinv.p;
    E.info = pe_info.p;
    E.delta = pe_delta.p;
    return E;
  }
};

namespace g2oc {

// Counts one kernel launch and, when timing is on, brackets it with CUDA
// events on the context's stream. Used as `G2OC_K(id) kernel<<<...>>>(...);`
struct LaunchScope {
  g2oc_ctx* c;
  int kid;
  bool done = false;
  cudaEvent_t e0 = nullptr;
  LaunchScope(g2oc_ctx* ctx, int id) : c(ctx), kid(id) {
    if (c->timing) {
      e0 = c->event();
      cudaEventRecord(e0, c->stream);
    }
  }
  ~LaunchScope() {
    c->kcount[kid]++;
    if (c->timing) {
      cudaEvent_t e1 = c->event();
      cudaEventRecord(e1, c->stream);
      c->pending.push_back(PendingTiming{kid, e0, e1});
      if (c->pending.size() > 8192) c->flush_timing();
    }
  }
};
#define G2OC_K(kid) for (::g2oc::LaunchScope _ls(c, ::g2oc::kid); !_ls.done; _ls.done = true)

// ------------------------------------------------------------ PCG driver
// Grid-barrier (cooperative) launches of different contexts on one device
// run one after another. Each such kernel sizes its grid to fill the GPU and
// its barrier needs every CTA resident at once, which two of them sharing the
// SMs (contexts on several host threads, or ranks emulated on one GPU) need
// not get: each waits for CTAs the other holds until its bounded spin gives
// up. While more than one context lives on the device, every cooperative
// launch therefore waits (on the device, cudaStreamWaitEvent) for the
// previous one of any context; the chain follows the host order of the
// launches, so it cannot form a cycle. One context alone pays nothing.
struct CoopChain {
  std::mutex m;
  int live = 0;               // contexts on this device
  const g2oc_ctx* owner = nullptr;
  cudaEvent_t last = nullptr;  // the owner's coop_done, recorded after its last launch
};
static CoopChain g_coop[64];

static void coop_register(g2oc_ctx* c, int delta) {
  if (c->device < 0 || c->device >= 64) return;
  CoopChain& ch = g_coop[c->device];
  std::lock_guard<std::mutex> lk(ch.m);
  ch.live += delta;
  if (delta < 0 && ch.owner == c) {
    ch.owner = nullptr;
    ch.last = nullptr;
  }
}

static int coop_launch(g2oc_ctx* c, const void* fn, int grid, int threads, void** args, size_t smem = 0) {
  cudaStream_t st = c->stream;
  if (c->device < 0 || c->device >= 64) {
    G2OC_CUDA_TRY(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(threads), args, smem, st));
    return G2OC_OK;
  }
  CoopChain& ch = g_coop[c->device];
  std::lock_guard<std::mutex> lk(ch.m);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  G2OC_CUDA_TRY(cudaStreamIsCapturing(st, &cap));
  if (ch.live <= 1 || cap != cudaStreamCaptureStatusNone) {  // alone, or inside a graph capture
    G2OC_CUDA_TRY(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(threads), args, smem, st));
    return G2OC_OK;
  }
  if (!c->coop_done) G2OC_CUDA_TRY(cudaEventCreateWithFlags(&c->coop_done, cudaEventDisableTiming));
  if (ch.last && ch.owner != c) G2OC_CUDA_TRY(cudaStreamWaitEvent(st, ch.last, 0));
  G2OC_CUDA_TRY(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(threads), args, smem, st));
  G2OC_CUDA_TRY(cudaEventRecord(c->coop_done, st));
  ch.owner = c;
  ch.last = c->coop_done;
  return G2OC_OK;
}

// Form of the PCG solve: one cooperative launch over dense tiles when the
// matrix is nearly full (6x6 blocks), else one cooperative launch over the
// sparse blocks. G2OC_PCG=sparse forces the sparse launch, G2OC_PCG=kernels
// the three-kernels-per-iteration form (host-polled).
// The variable is read at every solve.
enum PcgMode { PCG_AUTO = 0, PCG_KERNELS = 1, PCG_SPARSE = 2 };
static int pcg_mode() {
  const char* e = getenv("G2OC_PCG");
  if (e && strcmp(e, "kernels") == 0) return PCG_KERNELS;
  if (e && strcmp(e, "sparse") == 0) return PCG_SPARSE;
  return PCG_AUTO;
}
static bool kernels_pcg() { return pcg_mode() == PCG_KERNELS; }

// order of the Schur rows in their launches: 0 by pair work (longest
// first), 1 by camera index
static int schur_row_order() {
  static const int v = [] {
    const char* e = getenv("G2OC_SCHUR_ROW_ORDER");
    return e ? atoi(e) : 0;
  }();
  return v;
}

// entries between the staged BD blocks of a Schur row: 18 (packed, the
// default) or 24 (G2OC_SCHUR_BD_STRIDE=24: 16-byte aligned halves; measured
// slower, 417 vs 238 us per launch on the BA configuration, from 4-way bank
// conflicts of the staging stores)
static int schur_bd_stride() {
  static const int v = [] {
    const char* e = getenv("G2OC_SCHUR_BD_STRIDE");
    return e ? atoi(e) : 18;
  }();
  return v;
}

// FP32 Schur rows: gather each Hpl block with five aligned vector loads
// instead of nine 8-byte loads (the default: 229 vs 243 us per launch on the
// BA configuration; G2OC_SCHUR_VEC=0 for the 8-byte loads)
static bool schur_vec_loads() {
  static const int v = [] {
    const char* e = getenv("G2OC_SCHUR_VEC");
    return e ? atoi(e) : 1;
  }();
  return v != 0;
}

// tensor-core Cholesky substitutions: one cooperative launch per direction
// (the default) or two launches per tile step (G2OC_TC_SOLVE=launches)
static bool tc_solve_coop_on() {
  static const int v = [] {
    const char* e = getenv("G2OC_TC_SOLVE");
    return e && strcmp(e, "launches") == 0 ? 0 : 1;
  }();
  return v != 0;
}

// order of a Schur row's off-diagonal blocks over its lane groups: 0
// storage order (the default), 1 by pair count dealt in alternating rounds
// (measured slower: 249 vs 229 us per launch on the BA configuration, the
// scattered block order costing more in the stores than it saves in lane
// balance)
static int schur_block_order() {
  static const int v = [] {
    const char* e = getenv("G2OC_SCHUR_BLOCK_ORDER");
    return e ? atoi(e) : 0;
  }();
  return v;
}

// LinearSolverPCG::_maxIter (the system dimension when unset); an FP32-stored
// system (mixed path) is a correction step of the FP64 refinement, so its
// iterations are capped and the FP64 residual check decides whether another
// correction is needed
template <typename Real>
static int pcg_max_iter(const g2oc_ctx* c, int n) {
  int m = c->prm.pcg_max_iterations < 0 ? n : c->prm.pcg_max_iterations;
  if (sizeof(Real) == 4 && m > kMixedInnerMaxIter) m = kMixedInnerMaxIter;
  return m;
}

// The per-CTA partial sums: the multi-kernel PCG's column pass runs one CTA per
// block row and writes one slot each, so the buffer grows with the system (it
// never shrinks; the stream is drained first because queued kernels may still
// read the old buffer).
static int ensure_partials(g2oc_ctx* c, size_t slots) {
  if (c->partials.n >= slots) return G2OC_OK;
  G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return c->partials.alloc(slots);
}

template <typename Real, int BS>
static int run_pcg(g2oc_ctx* c, const SysDev<Real>& A, const double* minv, const double* rhs, double* xout,
                   double* r, double* s, double* d0, double* d1, double* q, double* qrow, double* tbuf,
                   bool fixed_d0, int* iters) {
  cudaStream_t st = c->stream;
  G2OC_TRY(ensure_partials(c, (size_t)A.nb));
  PcgState host;
  G2OC_CUDA_TRY(cudaMemcpyAsync(&host, c->pcg.p, sizeof(PcgState), cudaMemcpyDeviceToHost, st));
  G2OC_CUDA_TRY(cudaStreamSynchronize(st));
  PcgState cfg = host;  // keeps residual_carry and, for correction solves, d0
  cfg.tolerance = c->prm.pcg_tolerance;
  cfg.max_iter = c->prm.pcg_max_iterations < 0 ? A.nb * BS : c->prm.pcg_max_iterations;
  // FP32-stored system (mixed path): the inner solve is a correction step of
  // the FP64 refinement, so its iterations are capped; the FP64 residual
  // check decides whether another correction is needed
  if (sizeof(Real) == 4 && cfg.max_iter > kMixedInnerMaxIter) cfg.max_iter = kMixedInnerMaxIter;
  cfg.absolute_tolerance = c->prm.pcg_absolute_tolerance;
  cfg.fixed_d0 = fixed_d0 ? 1 : 0;
  cfg.counter = 0;
  cfg.done = 0;
  cfg.k = 0;
  cfg.breakdown = 0;
  G2OC_CUDA_TRY(cudaMemcpyAsync(c->pcg.p, &cfg, sizeof(PcgState), cudaMemcpyHostToDevice, st));
  const int nbv = cdiv(A.nb, 128);
  G2OC_K(K_PCG_INIT) pcg_init<BS><<<nbv, 128, 0, st>>>(A.nb, rhs, minv, r, s, xout, c->partials.p, c->pcg.p);
  G2OC_LAUNCH_CHECK();
  const bool wide = A.nnzb >= 64 * A.nb;  // dense-ish rows: 256 threads per row, else 32
  int chunk = 4;
  int launched = 0;
  for (;;) {
    for (int k = 0; k < chunk; ++k) {
      if (wide) {
        G2OC_K(K_PCG_SPMV) pcg_rowpass<Real, BS, 256><<<A.nb, 256, 0, st>>>(A, s, d0, d1, qrow, tbuf, c->pcg.p);
        G2OC_K(K_PCG_COLPASS) pcg_colpass<Real, BS, 256><<<A.nb, 256, 0, st>>>(A, d0, d1, qrow, tbuf, q,
                                                                                c->partials.p, c->pcg.p);
      } else {
        G2OC_K(K_PCG_SPMV) pcg_rowpass<Real, BS, 32><<<A.nb, 32, 0, st>>>(A, s, d0, d1, qrow, tbuf, c->pcg.p);
        G2OC_K(K_PCG_COLPASS) pcg_colpass<Real, BS, 32><<<A.nb, 32, 0, st>>>(A, d0, d1, qrow, tbuf, q,
                                                                              c->partials.p, c->pcg.p);
      }
      G2OC_K(K_PCG_UPDATE) pcg_update<BS><<<nbv, 128, 0, st>>>(A.nb, minv, d0, d1, q, r, s, xout, c->partials.p,
                                                               c->pcg.p);
    }
    G2OC_LAUNCH_CHECK();
    launched += chunk;
    G2OC_CUDA_TRY(cudaMemcpyAsync(&host, c->pcg.p, sizeof(PcgState), cudaMemcpyDeviceToHost, st));
    G2OC_CUDA_TRY(cudaStreamSynchronize(st));
    if (host.done) break;
    if (launched > cfg.max_iter + 2) {
      set_error("PCG did not report completion after %d iterations", launched);
      return G2OC_ERR_TIMEOUT;
    }
    chunk = chunk * 2 > kPcgChunkMax ? kPcgChunkMax : chunk * 2;
  }
  G2OC_K(K_PCG_CHECK) pcg_add_total<<<1, 32, 0, st>>>(c->pcg.p);
  G2OC_LAUNCH_CHECK();
  if (iters) *iters = host.iterations;
  return G2OC_OK;
}

// The whole PCG solve as one cooperative launch (pcg_solve_persistent), one
// CTA pair per SM; the host reads the state once at the end.
template <typename Real, int BS>
static int run_pcg_persistent(g2oc_ctx* c, const SysDev<Real>& A, const double* minv, const double* rhs,
                              double* xout, double* r, double* s, double* d, double* tbuf, double* cpart,
                              bool fixed_d0) {
  int& grid = c->pcg_grid[(sizeof(Real) == 4 ? 3 : 0) + (BS == 9 ? 2 : BS == 6 ? 1 : 0)];
  if (grid == 0) {
    int per_sm = 0, sms = 0;
    G2OC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_solve_persistent<Real, BS>,
                                                                kPcgThreads, 0));
    G2OC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    grid = (per_sm < 2 ? per_sm : 2) * sms;
    if (grid > 4096) grid = 4096;  // the per-CTA partials use half of `partials` each
    if (grid <= 0) {
      set_error("persistent PCG kernel cannot be resident");
      return G2OC_ERR_CUDA;
    }
  }
  double tol = c->prm.pcg_tolerance;
  int max_iter = pcg_max_iter<Real>(c, A.nb * BS);
  int abs_tol = c->prm.pcg_absolute_tolerance;
  int fixed = fixed_d0 ? 1 : 0;
  SysDev<Real> a = A;
  const int* chunk_ptr = c->sys_chunk_ptr.p;
  const int* chunk_row = c->sys_chunk_row.p;
  int nchunks = (int)c->S.sys_chunk_row.size();
  double* part_dq = c->partials.p;
  double* part_rs = c->partials.p + 4096;
  PcgState* stp = c->pcg.p;
  unsigned extra = c->barrier_extra;
  void* args[] = {&a,    &chunk_ptr, &chunk_row, &nchunks, &minv,    &rhs,    &xout, &r,       &s,
                  &d,    &tbuf,      &cpart,     &part_dq, &part_rs, &stp,    &tol,  &max_iter, &abs_tol,
                  &fixed, &extra};
  G2OC_K(K_PCG_SOLVE) { G2OC_TRY(coop_launch(c, (const void*)pcg_solve_persistent<Real, BS>, grid, kPcgThreads, args)); }
  return G2OC_OK;
}

// PCG over dense tiles (pcg_solve_tiles), one cooperative launch
template <typename Real>
static int run_pcg_tiles(g2oc_ctx* c, const Real* tiles, int nb, const double* minv, const double* rhs, double* xout,
                         double* r, double* s, double* dbuf0, double* dbuf1, double* part, bool fixed_d0) {
  int& grid = c->tile_grid[sizeof(Real) == 4 ? 1 : 0];
  if (grid == 0) {
    int per_sm = 0, sms = 0;
    G2OC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_solve_tiles<Real>, kTileThreads, 0));
    G2OC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    const int cap = sizeof(Real) == 4 ? 3 : 2;
    grid = (per_sm < cap ? per_sm : cap) * sms;
    if (grid > 4096) grid = 4096;
    if (grid <= 0) {
      set_error("dense-tile PCG kernel cannot be resident");
      return G2OC_ERR_CUDA;
    }
  }
  double tol = c->prm.pcg_tolerance;
  int max_iter = pcg_max_iter<Real>(c, nb * 6);
  int abs_tol = c->prm.pcg_absolute_tolerance;
  int fixed = fixed_d0 ? 1 : 0;
  const int2* tij = reinterpret_cast<const int2*>(c->tile_ij.p);
  int ntiles = (int)(c->S.tile_ij.size() / 2);
  int nbt = (nb + kTileBlocks - 1) / kTileBlocks;
  double* part_dq = c->partials.p;
  double* part_rs = c->partials.p + 4096;
  PcgState* stp = c->pcg.p;
  unsigned extra = c->barrier_extra;
  void* args[] = {&tiles, &tij,  &ntiles, &nbt,  &nb,      &minv,    &rhs, &xout,     &r,       &s,
                  &dbuf0, &dbuf1, &part,  &part_dq, &part_rs, &stp, &tol, &max_iter, &abs_tol, &fixed, &extra};
  G2OC_K(K_PCG_TILES) { G2OC_TRY(coop_launch(c, (const void*)pcg_solve_tiles<Real>, grid, kTileThreads, args)); }
  return G2OC_OK;
}

// sharded bundle adjustment: combine count elements across the ranks in place
// through the caller's all-reduce (a no-op for one rank)
static int shard_reduce(g2oc_ctx* c, void* p, long long count, int dtype, int op) {
  if (c->shard_world <= 1) return G2OC_OK;
  const int rc = c->shard_fn(c->shard_user, p, (int64_t)count, dtype, op, (void*)c->stream);
  if (rc != 0) {
    set_error("sharded bundle adjustment: the all-reduce returned %d", rc);
    return G2OC_ERR_STATE;
  }
  return G2OC_OK;
}

static int finalize_sum(g2oc_ctx* c, int nparts, int stride, double* out0, double* out1, double add0 = 0.0) {
  G2OC_K(K_REDUCE) finalize_sum_kernel<<<1, 256, 0, c->stream>>>(c->partials.p, nparts, stride, out0, out1, add0);
  G2OC_LAUNCH_CHECK();
  return G2OC_OK;
}

static int reset_pcg(g2oc_ctx* c);

// ---------------------------------------------------------- the engine
template <typename Real>
struct Engine final : EngineBase {
  g2oc_ctx* c;
  // Hessian
  DBuf<Real> hpp, hll, hpl, bdc, dinv, Sval, sysval;
  DBuf<double> minv, r, s, d0, d1, q, qrow, tbuf, cpart, tpart;
  DBuf<Real> tiles;  // dense-tile copy of the system (nearly full 6x6-block matrices), allocated on first use
  // Schur rows by lanes per off-diagonal block (2 / 8 / 16), from the row's
  // mean pair-list length (<= 12, <= 40, longer): a structural choice, so a
  // row gets the same arithmetic whatever else is in the graph
  DBuf<int> row_list[3];
  DBuf<int> block_order;  // per row: its off-diagonal blocks in processing order (empty: j order)
  int row_n[3] = {0, 0, 0};
  bool tiles_fresh = false;  // tiles hold the matrix of the current solve
  bool tiles_from_schur = false;  // the last Schur pass wrote the tiles, not the row-SoA values
  bool stage_in_smem = true;  // schur_rows: camera blocks staged in shared memory
  int bd_stride = 18;         // schur_rows: entries between staged BD blocks
  size_t schur_smem = 0;
  DBuf<Real> hcontrib;
  DBuf<double> bcontrib;
  DBuf<Real> phpp;  // the pose edge set's assembled blocks (storage order of hpp)
  DBuf<double> pb;  // and its gradient
  std::unique_ptr<TcChol> tc;  // tensor-core Cholesky of the reduced camera system (mixed precision)
  explicit Engine(g2oc_ctx* ctx) : c(ctx) {}

  int alloc() override {
    const Structure& S = c->S;
    const int pd = S.pd;
    G2OC_TRY(hpp.alloc((size_t)S.hpp_rc.size() / 2 * pd * pd));
    if (S.ba) {
      G2OC_TRY(hll.alloc((size_t)S.Pf * 6 + 1));
      G2OC_TRY(hpl.alloc((size_t)S.hpl_rc.size() / 2 * 18 + 1));
      G2OC_TRY(dinv.alloc((size_t)S.Pf * 9 + 1));
      G2OC_TRY(Sval.alloc((size_t)S.schur_rc.size() / 2 * 36 + 1));
      {
        // Schur rows by mean pair count, longest first (no Schur complement
        // when every landmark is fixed: the lists stay empty)
        std::vector<int> lists[3];
        std::vector<double> work(S.Cf);
        for (int r = 0; r < (S.schur ? S.Cf : 0); ++r) {
          const int k0 = S.sys_rptr[r], k1 = S.sys_rptr[r + 1];
          const double pairs = (double)(S.s_pair_ptr[k1] - S.s_pair_ptr[k0]);
          const double mean = k1 - k0 > 1 ? pairs / (k1 - k0 - 1) : 0.0;
          lists[mean <= 12.0 ? 0 : mean <= 40.0 ? 1 : 2].push_back(r);
          work[r] = pairs + 2.0 * (S.hc_ptr[r + 1] - S.hc_ptr[r]);
        }
        // rows with the most pair products first: the long rows start in
        // the first wave of CTAs (a row's result does not depend on when it
        // runs); G2OC_SCHUR_ROW_ORDER=1 keeps camera order instead, so the
        // rows in flight together are neighbours whose co-observed landmarks
        // (and so the gathered Hpl blocks) largely coincide
        const bool by_work = schur_row_order() == 0;
        for (int gi = 0; gi < 3; ++gi) {
          if (by_work)
            std::stable_sort(lists[gi].begin(), lists[gi].end(), [&](int a, int b) { return work[a] > work[b]; });
          row_n[gi] = (int)lists[gi].size();
          G2OC_TRY(row_list[gi].upload(lists[gi].empty() ? std::vector<int>{0} : lists[gi], c->stream));
        }
        // the order in which a row's off-diagonal blocks go to its lane
        // groups: by pair count, most first, dealt in rounds of one block per
        // group with the direction reversed every round, so the blocks a warp
        // runs side by side have nearly equal pair counts (a warp takes as
        // long as its longest block) and the groups' totals even out
        if (schur_block_order() != 0 && S.schur) {
          std::vector<int> ord(S.schur_rc.size() / 2 + 1, 0);
          std::vector<int> js;
          for (int gi = 0; gi < 3; ++gi) {
            const int groups = (sizeof(Real) == 4 ? 384 : 512) / (gi == 0 ? 2 : gi == 1 ? 8 : 16);
            for (int r : lists[gi]) {
              const int rb = S.sys_rptr[r], nb = S.sys_rptr[r + 1] - rb;
              js.resize(std::max(nb - 1, 0));
              for (int j = 1; j < nb; ++j) js[j - 1] = j;
              std::stable_sort(js.begin(), js.end(), [&](int a, int b) {
                return S.s_pair_ptr[rb + a + 1] - S.s_pair_ptr[rb + a] > S.s_pair_ptr[rb + b + 1] - S.s_pair_ptr[rb + b];
              });
              for (int q0 = 0; q0 < nb - 1; q0 += groups) {
                const int q1 = std::min(nb - 1, q0 + groups);
                if ((q0 / groups) & 1) std::reverse(js.begin() + q0, js.begin() + q1);
              }
              for (int q = 0; q < nb - 1; ++q) ord[rb + 1 + q] = js[q];
            }
          }
          G2OC_TRY(block_order.upload(ord, c->stream));
        } else {
          block_order.release();
        }
      }
      // FP32: BD blocks 24 floats apart when two CTAs of the row kernel still
      // fit on an SM (their halves then start on 16-byte boundaries): 228 KB
      // of shared memory per SM, 1 KB reserved and ~3 KB static per CTA
      bd_stride = schur_bd_stride() == 24 && sizeof(Real) == 4 &&
                          (size_t)S.max_blocks_per_cam * 24 * 4 <= 110 * 1024 ? 24 : 18;
      schur_smem = (size_t)S.max_blocks_per_cam * bd_stride * sizeof(Real);
      stage_in_smem = schur_smem <= 190 * 1024;
      if (!stage_in_smem) schur_smem = 0;
      if (!stage_in_smem) G2OC_TRY(bdc.alloc((size_t)S.hpl_rc.size() / 2 * 18 + 1));
      G2OC_TRY(c->db.alloc((size_t)S.Pf * 3 + 1));
      if (c->pose_edges()) {
        const size_t npa = S.pact.size();
        G2OC_TRY(hcontrib.alloc(npa * 3 * 36));
        G2OC_TRY(bcontrib.alloc(npa * 2 * 6));
        G2OC_TRY(phpp.alloc((size_t)(S.Cf + S.npp) * 36));
        G2OC_TRY(pb.alloc((size_t)S.Cf * 6 + 1));
      }
    } else {
      G2OC_TRY(hcontrib.alloc((size_t)S.act.size() * 3 * pd * pd));
      G2OC_TRY(bcontrib.alloc((size_t)S.act.size() * 2 * pd));
    }
    if (!(S.ba && S.schur)) G2OC_TRY(sysval.alloc((size_t)S.sys_nnzb * pd * pd + 1));
    const size_t n = (size_t)S.Cf * pd;
    G2OC_TRY(minv.alloc((size_t)S.Cf * pd * pd + 1));
    G2OC_TRY(r.alloc(n + 1));
    G2OC_TRY(s.alloc(n + 1));
    G2OC_TRY(d0.alloc(n + 1));
    G2OC_TRY(d1.alloc(n + 1));
    G2OC_TRY(q.alloc(n + 1));
    G2OC_TRY(qrow.alloc(n + 1));
    G2OC_TRY(tbuf.alloc((size_t)S.sys_nnzb * pd + 1));
    G2OC_TRY(cpart.alloc(S.sys_chunk_row.size() * pd + 1));

    return G2OC_OK;
  }

  SysDev<Real> sys(const Real* val) {
    SysDev<Real> A;
    A.nb = c->S.sys_nb;
    A.nnzb = c->S.sys_nnzb;
    A.rptr = c->sys_rptr.p;
    A.rcol = c->sys_rcol.p;
    A.brow = c->sys_brow.p;
    A.diag = c->sys_diag.p;
    A.cptr = c->sys_cptr.p;
    A.cblk = c->sys_cblk.p;
    A.perm = c->sys_perm.p;
    A.val = val;
    return A;
  }

  int build_system() override {
    const Structure& S = c->S;
    cudaStream_t st = c->stream;
    if (S.ba && S.D == 3) {
      if (S.Pf > 0) {
        G2OC_K(K_LANDMARK_PASS) st_landmark_pass<Real><<<cdiv(S.Pf, 128), 128, 0, st>>>(
            c->ba_edges(), c->ba_vertices(), c->l_ptr.p, S.Pf, hll.p, hpl.p, c->b.p + (size_t)S.Cf * 6);
        G2OC_LAUNCH_CHECK();
      }
      if (S.Cf > 0) {
        G2OC_K(K_CAMERA_PASS) st_camera_pass<Real, 128><<<S.Cf, 128, 0, st>>>(c->ba_cam_edges(), c->ba_vertices(),
                                                                              hpp.p, c->b.p);
        G2OC_LAUNCH_CHECK();
      }
    } else if (S.ba) {
      if (S.Pf > 0 && S.lm_warp_ok) {
        const int nch = (int)S.lm_chunk_ptr.size() - 1;
        G2OC_K(K_LANDMARK_PASS) ba_landmark_warp<Real><<<cdiv(nch, 8), 256, 0, st>>>(
            c->ba_edges(), c->ba_vertices(), c->lm_chunk_ptr.p, nch, c->e_lm.p, hll.p, hpl.p,
            c->b.p + (size_t)S.Cf * 6);
        G2OC_LAUNCH_CHECK();
      } else if (S.Pf > 0) {
        G2OC_K(K_LANDMARK_PASS) ba_landmark_pass<Real><<<cdiv(S.Pf, 128), 128, 0, st>>>(
            c->ba_edges(), c->ba_vertices(), c->l_ptr.p, S.Pf, hll.p, hpl.p, c->b.p + (size_t)S.Cf * 6);
        G2OC_LAUNCH_CHECK();
      }
      if (S.Cf > 0) {
        BACamEdges CE = c->ba_cam_edges();
        G2OC_K(K_CAMERA_PASS) ba_camera_pass<Real, 128><<<S.Cf, 128, 0, st>>>(CE, c->ba_vertices(), hpp.p, c->b.p);
        G2OC_LAUNCH_CHECK();
      }
    } else {
      const int n = (int)S.act.size();
      if (S.pose_type == G2OC_POSE_SE2) {
        G2OC_K(K_PG_LINEARIZE) pg_linearize<Real, G2OC_POSE_SE2><<<cdiv(n, 128), 128, 0, st>>>(c->pose.p, c->pg_edges(), c->pe_trans.p,
                                                                        hcontrib.p, bcontrib.p);
        G2OC_LAUNCH_CHECK();
        const int nnzb = (int)S.hpp_rc.size() / 2;
        G2OC_K(K_PG_ASSEMBLE_H) pg_assemble_h<Real, 3><<<cdiv((long long)nnzb * 3, 128), 128, 0, st>>>(nnzb, c->hb_src_ptr.p, c->hb_src.p,
                                                                               hcontrib.p, hpp.p);
        G2OC_K(K_PG_ASSEMBLE_B) pg_assemble_b<3><<<cdiv((long long)S.Cf * 3, 128), 128, 0, st>>>(S.Cf, c->bv_src_ptr.p, c->bv_src.p,
                                                                       bcontrib.p, c->b.p);
      } else {
        if (S.pose_type == G2OC_POSE_SE3EXPMAP)
          G2OC_K(K_PG_LINEARIZE) pg_linearize<Real, G2OC_POSE_SE3EXPMAP><<<cdiv(n, 64), 64, 0, st>>>(
              c->pose.p, c->pg_edges(), c->pe_trans.p, hcontrib.p, bcontrib.p);
        else
          G2OC_K(K_PG_LINEARIZE) pg_linearize<Real, G2OC_POSE_SE3><<<cdiv(n, 64), 64, 0, st>>>(
              c->pose.p, c->pg_edges(), c->pe_trans.p, hcontrib.p, bcontrib.p);
        G2OC_LAUNCH_CHECK();
        const int nnzb = (int)S.hpp_rc.size() / 2;
        G2OC_K(K_PG_ASSEMBLE_H) pg_assemble_h<Real, 6><<<cdiv((long long)nnzb * 6, 128), 128, 0, st>>>(nnzb, c->hb_src_ptr.p, c->hb_src.p,
                                                                               hcontrib.p, hpp.p);
        G2OC_K(K_PG_ASSEMBLE_B) pg_assemble_b<6><<<cdiv((long long)S.Cf * 6, 128), 128, 0, st>>>(S.Cf, c->bv_src_ptr.p, c->bv_src.p,
                                                                       bcontrib.p, c->b.p);
      }
      G2OC_LAUNCH_CHECK();
    }
    if (S.ba && c->pose_edges()) G2OC_TRY(pose_edge_system());
    return G2OC_OK;
  }

  // The pose edge set's part of buildSystem: the pose-graph kernels' edge
  // contributions (pg_linearize on the cameras in SE3Quat::toVector layout),
  // assembled per storage block and camera in edge order, then added to the
  // camera pass's blocks and gradient (ba_add_pose_system)
  int pose_edge_system() {
    const Structure& S = c->S;
    cudaStream_t st = c->stream;
    const int npa = (int)S.pact.size();
    G2OC_K(K_PG_LINEARIZE) ba_unpack_poses<<<cdiv((long long)S.C * 7, 256), 256, 0, st>>>(S.C, c->pose.p,
                                                                                        c->pgpose.p);
    G2OC_K(K_PG_LINEARIZE) pg_linearize<Real, G2OC_POSE_SE3EXPMAP><<<cdiv(npa, 64), 64, 0, st>>>(
        c->pgpose.p, c->ba_pose_edges(), c->pe_trans.p, hcontrib.p, bcontrib.p);
    G2OC_LAUNCH_CHECK();
    const int nblk = S.Cf + S.npp;
    G2OC_K(K_PG_ASSEMBLE_H) pg_assemble_h<Real, 6><<<cdiv((long long)nblk * 6, 128), 128, 0, st>>>(
        nblk, c->hb_src_ptr.p, c->hb_src.p, hcontrib.p, phpp.p);
    G2OC_K(K_PG_ASSEMBLE_B) pg_assemble_b<6><<<cdiv((long long)S.Cf * 6, 128), 128, 0, st>>>(
        S.Cf, c->bv_src_ptr.p, c->bv_src.p, bcontrib.p, pb.p);
    const long long tot = (long long)nblk * 36 + (long long)S.Cf * 6;
    G2OC_K(K_PG_ASSEMBLE_H) ba_add_pose_system<Real><<<cdiv(tot, 256), 256, 0, st>>>(S.Cf, S.npp, phpp.p, hpp.p,
                                                                                      pb.p, c->b.p);
    G2OC_LAUNCH_CHECK();
    return G2OC_OK;
  }

  // the pose edge set's part of the FP64 residual of the refinement:
  // r_p -= (J^T Om' J x)_p over the pose edges, matrix-free in FP64
  // (pg_hx_contrib), summed per camera in edge order
  int pose_edge_resid(double* rp) {
    const Structure& S = c->S;
    cudaStream_t st = c->stream;
    const int npa = (int)S.pact.size();
    G2OC_K(K_RESID_CAM) ba_unpack_poses<<<cdiv((long long)S.C * 7, 256), 256, 0, st>>>(S.C, c->pose.p,
                                                                                     c->pgpose.p);
    G2OC_K(K_RESID_CAM) pg_hx_contrib<G2OC_POSE_SE3EXPMAP><<<cdiv(npa, 64), 64, 0, st>>>(
        c->pgpose.p, c->ba_pose_edges(), c->pose_h.p, c->x.p, bcontrib.p);
    G2OC_K(K_RESID_CAM) pg_assemble_b<6><<<cdiv((long long)S.Cf * 6, 128), 128, 0, st>>>(
        S.Cf, c->bv_src_ptr.p, c->bv_src.p, bcontrib.p, pb.p);
    G2OC_K(K_RESID_CAM) axpy_kernel<<<cdiv((long long)S.Cf * 6, 256), 256, 0, st>>>(rp, pb.p, -1.0, S.Cf * 6);
    G2OC_LAUNCH_CHECK();
    return G2OC_OK;
  }

  int multiply_hessian(const double* src, double* dst) override {
    const Structure& S = c->S;
    cudaStream_t st = c->stream;
    const int n = c->vec_size();
    if (n <= 0) return G2OC_OK;

    if (S.Cf == 0) {
      G2OC_CUDA_TRY(cudaMemsetAsync(dst, 0, (size_t)n * sizeof(double), st));
      return G2OC_OK;
    }
    if (S.ba) {
      G2OC_K(K_LM_CONTROL) hpp_mult_diag6<Real><<<cdiv(n, 256), 256, 0, st>>>(S.Cf, hpp.p, src, dst, n);
      if (c->pose_edges())
        G2OC_K(K_LM_CONTROL) hpp_mult_pairs6<Real><<<cdiv(S.Cf * 6, 256), 256, 0, st>>>(
            S.Cf, c->pp_ptr.p, c->pp_ent.p, hpp.p, src, dst);
    }
    else if (S.pd == 3) G2OC_K(K_LM_CONTROL) hpp_mult_sym<Real, 3><<<cdiv(S.Cf, 128), 128, 0, st>>>(sys(nullptr), hpp.p, src, dst);
    else G2OC_K(K_LM_CONTROL) hpp_mult_sym<Real, 6><<<cdiv(S.Cf, 128), 128, 0, st>>>(sys(nullptr), hpp.p, src, dst);
    G2OC_LAUNCH_CHECK();
    return G2OC_OK;
  }

  int max_diag() override {
    const Structure& S = c->S;
    cudaStream_t st = c->stream;
    if (S.ba && c->shard_world > 1) {
      // the lambda of LM iteration 0 takes max |diag H| of the summed Hpp
      G2OC_TRY(c->shard_diag.alloc((size_t)S.Cf * 6 + 1));
      G2OC_K(K_MAX_DIAG) ba_hpp_diag<Real><<<cdiv(S.Cf * 6, 256), 256, 0, st>>>(hpp.p, S.Cf, c->shard_diag.p);
      G2OC_LAUNCH_CHECK();
      G2OC_TRY(shard_reduce(c, c->shard_diag.p, (long long)S.Cf * 6, G2OC_DT_F64, G2OC_RED_SUM));
      G2OC_K(K_MAX_DIAG) ba_max_diag_summed<Real><<<kRedBlocks, 256, 0, st>>>(c->shard_diag.p, S.Cf, hll.p, S.Pf,
                                                                              c->partials.p);
    } else if (S.ba) {
      G2OC_K(K_MAX_DIAG) ba_max_diag<Real><<<kRedBlocks, 256, 0, st>>>(hpp.p, S.Cf, hll.p, S.Pf, c->partials.p);
    }
    else if (S.pd == 3) G2OC_K(K_MAX_DIAG) pg_max_diag<Real, 3><<<kRedBlocks, 256, 0, st>>>(hpp.p, c->sys_diag.p, S.Cf, c->partials.p);
    else G2OC_K(K_MAX_DIAG) pg_max_diag<Real, 6><<<kRedBlocks, 256, 0, st>>>(hpp.p, c->sys_diag.p, S.Cf, c->partials.p);
    G2OC_LAUNCH_CHECK();
    G2OC_K(K_REDUCE) finalize_max_kernel<<<1, 256, 0, st>>>(c->partials.p, kRedBlocks, &c->sc.p->max_diag);
    G2OC_LAUNCH_CHECK();
    return shard_reduce(c, &c->sc.p->max_diag, 1, G2OC_DT_F64, G2OC_RED_MAX);
  }

  // S = Hpp + lambda - Hpl (H_ll + lambda)^-1 Hpl^T (internal row order) and,
  // when bs != nullptr, the reduced right-hand side of b
  // lam_c / lam_l: per camera row / per landmark damping (batched windows);
  // nullptr: lambda for all
  // to_tiles: write S into the tile PCG's dense tiles (tile_pcg_used());
  // to_windows: into the batched windows' dense matrices
  int schur(double lambda, double* bs, const double* lam_c = nullptr, const double* lam_l = nullptr,
            bool to_tiles = false, bool to_windows = false) {
    const Structure& S = c->S;
    cudaStream_t st = c->stream;
    if (to_tiles) G2OC_TRY(ensure_tiles());
    tiles_from_schur = to_tiles;
    if (to_tiles) tiles_fresh = true;
    if (S.Pf > 0) {
      G2OC_K(K_SCHUR_LANDMARK) schur_landmark<Real><<<cdiv(S.Pf, 128), 128, 0, st>>>(
          hll.p, hpl.p, c->hb_ptr.p, c->hc_index.p, S.Pf, lambda, lam_l, dinv.p, nullptr, c->flag.p);
      G2OC_LAUNCH_CHECK();
    }
    if (S.Cf == 0) return G2OC_OK;
    const double* bp = c->b.p;
    const double* bl = c->b.p + (size_t)S.Cf * 6;
    // sharded: the camera diagonal's lambda is added by rank 0 only (the
    // ranks' rows are summed); the landmarks' above is every rank's own
    lambda = (c->shard_world > 1 && c->shard_rank != 0) ? 0.0 : lambda;
    for (int gi = 0; gi < 3; ++gi) {
      if (row_n[gi] == 0) continue;
      const int* rows = row_list[gi].p;
      if (gi == 0) G2OC_TRY(launch_schur_rows<2>(rows, row_n[gi], lambda, lam_c, bp, bl, bs, to_tiles, to_windows));
      else if (gi == 1) G2OC_TRY(launch_schur_rows<8>(rows, row_n[gi], lambda, lam_c, bp, bl, bs, to_tiles, to_windows));
      else G2OC_TRY(launch_schur_rows<16>(rows, row_n[gi], lambda, lam_c, bp, bl, bs, to_tiles, to_windows));
    }
    return G2OC_OK;
  }

  // the PCG of a 6x6-block system runs on dense tiles (nearly full pattern,
  // automatic PCG form)
  bool tile_pcg_used() const { return c->S.pd == 6 && c->S.tile_ok && pcg_mode() == PCG_AUTO; }

  int ensure_tiles() {
    if (tiles.p) return G2OC_OK;
    const Structure& S = c->S;
    const size_t nt = S.tile_ij.size() / 2;
    G2OC_TRY(tiles.alloc(nt * kTileSize));
    G2OC_CUDA_TRY(cudaMemsetAsync(tiles.p, 0, tiles.bytes(), c->stream));  // blocks outside the pattern
    // per block row, one slot of 6 partial sums per tile index (zero for the
    // tiles outside the pattern)
    const size_t nbt = (S.sys_nb + kTileBlocks - 1) / kTileBlocks;
    G2OC_TRY(tpart.alloc((size_t)S.sys_nb * nbt * 6));
    G2OC_CUDA_TRY(cudaMemsetAsync(tpart.p, 0, tpart.bytes(), c->stream));
    return G2OC_OK;
  }

  // schur_rows over a list of camera rows with G lanes per off-diagonal block
  // (FP32 storage: 384 threads, two CTAs per SM; FP64: 512 threads, one)
  template <int G>
  int launch_schur_rows(const int* rows, int nrows, double lambda, const double* lam_c, const double* bp,
                        const double* bl, double* bs, bool to_tiles, bool to_windows) {
    constexpr int T = sizeof(Real) == 4 ? 384 : 512;
    cudaStream_t st = c->stream;
    Real* tl = to_tiles ? tiles.p : nullptr;
    const int* toff = to_tiles ? c->tile_off.p : nullptr;
    DenseOut dn{c->win_of_cam.p, c->win_cam.p, c->win_mat.p, to_windows ? c->win_scratch.p : nullptr};
    if (stage_in_smem) {
      auto kern = schur_vec_loads() ? schur_rows<Real, T, true, G, true> : schur_rows<Real, T, true, G, false>;
      G2OC_TRY(raise_dyn_smem((const void*)kern, schur_smem));
      G2OC_K(K_SCHUR_BLOCKS) kern<<<nrows, T, schur_smem, st>>>(
          rows, c->hc_ptr.p, c->hc_blk.p, c->hc_col.p, hpl.p, dinv.p, bdc.p, c->sys_rptr.p, c->sys_rcol.p,
          c->s_pair_ptr.p, c->s_pairs.p, block_order.p, c->s_hpp.p, hpp.p, lambda, lam_c, Sval.p, tl, toff, dn, bp,
          bl, bs, bd_stride);
    } else {
      G2OC_K(K_SCHUR_BLOCKS) schur_rows<Real, T, false, G><<<nrows, T, 0, st>>>(
          rows, c->hc_ptr.p, c->hc_blk.p, c->hc_col.p, hpl.p, dinv.p, bdc.p, c->sys_rptr.p, c->sys_rcol.p,
          c->s_pair_ptr.p, c->s_pairs.p, block_order.p, c->s_hpp.p, hpp.p, lambda, lam_c, Sval.p, tl, toff, dn, bp,
          bl, bs, bd_stride);
    }
    G2OC_LAUNCH_CHECK();
    return G2OC_OK;
  }

  int schur_rhs_from(const double* rp, const double* rl, double* bs) {
    const Structure& S = c->S;
    if (S.Pf > 0) {
      G2OC_K(K_SCHUR_DB) schur_db<Real><<<cdiv(S.Pf, 128), 128, 0, c->stream>>>(dinv.p, rl, S.Pf, c->db.p);
      G2OC_LAUNCH_CHECK();
    }
    G2OC_K(K_SCHUR_RHS) schur_rhs<Real, 256><<<S.Cf, 256, 0, c->stream>>>(c->hc_ptr.p, c->hc_blk.p, c->hc_col.p,
                                                                         hpl.p, c->db.p, rp, bs);
    G2OC_LAUNCH_CHECK();
    return G2OC_OK;
  }

  // fixed_d0: a correction solve of the refinement, stopping at the d0 of
  // the first solve (which set the preconditioner)
  int pcg_solve(const Real* val, const double* rhs, double* xout, bool fixed_d0) {
    const Structure& S = c->S;
    SysDev<Real> A = sys(val);
    // direct: the Schur pass wrote this system into the tiles (val unused)
    const bool direct = tiles_from_schur && val == Sval.p && tile_pcg_used();
    if (!fixed_d0 && !direct) tiles_fresh = false;
    if (S.pd == 6) {
      if (!fixed_d0) {
        if (direct)
          G2OC_K(K_PCG_DIAG_INV) pcg_diag_inv_tiles<Real><<<cdiv(A.nb, 20), 128, 0, c->stream>>>(
              tiles.p, c->tile_off.p, c->sys_diag.p, A.nb, minv.p, c->flag.p);
        else
          G2OC_K(K_PCG_DIAG_INV) pcg_diag_inv6_lanes<Real><<<cdiv(A.nb, 20), 128, 0, c->stream>>>(A, minv.p, c->flag.p);
        G2OC_LAUNCH_CHECK();
      }
      if (kernels_pcg())
        return run_pcg<Real, 6>(c, A, minv.p, rhs, xout, r.p, s.p, d0.p, d1.p, q.p, qrow.p, tbuf.p, fixed_d0, nullptr);
      if (tile_pcg_used()) {
        G2OC_TRY(ensure_tiles());
        if (!direct && (!fixed_d0 || !tiles_fresh)) {  // a correction solve reuses the tiles of its first solve
          G2OC_K(K_TILE_COPY) sys_to_tiles<Real><<<cdiv((long long)A.nnzb * 6, 256), 256, 0, c->stream>>>(
              A, c->tile_off.p, tiles.p);
          G2OC_LAUNCH_CHECK();
          tiles_fresh = true;
        }
        return run_pcg_tiles<Real>(c, tiles.p, A.nb, minv.p, rhs, xout, r.p, s.p, d0.p, d1.p, tpart.p, fixed_d0);
      }
      return run_pcg_persistent<Real, 6>(c, A, minv.p, rhs, xout, r.p, s.p, d0.p, tbuf.p, cpart.p, fixed_d0);
    }
    if (!fixed_d0) {
      G2OC_K(K_PCG_DIAG_INV) pcg_diag_inv<Real, 3><<<cdiv(A.nb, 128), 128, 0, c->stream>>>(A, minv.p, c->flag.p);
      G2OC_LAUNCH_CHECK();
    }
    if (kernels_pcg())
      return run_pcg<Real, 3>(c, A, minv.p, rhs, xout, r.p, s.p, d0.p, d1.p, q.p, qrow.p, tbuf.p, fixed_d0, nullptr);
    return run_pcg_persistent<Real, 3>(c, A, minv.p, rhs, xout, r.p, s.p, d0.p, tbuf.p, cpart.p, fixed_d0);
  }

  // a . b of two device vectors of length n, read on the host (one wait)
  int dev_dot_host(const double* a, const double* b, int n, double* out) {
    G2OC_K(K_LM_CONTROL) dot_partials<<<kRedBlocks, 256, 0, c->stream>>>(a, b, n, c->partials.p);
    G2OC_LAUNCH_CHECK();
    G2OC_TRY(finalize_sum(c, kRedBlocks, 1, &c->sc.p->refine_bnorm, nullptr));
    G2OC_CUDA_TRY(cudaMemcpyAsync(out, &c->sc.p->refine_bnorm, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return G2OC_OK;
  }

  // the Cholesky of a nearly full reduced camera system in mixed precision:
  // the tensor-core factorization of tc_chol.cuh (S written into the dense
  // tiles by the Schur pass)
  bool tc_chol_used() const {
    const Structure& S = c->S;
    return sizeof(Real) == 4 && S.ba && S.schur && S.pd == 6 && S.tile_ok &&
           c->prm.linear_solver == G2OC_LINEAR_CHOLESKY && c->shard_world <= 1;
  }

  int tc_factor(int* ok) {
    if constexpr (sizeof(Real) != 4) {
      set_error("the tensor-core Cholesky factors FP32-stored systems");
      return G2OC_ERR_NOT_SUPPORTED;
    } else {
      const Structure& S = c->S;
      cudaStream_t st = c->stream;
      if (!tc) {
        std::unique_ptr<TcChol> P(new TcChol());
        const int nbt = (S.sys_nb + kTileBlocks - 1) / kTileBlocks;
        G2OC_TRY(tc_chol_plan(*P, S.sys_nb * 6, nbt, S.tile_ij, st));
        tc = std::move(P);
      }
      G2OC_TRY(raise_dyn_smem((const void*)tc_tiles, kTcSmem));
      G2OC_TRY(raise_dyn_smem((const void*)tc_potrf, kTcPotrfSmem));
      TcChol& P = *tc;
      G2OC_CUDA_TRY(cudaMemsetAsync(P.info.p, 0, sizeof(int), st));
      G2OC_CUDA_TRY(cudaMemsetAsync(P.err.p, 0, sizeof(int), st));
      const long long total = (long long)P.np * P.np;
      G2OC_K(K_TC_EXPAND) tc_expand_tiles<<<cdiv(total, 256), 256, 0, st>>>(tiles.p, P.tile_index.p, P.nbt, P.n,
                                                                           P.np, P.A.p);
      G2OC_K(K_TC_EXPAND) chol_pivot_floor<float><<<1, 1024, 0, st>>>(P.A.p, P.np, P.n, P.floor.p);
      for (int k = 0; k < P.nt; ++k) {
        float* Wk = P.W.p + (size_t)k * kTc * kTc;
        G2OC_K(K_TC_POTRF) tc_potrf<<<1, 256, kTcPotrfSmem, st>>>(P.A.p, P.np, k, Wk, P.floor.p, P.info.p);
        const int p0 = P.list_ptr[2 * k], p1 = P.list_ptr[2 * k + 1], p2 = P.list_ptr[2 * k + 2];
        if (p1 > p0)
          G2OC_K(K_TC_TILES) tc_tiles<<<p1 - p0, 128, kTcSmem, st>>>(P.A.p, P.np, k, P.lists.p + p0, Wk, P.err.p);
        if (p2 > p1)
          G2OC_K(K_TC_TILES) tc_tiles<<<p2 - p1, 128, kTcSmem, st>>>(P.A.p, P.np, k, P.lists.p + p1, Wk, P.err.p);
      }
      G2OC_LAUNCH_CHECK();
      int h[2];
      G2OC_CUDA_TRY(cudaMemcpyAsync(&h[0], P.info.p, sizeof(int), cudaMemcpyDeviceToHost, st));
      G2OC_CUDA_TRY(cudaMemcpyAsync(&h[1], P.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
      G2OC_CUDA_TRY(cudaStreamSynchronize(st));
      if (h[1]) {
        set_error("tensor-core Cholesky: a bounded wait for the tile products gave up");
        return G2OC_ERR_TIMEOUT;
      }
      *ok = h[0] == 0;
      return G2OC_OK;
    }
  }

  // x = S^-1 rhs with the factor of tc_factor (FP64 substitutions)
  int tc_resolve(const double* rhs, double* xout) {
    TcChol& P = *tc;
    cudaStream_t st = c->stream;
    G2OC_K(K_TC_SOLVE) tc_load_rhs<<<cdiv(P.np, 256), 256, 0, st>>>(rhs, P.n, P.np, P.y.p);
    if (tc_solve_coop_on()) {
      // one cooperative launch per direction (a grid barrier per tile step)
      int sms = 0;
      G2OC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
      G2OC_TRY(raise_dyn_smem((const void*)tc_solve_coop, kTcSolveSmem));
      int grid = std::min(sms, std::max(4 * (P.nt - 1), 1));
      const float* A = P.A.p;
      const float* W = P.W.p;
      int np = P.np, nt = P.nt;
      double* y = P.y.p;
      PcgState* stp = P.sync.p;
      unsigned extra = c->barrier_extra;
      for (int dir = 0; dir < 2; ++dir) {
        G2OC_CUDA_TRY(cudaMemsetAsync(P.sync.p, 0, sizeof(PcgState), st));
        void* args[] = {&A, &W, &np, &nt, &y, &stp, &extra, &dir};
        G2OC_K(K_TC_SOLVE) {
          G2OC_TRY(coop_launch(c, (const void*)tc_solve_coop, grid, kTcSolveThreads, args, kTcSolveSmem));
        }
      }
      G2OC_LAUNCH_CHECK();
      int bad = 0;
      G2OC_CUDA_TRY(cudaMemcpyAsync(&bad, &P.sync.p->sync_error, sizeof(int), cudaMemcpyDeviceToHost, st));
      G2OC_CUDA_TRY(cudaStreamSynchronize(st));
      if (bad) {
        set_error("tensor-core Cholesky: a grid barrier of the substitutions gave up");
        return G2OC_ERR_TIMEOUT;
      }
      G2OC_CUDA_TRY(cudaMemcpyAsync(xout, P.y.p, (size_t)P.n * sizeof(double), cudaMemcpyDeviceToDevice, st));
      return G2OC_OK;
    }
    for (int k = 0; k < P.nt; ++k) {
      G2OC_K(K_TC_SOLVE) tc_apply_w<<<1, kTc, 0, st>>>(P.W.p + (size_t)k * kTc * kTc, P.y.p, k, false);
      if (k + 1 < P.nt) G2OC_K(K_TC_SOLVE) tc_fwd_update<<<P.nt - k - 1, kTc, 0, st>>>(P.A.p, P.np, k, P.y.p);
    }
    for (int k = P.nt - 1; k >= 0; --k) {
      G2OC_K(K_TC_SOLVE) tc_apply_w<<<1, kTc, 0, st>>>(P.W.p + (size_t)k * kTc * kTc, P.y.p, k, true);
      if (k > 0) G2OC_K(K_TC_SOLVE) tc_bwd_update<<<k, kTc, 0, st>>>(P.A.p, P.np, k, P.y.p);
    }
    G2OC_LAUNCH_CHECK();
    G2OC_CUDA_TRY(cudaMemcpyAsync(xout, P.y.p, (size_t)P.n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    return G2OC_OK;
  }

  int chol_solve(const Real* val, const double* rhs, double* xout, int* ok) {
    const Structure& S = c->S;
    if (!c->chol) {
      const std::vector<int32_t>& rc = S.ba && S.schur ? S.schur_rc : S.hpp_rc;
      std::unique_ptr<CholPlan> P(new CholPlan());
      G2OC_TRY(chol_plan_build(*P, S.sys_nb, S.pd, rc, !S.ba, c->stream));
      c->chol = std::move(P);
    }
    return g2oc::chol_solve<Real>(*c->chol, c->stream, sys(val), rhs, xout, ok, &c->kcount[K_CHOLESKY]);
  }

  int solve(double lambda) override {
    const Structure& S = c->S;
    cudaStream_t st = c->stream;
    int ok = 1;
    const bool use_chol = c->prm.linear_solver == G2OC_LINEAR_CHOLESKY ||
                          (c->prm.linear_solver == 2 && !S.ba);
    if (S.Cf == 0) {
      // every pose fixed: only the landmarks move, x_l = (H_ll + lambda)^-1 b_l
      G2OC_CUDA_TRY(cudaMemsetAsync(c->x.p, 0, c->x.bytes(), st));
      if (S.ba && S.Pf > 0) {
        if (S.schur) {
          G2OC_K(K_SCHUR_LANDMARK) schur_landmark<Real><<<cdiv(S.Pf, 128), 128, 0, st>>>(
              hll.p, hpl.p, c->hb_ptr.p, c->hc_index.p, S.Pf, lambda, nullptr, dinv.p, nullptr, c->flag.p);
          G2OC_LAUNCH_CHECK();
          G2OC_TRY(backsub(c->b.p, c->xs.p, c->x.p));
        }
      }
    } else if (S.ba && S.schur) {
      cudaEvent_t ts = c->cur_stats ? c->mark() : nullptr;
      if (c->shard_world > 1) {
        // every rank forms its landmarks' part of S and b_schur (its Hpp and
        // b_p parts included; the cameras' lambda on rank 0 only, the
        // landmarks' on every rank) into zeroed tiles, then the ranks sum
        // them: all hold the same reduced system
        G2OC_TRY(ensure_tiles());
        G2OC_CUDA_TRY(cudaMemsetAsync(tiles.p, 0, tiles.bytes(), st));
        G2OC_TRY(schur(lambda, c->rhs.p, nullptr, nullptr, true));
        G2OC_TRY(shard_reduce(c, tiles.p, (long long)tiles.n, sizeof(Real) == 4 ? G2OC_DT_F32 : G2OC_DT_F64,
                              G2OC_RED_SUM));
        G2OC_TRY(shard_reduce(c, c->rhs.p, (long long)S.Cf * 6, G2OC_DT_F64, G2OC_RED_SUM));
      } else {
        G2OC_TRY(schur(lambda, c->rhs.p, nullptr, nullptr, (!use_chol && tile_pcg_used()) || tc_chol_used()));
      }
      const double* bp = c->b.p;
      const double* bl = c->b.p + (size_t)S.Cf * 6;
      if (ts) c->span(ts, &c->cur_stats->time_schur_complement, &c->cur_stats->time_linear_solver);
      const bool tc_chol = use_chol && tc_chol_used();
      if (tc_chol) {
        G2OC_TRY(tc_factor(&ok));
        G2OC_TRY(tc_resolve(c->rhs.p, c->xs.p));
      } else if (use_chol) {
        G2OC_TRY(chol_solve(Sval.p, c->rhs.p, c->xs.p, &ok));
      } else {
        G2OC_TRY(pcg_solve(Sval.p, c->rhs.p, c->xs.p, false));
      }
      G2OC_CUDA_TRY(cudaMemcpyAsync(c->x.p, c->xs.p, (size_t)S.Cf * 6 * sizeof(double), cudaMemcpyDeviceToDevice, st));
      G2OC_TRY(backsub(bl, c->xs.p, c->x.p + (size_t)S.Cf * 6));
      // mixed precision: FP64 iterative refinement on the true residual of
      // the damped normal equations, r = b - (J^T Om' J + lambda I) x, formed
      // matrix-free from the edges in FP64. A correction is solved (FP32
      // Schur + PCG, stopping at the d0 of the first solve) only while the
      // reduced residual's M-norm is above that d0, i.e. while the FP32
      // storage of H / S / Dinv, not the PCG tolerance, limits the step; a
      // correction that raises the residual is undone and ends the loop.
      // With the tensor-core Cholesky the same loop runs with corrections
      // from the kept factor, stopping when |r_s| / |b_s| of the reduced
      // system is at or below refine_tolerance.
      if (sizeof(Real) == 4 && ok && (!use_chol || tc_chol) && c->prm.refine_max_iterations >= 0) {
        const int n = c->vec_size();
        double prev = -1.0;
        double bs2 = 0.0;
        if (tc_chol) G2OC_TRY(dev_dot_host(c->rhs.p, c->rhs.p, S.Cf * 6, &bs2));
        for (int k = 0; k <= c->prm.refine_max_iterations; ++k) {
          double* rp = c->resid.p;
          double* rl = c->resid.p + (size_t)S.Cf * 6;
          if (S.D == 3) {
            if (S.Pf > 0)
              G2OC_K(K_RESID_LM) st_resid64_landmark<<<cdiv(S.Pf, 128), 128, 0, st>>>(
                  c->ba_edges(), c->ba_vertices(), c->l_ptr.p, S.Pf, c->pose_h.p, lambda, bl, c->x.p,
                  c->x.p + (size_t)S.Cf * 6, rl);
          } else if (S.Pf > 0 && S.lm_warp_ok) {
            const int nch = (int)S.lm_chunk_ptr.size() - 1;
            G2OC_K(K_RESID_LM) ba_resid64_landmark_warp<<<cdiv(nch, 8), 256, 0, st>>>(
                c->ba_edges(), c->ba_vertices(), c->lm_chunk_ptr.p, nch, c->e_lm.p, c->pose_h.p, lambda, bl, c->x.p,
                c->x.p + (size_t)S.Cf * 6, rl);
          } else if (S.Pf > 0) {
            G2OC_K(K_RESID_LM) ba_resid64_landmark<<<cdiv(S.Pf, 128), 128, 0, st>>>(
                c->ba_edges(), c->ba_vertices(), c->l_ptr.p, S.Pf, c->pose_h.p, lambda, bl, c->x.p,
                c->x.p + (size_t)S.Cf * 6, rl);
          }
          BACamEdges CE = c->ba_cam_edges();
          if (S.D == 3)
            G2OC_K(K_RESID_CAM) st_resid64_camera<128><<<S.Cf, 128, 0, st>>>(CE, c->ba_vertices(), c->point_l.p,
                                                                             lambda, bp, c->x.p,
                                                                             c->x.p + (size_t)S.Cf * 6, rp);
          else
            G2OC_K(K_RESID_CAM) ba_resid64_camera<128><<<S.Cf, 128, 0, st>>>(CE, c->ba_vertices(), c->point_l.p,
                                                                             lambda, bp, c->x.p,
                                                                             c->x.p + (size_t)S.Cf * 6, rp);
          G2OC_LAUNCH_CHECK();
          if (c->pose_edges()) G2OC_TRY(pose_edge_resid(rp));
          G2OC_TRY(schur_rhs_from(rp, rl, c->rhs.p));
          double check = 0.0, bound = 0.0;
          if (tc_chol) {
            double rs2 = 0.0;
            G2OC_TRY(dev_dot_host(c->rhs.p, c->rhs.p, S.Cf * 6, &rs2));
            check = bs2 > 0.0 ? std::sqrt(rs2 / bs2) : 0.0;
            bound = c->prm.refine_tolerance;
          } else {
            G2OC_K(K_PCG_CHECK) pcg_check_dn<6><<<cdiv(S.Cf, 128), 128, 0, st>>>(S.Cf, minv.p, c->rhs.p,
                                                                                 c->partials.p, c->pcg.p);
            G2OC_LAUNCH_CHECK();
            PcgState ps;
            G2OC_CUDA_TRY(cudaMemcpyAsync(&ps, c->pcg.p, sizeof(PcgState), cudaMemcpyDeviceToHost, st));
            G2OC_CUDA_TRY(cudaStreamSynchronize(st));
            check = ps.check_dn;
            bound = ps.d0;
          }
          c->last_refine_dn = check;
          if (prev >= 0.0 && !(check < prev)) {
            // the last correction did not reduce the true residual: undo it
            G2OC_K(K_AXPY) axpy_kernel<<<cdiv(n, 256), 256, 0, st>>>(c->x.p, c->dx.p, -1.0, n);
            G2OC_LAUNCH_CHECK();
            break;
          }
          if (!(check > bound) || k == c->prm.refine_max_iterations) break;
          prev = check;
          if (tc_chol) G2OC_TRY(tc_resolve(c->rhs.p, c->xs.p));
          else G2OC_TRY(pcg_solve(Sval.p, c->rhs.p, c->xs.p, true));
          c->refine_steps++;
          G2OC_CUDA_TRY(cudaMemcpyAsync(c->dx.p, c->xs.p, (size_t)S.Cf * 6 * sizeof(double), cudaMemcpyDeviceToDevice, st));
          G2OC_TRY(backsub(rl, c->xs.p, c->dx.p + (size_t)S.Cf * 6));
          G2OC_K(K_AXPY) axpy_kernel<<<cdiv(n, 256), 256, 0, st>>>(c->x.p, c->dx.p, 1.0, n);
          G2OC_LAUNCH_CHECK();
        }
      }
    } else {
      const int nnzb = S.sys_nnzb;
      const long long nel = (long long)nnzb * S.pd * S.pd;
      if (S.pd == 3)
        G2OC_K(K_DAMP) sys_gather_damped<Real, 3><<<cdiv(nel, 256), 256, 0, st>>>(
            hpp.p, c->sys_perm.p, c->sys_brow.p, c->sys_rptr.p, c->sys_rcol.p, nnzb, lambda, sysval.p);
      else
        G2OC_K(K_DAMP) sys_gather_damped<Real, 6><<<cdiv(nel, 256), 256, 0, st>>>(
            hpp.p, c->sys_perm.p, c->sys_brow.p, c->sys_rptr.p, c->sys_rcol.p, nnzb, lambda, sysval.p);
      G2OC_LAUNCH_CHECK();
      if (use_chol) G2OC_TRY(chol_solve(sysval.p, c->b.p, c->x.p, &ok));
      else G2OC_TRY(pcg_solve(sysval.p, c->b.p, c->x.p, false));
      if (sizeof(Real) == 4 && ok && use_chol && !S.ba && c->prm.refine_max_iterations >= 0)
        G2OC_TRY(refine_pose_graph(lambda));
    }
    G2OC_K(K_LM_CONTROL) set_solve_ok<<<1, 32, 0, st>>>(c->sc.p, ok);
    G2OC_LAUNCH_CHECK();
    return G2OC_OK;
  }

  // Mixed precision on the pose graphs (FP32 Hessian, FP64 Cholesky of it):
  // FP64 iterative refinement on the true residual of the damped system,
  // r = b - (J^T Om' J + lambda I) x, formed matrix-free from the edges in
  // FP64 (pg_hx_contrib). While |r| / |b| is above refine_tolerance a
  // correction is solved with the same factor, up to refine_max_iterations;
  // a correction that does not reduce the residual is undone and ends the loop.
  int refine_pose_graph(double lambda) {
    const Structure& S = c->S;
    cudaStream_t st = c->stream;
    const int n = c->vec_size();
    const int ne = (int)S.act.size();
    double prev = -1.0;
    for (int k = 0;; ++k) {
      if (S.pose_type == G2OC_POSE_SE2) {
        G2OC_K(K_PG_RESID) pg_hx_contrib<G2OC_POSE_SE2><<<cdiv(ne, 128), 128, 0, st>>>(
            c->pose.p, c->pg_edges(), c->pose_h.p, c->x.p, bcontrib.p);
        G2OC_K(K_PG_RESID) pg_assemble_b<3><<<cdiv((long long)S.Cf * 3, 128), 128, 0, st>>>(
            S.Cf, c->bv_src_ptr.p, c->bv_src.p, bcontrib.p, c->xs.p);
      } else {
        if (S.pose_type == G2OC_POSE_SE3EXPMAP)
          G2OC_K(K_PG_RESID) pg_hx_contrib<G2OC_POSE_SE3EXPMAP><<<cdiv(ne, 64), 64, 0, st>>>(
              c->pose.p, c->pg_edges(), c->pose_h.p, c->x.p, bcontrib.p);
        else
          G2OC_K(K_PG_RESID) pg_hx_contrib<G2OC_POSE_SE3><<<cdiv(ne, 64), 64, 0, st>>>(
              c->pose.p, c->pg_edges(), c->pose_h.p, c->x.p, bcontrib.p);
        G2OC_K(K_PG_RESID) pg_assemble_b<6><<<cdiv((long long)S.Cf * 6, 128), 128, 0, st>>>(
            S.Cf, c->bv_src_ptr.p, c->bv_src.p, bcontrib.p, c->xs.p);
      }
      G2OC_K(K_PG_RESID) pg_resid_finish<<<kRedBlocks, 256, 0, st>>>(n, c->b.p, c->xs.p, c->x.p, lambda,
                                                                     c->resid.p, c->partials.p);
      G2OC_LAUNCH_CHECK();
      G2OC_TRY(finalize_sum(c, kRedBlocks, 2, &c->sc.p->refine_rnorm, &c->sc.p->refine_bnorm));
      double rb[2];
      G2OC_CUDA_TRY(cudaMemcpyAsync(rb, &c->sc.p->refine_rnorm, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
      G2OC_CUDA_TRY(cudaStreamSynchronize(st));
      const double rel = rb[1] > 0.0 ? std::sqrt(rb[0] / rb[1]) : 0.0;
      c->last_refine_dn = rel;
      if (prev >= 0.0 && !(rel < prev)) {
        G2OC_K(K_AXPY) axpy_kernel<<<cdiv(n, 256), 256, 0, st>>>(c->x.p, c->dx.p, -1.0, n);
        G2OC_LAUNCH_CHECK();
        break;
      }
      if (!(rel > c->prm.refine_tolerance) || k == c->prm.refine_max_iterations) break;
      prev = rel;
      G2OC_TRY(chol_resolve(*c->chol, st, c->resid.p, c->dx.p, &c->kcount[K_CHOLESKY]));
      c->refine_steps++;
      G2OC_K(K_AXPY) axpy_kernel<<<cdiv(n, 256), 256, 0, st>>>(c->x.p, c->dx.p, 1.0, n);
      G2OC_LAUNCH_CHECK();
    }
    return G2OC_OK;
  }

  const int* hpl_row() { return c->hpl_row.p; }

  // x_l = Dinv (r_l - sum_a B_a^T x_p(row a)) (block_solver.hpp:449-474)
  int backsub(const double* rl, const double* xp, double* xl) {
    const Structure& S = c->S;
    cudaStream_t st = c->stream;
    if (S.Pf == 0) return G2OC_OK;
    if (S.lm_warp_ok) {
      const int nch = (int)S.lm_chunk_ptr.size() - 1;
      G2OC_K(K_BACKSUB) ba_backsub_warp<Real><<<cdiv(nch, 8), 256, 0, st>>>(
          c->e_hpl.p, c->hpl_row.p, c->lm_chunk_ptr.p, nch, c->e_lm.p, hpl.p, dinv.p, rl, xp, xl);
    } else {
      G2OC_K(K_BACKSUB) ba_backsub<Real><<<cdiv(S.Pf, 128), 128, 0, st>>>(c->hb_ptr.p, c->hpl_row.p, S.Pf, hpl.p,
                                                                         dinv.p, rl, xp, xl);
    }
    G2OC_LAUNCH_CHECK();
    return G2OC_OK;
  }

  template <typename T>
  static void to_double(const std::vector<T>& in, double* out) {
    for (size_t i = 0; i < in.size(); ++i) out[i] = (double)in[i];
  }

  int get_hessian(double* hpp_out, double* hll_out, double* hpl_out) override {
    const Structure& S = c->S;
    G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (hpp_out) {
      std::vector<Real> h(hpp.n);
      G2OC_CUDA_TRY(cudaMemcpy(h.data(), hpp.p, hpp.bytes(), cudaMemcpyDeviceToHost));
      if (S.ba && S.npp > 0) {  // storage (diagonal blocks, then pose-pose blocks) to hpp_rc order
        for (size_t i = 0; i < S.hpp_store.size(); ++i)
          for (int e = 0; e < 36; ++e) hpp_out[i * 36 + e] = (double)h[(size_t)S.hpp_store[i] * 36 + e];
      } else {
        to_double(h, hpp_out);
      }
    }
    if (S.ba && hll_out && S.Pf > 0) {
      std::vector<Real> h((size_t)S.Pf * 6);
      G2OC_CUDA_TRY(cudaMemcpy(h.data(), hll.p, h.size() * sizeof(Real), cudaMemcpyDeviceToHost));
      for (int l = 0; l < S.Pf; ++l) {
        const Real* a = h.data() + (size_t)l * 6;
        double* o = hll_out + (size_t)l * 9;
        o[0] = a[0]; o[1] = a[1]; o[2] = a[2];
        o[3] = a[1]; o[4] = a[3]; o[5] = a[4];
        o[6] = a[2]; o[7] = a[4]; o[8] = a[5];
      }
    }
    if (S.ba && hpl_out && !S.hpl_rc.empty()) {
      std::vector<Real> h(S.hpl_rc.size() / 2 * 18);
      G2OC_CUDA_TRY(cudaMemcpy(h.data(), hpl.p, h.size() * sizeof(Real), cudaMemcpyDeviceToHost));
      to_double(h, hpl_out);
    }
    return G2OC_OK;
  }

  int batch_lambda_init(double user_lambda, double tau) override {
    G2OC_K(K_LM_CONTROL) win_lambda_init<Real, 256><<<c->nw, 256, 0, c->stream>>>(hpp.p, hll.p, c->windev(),
                                                                                 c->win_state.p, user_lambda, tau);
    G2OC_LAUNCH_CHECK();
    return G2OC_OK;
  }

  // one launch of the dense per-window solve with THREADS threads per window
  template <int T>
  int launch_win_chol(const int* list, int nlist, int nmax) {
    if (nlist == 0) return G2OC_OK;
    const size_t smem = win_chol_smem(nmax);
    if (smem > 48 * 1024) G2OC_TRY(raise_dyn_smem((const void*)win_chol_solve<T>, smem));
    G2OC_K(K_CHOLESKY) win_chol_solve<T><<<nlist, T, smem, c->stream>>>(list, nlist, c->windev(), c->rhs.p, c->xs.p,
                                                                          c->win_scratch.p, c->win_state.p);
    G2OC_LAUNCH_CHECK();
    return G2OC_OK;
  }
  int launch_win_chol_t(int t, const int* list, int nlist, int nmax) {
    if (t == 0) return launch_win_chol<128>(list, nlist, nmax);
    if (t == 1) return launch_win_chol<256>(list, nlist, nmax);
    return launch_win_chol<512>(list, nlist, nmax);
  }

  // Times the dense solve with 128 / 256 / 512 threads per window on each
  // window-size class (n < 96, < 192, >= 192 unknowns) and keeps the fastest;
  // the windows are then solved in three launches, one per thread count.
  int batch_autotune() {
    const Structure& S = c->S;
    (void)S;
    cudaStream_t st = c->stream;
    // windows largest first within a launch (the long factorizations start
    // in the first wave)
    auto wn = [&](int w) { return 6 * (c->win_cam_h[w + 1] - c->win_cam_h[w]); };
    auto by_size = [&](std::vector<int>& v) {
      std::stable_sort(v.begin(), v.end(), [&](int a, int b) { return wn(a) > wn(b); });
    };
    std::vector<int> cls[3];
    int cls_nmax[3] = {0, 0, 0};
    for (int w = 0; w < c->nw; ++w) {
      const int n = wn(w);
      const int k = n < 96 ? 0 : n < 192 ? 1 : 2;
      cls[k].push_back(w);
      cls_nmax[k] = std::max(cls_nmax[k], n);
    }
    for (auto& v : cls) by_size(v);
    DBuf<int> tmp;
    // the solve factors the windows' matrices in place: every trial starts
    // from a copy of them, and the copy is put back for the real solve
    DBuf<double> saved;
    const size_t mbytes = c->win_scratch.bytes();
    G2OC_TRY(saved.alloc(c->win_scratch.n));
    G2OC_CUDA_TRY(cudaMemcpyAsync(saved.p, c->win_scratch.p, mbytes, cudaMemcpyDeviceToDevice, st));
    auto restore = [&]() -> int {
      G2OC_CUDA_TRY(cudaMemcpyAsync(c->win_scratch.p, saved.p, mbytes, cudaMemcpyDeviceToDevice, st));
      return G2OC_OK;
    };
    cudaEvent_t a, b;
    G2OC_CUDA_TRY(cudaEventCreate(&a));
    G2OC_CUDA_TRY(cudaEventCreate(&b));
    std::vector<int> lists[3];
    c->win_threads.assign(c->nw, 0);
    for (int k = 0; k < 3; ++k) {
      if (cls[k].empty()) continue;
      G2OC_TRY(tmp.upload(cls[k], st));
      int best = 1;
      float best_ms = 1e30f;
      for (int t = 0; t < 3; ++t) {
        G2OC_TRY(restore());
        G2OC_TRY(launch_win_chol_t(t, tmp.p, (int)cls[k].size(), cls_nmax[k]));  // warm
        G2OC_TRY(restore());
        G2OC_CUDA_TRY(cudaEventRecord(a, st));
        G2OC_TRY(launch_win_chol_t(t, tmp.p, (int)cls[k].size(), cls_nmax[k]));
        G2OC_CUDA_TRY(cudaEventRecord(b, st));
        G2OC_CUDA_TRY(cudaEventSynchronize(b));
        float ms = 0.f;
        G2OC_CUDA_TRY(cudaEventElapsedTime(&ms, a, b));
        if (ms < best_ms) {
          best_ms = ms;
          best = t;
        }
      }
      c->win_threads_of_class[k] = 128 << best;
      for (int w : cls[k]) {
        lists[best].push_back(w);
        c->win_threads[w] = 128 << best;
      }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    G2OC_TRY(restore());
    for (int t = 0; t < 3; ++t) {
      by_size(lists[t]);
      c->win_list_n[t] = (int)lists[t].size();
      c->win_list_nmax[t] = lists[t].empty() ? 0 : wn(lists[t][0]);
      G2OC_TRY(c->win_list[t].upload(lists[t].empty() ? std::vector<int>{0} : lists[t], st));
    }
    G2OC_CUDA_TRY(cudaStreamSynchronize(st));
    c->win_tuned = true;
    return G2OC_OK;
  }

  int batch_solve(bool autotune) override {
    const Structure& S = c->S;
    cudaStream_t st = c->stream;
    if (c->win_sparse)
      G2OC_CUDA_TRY(cudaMemsetAsync(c->win_scratch.p, 0, c->win_scratch.bytes(), st));
    G2OC_TRY(schur(0.0, c->rhs.p, c->lam_c.p, c->lam_l.p, false, true));
    if (autotune && !c->win_tuned) G2OC_TRY(batch_autotune());
    for (int t = 0; t < 3; ++t)
      G2OC_TRY(launch_win_chol_t(t, c->win_list[t].p, c->win_list_n[t], c->win_list_nmax[t]));
    G2OC_CUDA_TRY(cudaMemcpyAsync(c->x.p, c->xs.p, (size_t)S.Cf * 6 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    return backsub(c->b.p + (size_t)S.Cf * 6, c->xs.p, c->x.p + (size_t)S.Cf * 6);
  }

  int solve_rhs(const double* rhs, double* out, bool reuse_schur = false) override {
    const Structure& S = c->S;
    cudaStream_t st = c->stream;
    if (!(S.ba && S.schur) || S.Cf == 0) {
      set_error("the adjoint solve needs a bundle adjustment with free cameras and landmarks");
      return G2OC_ERR_NOT_SUPPORTED;
    }
    const bool use_chol = c->prm.linear_solver == G2OC_LINEAR_CHOLESKY;
    if (!reuse_schur) G2OC_TRY(schur(0.0, nullptr, nullptr, nullptr, !use_chol && tile_pcg_used()));
    const double* rp = rhs;
    const double* rl = rhs + (size_t)S.Cf * 6;
    G2OC_TRY(schur_rhs_from(rp, rl, c->rhs.p));
    int ok = 1;
    if (use_chol) {
      G2OC_TRY(chol_solve(Sval.p, c->rhs.p, c->xs.p, &ok));
      if (!ok) {
        set_error("adjoint solve: the reduced system is not positive definite");
        return G2OC_ERR_NOT_PD;
      }
    } else {
      // no carried threshold (LinearSolverPCG::_residual) between these solves
      static const double kNoCarry = -1.0;
      G2OC_CUDA_TRY(cudaMemcpyAsync(&c->pcg.p->residual_carry, &kNoCarry, sizeof(double), cudaMemcpyHostToDevice, st));
      G2OC_TRY(pcg_solve(Sval.p, c->rhs.p, c->xs.p, false));
    }
    G2OC_CUDA_TRY(cudaMemcpyAsync(out, c->xs.p, (size_t)S.Cf * 6 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    return backsub(rl, c->xs.p, out + (size_t)S.Cf * 6);
  }

  int schur_export(double lambda, double* S_out, double* bs_out) override {
    const Structure& S = c->S;
    if (!S.ba || !S.schur) {
      set_error("the graph has no Schur complement (no marginalized vertices)");
      return G2OC_ERR_NOT_SUPPORTED;
    }
    G2OC_TRY(schur(lambda, c->rhs.p));
    G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (S_out) {
      std::vector<Real> h((size_t)S.sys_nnzb * 36);
      G2OC_CUDA_TRY(cudaMemcpy(h.data(), Sval.p, h.size() * sizeof(Real), cudaMemcpyDeviceToHost));
      for (int k = 0; k < S.sys_nnzb; ++k) {
        const int r = S.sys_brow[k], rb = S.sys_rptr[r], nblk = S.sys_rptr[r + 1] - rb;
        for (int e = 0; e < 36; ++e)
          S_out[(size_t)S.sys_perm[k] * 36 + e] = (double)h[sys_offset<6>(rb, nblk, k - rb, e)];
      }
    }
    if (bs_out) G2OC_CUDA_TRY(cudaMemcpy(bs_out, c->rhs.p, (size_t)S.Cf * 6 * sizeof(double), cudaMemcpyDeviceToHost));
    return G2OC_OK;
  }
};

// BlockSolver<9,3> of the BAL path (g2o/examples/bal/bal_example.cpp:227-250,
// g2o/core/block_solver.hpp): landmark and camera passes of buildSystem, the
// Schur complement of the 9 x 9 camera blocks, block-Jacobi PCG
// (LinearSolverPCG) or the dense Cholesky on it, landmark back-substitution.
// FP64.
struct BalEngine final : EngineBase {
  g2oc_ctx* c;
  DBuf<double> hpp, hll, hpl, dinv, Y, Sval, minv, r, s, d, tbuf, cpart, part;
  // the Schur complement's work plan: chunks (block, first item, end, slot or
  // -1) and the blocks cut into several chunks (block, first slot, slots)
  DBuf<int4> chunks, reds, cch;
  DBuf<int> cch_ptr;
  DBuf<double> ccpart;
  int ncch = 0;
  DBuf<int2> pairs;  // co-observation pairs as absolute Hpl block indices (a of the row camera, b)
  DBuf<double> rpart;  // the diagonal chunks' sums of Y_a b_l (reduced right-hand side), 9 per slot
  int nchunks = 0, nreds = 0;
  explicit BalEngine(g2oc_ctx* ctx) : c(ctx) {}

  int plan_schur() {
    const Structure& S = c->S;
    std::vector<int4> ch, rd;
    int nslots = 0;
    for (int k = 0; k < S.sys_nnzb; ++k) {
      const int r = S.sys_brow[k];
      const bool diag = S.sys_rcol[k] == r;
      const int q0 = diag ? S.hc_ptr[r] : S.s_pair_ptr[k];
      const int q1 = diag ? S.hc_ptr[r + 1] : S.s_pair_ptr[k + 1];
      const int n = std::max(1, (q1 - q0 + kBalChunk - 1) / kBalChunk);
      if (n == 1) {
        ch.push_back(make_int4(k, q0, q1, -1));
        continue;
      }
      rd.push_back(make_int4(k, nslots, n, 0));
      for (int t = 0; t < n; ++t)
        ch.push_back(make_int4(k, q0 + t * kBalChunk, std::min(q1, q0 + (t + 1) * kBalChunk), nslots++));
    }
    nchunks = (int)ch.size();
    nreds = (int)rd.size();
    {
      std::vector<int2> pa(S.s_pairs.size() / 2 + 1, make_int2(0, 0));
      for (int k = 0; k < S.sys_nnzb; ++k) {
        const int r = S.sys_brow[k];
        if (S.sys_rcol[k] == r) continue;
        for (int q = S.s_pair_ptr[k]; q < S.s_pair_ptr[k + 1]; ++q)
          pa[q] = make_int2(S.hc_blk[S.hc_ptr[r] + S.s_pairs[2 * (size_t)q]], S.s_pairs[2 * (size_t)q + 1]);
      }
      G2OC_TRY(pairs.upload(pa, c->stream));
    }
    // the camera pass: each camera's edges in chunks
    {
      std::vector<int4> cc;
      std::vector<int> cp(S.Cf + 1, 0);
      for (int h = 0; h < S.Cf; ++h) {
        const int j0 = S.c_ptr[h], j1 = S.c_ptr[h + 1];
        if (j1 == j0) cc.push_back(make_int4(h, j0, j1, 0));
        for (int j = j0; j < j1; j += kBalCamChunk) cc.push_back(make_int4(h, j, std::min(j1, j + kBalCamChunk), 0));
        cp[h + 1] = (int)cc.size();
      }
      ncch = (int)cc.size();
      G2OC_TRY(cch.upload(cc.empty() ? std::vector<int4>{make_int4(0, 0, 0, 0)} : cc, c->stream));
      G2OC_TRY(cch_ptr.upload(cp, c->stream));
      G2OC_TRY(ccpart.alloc((size_t)ncch * 54 + 1));
    }
    G2OC_TRY(chunks.upload(ch.empty() ? std::vector<int4>{make_int4(0, 0, 0, -1)} : ch, c->stream));
    G2OC_TRY(reds.upload(rd.empty() ? std::vector<int4>{make_int4(0, 0, 0, 0)} : rd, c->stream));
    G2OC_TRY(part.alloc((size_t)nslots * 81 + 1));
    G2OC_TRY(rpart.alloc((size_t)nslots * 9 + 1));
    return G2OC_OK;
  }

  int alloc() override {
    const Structure& S = c->S;
    const size_t nh = S.hpl_rc.size() / 2;
    G2OC_TRY(hpp.alloc((size_t)S.Cf * 81 + 1));
    G2OC_TRY(hll.alloc((size_t)S.Pf * 6 + 1));
    G2OC_TRY(hpl.alloc(nh * kBalBlk + 1));
    G2OC_TRY(dinv.alloc((size_t)S.Pf * 9 + 1));
    G2OC_TRY(Y.alloc(nh * kBalBlk + 1));
    G2OC_TRY(Sval.alloc((size_t)S.sys_nnzb * 81 + 1));
    const size_t n = (size_t)S.Cf * 9;
    G2OC_TRY(minv.alloc((size_t)S.Cf * 81 + 1));
    G2OC_TRY(r.alloc(n + 1));
    G2OC_TRY(s.alloc(n + 1));
    G2OC_TRY(d.alloc(n + 1));
    G2OC_TRY(tbuf.alloc((size_t)S.sys_nnzb * 9 + 1));
    G2OC_TRY(cpart.alloc(S.sys_chunk_row.size() * 9 + 1));
    return plan_schur();
  }

  SysDev<double> sys(const double* val) {
    SysDev<double> A;
    A.nb = c->S.sys_nb;
    A.nnzb = c->S.sys_nnzb;
    A.rptr = c->sys_rptr.p;
    A.rcol = c->sys_rcol.p;
    A.brow = c->sys_brow.p;
    A.diag = c->sys_diag.p;
    A.cptr = c->sys_cptr.p;
    A.cblk = c->sys_cblk.p;
    A.perm = c->sys_perm.p;
    A.val = val;
    return A;
  }

  int build_system() override {
    const Structure& S = c->S;
    cudaStream_t st = c->stream;
    if (S.Pf > 0 && S.lm_warp_ok) {
      const int nch = (int)S.lm_chunk_ptr.size() - 1;
      G2OC_K(K_LANDMARK_PASS) bal_landmark_warp<<<cdiv(nch, kBalLmWarps), kBalLmWarps * 32, 0, st>>>(
          c->ba_edges(), c->ba_vertices(), c->lm_chunk_ptr.p, nch, c->e_lm.p, hll.p, hpl.p,
          c->b.p + (size_t)S.Cf * 9);
      G2OC_LAUNCH_CHECK();
    } else if (S.Pf > 0) {
      G2OC_K(K_LANDMARK_PASS) bal_landmark_pass<<<cdiv(S.Pf, 128), 128, 0, st>>>(
          c->ba_edges(), c->ba_vertices(), c->l_ptr.p, S.Pf, hll.p, hpl.p, c->b.p + (size_t)S.Cf * 9);
      G2OC_LAUNCH_CHECK();
    }
    if (S.Cf > 0 && ncch > 0) {
      G2OC_K(K_CAMERA_PASS) bal_camera_chunks<128><<<ncch, 128, 0, st>>>(c->ba_cam_edges(), c->ba_vertices(), cch.p,
                                                                         ccpart.p);
      G2OC_K(K_CAMERA_PASS) bal_camera_reduce<<<cdiv(S.Cf * 54, 256), 256, 0, st>>>(S.Cf, cch_ptr.p, ccpart.p, hpp.p,
                                                                                    c->b.p);
      G2OC_LAUNCH_CHECK();
    }
    return G2OC_OK;
  }

  int max_diag() override {
    const Structure& S = c->S;
    cudaStream_t st = c->stream;
    G2OC_K(K_MAX_DIAG) bal_max_diag<<<kRedBlocks, 256, 0, st>>>(hpp.p, S.Cf, hll.p, S.Pf, c->partials.p);
    G2OC_LAUNCH_CHECK();
    G2OC_K(K_REDUCE) finalize_max_kernel<<<1, 256, 0, st>>>(c->partials.p, kRedBlocks, &c->sc.p->max_diag);
    G2OC_LAUNCH_CHECK();
    return G2OC_OK;
  }

  int multiply_hessian(const double* src, double* dst) override {
    const int n = c->vec_size();
    if (n <= 0) return G2OC_OK;
    G2OC_K(K_LM_CONTROL) bal_hpp_mult<<<cdiv(n, 256), 256, 0, c->stream>>>(c->S.Cf, hpp.p, src, dst, n);
    G2OC_LAUNCH_CHECK();
    return G2OC_OK;
  }

  // Dinv, Y and S = Hpp + lambda - Hpl (H_ll + lambda)^-1 Hpl^T with the
  // reduced right-hand side bs (optional)
  int schur(double lambda, double* bs) {
    const Structure& S = c->S;
    cudaStream_t st = c->stream;
    if (S.Pf > 0) {
      G2OC_K(K_SCHUR_LANDMARK) bal_schur_landmark<<<cdiv(S.Pf, 128), 128, 0, st>>>(hll.p, S.Pf, lambda, dinv.p,
                                                                                c->flag.p);
      G2OC_LAUNCH_CHECK();
      const int nh = (int)(S.hpl_rc.size() / 2);
      if (nh > 0) {
        G2OC_K(K_SCHUR_LANDMARK) bal_schur_y<<<cdiv(nh, kBalYBlocks), kBalYBlocks, 0, st>>>(
            nh, c->hpl_col.p, hpl.p, dinv.p, c->b.p + (size_t)S.Cf * 9, Y.p);
        G2OC_LAUNCH_CHECK();
      }
    }
    if (S.Cf == 0) return G2OC_OK;
    G2OC_K(K_SCHUR_BLOCKS) bal_schur_chunks<<<cdiv(nchunks, kBalChunkWarps), kBalChunkWarps * 32, 0, st>>>(
        nchunks, chunks.p, c->sys_brow.p, c->sys_rptr.p, c->sys_rcol.p, pairs.p, c->hc_blk.p, hpp.p, hpl.p, Y.p,
        lambda, Sval.p, part.p, c->b.p, bs, rpart.p);
    G2OC_LAUNCH_CHECK();
    if (nreds > 0) {
      G2OC_K(K_SCHUR_RHS) bal_schur_reduce<<<cdiv((long long)nreds * 81, 256), 256, 0, st>>>(
          nreds, reds.p, c->sys_brow.p, c->sys_rptr.p, c->sys_rcol.p, hpp.p, lambda, part.p, Sval.p, rpart.p, c->b.p,
          bs);
      G2OC_LAUNCH_CHECK();
    }
    return G2OC_OK;
  }

  int backsub(const double* rl, const double* xp, double* xl) {
    const Structure& S = c->S;
    if (S.Pf == 0) return G2OC_OK;
    if (S.lm_warp_ok) {
      const int nch = (int)S.lm_chunk_ptr.size() - 1;
      G2OC_K(K_BACKSUB) bal_backsub_warp<<<cdiv(nch, 8), 256, 0, c->stream>>>(
          c->e_hpl.p, c->hpl_row.p, c->lm_chunk_ptr.p, nch, c->e_lm.p, hpl.p, dinv.p, rl, xp, xl);
    } else {
      G2OC_K(K_BACKSUB) bal_backsub<<<cdiv(S.Pf, 128), 128, 0, c->stream>>>(c->hb_ptr.p, c->hpl_row.p, S.Pf, hpl.p,
                                                                            dinv.p, rl, xp, xl);
    }
    G2OC_LAUNCH_CHECK();
    return G2OC_OK;
  }

  int solve(double lambda) override {
    const Structure& S = c->S;
    cudaStream_t st = c->stream;
    int ok = 1;
    const double* bl = c->b.p + (size_t)S.Cf * 9;
    if (S.Cf == 0) {
      // every camera fixed: x_l = (H_ll + lambda I)^-1 b_l
      G2OC_CUDA_TRY(cudaMemsetAsync(c->x.p, 0, c->x.bytes(), st));
      G2OC_TRY(schur(lambda, nullptr));
      G2OC_TRY(backsub(bl, c->xs.p, c->x.p));
    } else {
      cudaEvent_t ts = c->cur_stats ? c->mark() : nullptr;
      G2OC_TRY(schur(lambda, c->rhs.p));
      if (ts) c->span(ts, &c->cur_stats->time_schur_complement, &c->cur_stats->time_linear_solver);
      SysDev<double> A = sys(Sval.p);
      if (c->prm.linear_solver == G2OC_LINEAR_CHOLESKY) {
        if (!c->chol) {
          std::unique_ptr<CholPlan> P(new CholPlan());
          G2OC_TRY(chol_plan_build(*P, S.sys_nb, 9, S.schur ? S.schur_rc : S.hpp_rc, false, st));
          c->chol = std::move(P);
        }
        G2OC_TRY(g2oc::chol_solve<double>(*c->chol, st, A, c->rhs.p, c->xs.p, &ok, &c->kcount[K_CHOLESKY]));
      } else {
        G2OC_K(K_PCG_DIAG_INV) pcg_diag_inv_lanes<double, 9><<<cdiv(A.nb, 3 * 4), 128, 0, st>>>(A, minv.p,
                                                                                             c->flag.p);
        G2OC_LAUNCH_CHECK();
        const int rc = run_pcg_persistent<double, 9>(c, A, minv.p, c->rhs.p, c->xs.p, r.p, s.p, d.p, tbuf.p,
                                                     cpart.p, false);
        if (rc != G2OC_OK) return rc;
      }
      G2OC_CUDA_TRY(cudaMemcpyAsync(c->x.p, c->xs.p, (size_t)S.Cf * 9 * sizeof(double), cudaMemcpyDeviceToDevice,
                                    st));
      G2OC_TRY(backsub(bl, c->xs.p, c->x.p + (size_t)S.Cf * 9));
    }
    G2OC_K(K_LM_CONTROL) set_solve_ok<<<1, 32, 0, st>>>(c->sc.p, ok);
    G2OC_LAUNCH_CHECK();
    return G2OC_OK;
  }

  int get_hessian(double* hpp_out, double* hll_out, double* hpl_out) override {
    const Structure& S = c->S;
    G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (hpp_out && S.Cf > 0)
      G2OC_CUDA_TRY(cudaMemcpy(hpp_out, hpp.p, (size_t)S.Cf * 81 * sizeof(double), cudaMemcpyDeviceToHost));
    if (hll_out && S.Pf > 0) {
      std::vector<double> h((size_t)S.Pf * 6);
      G2OC_CUDA_TRY(cudaMemcpy(h.data(), hll.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
      for (int l = 0; l < S.Pf; ++l) {
        const double* a = h.data() + (size_t)l * 6;
        double* o = hll_out + (size_t)l * 9;
        o[0] = a[0]; o[1] = a[1]; o[2] = a[2];
        o[3] = a[1]; o[4] = a[3]; o[5] = a[4];
        o[6] = a[2]; o[7] = a[4]; o[8] = a[5];
      }
    }
    if (hpl_out && !S.hpl_rc.empty()) {
      const size_t nh = S.hpl_rc.size() / 2;
      std::vector<double> h(nh * kBalBlk);
      G2OC_CUDA_TRY(cudaMemcpy(h.data(), hpl.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
      for (size_t a = 0; a < nh; ++a)
        for (int r = 0; r < 9; ++r)
          for (int cc = 0; cc < 3; ++cc) hpl_out[a * 27 + r * 3 + cc] = h[a * kBalBlk + bal_bt(r, cc)];
    }
    return G2OC_OK;
  }

  int schur_export(double lambda, double* S_out, double* bs_out) override {
    const Structure& S = c->S;
    if (!S.schur) {
      set_error("the graph has no Schur complement (no marginalized vertices)");
      return G2OC_ERR_NOT_SUPPORTED;
    }
    G2OC_TRY(schur(lambda, c->rhs.p));
    G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (S_out) {
      std::vector<double> h((size_t)S.sys_nnzb * 81);
      G2OC_CUDA_TRY(cudaMemcpy(h.data(), Sval.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
      for (int k = 0; k < S.sys_nnzb; ++k) {
        const int rr = S.sys_brow[k], rb = S.sys_rptr[rr], nblk = S.sys_rptr[rr + 1] - rb;
        for (int e = 0; e < 81; ++e) S_out[(size_t)S.sys_perm[k] * 81 + e] = h[sys_offset<9>(rb, nblk, k - rb, e)];
      }
    }
    if (bs_out) G2OC_CUDA_TRY(cudaMemcpy(bs_out, c->rhs.p, (size_t)S.Cf * 9 * sizeof(double), cudaMemcpyDeviceToHost));
    return G2OC_OK;
  }

  int solve_rhs(const double*, double*, bool) override {
    set_error("the adjoint solve is built for the SE3 bundle adjustment, not for BAL cameras");
    return G2OC_ERR_NOT_SUPPORTED;
  }
  int batch_lambda_init(double, double) override {
    set_error("batched windows take SE3 bundle adjustments");
    return G2OC_ERR_NOT_SUPPORTED;
  }
  int batch_solve(bool) override {
    set_error("batched windows take SE3 bundle adjustments");
    return G2OC_ERR_NOT_SUPPORTED;
  }
};

// ------------------------------------------------------------ driver ops
static int chi2_to(g2oc_ctx* c, double* out_plain, double* out_robust) {
  const Structure& S = c->S;
  cudaStream_t st = c->stream;
  if (S.bal)
    G2OC_K(K_CHI2) bal_chi2_kernel<<<kChi2Blocks, 256, 0, st>>>(c->ba_edges(), c->ba_vertices(), c->partials.p);
  else if (S.ba && S.D == 3)
    G2OC_K(K_CHI2) st_chi2_kernel<<<kChi2Blocks, 256, 0, st>>>(c->ba_edges(), c->ba_vertices(), c->partials.p);
  else if (S.ba) G2OC_K(K_CHI2) ba_chi2_kernel<<<kChi2Blocks, 256, 0, st>>>(c->ba_edges(), c->ba_vertices(), c->partials.p);
  else if (S.pose_type == G2OC_POSE_SE2)
    G2OC_K(K_CHI2) pg_chi2_kernel<G2OC_POSE_SE2><<<kRedBlocks, 256, 0, st>>>(c->pose.p, c->pg_edges(), c->partials.p);
  else if (S.pose_type == G2OC_POSE_SE3EXPMAP)
    G2OC_K(K_CHI2) pg_chi2_kernel<G2OC_POSE_SE3EXPMAP><<<kRedBlocks, 128, 0, st>>>(c->pose.p, c->pg_edges(), c->partials.p);
  else G2OC_K(K_CHI2) pg_chi2_kernel<G2OC_POSE_SE3><<<kRedBlocks, 128, 0, st>>>(c->pose.p, c->pg_edges(), c->partials.p);
  G2OC_LAUNCH_CHECK();
  int nparts = S.ba ? kChi2Blocks : kRedBlocks;
  if (S.ba && c->pose_edges()) {
    // the pose edge set's chi2 in the partials after the projection edges'
    G2OC_K(K_CHI2) ba_unpack_poses<<<cdiv((long long)S.C * 7, 256), 256, 0, st>>>(S.C, c->pose.p, c->pgpose.p);
    G2OC_K(K_CHI2) pg_chi2_kernel<G2OC_POSE_SE3EXPMAP><<<kRedBlocks, 128, 0, st>>>(c->pgpose.p, c->ba_pose_edges(),
                                                                                 c->partials.p + 2 * nparts);
    G2OC_LAUNCH_CHECK();
    nparts += kRedBlocks;
  }
  G2OC_TRY(finalize_sum(c, nparts, 2, out_plain, out_robust));
  G2OC_TRY(shard_reduce(c, out_plain, 1, G2OC_DT_F64, G2OC_RED_SUM));
  return shard_reduce(c, out_robust, 1, G2OC_DT_F64, G2OC_RED_SUM);
}

static int oplus(g2oc_ctx* c) {
  const Structure& S = c->S;
  cudaStream_t st = c->stream;
  if (S.bal)
    G2OC_K(K_OPLUS) bal_oplus<<<cdiv((long long)S.Cf * 9 + (long long)S.Pf * 3, 256), 256, 0, st>>>(
        c->ba_vertices(), S.Cf, S.Pf, c->x.p, c->flag.p);
  else if (S.ba) G2OC_K(K_OPLUS) ba_oplus<<<cdiv(S.Cf + S.Pf, 256), 256, 0, st>>>(c->ba_vertices(), S.Cf, S.Pf, c->x.p, c->flag.p);
  else if (S.pose_type == G2OC_POSE_SE2)
    G2OC_K(K_OPLUS) pg_oplus<G2OC_POSE_SE2><<<cdiv(S.Cf, 128), 128, 0, st>>>(c->pose.p, c->free_pose.p, S.Cf, c->x.p,
                                                             c->oplus_count.p, c->flag.p);
  else if (S.pose_type == G2OC_POSE_SE3EXPMAP)
    G2OC_K(K_OPLUS) pg_oplus<G2OC_POSE_SE3EXPMAP><<<cdiv(S.Cf, 128), 128, 0, st>>>(c->pose.p, c->free_pose.p, S.Cf,
                                                                                  c->x.p, c->oplus_count.p, c->flag.p);
  else G2OC_K(K_OPLUS) pg_oplus<G2OC_POSE_SE3><<<cdiv(S.Cf, 128), 128, 0, st>>>(c->pose.p, c->free_pose.p, S.Cf, c->x.p,
                                                                c->oplus_count.p, c->flag.p);
  G2OC_LAUNCH_CHECK();
  return G2OC_OK;
}

static int push(g2oc_ctx* c) {
  G2OC_CUDA_TRY(cudaMemcpyAsync(c->pose_bak.p, c->pose.p, c->pose.bytes(), cudaMemcpyDeviceToDevice, c->stream));
  if (c->point.n)
    G2OC_CUDA_TRY(cudaMemcpyAsync(c->point_bak.p, c->point.p, c->point.bytes(), cudaMemcpyDeviceToDevice, c->stream));
  return G2OC_OK;
}

static int pop(g2oc_ctx* c) {
  G2OC_CUDA_TRY(cudaMemcpyAsync(c->pose.p, c->pose_bak.p, c->pose.bytes(), cudaMemcpyDeviceToDevice, c->stream));
  if (c->point.n)
    G2OC_CUDA_TRY(cudaMemcpyAsync(c->point.p, c->point_bak.p, c->point.bytes(), cudaMemcpyDeviceToDevice, c->stream));
  return G2OC_OK;
}

static int reset_pcg(g2oc_ctx* c);

// DevScalars and PcgState after the queued work (the one wait of an LM
// trial): PCG iterations since the last read go to stv
static int read_state(g2oc_ctx* c, DevScalars* h, g2oc_iteration_stats* stv) {
  if (!c->ev_read) {
    G2OC_TRY(c->h_sc.resize(1));
    G2OC_TRY(c->h_pcg.resize(1));
    G2OC_CUDA_TRY(cudaEventCreateWithFlags(&c->ev_read, cudaEventDisableTiming));
  }
  G2OC_CUDA_TRY(cudaMemcpyAsync(c->h_sc.data(), c->sc.p, sizeof(DevScalars), cudaMemcpyDeviceToHost, c->stream));
  G2OC_CUDA_TRY(cudaMemcpyAsync(c->h_pcg.data(), c->pcg.p, sizeof(PcgState), cudaMemcpyDeviceToHost, c->stream));
  G2OC_CUDA_TRY(cudaEventRecord(c->ev_read, c->stream));
  // the host polls (the trial's work is a few hundred microseconds at most;
  // a blocking wait would add its wake-up latency to every trial)
  cudaError_t q;
  while ((q = cudaEventQuery(c->ev_read)) == cudaErrorNotReady) {
  }
  G2OC_CUDA_TRY(q);
  cudaGetLastError();  // the not-ready answers are not errors of later launches
  *h = *c->h_sc.data();
  const PcgState ps = *c->h_pcg.data();
  if (ps.sync_error) {
    G2OC_TRY(reset_pcg(c));
    set_error("PCG: a grid barrier wait ran out");
    return G2OC_ERR_TIMEOUT;
  }
  if (stv) stv->iterations_linear_solver += (int)(ps.total_iterations - c->pcg_seen);
  c->pcg_seen = ps.total_iterations;
  c->lambda_host = h->lambda;
  return G2OC_OK;
}

// OptimizationAlgorithmLevenberg::solve (optimization_algorithm_levenberg.cpp:60-153).
// The errors of the state an iteration starts from are those of the trial
// accepted last (same estimates, same kernel), so their chi2 is carried over
// instead of recomputed; the host waits for the device once per trial.
static int lm_iteration(g2oc_ctx* c, int iteration, g2oc_iteration_stats* stv, int* result) {
  cudaStream_t st = c->stream;
  DevScalars* sc = c->sc.p;
  c->cur_stats = stv;
  cudaEvent_t t0 = c->mark();
  if (!c->chi2_carry) G2OC_TRY(chi2_to(c, &sc->chi2_plain, &sc->chi2_current));
  c->span(t0, &stv->time_residuals);
  t0 = c->mark();
  G2OC_TRY(c->eng->build_system());
  c->system_built = true;
  c->span(t0, &stv->time_quadratic_form);
  DevScalars h{};
  if (iteration == 0) {
    G2OC_TRY(c->eng->max_diag());
    G2OC_K(K_LM_CONTROL) lm_init_lambda<<<1, 32, 0, st>>>(sc, c->prm.initial_lambda, c->prm.tau);
    G2OC_LAUNCH_CHECK();
    G2OC_TRY(read_state(c, &h, stv));
  }
  const int n = c->vec_size();
  double rho = 0;
  int qmax = 0;
  bool accepted = false;
  do {
    G2OC_TRY(push(c));
    t0 = c->mark();
    G2OC_TRY(c->eng->solve(c->lambda_host));
    c->span(t0, &stv->time_linear_solver);
    t0 = c->mark();
    G2OC_TRY(oplus(c));
    c->span(t0, &stv->time_update);
    G2OC_TRY(chi2_to(c, &sc->chi2_temp_plain, &sc->chi2_temp));
    {
      // sharded: the camera entries are the same on every rank, their lambda
      // term (and the 1e-3) counted on rank 0 only; b's camera part is each
      // rank's share
      const bool other = c->shard_world > 1 && c->shard_rank != 0;
      G2OC_K(K_LM_CONTROL) lm_scale_partials<<<kRedBlocks, 256, 0, st>>>(c->x.p, c->b.p, n, sc, c->partials.p,
                                                                         other ? c->S.Cf * 6 : 0);
      G2OC_LAUNCH_CHECK();
      G2OC_TRY(finalize_sum(c, kRedBlocks, 1, &sc->scale, nullptr, other ? 0.0 : 1e-3));
      G2OC_TRY(shard_reduce(c, &sc->scale, 1, G2OC_DT_F64, G2OC_RED_SUM));
    }
    G2OC_K(K_LM_CONTROL) lm_decide<<<1, 32, 0, st>>>(sc);
    G2OC_LAUNCH_CHECK();
    G2OC_TRY(read_state(c, &h, stv));
    rho = h.rho;
    accepted = h.accept != 0;
    if (!accepted) {
      G2OC_TRY(pop(c));
      if (!std::isfinite(h.lambda)) {
        qmax++;
        stv->levenberg_iterations = qmax;
        break;
      }
    }
    qmax++;
    stv->levenberg_iterations = qmax;
  } while (rho < 0 && qmax < c->prm.max_trials_after_failure);
  c->chi2_carry = accepted;
  stv->lambda = h.lambda;
  stv->chi2 = h.chi2_current;  // activeRobustChi2 of the state the iteration ends in (G2OBatchStatistics::chi2)
  c->resolve_spans();
  c->cur_stats = nullptr;
  if (qmax == c->prm.max_trials_after_failure || rho == 0 || !std::isfinite(h.lambda)) *result = G2OC_RESULT_TERMINATE;
  else *result = G2OC_RESULT_OK;
  return G2OC_OK;
}

// OptimizationAlgorithmGaussNewton::solve (optimization_algorithm_gauss_newton.cpp:48-93)
static int gn_iteration(g2oc_ctx* c, int iteration, g2oc_iteration_stats* stv, int* result) {
  (void)iteration;
  c->cur_stats = stv;
  c->chi2_carry = false;
  cudaEvent_t t0 = c->mark();
  G2OC_TRY(chi2_to(c, &c->sc.p->chi2_plain, &c->sc.p->chi2_current));
  c->span(t0, &stv->time_residuals);
  t0 = c->mark();
  G2OC_TRY(c->eng->build_system());
  c->system_built = true;
  c->span(t0, &stv->time_quadratic_form);
  t0 = c->mark();
  G2OC_TRY(c->eng->solve(0.0));
  c->span(t0, &stv->time_linear_solver);
  t0 = c->mark();
  G2OC_TRY(oplus(c));
  c->span(t0, &stv->time_update);
  G2OC_TRY(chi2_to(c, nullptr, &c->sc.p->chi2_temp));
  DevScalars h;
  G2OC_TRY(read_state(c, &h, stv));
  stv->chi2 = h.chi2_temp;  // activeRobustChi2 after the update (G2OBatchStatistics::chi2)
  c->resolve_spans();
  c->cur_stats = nullptr;
  *result = h.solve_ok ? G2OC_RESULT_OK : G2OC_RESULT_FAIL;
  return G2OC_OK;
}

// a . b of device vectors, on the host (one wait), fixed summation order
static int dl_dot(g2oc_ctx* c, const double* a, const double* b, int n, double* out) {
  G2OC_K(K_LM_CONTROL) dot_partials<<<kRedBlocks, 256, 0, c->stream>>>(a, b, n, c->partials.p);
  G2OC_LAUNCH_CHECK();
  G2OC_TRY(finalize_sum(c, kRedBlocks, 1, &c->sc.p->refine_rnorm, nullptr));
  G2OC_CUDA_TRY(cudaMemcpyAsync(out, &c->sc.p->refine_rnorm, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return G2OC_OK;
}

static int dl_combine(g2oc_ctx* c, int n, double a, const double* x, double b, const double* y, double* out) {
  if (n <= 0) return G2OC_OK;
  G2OC_K(K_AXPY) dl_axpby<<<cdiv(n, 256), 256, 0, c->stream>>>(n, a, x, b, y, out);
  G2OC_LAUNCH_CHECK();
  return G2OC_OK;
}

// OptimizationAlgorithmDogleg::solve (g2o/core/optimization_algorithm_dogleg.cpp:62-180):
// steepest-descent step alpha b with alpha = |b|^2 / b^T Hpp b, Gauss-Newton
// step H^-1 b (damped with lambda once a solve was not positive definite),
// the dogleg between them inside the trust radius Delta; the step is kept
// when the gain ratio rho > 0; Delta grows (rho > 0.75) or halves
// (rho < 0.25). The control runs on the host from device dot products.
static int dl_iteration(g2oc_ctx* c, int iteration, g2oc_iteration_stats* stv, int* result) {
  cudaStream_t st = c->stream;
  DevScalars* sc = c->sc.p;
  c->cur_stats = stv;
  const int n = c->vec_size();
  if (iteration == 0) {
    c->dl_delta = c->prm.initial_delta;
    c->dl_lambda = c->prm.initial_lambda > 0 ? c->prm.initial_lambda : 1e-7;
    c->dl_was_pd = true;
  }
  if (c->dl_buf.n < (size_t)3 * n) G2OC_TRY(c->dl_buf.alloc((size_t)3 * n));
  double* hsd = c->dl_buf.p;
  double* hgn = c->dl_buf.p + n;
  double* aux = c->dl_buf.p + 2 * (size_t)n;
  double* hdl = c->x.p;  // the update oplus applies
  const double* b = c->b.p;
  cudaEvent_t t0 = c->mark();
  G2OC_TRY(chi2_to(c, &sc->chi2_plain, &sc->chi2_current));
  c->span(t0, &stv->time_residuals);
  t0 = c->mark();
  G2OC_TRY(c->eng->build_system());
  c->system_built = true;
  c->span(t0, &stv->time_quadratic_form);
  DevScalars h{};
  G2OC_TRY(read_state(c, &h, stv));
  const double current_chi = h.chi2_current;
  // alpha = |b|^2 / (b^T Hpp b); hsd = alpha b
  G2OC_TRY(c->eng->multiply_hessian(b, aux));
  double bb = 0, ab = 0;
  G2OC_TRY(dl_dot(c, b, b, n, &bb));
  G2OC_TRY(dl_dot(c, aux, b, n, &ab));
  const double alpha = bb / ab;
  G2OC_TRY(dl_combine(c, n, alpha, b, 0.0, nullptr, hsd));
  double hsd2 = 0;
  G2OC_TRY(dl_dot(c, hsd, hsd, n, &hsd2));
  const double hsd_norm = std::sqrt(hsd2);
  double hgn_norm = -1.0, new_chi = current_chi;
  bool solved = false, good = false;
  int tries = 0, step = 0;
  const int max_trials = c->prm.max_trials_after_failure;
  do {
    ++tries;
    if (!solved) {
      solved = true;
      bool ok = false;
      while (!ok) {
        t0 = c->mark();
        G2OC_TRY(c->eng->solve(c->dl_was_pd ? 0.0 : c->dl_lambda));
        c->span(t0, &stv->time_linear_solver);
        G2OC_TRY(read_state(c, &h, stv));
        ok = h.solve_ok != 0;
        c->dl_was_pd = c->dl_was_pd && ok;
        if (!c->dl_was_pd) {
          if (ok) {
            c->dl_lambda = std::max(1e-12, c->dl_lambda / (0.5 * c->prm.lambda_factor));
          } else {
            c->dl_lambda *= c->prm.lambda_factor;
            if (c->dl_lambda > 1e3) {
              c->dl_lambda = 1e3;
              stv->levenberg_iterations = tries;
              stv->lambda = c->dl_lambda;
              stv->trust_radius = c->dl_delta;
              stv->chi2 = current_chi;
              c->resolve_spans();
              c->cur_stats = nullptr;
              *result = G2OC_RESULT_FAIL;
              return G2OC_OK;
            }
          }
        }
      }
      G2OC_CUDA_TRY(cudaMemcpyAsync(hgn, c->x.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st));
      double g2 = 0;
      G2OC_TRY(dl_dot(c, hgn, hgn, n, &g2));
      hgn_norm = std::sqrt(g2);
    }
    const double delta = c->dl_delta;
    if (hgn_norm < delta) {
      G2OC_CUDA_TRY(cudaMemcpyAsync(hdl, hgn, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st));
      step = 2;
    } else if (hsd_norm > delta) {
      G2OC_TRY(dl_combine(c, n, delta / hsd_norm, hsd, 0.0, nullptr, hdl));
      step = 1;
    } else {
      G2OC_TRY(dl_combine(c, n, 1.0, hgn, -1.0, hsd, aux));  // b - a
      double cc = 0, bma2 = 0;
      G2OC_TRY(dl_dot(c, hsd, aux, n, &cc));
      G2OC_TRY(dl_dot(c, aux, aux, n, &bma2));
      double beta;
      if (cc <= 0.) beta = (-cc + std::sqrt(cc * cc + bma2 * (delta * delta - hsd2))) / bma2;
      else beta = (delta * delta - hsd2) / (cc + std::sqrt(cc * cc + bma2 * (delta * delta - hsd2)));
      G2OC_TRY(dl_combine(c, n, 1.0, hsd, beta, aux, hdl));
      step = 3;
    }
    // linear gain -hdl^T Hpp hdl + 2 b^T hdl
    G2OC_TRY(c->eng->multiply_hessian(hdl, aux));
    double hh = 0, bh = 0;
    G2OC_TRY(dl_dot(c, aux, hdl, n, &hh));
    G2OC_TRY(dl_dot(c, b, hdl, n, &bh));
    double linear_gain = -1 * hh + 2 * bh;
    G2OC_TRY(push(c));
    t0 = c->mark();
    G2OC_TRY(oplus(c));
    c->span(t0, &stv->time_update);
    G2OC_TRY(chi2_to(c, &sc->chi2_temp_plain, &sc->chi2_temp));
    G2OC_TRY(read_state(c, &h, stv));
    new_chi = h.chi2_temp;
    const double nonlinear_gain = current_chi - new_chi;
    if (std::fabs(linear_gain) < 1e-12) linear_gain = 1e-12;
    const double rho = nonlinear_gain / linear_gain;
    if (rho > 0) {
      good = true;
    } else {
      G2OC_TRY(pop(c));
    }
    if (rho > 0.75) {
      double d2 = 0;
      G2OC_TRY(dl_dot(c, hdl, hdl, n, &d2));
      c->dl_delta = std::max(c->dl_delta, 3 * std::sqrt(d2));
    } else if (rho < 0.25) {
      c->dl_delta *= 0.5;
    }
  } while (!good && tries < max_trials);
  stv->levenberg_iterations = tries;
  stv->lambda = c->dl_was_pd ? 0.0 : c->dl_lambda;
  stv->trust_radius = c->dl_delta;
  stv->dogleg_step = step;
  stv->chi2 = good ? new_chi : current_chi;  // activeRobustChi2 of the state the iteration ends in
  c->chi2_carry = false;
  c->resolve_spans();
  c->cur_stats = nullptr;
  *result = (tries == max_trials || !good) ? G2OC_RESULT_TERMINATE : G2OC_RESULT_OK;
  return G2OC_OK;
}

static int structure_only(g2oc_ctx* c, int num_iters, int num_max_trials) {
  const Structure& S = c->S;
  if (!S.ba || S.D != 2 || S.bal) {
    set_error("the structure-only solver optimizes the landmarks of an SE3 bundle adjustment with two-row projection edges");
    return G2OC_ERR_NOT_SUPPORTED;
  }
  if (S.Pf == 0 || num_iters <= 0) return G2OC_OK;
  G2OC_K(K_OPLUS) ba_structure_only<<<cdiv(S.Pf, 128), 128, 0, c->stream>>>(c->ba_edges(), c->ba_vertices(),
                                                                              c->l_ptr.p, S.Pf, num_iters,
                                                                              num_max_trials);
  G2OC_LAUNCH_CHECK();
  c->chi2_carry = false;
  c->system_built = false;
  return G2OC_OK;
}

// StructureOnlySolver::solve (structure_only_solver.h:62-65): calc(points, 1)
static int so_iteration(g2oc_ctx* c, g2oc_iteration_stats* stv, int* result) {
  cudaEvent_t t0 = c->mark();
  G2OC_TRY(structure_only(c, 1, c->prm.max_trials_after_failure));
  c->span(t0, &stv->time_update);
  G2OC_TRY(chi2_to(c, &c->sc.p->chi2_plain, &c->sc.p->chi2_current));
  DevScalars h{};
  G2OC_TRY(read_state(c, &h, stv));
  stv->chi2 = h.chi2_current;
  c->resolve_spans();
  *result = G2OC_RESULT_OK;
  return G2OC_OK;
}

static int reset_pcg(g2oc_ctx* c) {
  PcgState p{};
  p.residual_carry = -1.0;
  G2OC_CUDA_TRY(cudaMemcpyAsync(c->pcg.p, &p, sizeof(PcgState), cudaMemcpyHostToDevice, c->stream));
  c->pcg_seen = 0;
  return G2OC_OK;
}

static int check_ctx(g2oc_ctx* c, bool need_upload) {
  if (!c) {
    set_error("context is NULL");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  if (need_upload && !c->uploaded) {
    set_error("no graph uploaded");
    return G2OC_ERR_STATE;
  }
  G2OC_CUDA_TRY(cudaSetDevice(c->device));
  return G2OC_OK;
}

// inverse measurement on the host, once per upload
static void inverse_measurement(int et, const double* m, double* out) {
  if (et == G2OC_EDGE_SE2) {
    se2_inv(m, out);
  } else if (et == G2OC_EDGE_SE3_EXPMAP) {
    memcpy(out, m, 7 * sizeof(double));  // EdgeSE3Expmap's error uses the measurement itself
  } else {
    iso_inv(m, out);
  }
}

}  // namespace g2oc

using namespace g2oc;

extern "C" {

int g2oc_abi_version(void) { return G2OC_ABI_VERSION; }

const char* g2oc_last_error(void) { return g_err; }

void g2oc_default_params(g2oc_params* p) {
  if (!p) return;
  p->algorithm = G2OC_ALGO_LEVENBERG;
  p->linear_solver = G2OC_LINEAR_PCG;
  p->precision = G2OC_PREC_FP64;
  p->pcg_max_iterations = -1;
  p->pcg_tolerance = 1e-6;
  p->pcg_absolute_tolerance = 1;
  p->max_trials_after_failure = 10;
  p->initial_lambda = 0.0;
  p->tau = 1e-5;
  p->refine_max_iterations = 2;
  p->refine_tolerance = 1e-10;
  p->initial_delta = 1e4;
  p->lambda_factor = 10.0;
}

// names registered by this library, "<gn|lm|dl>_cuda[_<variant>]"
static const char* kSolvers[][2] = {
    {"gn_cuda", "Gauss-Newton: B200 block solver, FP64, PCG with Schur / Cholesky without"},
    {"lm_cuda", "Levenberg: B200 block solver, FP64, PCG with Schur / Cholesky without"},
    {"gn_cuda_pcg", "Gauss-Newton: B200 block solver, FP64, block-Jacobi PCG"},
    {"lm_cuda_pcg", "Levenberg: B200 block solver, FP64, block-Jacobi PCG"},
    {"gn_cuda_pcg6_3", "Gauss-Newton: B200 BlockSolver<6,3>, FP64, block-Jacobi PCG"},
    {"lm_cuda_pcg6_3", "Levenberg: B200 BlockSolver<6,3>, FP64, block-Jacobi PCG"},
    {"gn_cuda_pcg3_3", "Gauss-Newton: B200 BlockSolver<3,3>, FP64, block-Jacobi PCG"},
    {"lm_cuda_pcg3_3", "Levenberg: B200 BlockSolver<3,3>, FP64, block-Jacobi PCG"},
    {"gn_cuda_pcg9_3", "Gauss-Newton: B200 BlockSolver<9,3> (BAL cameras), FP64, block-Jacobi PCG"},
    {"lm_cuda_pcg9_3", "Levenberg: B200 BlockSolver<9,3> (BAL cameras), FP64, block-Jacobi PCG"},
    {"gn_cuda_chol", "Gauss-Newton: B200 block solver, FP64, dense Cholesky"},
    {"lm_cuda_chol", "Levenberg: B200 block solver, FP64, dense Cholesky"},
    {"gn_cuda_mixed", "Gauss-Newton: B200 block solver, FP32 Hessian/Schur/PCG with FP64 refinement"},
    {"lm_cuda_mixed", "Levenberg: B200 block solver, FP32 Hessian/Schur/PCG with FP64 refinement"},
    {"gn_cuda_mixed_fast", "Gauss-Newton: B200 block solver, FP32 Hessian/Schur/PCG steps, FP64 errors and control"},
    {"lm_cuda_mixed_fast", "Levenberg: B200 block solver, FP32 Hessian/Schur/PCG steps, FP64 errors and control"},
    {"gn_cuda_chol_mixed", "Gauss-Newton: B200 block solver, FP32 Hessian, FP64 Cholesky, FP64 refinement"},
    {"lm_cuda_chol_mixed", "Levenberg: B200 block solver, FP32 Hessian, FP64 Cholesky, FP64 refinement"},
    {"gn_cuda_chol_mixed_fast", "Gauss-Newton: B200 block solver, FP32 Hessian, FP64 Cholesky of it"},
    {"lm_cuda_chol_mixed_fast", "Levenberg: B200 block solver, FP32 Hessian, FP64 Cholesky of it"},
    {"dl_cuda", "Dogleg: B200 block solver, FP64, PCG with Schur / Cholesky without"},
    {"dl_cuda_pcg", "Dogleg: B200 block solver, FP64, block-Jacobi PCG"},
    {"dl_cuda_chol", "Dogleg: B200 block solver, FP64, dense Cholesky"},
    {"structure_only_cuda_3", "Optimize the landmark positions (3D), cameras fixed: one small LM per landmark"},
};

int g2oc_list_solvers(char* buf, size_t size) {
  std::string s;
  for (auto& e : kSolvers) {
    if (!s.empty()) s += ";";
    s += e[0];
  }
  if (!buf || size < s.size() + 1) {
    set_error("buffer too small: %zu bytes needed", s.size() + 1);
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  memcpy(buf, s.c_str(), s.size() + 1);
  return G2OC_OK;
}

int g2oc_construct(const char* name, g2oc_params* p) {
  if (!name || !p) {
    set_error("name or params is NULL");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  bool found = false;
  for (auto& e : kSolvers)
    if (strcmp(e[0], name) == 0) found = true;
  if (!found) {
    set_error("SOLVER FACTORY: Unable to create solver %s", name);
    return G2OC_ERR_UNKNOWN_SOLVER;
  }
  const std::string n(name);
  g2oc_default_params(p);
  if (n == "structure_only_cuda_3") {
    p->algorithm = G2OC_ALGO_STRUCTURE_ONLY;  // StructureOnlyCreator (g2o/solvers/structure_only/structure_only.cpp)
    return G2OC_OK;
  }
  p->algorithm = n.substr(0, 2) == "gn"   ? G2OC_ALGO_GAUSS_NEWTON
                 : n.substr(0, 2) == "dl" ? G2OC_ALGO_DOGLEG
                                          : G2OC_ALGO_LEVENBERG;
  if (p->algorithm == G2OC_ALGO_DOGLEG) {
    // OptimizationAlgorithmDogleg's properties (optimization_algorithm_dogleg.cpp:44-51)
    p->max_trials_after_failure = 100;
    p->initial_lambda = 1e-7;
  }
  const std::string v = n.size() > 7 ? n.substr(8) : "";
  if (v.empty()) p->linear_solver = 2;  // PCG with Schur, Cholesky without
  else if (v.rfind("chol", 0) == 0) {
    p->linear_solver = G2OC_LINEAR_CHOLESKY;
    // FP32 Hessian, FP64 factorization of it; FP64 refinement of every step
    // on pose graphs unless _fast
    if (v == "chol_mixed" || v == "chol_mixed_fast") p->precision = G2OC_PREC_MIXED;
    if (v == "chol_mixed_fast") p->refine_max_iterations = -1;
  }
  else if (v == "mixed" || v == "mixed_fast") {
    p->linear_solver = G2OC_LINEAR_PCG;
    p->precision = G2OC_PREC_MIXED;
    if (v == "mixed_fast") p->refine_max_iterations = -1;  // the FP32-stored system's solution is the step
  } else p->linear_solver = G2OC_LINEAR_PCG;
  return G2OC_OK;
}

int g2oc_create(int device, g2oc_ctx** out) {
  if (!out) {
    set_error("out is NULL");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    set_error("no CUDA device");
    return G2OC_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= n) {
    set_error("device %d out of range (%d devices)", device, n);
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  cudaDeviceProp prop;
  G2OC_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) {
    set_error("device %d is sm_%d%d; this library is built for sm_100a", device, prop.major, prop.minor);
    return G2OC_ERR_NO_DEVICE;
  }
  G2OC_CUDA_TRY(cudaSetDevice(device));
  std::unique_ptr<g2oc_ctx> c(new g2oc_ctx());
  c->device = device;
  if (const char* e = getenv("G2OC_TEST_BARRIER_EXTRA")) c->barrier_extra = atoi(e) > 0 ? 1u : 0u;
  G2OC_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  g2oc_default_params(&c->prm);
  G2OC_TRY(c->sc.alloc(1));
  G2OC_TRY(c->pcg.alloc(1));
  G2OC_TRY(c->flag.alloc(1));
  G2OC_TRY(c->partials.alloc(2 * 8192));
  G2OC_CUDA_TRY(cudaMemsetAsync(c->sc.p, 0, sizeof(DevScalars), c->stream));
  G2OC_CUDA_TRY(cudaMemsetAsync(c->flag.p, 0, sizeof(int), c->stream));
  G2OC_TRY(reset_pcg(c.get()));
  G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
  coop_register(c.get(), +1);
  *out = c.release();
  return G2OC_OK;
}

void g2oc_destroy(g2oc_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  coop_register(c, -1);
  delete c;
}

static int make_engine(g2oc_ctx* c) {
  if (c->pose_edges() && c->prm.algorithm == G2OC_ALGO_STRUCTURE_ONLY) {
    set_error("a graph with a pose edge set runs Gauss-Newton, Levenberg-Marquardt or Dogleg");
    return G2OC_ERR_NOT_SUPPORTED;
  }
  if (c->pose_edges() && c->shard_world > 1 && c->shard_rank != 0) {
    // the ranks sum their parts of the reduced camera system, the gradient
    // and chi2: the pose edges' terms are added once, by rank 0
    set_error("sharded mode: the pose edge set belongs to rank 0's graph (rank %d has %d pose edges)", c->shard_rank,
              (int)c->S.pact.size());
    return G2OC_ERR_NOT_SUPPORTED;
  }
  if (c->S.bal) {
    if (c->prm.precision == G2OC_PREC_MIXED) {
      set_error("the BAL block solver runs in FP64 (no mixed-precision form)");
      return G2OC_ERR_NOT_SUPPORTED;
    }
    c->eng.reset(new BalEngine(c));
  } else if (c->prm.precision == G2OC_PREC_MIXED) c->eng.reset(new Engine<float>(c));
  else c->eng.reset(new Engine<double>(c));
  G2OC_TRY(c->eng->alloc());
  c->system_built = false;
  return G2OC_OK;
}

int g2oc_set_params(g2oc_ctx* c, const g2oc_params* p) {
  G2OC_TRY(check_ctx(c, false));
  if (!p) {
    set_error("params is NULL");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  if (p->algorithm < 0 || p->algorithm > 3 || p->linear_solver < 0 || p->linear_solver > 2 || p->precision < 0 ||
      p->precision > 1 || p->max_trials_after_failure < 1 || p->pcg_tolerance < 0 ||
      (p->algorithm == G2OC_ALGO_DOGLEG && (!(p->initial_delta > 0) || !(p->lambda_factor > 0)))) {
    set_error("invalid parameter value");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  const bool prec_changed = p->precision != c->prm.precision;
  c->prm = *p;
  if (c->win_graph) {  // the captured window round holds the old parameters
    cudaGraphExecDestroy(c->win_graph);
    c->win_graph = nullptr;
  }
  if (c->uploaded && prec_changed) G2OC_TRY(make_engine(c));
  return G2OC_OK;
}

static bool same_topology(const g2oc_ctx::Topology& t, const g2oc_graph* g) {
  if (!t.valid || t.pose_type != g->pose_type || t.num_poses != g->num_poses || t.num_points != g->num_points ||
      t.edge_type != g->edge_type || t.num_edges != g->num_edges || !g->edge_vertex)
    return false;
  if (t.has_pose_fixed != (g->pose_fixed != nullptr) || t.has_point_fixed != (g->point_fixed != nullptr)) return false;
  if ((int32_t)(t.pose_edge_vertex.size() / 2) != g->num_pose_edges) return false;
  if (g->num_pose_edges > 0 &&
      (!g->pose_edge_vertex ||
       memcmp(t.pose_edge_vertex.data(), g->pose_edge_vertex, t.pose_edge_vertex.size() * sizeof(int32_t))))
    return false;
  if (!t.edge_vertex.empty()) {
    // compared in parallel chunks (tens of MB for large graphs)
    const size_t n = t.edge_vertex.size(), chunk = 1 << 20;
    const long long nch = (long long)((n + chunk - 1) / chunk);
    int differ = 0;
#pragma omp parallel for schedule(static) reduction(| : differ) if (nch > 1)
    for (long long q = 0; q < nch; ++q) {
      const size_t a = (size_t)q * chunk, len = std::min(chunk, n - a);
      if (memcmp(t.edge_vertex.data() + a, g->edge_vertex + a, len * sizeof(int32_t))) differ |= 1;
    }
    if (differ) return false;
  }
  if (t.has_pose_fixed && !t.pose_fixed.empty() && memcmp(t.pose_fixed.data(), g->pose_fixed, t.pose_fixed.size()))
    return false;
  if (t.has_point_fixed && !t.point_fixed.empty() && memcmp(t.point_fixed.data(), g->point_fixed, t.point_fixed.size()))
    return false;
  return true;
}

static void save_topology(g2oc_ctx::Topology& t, const g2oc_graph* g) {
  t.pose_type = g->pose_type;
  t.num_poses = g->num_poses;
  t.num_points = g->num_points;
  t.edge_type = g->edge_type;
  t.num_edges = g->num_edges;
  t.edge_vertex.assign(g->edge_vertex, g->edge_vertex + 2 * (size_t)g->num_edges);
  if (g->num_pose_edges > 0)
    t.pose_edge_vertex.assign(g->pose_edge_vertex, g->pose_edge_vertex + 2 * (size_t)g->num_pose_edges);
  else
    t.pose_edge_vertex.clear();
  t.has_pose_fixed = g->pose_fixed != nullptr;
  t.has_point_fixed = g->point_fixed != nullptr;
  t.pose_fixed.assign(g->pose_fixed ? g->pose_fixed : nullptr, g->pose_fixed ? g->pose_fixed + g->num_poses : nullptr);
  if (g->point_fixed && g->num_points > 0) t.point_fixed.assign(g->point_fixed, g->point_fixed + g->num_points);
  else t.point_fixed.clear();
  t.valid = true;
}

// Everything that depends on the topology alone (vertex counts and types,
// fixed flags, edge list): SparseOptimizer::initializeOptimization and
// BlockSolver::buildStructure (g2o/core/sparse_optimizer.cpp:175-287,
// g2o/core/block_solver.hpp:110-269), the device index lists and the buffers.
static int upload_topology(g2oc_ctx* c, const g2oc_graph* g) {
  c->topo.valid = false;
  c->eng.reset();
  c->chol.reset();
  Structure& S = c->S;
  S = Structure();
  S.shard_world = c->shard_world;
  G2OC_TRY(build_structure(g, S));
  cudaStream_t st = c->stream;
  const int na = (int)S.act.size();
  if (S.ba) {
    // SE3Quat cameras packed 8 doubles apart; BAL cameras as given (9)
    G2OC_TRY(c->pose.alloc((size_t)S.C * (S.bal ? kBalCam : 8)));
    G2OC_TRY(c->point.alloc((size_t)S.P * 4));
    G2OC_TRY(c->point_bak.alloc(c->point.n));
    G2OC_TRY(c->point_init.alloc(c->point.n));
    G2OC_TRY(c->raw_pose.alloc(S.bal ? 1 : (size_t)S.C * 7));
    G2OC_TRY(c->raw_point.alloc((size_t)S.P * 3));
  } else {
    G2OC_TRY(c->pose.alloc((size_t)S.C * S.ped));
    c->point.release();
    c->point_bak.release();
    c->point_init.release();
  }
  G2OC_TRY(c->pose_bak.alloc(c->pose.n));
  G2OC_TRY(c->pose_init.alloc(c->pose.n));
  G2OC_TRY(c->oplus_count.alloc(S.C));
  G2OC_TRY(c->free_pose.upload(S.free_pose_of_h, st));
  G2OC_TRY(c->free_point.upload(S.free_point_of_l, st));
  G2OC_TRY(c->pose_h.upload(S.pose_h, st));
  if (S.ba) G2OC_TRY(c->point_l.upload(S.point_l, st));
  if (S.ba) {
    const size_t nc = S.c_edge.size();
    std::vector<int2> ev(na), cv(nc);
    std::vector<int> scam(nc);
    for (int k = 0; k < na; ++k) {
      const int e = S.dev_edge[k];
      ev[k] = make_int2(g->edge_vertex[2 * e], g->edge_vertex[2 * e + 1]);
    }
    for (size_t j = 0; j < nc; ++j) {
      cv[j] = ev[S.c_edge[j]];
      scam[j] = S.dev_edge[S.c_edge[j]];
    }
    G2OC_TRY(c->e_v.upload(ev, st));
    G2OC_TRY(c->c_v.upload(cv, st));
    G2OC_TRY(c->src_dev.upload(S.dev_edge, st));
    G2OC_TRY(c->src_cam.upload(scam, st));
    G2OC_TRY(c->e_z.alloc(na));
    G2OC_TRY(c->e_om.alloc(na));
    G2OC_TRY(c->c_z.alloc(nc));
    G2OC_TRY(c->c_om.alloc(nc));
    G2OC_TRY(c->raw_meas.alloc((size_t)S.E * S.md));
    G2OC_TRY(c->raw_info.alloc((size_t)S.E * S.D * S.D));
    if (S.D == 3) {
      G2OC_TRY(c->e_z3.alloc(na));
      G2OC_TRY(c->e_oa3.alloc(na));
      G2OC_TRY(c->e_ob3.alloc(na));
      G2OC_TRY(c->c_z3.alloc(nc));
      G2OC_TRY(c->c_oa3.alloc(nc));
      G2OC_TRY(c->c_ob3.alloc(nc));
    } else {
      for (auto* b : {&c->e_z3, &c->e_oa3, &c->c_z3, &c->c_oa3}) b->release();
      c->e_ob3.release();
      c->c_ob3.release();
    }
    G2OC_TRY(c->raw_delta.alloc((size_t)S.E));
    G2OC_TRY(c->e_hpl.upload(S.e_hpl, st));
    G2OC_TRY(c->l_ptr.upload(S.l_ptr, st));
    if (S.lm_warp_ok) {
      G2OC_TRY(c->e_lm.upload(S.e_lm, st));
      G2OC_TRY(c->lm_chunk_ptr.upload(S.lm_chunk_ptr, st));
    }
    G2OC_TRY(c->c_ptr.upload(S.c_ptr, st));
    G2OC_TRY(c->hb_ptr.upload(S.hb_ptr, st));
    const size_t nh = S.hpl_rc.size() / 2;
    std::vector<int> hr(nh), hcl(nh);
    for (size_t b = 0; b < nh; ++b) {
      hr[b] = S.hpl_rc[2 * b];
      hcl[b] = S.hpl_rc[2 * b + 1];
    }
    G2OC_TRY(c->hpl_row.upload(hr, st));
    G2OC_TRY(c->hpl_col.upload(hcl, st));
    G2OC_TRY(c->hc_ptr.upload(S.hc_ptr, st));
    G2OC_TRY(c->hc_blk.upload(S.hc_blk, st));
    std::vector<int> hcidx(S.hc_blk.size()), hccol(S.hc_blk.size());
    for (size_t p = 0; p < S.hc_blk.size(); ++p) {
      hcidx[S.hc_blk[p]] = (int)p;
      hccol[p] = S.hpl_rc[2 * (size_t)S.hc_blk[p] + 1];
    }
    G2OC_TRY(c->hc_index.upload(hcidx, st));
    G2OC_TRY(c->hc_col.upload(hccol, st));
    G2OC_TRY(c->s_pair_ptr.upload(S.s_pair_ptr, st));
    std::vector<int2> ab(S.s_pairs.size() / 2);
    for (size_t i = 0; i < ab.size(); ++i) ab[i] = make_int2(S.s_pairs[2 * i], S.s_pairs[2 * i + 1]);
    G2OC_TRY(c->s_pairs.upload(ab, st));
    G2OC_TRY(c->s_hpp.upload(S.s_hpp, st));
    if (!S.pact.empty()) {
      // the pose edge set, on the pose-graph kernels' arrays
      const int npa = (int)S.pact.size();
      std::vector<int2> pv(npa);
      for (int k = 0; k < npa; ++k) {
        const int e = S.pact[k];
        pv[k] = make_int2(g->pose_edge_vertex[2 * e], g->pose_edge_vertex[2 * e + 1]);
      }
      G2OC_TRY(c->pe_v.upload(pv, st));
      G2OC_TRY(c->pe_zinv.alloc((size_t)npa * 7));
      G2OC_TRY(c->pe_info.alloc((size_t)npa * 36));
      G2OC_TRY(c->pe_delta.alloc(npa));
      G2OC_TRY(c->pe_trans.upload(S.pe_trans, st));
      G2OC_TRY(c->hb_src_ptr.upload(S.hb_src_ptr, st));
      G2OC_TRY(c->hb_src.upload(S.hb_src.empty() ? std::vector<int>{0} : S.hb_src, st));
      G2OC_TRY(c->bv_src_ptr.upload(S.bv_src_ptr, st));
      G2OC_TRY(c->bv_src.upload(S.bv_src.empty() ? std::vector<int>{0} : S.bv_src, st));
      G2OC_TRY(c->pgpose.alloc((size_t)S.C * 7));
      G2OC_TRY(c->pp_ptr.upload(S.pp_ptr, st));
      std::vector<int4> pe4(S.pp_ent.size() / 4 + 1, make_int4(0, 0, 0, 0));
      for (size_t q = 0; q < S.pp_ent.size() / 4; ++q)
        pe4[q] = make_int4(S.pp_ent[4 * q], S.pp_ent[4 * q + 1], S.pp_ent[4 * q + 2], 0);
      G2OC_TRY(c->pp_ent.upload(pe4, st));
    }
  } else {
    std::vector<int2> ev(na);
    for (int k = 0; k < na; ++k) {
      const int e = S.act[k];
      ev[k] = make_int2(g->edge_vertex[2 * e], g->edge_vertex[2 * e + 1]);
    }
    G2OC_TRY(c->pe_v.upload(ev, st));
    G2OC_TRY(c->pe_zinv.alloc((size_t)na * S.md));
    G2OC_TRY(c->pe_info.alloc((size_t)na * S.D * S.D));
    G2OC_TRY(c->pe_delta.alloc(na));
    G2OC_TRY(c->pe_trans.upload(S.pe_trans, st));
    G2OC_TRY(c->hb_src_ptr.upload(S.hb_src_ptr, st));
    G2OC_TRY(c->hb_src.upload(S.hb_src, st));
    G2OC_TRY(c->bv_src_ptr.upload(S.bv_src_ptr, st));
    G2OC_TRY(c->bv_src.upload(S.bv_src, st));
  }
  G2OC_TRY(c->sys_perm.upload(S.sys_perm, st));
  G2OC_TRY(c->sys_rptr.upload(S.sys_rptr, st));
  G2OC_TRY(c->sys_rcol.upload(S.sys_rcol, st));
  G2OC_TRY(c->sys_brow.upload(S.sys_brow, st));
  G2OC_TRY(c->sys_diag.upload(S.sys_diag, st));
  G2OC_TRY(c->sys_cptr.upload(S.sys_cptr, st));
  G2OC_TRY(c->sys_cblk.upload(S.sys_cblk, st));
  G2OC_TRY(c->sys_chunk_ptr.upload(S.sys_chunk_ptr, st));
  G2OC_TRY(c->sys_chunk_row.upload(S.sys_chunk_row, st));
  if (S.tile_ok) {
    G2OC_TRY(c->tile_ij.upload(S.tile_ij, st));
    G2OC_TRY(c->tile_off.upload(S.tile_off, st));
  }
  const int n = c->vec_size();
  G2OC_TRY(c->b.alloc(n));
  G2OC_TRY(c->x.alloc(n));
  G2OC_TRY(c->dx.alloc(n));
  G2OC_TRY(c->resid.alloc(n));
  G2OC_TRY(c->xs.alloc((size_t)S.Cf * S.pd));
  G2OC_TRY(c->rhs.alloc((size_t)S.Cf * S.pd));
  G2OC_TRY(c->errbuf.alloc(std::max((size_t)na * 36, (size_t)na * S.D + S.pact.size() * 6)));
  G2OC_TRY(make_engine(c));
  save_topology(c->topo, g);
  return G2OC_OK;
}

// BA vertex estimates from the caller's layout (copied as-is, reordered on the device)
static int upload_ba_estimates(g2oc_ctx* c, const double* pose, const double* point) {
  const Structure& S = c->S;
  cudaStream_t st = c->stream;
  if (pose && S.C > 0 && S.bal) {
    G2OC_CUDA_TRY(cudaMemcpyAsync(c->pose.p, pose, c->pose.bytes(), cudaMemcpyHostToDevice, st));
  } else if (pose && S.C > 0) {
    G2OC_CUDA_TRY(cudaMemcpyAsync(c->raw_pose.p, pose, c->raw_pose.bytes(), cudaMemcpyHostToDevice, st));
    G2OC_K(K_IO) ba_pack_poses<<<cdiv((long long)S.C * 8, 256), 256, 0, st>>>(S.C, c->raw_pose.p, c->pose.p);
    G2OC_LAUNCH_CHECK();
  }
  if (point && S.P > 0) {
    G2OC_CUDA_TRY(cudaMemcpyAsync(c->raw_point.p, point, c->raw_point.bytes(), cudaMemcpyHostToDevice, st));
    G2OC_K(K_IO) ba_pack_points<<<cdiv((long long)S.P * 4, 256), 256, 0, st>>>(S.P, c->raw_point.p, c->point.p);
    G2OC_LAUNCH_CHECK();
  }
  return G2OC_OK;
}

// Everything that depends on the values: estimates, measurements, information
// matrices, robust kernels, camera parameters.
static int upload_data(g2oc_ctx* c, const g2oc_graph* g) {
  const Structure& S = c->S;
  cudaStream_t st = c->stream;
  const int na = (int)S.act.size();
  c->fx = g->focal_length;
  c->fy = (g->edge_type == G2OC_EDGE_SE3_PROJECT_XYZ || g->edge_type == G2OC_EDGE_STEREO_SE3_PROJECT_XYZ)
              ? g->focal_length_y
              : g->focal_length;
  c->bf = g->edge_type == G2OC_EDGE_STEREO_SE3_PROJECT_XYZ ? g->stereo_bf : 0.0;
  c->cx = g->principal_point[0];
  c->cy = g->principal_point[1];
  if (S.ba) {
    G2OC_TRY(upload_ba_estimates(c, g->pose_estimate, g->point_estimate));
    if (S.E > 0) {
      G2OC_CUDA_TRY(cudaMemcpyAsync(c->raw_meas.p, g->measurement, c->raw_meas.bytes(), cudaMemcpyHostToDevice, st));
      G2OC_CUDA_TRY(cudaMemcpyAsync(c->raw_info.p, g->information, c->raw_info.bytes(), cudaMemcpyHostToDevice, st));
      if (g->robust_delta)
        G2OC_CUDA_TRY(cudaMemcpyAsync(c->raw_delta.p, g->robust_delta, c->raw_delta.bytes(), cudaMemcpyHostToDevice, st));
      const int nc = (int)S.c_edge.size();
      if (na + nc > 0 && S.D == 3) {
        G2OC_K(K_IO) st_gather_edges<<<cdiv((long long)na + nc, 256), 256, 0, st>>>(
            na, nc, c->src_dev.p, c->src_cam.p, c->raw_meas.p, c->raw_info.p, g->robust_delta ? c->raw_delta.p : nullptr,
            c->e_z3.p, c->e_oa3.p, c->e_ob3.p, c->c_z3.p, c->c_oa3.p, c->c_ob3.p);
        G2OC_LAUNCH_CHECK();
      } else if (na + nc > 0) {
        // uniform information and Huber delta: one record for the graph
        const double* I = g->information;
        const double* dl = g->robust_delta;
        const double d0 = dl ? dl[0] : 0.0;
        bool uniform = true;
#pragma omp parallel for schedule(static) reduction(&& : uniform) if (S.E > 65536)
        for (int e = 0; e < S.E; ++e) {
          const double* Ie = I + (size_t)e * 4;
          uniform = uniform && Ie[0] == I[0] && Ie[1] == I[1] && Ie[3] == I[3] && (dl ? dl[e] : 0.0) == d0;
        }
        c->om_uniform = uniform;
        c->om_const = make_double4(I[0], I[1], I[3], d0);
        G2OC_K(K_IO) ba_gather_edges<<<cdiv((long long)na + nc, 256), 256, 0, st>>>(
            na, nc, c->src_dev.p, c->src_cam.p, c->raw_meas.p, c->raw_info.p, g->robust_delta ? c->raw_delta.p : nullptr,
            c->e_z.p, c->e_om.p, c->c_z.p, c->c_om.p);
        G2OC_LAUNCH_CHECK();
      }
    }
    if (!S.pact.empty()) {
      // the pose edge set's values (EdgeSE3Expmap: the error uses the measurement C itself)
      const int npa = (int)S.pact.size();
      std::vector<double> zi((size_t)npa * 7), info((size_t)npa * 36), dl(npa);
      for (int k = 0; k < npa; ++k) {
        const int e = S.pact[k];
        memcpy(zi.data() + (size_t)k * 7, g->pose_edge_measurement + (size_t)e * 7, 7 * sizeof(double));
        memcpy(info.data() + (size_t)k * 36, g->pose_edge_information + (size_t)e * 36, 36 * sizeof(double));
        dl[k] = g->pose_edge_robust_delta ? g->pose_edge_robust_delta[e] : 0.0;
      }
      G2OC_TRY(c->pe_zinv.upload(zi, st));
      G2OC_TRY(c->pe_info.upload(info, st));
      G2OC_TRY(c->pe_delta.upload(dl, st));
    }
  } else {
    if (S.C > 0)
      G2OC_CUDA_TRY(cudaMemcpyAsync(c->pose.p, g->pose_estimate, c->pose.bytes(), cudaMemcpyHostToDevice, st));
    const int D = S.D, ZD = S.md;
    std::vector<double> zi((size_t)na * ZD), info((size_t)na * D * D), dl(na);
#pragma omp parallel for schedule(static) if (na > 65536)
    for (int k = 0; k < na; ++k) {
      const int e = S.act[k];
      inverse_measurement(S.edge_type, g->measurement + (size_t)e * ZD, zi.data() + (size_t)k * ZD);
      memcpy(info.data() + (size_t)k * D * D, g->information + (size_t)e * D * D, D * D * sizeof(double));
      dl[k] = g->robust_delta ? g->robust_delta[e] : 0.0;
    }
    G2OC_TRY(c->pe_zinv.upload(zi, st));
    G2OC_TRY(c->pe_info.upload(info, st));
    G2OC_TRY(c->pe_delta.upload(dl, st));
  }
  G2OC_CUDA_TRY(cudaMemcpyAsync(c->pose_init.p, c->pose.p, c->pose.bytes(), cudaMemcpyDeviceToDevice, st));
  if (c->point.n)
    G2OC_CUDA_TRY(cudaMemcpyAsync(c->point_init.p, c->point.p, c->point.bytes(), cudaMemcpyDeviceToDevice, st));
  if (S.C > 0) G2OC_CUDA_TRY(cudaMemsetAsync(c->oplus_count.p, 0, S.C * sizeof(int), st));
  const int n = c->vec_size();
  if (n > 0) {
    G2OC_CUDA_TRY(cudaMemsetAsync(c->x.p, 0, n * sizeof(double), st));
    G2OC_CUDA_TRY(cudaMemsetAsync(c->b.p, 0, n * sizeof(double), st));
  }
  G2OC_TRY(reset_pcg(c));
  c->system_built = false;
  return G2OC_OK;
}

static void drop_windows(g2oc_ctx* c) {
  c->batch = false;
  c->nw = 0;
  c->win_tuned = false;
  if (c->win_graph) {
    cudaGraphExecDestroy(c->win_graph);
    c->win_graph = nullptr;
  }
}

int g2oc_upload(g2oc_ctx* c, const g2oc_graph* g) {
  G2OC_TRY(check_ctx(c, false));
  c->chi2_carry = false;
  drop_windows(c);
  if (!g) {
    set_error("graph is NULL");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  const bool reuse = c->eng && same_topology(c->topo, g);
  c->uploaded = false;
  c->last_upload_reused = false;
  if (reuse) {
    // the null checks build_structure makes for a new topology
    if (!g->pose_estimate || !g->measurement || !g->information || (c->S.ba && g->num_points > 0 && !g->point_estimate) ||
        (g->num_pose_edges > 0 && (!g->pose_edge_measurement || !g->pose_edge_information))) {
      set_error("graph array is NULL");
      return G2OC_ERR_INVALID_ARGUMENT;
    }
  } else {
    G2OC_TRY(upload_topology(c, g));
  }
  G2OC_TRY(upload_data(c, g));
  G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->uploaded = true;
  c->last_upload_reused = reuse;
  return G2OC_OK;
}

int g2oc_get_hessian_info(g2oc_ctx* c, g2oc_hessian_info* info) {
  G2OC_TRY(check_ctx(c, true));
  if (!info) return G2OC_ERR_INVALID_ARGUMENT;
  const Structure& S = c->S;
  info->num_free_poses = S.Cf;
  info->num_free_points = S.Pf;
  info->pose_dim = S.pd;
  info->point_dim = S.ba ? 3 : 0;
  info->hpp_nnzb = (int)(S.hpp_rc.size() / 2);
  info->hpl_nnzb = (int)(S.hpl_rc.size() / 2);
  info->schur_nnzb = (int)(S.schur_rc.size() / 2);
  info->num_active_edges = (int)S.act.size();
  info->vector_size = c->vec_size();
  info->schur_pairs = S.num_pairs;
  info->num_active_pose_edges = (int32_t)S.pact.size();
  return G2OC_OK;
}

int g2oc_set_estimates(g2oc_ctx* c, const double* pose, const double* point) {
  G2OC_TRY(check_ctx(c, true));
  c->chi2_carry = false;
  const Structure& S = c->S;
  if (S.ba) {
    G2OC_TRY(upload_ba_estimates(c, pose, point));
  } else if (pose && S.C > 0) {
    G2OC_CUDA_TRY(cudaMemcpyAsync(c->pose.p, pose, c->pose.bytes(), cudaMemcpyHostToDevice, c->stream));
  }
  G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->system_built = false;
  return G2OC_OK;
}

int g2oc_download(g2oc_ctx* c, double* pose, double* point) {
  G2OC_TRY(check_ctx(c, true));
  const Structure& S = c->S;
  cudaStream_t st = c->stream;
  if (S.ba) {
    // reorder into the caller's layout on the device, then one copy each
    if (pose && S.C > 0 && S.bal) {
      G2OC_CUDA_TRY(cudaMemcpyAsync(pose, c->pose.p, c->pose.bytes(), cudaMemcpyDeviceToHost, st));
    } else if (pose && S.C > 0) {
      G2OC_K(K_IO) ba_unpack_poses<<<cdiv((long long)S.C * 7, 256), 256, 0, st>>>(S.C, c->pose.p, c->raw_pose.p);
      G2OC_LAUNCH_CHECK();
      G2OC_CUDA_TRY(cudaMemcpyAsync(pose, c->raw_pose.p, c->raw_pose.bytes(), cudaMemcpyDeviceToHost, st));
    }
    if (point && S.P > 0) {
      G2OC_K(K_IO) ba_unpack_points<<<cdiv((long long)S.P * 3, 256), 256, 0, st>>>(S.P, c->point.p, c->raw_point.p);
      G2OC_LAUNCH_CHECK();
      G2OC_CUDA_TRY(cudaMemcpyAsync(point, c->raw_point.p, c->raw_point.bytes(), cudaMemcpyDeviceToHost, st));
    }
  } else if (pose && S.C > 0) {
    G2OC_CUDA_TRY(cudaMemcpyAsync(pose, c->pose.p, c->pose.bytes(), cudaMemcpyDeviceToHost, st));
  }
  G2OC_CUDA_TRY(cudaStreamSynchronize(st));
  return G2OC_OK;
}

static int check_sharding(g2oc_ctx* c) {
  if (c->shard_world <= 1) return G2OC_OK;
  const Structure& S = c->S;
  if (!S.ba || !S.schur || !S.tile_ok || c->prm.linear_solver == G2OC_LINEAR_CHOLESKY ||
      pcg_mode() != PCG_AUTO ||
      c->prm.algorithm == G2OC_ALGO_DOGLEG || c->prm.algorithm == G2OC_ALGO_STRUCTURE_ONLY ||
      (c->prm.precision == G2OC_PREC_MIXED && c->prm.refine_max_iterations >= 0)) {
    set_error("sharded mode runs bundle adjustments with >= %d free cameras and landmarks, the PCG solver, FP64 or "
              "mixed precision without FP64 refinement",
              2 * kTileBlocks);
    return G2OC_ERR_NOT_SUPPORTED;
  }
  return G2OC_OK;
}

int g2oc_set_sharding(g2oc_ctx* c, int32_t rank, int32_t world, g2oc_allreduce_fn allreduce, void* user) {
  G2OC_TRY(check_ctx(c, false));
  if (world < 1 || rank < 0 || rank >= world || (world > 1 && !allreduce)) {
    set_error("sharding: rank %d of %d (an all-reduce is needed for more than one rank)", rank, world);
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  if (c->uploaded || c->batch) {
    set_error("g2oc_set_sharding comes before g2oc_upload");
    return G2OC_ERR_STATE;
  }
  c->shard_rank = rank;
  c->shard_world = world;
  c->shard_fn = allreduce;
  c->shard_user = user;
  c->topo.valid = false;  // the next upload builds the structure for this world size
  return G2OC_OK;
}

static int optimize_impl(g2oc_ctx* c, int iterations, g2oc_iteration_stats* stats, int* done) {
  if (iterations < 0) {
    set_error("iterations < 0");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  G2OC_TRY(check_sharding(c));
  G2OC_TRY(reset_pcg(c));  // LinearSolverPCG::init via BlockSolver::init
  int result = G2OC_RESULT_OK;
  int it = 0;
  for (int i = 0; i < iterations && result == G2OC_RESULT_OK; ++i) {
    g2oc_iteration_stats stv;
    memset(&stv, 0, sizeof(stv));
    cudaEvent_t t0 = c->mark();
    if (c->prm.algorithm == G2OC_ALGO_LEVENBERG) G2OC_TRY(lm_iteration(c, i, &stv, &result));
    else if (c->prm.algorithm == G2OC_ALGO_DOGLEG) G2OC_TRY(dl_iteration(c, i, &stv, &result));
    else if (c->prm.algorithm == G2OC_ALGO_STRUCTURE_ONLY) G2OC_TRY(so_iteration(c, &stv, &result));
    else G2OC_TRY(gn_iteration(c, i, &stv, &result));
    stv.iteration = i;
    stv.result = result;
    c->span(t0, &stv.time_iteration);
    c->resolve_spans();
    if (stats) stats[i] = stv;
    ++it;
  }
  G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (done) *done = (result == G2OC_RESULT_FAIL) ? 0 : it;
  return G2OC_OK;
}

static int iterate_impl(g2oc_ctx* c, int iteration, g2oc_iteration_stats* stats, int* result) {
  if (iteration < 0 || !result) {
    set_error("iteration < 0 or result is NULL");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  if (iteration == 0) G2OC_TRY(reset_pcg(c));
  g2oc_iteration_stats stv;
  memset(&stv, 0, sizeof(stv));
  cudaEvent_t t0 = c->mark();
  if (c->prm.algorithm == G2OC_ALGO_LEVENBERG) G2OC_TRY(lm_iteration(c, iteration, &stv, result));
  else if (c->prm.algorithm == G2OC_ALGO_DOGLEG) G2OC_TRY(dl_iteration(c, iteration, &stv, result));
  else if (c->prm.algorithm == G2OC_ALGO_STRUCTURE_ONLY) G2OC_TRY(so_iteration(c, &stv, result));
  else G2OC_TRY(gn_iteration(c, iteration, &stv, result));
  stv.iteration = iteration;
  stv.result = *result;
  c->span(t0, &stv.time_iteration);
  c->resolve_spans();
  if (stats) *stats = stv;
  G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return G2OC_OK;
}

// the iteration paths record phase-time spans aimed at a stats record on
// their own stack; a failure half-way must not leave those behind
int g2oc_optimize(g2oc_ctx* c, int iterations, g2oc_iteration_stats* stats, int* done) {
  G2OC_TRY(check_ctx(c, true));
  const int st = optimize_impl(c, iterations, stats, done);
  if (st != G2OC_OK) c->drop_spans();
  return st;
}

int g2oc_iterate(g2oc_ctx* c, int iteration, g2oc_iteration_stats* stats, int* result) {
  G2OC_TRY(check_ctx(c, true));
  const int st = iterate_impl(c, iteration, stats, result);
  if (st != G2OC_OK) c->drop_spans();
  return st;
}

int g2oc_structure_only(g2oc_ctx* c, int32_t num_iters, int32_t num_max_trials) {
  G2OC_TRY(check_ctx(c, true));
  if (num_iters < 0 || num_max_trials < 1) {
    set_error("num_iters < 0 or num_max_trials < 1");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  if (c->batch || c->shard_world > 1) {
    set_error("the structure-only solver runs on a single bundle adjustment context");
    return G2OC_ERR_NOT_SUPPORTED;
  }
  G2OC_TRY(structure_only(c, num_iters, num_max_trials));
  G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return G2OC_OK;
}

int g2oc_chi2(g2oc_ctx* c, double* chi2, double* robust) {
  G2OC_TRY(check_ctx(c, true));
  G2OC_TRY(chi2_to(c, &c->sc.p->chi2_plain, &c->sc.p->chi2_temp));
  DevScalars h;
  G2OC_CUDA_TRY(cudaMemcpyAsync(&h, c->sc.p, sizeof(DevScalars), cudaMemcpyDeviceToHost, c->stream));
  G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (chi2) *chi2 = h.chi2_plain;
  if (robust) *robust = h.chi2_temp;
  return G2OC_OK;
}

int g2oc_errors(g2oc_ctx* c, double* out) {
  G2OC_TRY(check_ctx(c, true));
  if (!out) return G2OC_ERR_INVALID_ARGUMENT;
  const Structure& S = c->S;
  const int na = (int)S.act.size();
  if (S.bal)
    G2OC_K(K_ERRORS) bal_errors_kernel<<<cdiv(na, 128), 128, 0, c->stream>>>(c->ba_edges(), c->ba_vertices(), c->errbuf.p);
  else if (S.ba && S.D == 3)
    G2OC_K(K_ERRORS) st_errors_kernel<<<cdiv(na, 128), 128, 0, c->stream>>>(c->ba_edges(), c->ba_vertices(), c->errbuf.p);
  else if (S.ba) G2OC_K(K_ERRORS) ba_errors_kernel<<<cdiv(na, 128), 128, 0, c->stream>>>(c->ba_edges(), c->ba_vertices(), c->errbuf.p);
  else if (S.pose_type == G2OC_POSE_SE2)
    G2OC_K(K_ERRORS) pg_errors_kernel<G2OC_POSE_SE2><<<cdiv(na, 128), 128, 0, c->stream>>>(c->pose.p, c->pg_edges(), c->errbuf.p);
  else if (S.pose_type == G2OC_POSE_SE3EXPMAP)
    G2OC_K(K_ERRORS) pg_errors_kernel<G2OC_POSE_SE3EXPMAP><<<cdiv(na, 128), 128, 0, c->stream>>>(c->pose.p, c->pg_edges(),
                                                                                                c->errbuf.p);
  else G2OC_K(K_ERRORS) pg_errors_kernel<G2OC_POSE_SE3><<<cdiv(na, 128), 128, 0, c->stream>>>(c->pose.p, c->pg_edges(), c->errbuf.p);
  G2OC_LAUNCH_CHECK();
  const size_t npe = S.ba ? S.pact.size() : 0;
  if (npe > 0) {
    // the pose edge set's errors follow the projection edges'
    G2OC_K(K_ERRORS) ba_unpack_poses<<<cdiv((long long)S.C * 7, 256), 256, 0, c->stream>>>(S.C, c->pose.p,
                                                                                          c->pgpose.p);
    G2OC_K(K_ERRORS) pg_errors_kernel<G2OC_POSE_SE3EXPMAP><<<cdiv((long long)npe, 128), 128, 0, c->stream>>>(
        c->pgpose.p, c->ba_pose_edges(), c->errbuf.p + (size_t)na * S.D);
    G2OC_LAUNCH_CHECK();
  }
  std::vector<double> h((size_t)na * S.D + npe * 6);
  G2OC_CUDA_TRY(cudaMemcpyAsync(h.data(), c->errbuf.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
  for (int a = 0; a < na; ++a)
    memcpy(out + (size_t)a * S.D, h.data() + (size_t)S.dev_of_act[a] * S.D, S.D * sizeof(double));
  if (npe > 0) memcpy(out + (size_t)na * S.D, h.data() + (size_t)na * S.D, npe * 6 * sizeof(double));
  return G2OC_OK;
}

int g2oc_jacobians(g2oc_ctx* c, double* j0, double* j1) {
  G2OC_TRY(check_ctx(c, true));
  if (!j0 || !j1) return G2OC_ERR_INVALID_ARGUMENT;
  const Structure& S = c->S;
  const int na = (int)S.act.size();
  const int d0 = S.ba ? 3 : S.pd, d1 = S.pd, D = S.D;
  DBuf<double> a, b;
  G2OC_TRY(a.alloc((size_t)na * D * d0));
  G2OC_TRY(b.alloc((size_t)na * D * d1));
  if (S.bal)
    G2OC_K(K_JACOBIANS) bal_jacobians_kernel<<<cdiv(na, 128), 128, 0, c->stream>>>(c->ba_edges(), c->ba_vertices(), a.p, b.p);
  else if (S.ba && S.D == 3)
    G2OC_K(K_JACOBIANS) st_jacobians_kernel<<<cdiv(na, 128), 128, 0, c->stream>>>(c->ba_edges(), c->ba_vertices(), a.p, b.p);
  else if (S.ba) G2OC_K(K_JACOBIANS) ba_jacobians_kernel<<<cdiv(na, 128), 128, 0, c->stream>>>(c->ba_edges(), c->ba_vertices(), a.p, b.p);
  else if (S.pose_type == G2OC_POSE_SE2)
    G2OC_K(K_JACOBIANS) pg_jacobians_kernel<G2OC_POSE_SE2><<<cdiv(na, 128), 128, 0, c->stream>>>(c->pose.p, c->pg_edges(), a.p, b.p);
  else if (S.pose_type == G2OC_POSE_SE3EXPMAP)
    G2OC_K(K_JACOBIANS) pg_jacobians_kernel<G2OC_POSE_SE3EXPMAP><<<cdiv(na, 64), 64, 0, c->stream>>>(c->pose.p, c->pg_edges(),
                                                                                                    a.p, b.p);
  else G2OC_K(K_JACOBIANS) pg_jacobians_kernel<G2OC_POSE_SE3><<<cdiv(na, 64), 64, 0, c->stream>>>(c->pose.p, c->pg_edges(), a.p, b.p);
  G2OC_LAUNCH_CHECK();
  std::vector<double> ha(a.n), hb(b.n);
  G2OC_CUDA_TRY(cudaMemcpyAsync(ha.data(), a.p, a.bytes(), cudaMemcpyDeviceToHost, c->stream));
  G2OC_CUDA_TRY(cudaMemcpyAsync(hb.data(), b.p, b.bytes(), cudaMemcpyDeviceToHost, c->stream));
  G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < na; ++k) {
    const size_t dev = S.dev_of_act[k];
    memcpy(j0 + (size_t)k * D * d0, ha.data() + dev * D * d0, D * d0 * sizeof(double));
    memcpy(j1 + (size_t)k * D * d1, hb.data() + dev * D * d1, D * d1 * sizeof(double));
  }
  return G2OC_OK;
}

int g2oc_build_system(g2oc_ctx* c) {
  G2OC_TRY(check_ctx(c, true));
  G2OC_TRY(c->eng->build_system());
  G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->system_built = true;
  return G2OC_OK;
}

int g2oc_get_pattern(g2oc_ctx* c, int32_t* hpp_rc, int32_t* hpl_rc, int32_t* schur_rc) {
  G2OC_TRY(check_ctx(c, true));
  const Structure& S = c->S;
  if (hpp_rc) memcpy(hpp_rc, S.hpp_rc.data(), S.hpp_rc.size() * sizeof(int32_t));
  if (hpl_rc) memcpy(hpl_rc, S.hpl_rc.data(), S.hpl_rc.size() * sizeof(int32_t));
  if (schur_rc) memcpy(schur_rc, S.schur_rc.data(), S.schur_rc.size() * sizeof(int32_t));
  return G2OC_OK;
}

int g2oc_get_hessian(g2oc_ctx* c, double* hpp, double* hll, double* hpl, double* b) {
  G2OC_TRY(check_ctx(c, true));
  if (!c->system_built) {
    set_error("call g2oc_build_system first");
    return G2OC_ERR_STATE;
  }
  G2OC_TRY(c->eng->get_hessian(hpp, hll, hpl));
  if (b) G2OC_CUDA_TRY(cudaMemcpy(b, c->b.p, c->b.bytes(), cudaMemcpyDeviceToHost));
  return G2OC_OK;
}

int g2oc_schur(g2oc_ctx* c, double lambda, double* S_out, double* bs) {
  G2OC_TRY(check_ctx(c, true));
  if (!c->system_built) {
    set_error("call g2oc_build_system first");
    return G2OC_ERR_STATE;
  }
  return c->eng->schur_export(lambda, S_out, bs);
}

int g2oc_solve(g2oc_ctx* c, double lambda, double* x, int32_t* iters) {
  G2OC_TRY(check_ctx(c, true));
  if (!c->system_built) {
    set_error("call g2oc_build_system first");
    return G2OC_ERR_STATE;
  }
  G2OC_TRY(c->eng->solve(lambda));
  DevScalars h;
  g2oc_iteration_stats stv;
  memset(&stv, 0, sizeof(stv));
  G2OC_TRY(read_state(c, &h, &stv));
  if (iters) *iters = stv.iterations_linear_solver;
  if (x) G2OC_CUDA_TRY(cudaMemcpy(x, c->x.p, c->x.bytes(), cudaMemcpyDeviceToHost));
  return h.solve_ok ? G2OC_OK : G2OC_ERR_NOT_PD;
}

int g2oc_solver_init(g2oc_ctx* c) {
  G2OC_TRY(check_ctx(c, true));
  G2OC_TRY(reset_pcg(c));
  G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return G2OC_OK;
}

int g2oc_multiply_hessian(g2oc_ctx* c, const double* src, double* dest) {
  G2OC_TRY(check_ctx(c, true));
  if (!c->system_built) {
    set_error("call g2oc_build_system first");
    return G2OC_ERR_STATE;
  }
  if (!src || !dest) {
    set_error("src or dest is NULL");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  const Structure& S = c->S;
  const size_t np = (size_t)S.Cf * S.pd;
  if (np == 0) return G2OC_OK;
  cudaStream_t st = c->stream;
  // src in the first np entries of the residual scratch, the product in dx
  // (both hold the whole Hessian-order vector; the product's landmark part
  // is zero and not returned)
  G2OC_CUDA_TRY(cudaMemcpyAsync(c->resid.p, src, np * sizeof(double), cudaMemcpyHostToDevice, st));
  G2OC_TRY(c->eng->multiply_hessian(c->resid.p, c->dx.p));
  G2OC_CUDA_TRY(cudaMemcpyAsync(dest, c->dx.p, np * sizeof(double), cudaMemcpyDeviceToHost, st));
  G2OC_CUDA_TRY(cudaStreamSynchronize(st));
  return G2OC_OK;
}

// ------------------------------------------------------------ adjoint
// a . b of device vectors, on the host (one wait)
static int dev_dot(g2oc_ctx* c, const double* a, const double* b, int n, double* out) {
  G2OC_K(K_LM_CONTROL) dot_partials<<<kRedBlocks, 256, 0, c->stream>>>(a, b, n, c->partials.p);
  G2OC_LAUNCH_CHECK();
  G2OC_TRY(finalize_sum(c, kRedBlocks, 1, &c->sc.p->refine_rnorm, nullptr));
  G2OC_CUDA_TRY(cudaMemcpyAsync(out, &c->sc.p->refine_rnorm, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return G2OC_OK;
}

// q = H p for the exact Hessian of F at x* (forward-mode dual numbers,
// adjoint_kernels.cuh)
static int adj_hessian_product(g2oc_ctx* c, const double* p, double* q) {
  const Structure& S = c->S;
  cudaStream_t st = c->stream;
  if (S.Pf > 0 && S.lm_warp_ok) {
    const int nch = (int)S.lm_chunk_ptr.size() - 1;
    G2OC_K(K_BACKWARD) ba_hvp_landmark_warp<<<cdiv(nch, 8), 256, 0, st>>>(
        c->ba_edges(), c->ba_vertices(), c->lm_chunk_ptr.p, nch, c->e_lm.p, c->pose_h.p, S.Cf, p, q);
  } else if (S.Pf > 0) {
    G2OC_K(K_BACKWARD) ba_hvp_landmark<<<cdiv(S.Pf, 128), 128, 0, st>>>(c->ba_edges(), c->ba_vertices(), c->l_ptr.p,
                                                                        S.Pf, c->pose_h.p, S.Cf, p, q);
  }
  BACamEdges CE = c->ba_cam_edges();
  G2OC_K(K_BACKWARD) ba_hvp_camera<128><<<S.Cf, 128, 0, st>>>(CE, c->ba_vertices(), c->point_l.p, S.Cf, p, q);
  G2OC_LAUNCH_CHECK();
  return G2OC_OK;
}

// preconditioner: the Gauss-Newton Schur solve at x*. The Gauss-Newton
// system is the same for every application within one
// backward call (same estimates, lambda 0): H and its Schur complement are
// built on the first, the later ones form the reduced right-hand side only.
static int adj_precondition(g2oc_ctx* c, const double* r, double* z) {
  if (c->adj_schur_ready) return c->eng->solve_rhs(r, z, true);
  G2OC_TRY(c->eng->build_system());
  G2OC_TRY(c->eng->solve_rhs(r, z, false));
  c->adj_schur_ready = true;
  return G2OC_OK;
}

int g2oc_backward(g2oc_ctx* c, const double* dL_dx, double* dL_dmeas, double* dL_dlogw, g2oc_backward_stats* stats) {
  G2OC_TRY(check_ctx(c, true));
  if (c->shard_world > 1) {
    set_error("g2oc_backward runs on one rank (no sharding)");
    return G2OC_ERR_NOT_SUPPORTED;
  }
  if (!dL_dx || !dL_dmeas || !dL_dlogw) {
    set_error("dL_dx, dL_dmeas and dL_dlogw must be given");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  const Structure& S = c->S;
  if (!S.ba || !S.schur || S.Cf == 0 || S.D != 2 || S.bal || c->pose_edges()) {
    set_error("g2oc_backward supports SE3 bundle adjustment with two-row projection edges, free cameras and landmarks");
    return G2OC_ERR_NOT_SUPPORTED;
  }
  cudaStream_t st = c->stream;
  const int n = c->vec_size();
  // dL/dx in Hessian order (free cameras, then free landmarks)
  std::vector<double> g(n);
  for (int h = 0; h < S.Cf; ++h)
    for (int a = 0; a < 6; ++a) g[(size_t)h * 6 + a] = dL_dx[(size_t)S.free_pose_of_h[h] * 6 + a];
  for (int l = 0; l < S.Pf; ++l)
    for (int a = 0; a < 3; ++a)
      g[(size_t)S.Cf * 6 + l * 3 + a] = dL_dx[(size_t)S.C * 6 + (size_t)S.free_point_of_l[l] * 3 + a];
  G2OC_TRY(c->adj_g.upload(g, st));
  for (auto* bf : {&c->adj_v, &c->adj_r, &c->adj_dv, &c->adj_p, &c->adj_q, &c->adj_rold})
    G2OC_TRY(bf->alloc(n));
  const size_t nb = (size_t)n * sizeof(double);
  // v = H^-1 g by flexible preconditioned conjugate gradients on the exact
  // Hessian of F (FP64 products by forward-mode differentiation),
  // preconditioned by the Gauss-Newton Schur solve in the context's
  // precision and linear solver; Polak-Ribiere beta, since the inner solve
  // is itself iterative
  G2OC_CUDA_TRY(cudaMemsetAsync(c->adj_v.p, 0, nb, st));
  G2OC_CUDA_TRY(cudaMemcpyAsync(c->adj_r.p, c->adj_g.p, nb, cudaMemcpyDeviceToDevice, st));
  double gg = 0.0;
  G2OC_TRY(dev_dot(c, c->adj_g.p, c->adj_g.p, n, &gg));
  int steps = 0;
  double rel = gg > 0.0 ? 1.0 : 0.0;
  G2OC_TRY(reset_pcg(c));
  c->adj_schur_ready = false;
  if (gg > 0.0) {
    G2OC_TRY(adj_precondition(c, c->adj_r.p, c->adj_dv.p));  // z
    G2OC_CUDA_TRY(cudaMemcpyAsync(c->adj_p.p, c->adj_dv.p, nb, cudaMemcpyDeviceToDevice, st));
    double rz = 0.0;
    G2OC_TRY(dev_dot(c, c->adj_r.p, c->adj_dv.p, n, &rz));
    while (steps < kAdjointMaxSteps) {
      G2OC_TRY(adj_hessian_product(c, c->adj_p.p, c->adj_q.p));
      double pq = 0.0;
      G2OC_TRY(dev_dot(c, c->adj_p.p, c->adj_q.p, n, &pq));
      ++steps;
      if (!(pq > 0.0) || !(rz > 0.0)) break;  // not positive definite along p: not at a minimum
      const double alpha = rz / pq;
      G2OC_K(K_AXPY) axpy_kernel<<<cdiv(n, 256), 256, 0, st>>>(c->adj_v.p, c->adj_p.p, alpha, n);
      G2OC_CUDA_TRY(cudaMemcpyAsync(c->adj_rold.p, c->adj_r.p, nb, cudaMemcpyDeviceToDevice, st));
      G2OC_K(K_AXPY) axpy_kernel<<<cdiv(n, 256), 256, 0, st>>>(c->adj_r.p, c->adj_q.p, -alpha, n);
      G2OC_LAUNCH_CHECK();
      double rr = 0.0;
      G2OC_TRY(dev_dot(c, c->adj_r.p, c->adj_r.p, n, &rr));
      rel = std::sqrt(rr / gg);
      if (rel <= kAdjointTolerance) break;
      G2OC_TRY(adj_precondition(c, c->adj_r.p, c->adj_dv.p));
      double rz_new = 0.0, zr_old = 0.0;
      G2OC_TRY(dev_dot(c, c->adj_r.p, c->adj_dv.p, n, &rz_new));
      G2OC_TRY(dev_dot(c, c->adj_rold.p, c->adj_dv.p, n, &zr_old));
      const double beta = (rz_new - zr_old) / rz;
      G2OC_K(K_AXPY) xpay_kernel<<<cdiv(n, 256), 256, 0, st>>>(c->adj_p.p, c->adj_dv.p, beta, n);
      G2OC_LAUNCH_CHECK();
      rz = rz_new;
    }
    // the true residual |g - H v| / |g|
    G2OC_TRY(adj_hessian_product(c, c->adj_v.p, c->adj_q.p));
    G2OC_CUDA_TRY(cudaMemcpyAsync(c->adj_r.p, c->adj_g.p, nb, cudaMemcpyDeviceToDevice, st));
    G2OC_K(K_AXPY) axpy_kernel<<<cdiv(n, 256), 256, 0, st>>>(c->adj_r.p, c->adj_q.p, -1.0, n);
    G2OC_LAUNCH_CHECK();
    double rr = 0.0;
    G2OC_TRY(dev_dot(c, c->adj_r.p, c->adj_r.p, n, &rr));
    rel = std::sqrt(rr / gg);
  }
  c->system_built = false;  // the preconditioner rebuilt the engine's H
  DevScalars h;
  g2oc_iteration_stats tmp;
  memset(&tmp, 0, sizeof(tmp));
  G2OC_TRY(read_state(c, &h, &tmp));
  // per-edge gradients, caller's edge order (zero for inactive edges)
  G2OC_TRY(c->adj_dmeas.alloc((size_t)S.E * 2 + 1));
  G2OC_TRY(c->adj_dlogw.alloc((size_t)S.E + 1));
  G2OC_CUDA_TRY(cudaMemsetAsync(c->adj_dmeas.p, 0, c->adj_dmeas.bytes(), st));
  G2OC_CUDA_TRY(cudaMemsetAsync(c->adj_dlogw.p, 0, c->adj_dlogw.bytes(), st));
  const int na = (int)S.act.size();
  if (na > 0) {
    G2OC_K(K_BACKWARD) ba_backward_edges<<<cdiv(na, 128), 128, 0, st>>>(
        c->ba_edges(), c->ba_vertices(), c->pose_h.p, c->point_l.p, S.Cf, c->adj_v.p, c->src_dev.p, c->adj_dmeas.p,
        c->adj_dlogw.p);
    G2OC_LAUNCH_CHECK();
  }
  if (S.E > 0) {
    G2OC_CUDA_TRY(cudaMemcpyAsync(dL_dmeas, c->adj_dmeas.p, (size_t)S.E * 2 * sizeof(double), cudaMemcpyDeviceToHost,
                                  st));
    G2OC_CUDA_TRY(cudaMemcpyAsync(dL_dlogw, c->adj_dlogw.p, (size_t)S.E * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  G2OC_CUDA_TRY(cudaStreamSynchronize(st));
  if (stats) {
    stats->refinement_steps = steps;
    stats->pcg_iterations = tmp.iterations_linear_solver;
    stats->relative_residual = rel;
  }
  if (rel > kAdjointAcceptance) {
    set_error("adjoint solve stopped at relative residual %.3e after %d steps", rel, steps);
    return G2OC_ERR_NOT_CONVERGED;
  }
  return G2OC_OK;
}

// ------------------------------------------------------- batched windows
int g2oc_upload_windows(g2oc_ctx* c, int32_t num_windows, const g2oc_graph* w) {
  G2OC_TRY(check_ctx(c, false));
  if (c->shard_world > 1) {
    set_error("batched windows shard by window (one context per rank), not by landmark");
    return G2OC_ERR_NOT_SUPPORTED;
  }
  if (num_windows <= 0 || !w) {
    set_error("num_windows must be positive and windows non-NULL");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  for (int i = 0; i < num_windows; ++i) {
    const g2oc_graph& g = w[i];
    if (g.pose_type != G2OC_POSE_SE3EXPMAP ||
        (g.edge_type != G2OC_EDGE_PROJECT_XYZ2UV && g.edge_type != G2OC_EDGE_SE3_PROJECT_XYZ)) {
      set_error("window %d: batched windows are bundle adjustments (VertexSE3Expmap, EdgeProjectXYZ2UV or "
                "EdgeSE3ProjectXYZ)", i);
      return G2OC_ERR_NOT_SUPPORTED;
    }
    const double fy_i = g.edge_type == G2OC_EDGE_SE3_PROJECT_XYZ ? g.focal_length_y : g.focal_length;
    const double fy_0 = w[0].edge_type == G2OC_EDGE_SE3_PROJECT_XYZ ? w[0].focal_length_y : w[0].focal_length;
    if (g.focal_length != w[0].focal_length || fy_i != fy_0 || g.principal_point[0] != w[0].principal_point[0] ||
        g.principal_point[1] != w[0].principal_point[1]) {
      set_error("window %d: every window must use the same camera parameters", i);
      return G2OC_ERR_NOT_SUPPORTED;
    }
    if (!g.pose_estimate || !g.edge_vertex || !g.measurement || !g.information ||
        (g.num_points > 0 && !g.point_estimate)) {
      set_error("window %d: graph array is NULL", i);
      return G2OC_ERR_INVALID_ARGUMENT;
    }
  }
  // pack: vertices and edges window after window, vertex indices offset
  std::vector<int> pose_off(num_windows + 1, 0), point_off(num_windows + 1, 0), edge_off(num_windows + 1, 0);
  for (int i = 0; i < num_windows; ++i) {
    pose_off[i + 1] = pose_off[i] + w[i].num_poses;
    point_off[i + 1] = point_off[i] + w[i].num_points;
    edge_off[i + 1] = edge_off[i] + w[i].num_edges;
  }
  const int C = pose_off[num_windows], P = point_off[num_windows], E = edge_off[num_windows];
  g2oc::PinnedVec<double>&pose = c->pk_pose, &point = c->pk_point, &meas = c->pk_meas, &info = c->pk_info,
                          &delta = c->pk_delta;
  g2oc::PinnedVec<uint8_t>&pf = c->pk_pf, &qf = c->pk_qf;
  g2oc::PinnedVec<int32_t>& ev = c->pk_ev;
  G2OC_TRY(pose.resize((size_t)C * 7));
  G2OC_TRY(point.resize((size_t)P * 3));
  G2OC_TRY(meas.resize((size_t)E * 2));
  G2OC_TRY(info.resize((size_t)E * 4));
  G2OC_TRY(delta.resize(E));
  G2OC_TRY(pf.resize(C));
  G2OC_TRY(qf.resize(P));
  G2OC_TRY(ev.resize((size_t)E * 2));
  bool robust = false;
  for (int i = 0; i < num_windows; ++i) robust |= w[i].robust_delta != nullptr;
  // windows in parallel (each writes its own ranges); the first window with
  // an out-of-range vertex index is reported
  int bad_window = num_windows, bad_edge = 0;
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = 0; i < num_windows; ++i) {
    const g2oc_graph& g = w[i];
    memcpy(pose.data() + (size_t)pose_off[i] * 7, g.pose_estimate, (size_t)g.num_poses * 7 * sizeof(double));
    if (g.num_points)
      memcpy(point.data() + (size_t)point_off[i] * 3, g.point_estimate, (size_t)g.num_points * 3 * sizeof(double));
    if (g.pose_fixed) memcpy(pf.data() + pose_off[i], g.pose_fixed, g.num_poses);
    else memset(pf.data() + pose_off[i], 0, g.num_poses);
    if (g.point_fixed) memcpy(qf.data() + point_off[i], g.point_fixed, g.num_points);
    else memset(qf.data() + point_off[i], 0, g.num_points);
    memcpy(meas.data() + (size_t)edge_off[i] * 2, g.measurement, (size_t)g.num_edges * 2 * sizeof(double));
    memcpy(info.data() + (size_t)edge_off[i] * 4, g.information, (size_t)g.num_edges * 4 * sizeof(double));
    int32_t* evw = ev.data() + 2 * (size_t)edge_off[i];
    double* dw = delta.data() + edge_off[i];
    for (int e = 0; e < g.num_edges; ++e) {
      const int v0 = g.edge_vertex[2 * e], v1 = g.edge_vertex[2 * e + 1];
      if (v0 < 0 || v0 >= g.num_points || v1 < 0 || v1 >= g.num_poses) {
#pragma omp critical(g2oc_bad_window)
        if (i < bad_window) {
          bad_window = i;
          bad_edge = e;
        }
        break;
      }
      evw[2 * e] = v0 + point_off[i];
      evw[2 * e + 1] = v1 + pose_off[i];
      dw[e] = g.robust_delta ? g.robust_delta[e] : 0.0;
    }
  }
  if (bad_window < num_windows) {
    set_error("window %d edge %d: vertex index out of range", bad_window, bad_edge);
    return G2OC_ERR_BAD_GRAPH;
  }
  g2oc_graph packed;
  memset(&packed, 0, sizeof(packed));
  packed.pose_type = G2OC_POSE_SE3EXPMAP;
  packed.num_poses = C;
  packed.pose_estimate = pose.data();
  packed.pose_fixed = pf.data();
  packed.num_points = P;
  packed.point_estimate = point.data();
  packed.point_fixed = qf.data();
  packed.edge_type = w[0].edge_type;
  packed.num_edges = E;
  packed.edge_vertex = ev.data();
  packed.measurement = meas.data();
  packed.information = info.data();
  packed.robust_delta = robust ? delta.data() : nullptr;
  packed.focal_length = w[0].focal_length;
  packed.focal_length_y = w[0].focal_length_y;
  packed.principal_point[0] = w[0].principal_point[0];
  packed.principal_point[1] = w[0].principal_point[1];
  // a re-upload of the same windows (same topology, same window ranges) keeps
  // the tuned dense-solve schedule and the captured LM round: every device
  // buffer they use keeps its size and address
  struct Kept {
    cudaGraphExec_t graph = nullptr;
    ~Kept() {
      if (graph) cudaGraphExecDestroy(graph);
    }
  } kept;
  kept.graph = c->win_graph;
  c->win_graph = nullptr;
  const bool was_batch = c->batch, was_tuned = c->win_tuned;
  const int old_nw = c->nw;
  const std::vector<int> old_pose = c->win_pose_h, old_point = c->win_point_h;
  G2OC_TRY(g2oc_upload(c, &packed));
  const bool same_windows = was_batch && c->last_upload_reused && old_nw == num_windows && old_pose == pose_off &&
                            old_point == point_off;
  const Structure& S = c->S;
  if (!S.ba || !S.schur || S.bal) {
    set_error("batched windows need SE3 cameras and free landmarks (Schur complement)");
    return G2OC_ERR_NOT_SUPPORTED;
  }
  // window ranges: free cameras and landmarks are numbered in vertex order, so
  // each window's are contiguous
  const int nw = num_windows;
  std::vector<int> wc(nw + 1, 0), wl(nw + 1, 0), we(nw + 1, 0), ofc(std::max(S.Cf, 1)), ofl(std::max(S.Pf, 1)),
      ofp(std::max(C, 1)), ofq(std::max(P, 1));
  for (int i = 0; i < nw; ++i) {
    int nc = 0, nl = 0;
    for (int v = pose_off[i]; v < pose_off[i + 1]; ++v) {
      ofp[v] = i;
      if (S.pose_h[v] >= 0) ofc[S.pose_h[v]] = i, ++nc;
    }
    for (int v = point_off[i]; v < point_off[i + 1]; ++v) {
      ofq[v] = i;
      if (S.point_l[v] >= 0) ofl[S.point_l[v]] = i, ++nl;
    }
    wc[i + 1] = wc[i] + nc;
    wl[i + 1] = wl[i] + nl;
  }
  // device edges of a window must be contiguous (they are, unless a window has
  // fixed points, whose edges the device order puts after all free landmarks)
  const int na = (int)S.act.size();
  std::vector<int> win_of_edge(E);
  for (int i = 0; i < nw; ++i)
    for (int e = edge_off[i]; e < edge_off[i + 1]; ++e) win_of_edge[e] = i;
  int prev = 0;
  for (int k = 0; k < na; ++k) {
    const int wi = win_of_edge[S.dev_edge[k]];
    if (wi < prev) {
      set_error("batched windows with fixed points are not supported");
      return G2OC_ERR_NOT_SUPPORTED;
    }
    for (int j = prev + 1; j <= wi; ++j) we[j] = k;
    prev = wi;
  }
  for (int j = prev + 1; j <= nw; ++j) we[j] = na;
  // each window's dense (n + 1) x n matrix: the reduced system's lower
  // triangle, then the right-hand side row
  std::vector<long long> mat(nw);
  long long off = 0;
  int nmax = 0;
  for (int i = 0; i < nw; ++i) {
    const int n = 6 * (wc[i + 1] - wc[i]);
    mat[i] = off;
    off += (long long)n * (n + 1);
    nmax = std::max(nmax, n);
  }
  if (win_chol_smem(nmax) > 227 * 1024) {
    set_error("a window has %d free camera unknowns; the dense window solve takes at most %d", nmax,
              (int)((227 * 1024 / sizeof(double) - kWinGroups * kWinNB - 2 * kWinNB) / (kWinNB + 2)));
    return G2OC_ERR_NOT_SUPPORTED;
  }
  cudaStream_t st = c->stream;
  c->nw = nw;
  c->win_cam_h = wc;
  c->win_lm_h = wl;
  c->win_pose_h = pose_off;
  c->win_point_h = point_off;
  c->win_nmax = nmax;
  // a window whose cameras do not all co-observe has zero blocks in its dense
  // matrix, which the Schur rows do not write
  c->win_sparse = false;
  for (int i = 0; i < nw; ++i) {
    const int nb = wc[i + 1] - wc[i];
    const long long blocks = nb > 0 ? (long long)S.sys_rptr[wc[i + 1]] - S.sys_rptr[wc[i]] : 0;
    if (blocks != (long long)nb * (nb + 1) / 2) c->win_sparse = true;
  }
  G2OC_TRY(c->win_cam.upload(wc, st));
  G2OC_TRY(c->win_lm.upload(wl, st));
  G2OC_TRY(c->win_edge.upload(we, st));
  {
    std::vector<int> cw, ce0, cptr(nw + 1, 0);
    for (int i = 0; i < nw; ++i) {
      for (int e0 = we[i]; e0 < we[i + 1]; e0 += kWinChi2Chunk) {
        cw.push_back(i);
        ce0.push_back(e0);
      }
      cptr[i + 1] = (int)cw.size();
    }
    c->win_nchunks = (int)cw.size();
    if (cw.empty()) {
      cw.push_back(0);
      ce0.push_back(0);
    }
    G2OC_TRY(c->win_chunk_w.upload(cw, st));
    G2OC_TRY(c->win_chunk_e0.upload(ce0, st));
    G2OC_TRY(c->win_chunk_ptr.upload(cptr, st));
    G2OC_TRY(c->win_chunk_sum.alloc(cw.size()));
  }
  G2OC_TRY(c->win_pose.upload(pose_off, st));
  G2OC_TRY(c->win_point.upload(point_off, st));
  G2OC_TRY(c->win_of_cam.upload(ofc, st));
  G2OC_TRY(c->win_of_lm.upload(ofl, st));
  G2OC_TRY(c->win_of_pose.upload(ofp, st));
  G2OC_TRY(c->win_of_point.upload(ofq, st));
  G2OC_TRY(c->win_mat.upload(mat, st));
  G2OC_TRY(c->win_scratch.alloc((size_t)std::max(off, 1LL)));
  G2OC_TRY(c->lam_c.alloc(std::max(S.Cf, 1)));
  G2OC_TRY(c->lam_l.alloc(std::max(S.Pf, 1)));
  G2OC_TRY(c->win_state.alloc(nw));
  G2OC_TRY(c->win_active.alloc(1));
  G2OC_CUDA_TRY(cudaStreamSynchronize(st));
  c->batch = true;
  if (same_windows) {
    c->win_tuned = was_tuned;
    c->win_graph = kept.graph;
    kept.graph = nullptr;
  }
  return G2OC_OK;
}

// robust chi2 of every window (which = 0: into chi2_cur at an iteration's
// start; 1: into chi2_temp after a trial step)
static int window_chi2(g2oc_ctx* c, int which) {
  cudaStream_t st = c->stream;
  if (c->win_nchunks > 0) {
    G2OC_K(K_CHI2) win_chi2_chunks<512><<<c->win_nchunks, 512, 0, st>>>(
        c->ba_edges(), c->ba_vertices(), c->windev(), c->win_chunk_w.p, c->win_chunk_e0.p, c->win_state.p, which,
        c->win_chunk_sum.p);
    G2OC_LAUNCH_CHECK();
  }
  G2OC_K(K_CHI2) win_chi2_finish<<<cdiv(c->nw, 128), 128, 0, st>>>(c->win_chunk_ptr.p, c->nw, c->win_chunk_sum.p,
                                                                    c->win_state.p, which);
  G2OC_LAUNCH_CHECK();
  return G2OC_OK;
}

// one LM round of every unfinished window (only stream-ordered work: this is
// what the CUDA graph captures)
static int window_round(g2oc_ctx* c, bool autotune) {
  const Structure& S = c->S;
  cudaStream_t st = c->stream;
  const WinDev W = c->windev();
  const int n = c->vec_size();
  G2OC_CUDA_TRY(cudaMemsetAsync(c->win_active.p, 0, sizeof(int), st));
  G2OC_TRY(window_chi2(c, 0));
  G2OC_LAUNCH_CHECK();
  G2OC_TRY(c->eng->build_system());
  G2OC_TRY(c->eng->batch_lambda_init(c->prm.initial_lambda, c->prm.tau));
  G2OC_K(K_LM_CONTROL) win_spread_lambda<<<cdiv(S.Cf + S.Pf, 256), 256, 0, st>>>(
      c->win_of_cam.p, S.Cf, c->win_of_lm.p, S.Pf, c->win_state.p, c->lam_c.p, c->lam_l.p);
  G2OC_LAUNCH_CHECK();
  G2OC_TRY(push(c));
  G2OC_TRY(c->eng->batch_solve(autotune));
  G2OC_K(K_LM_CONTROL) win_mask_step<<<cdiv(n, 256), 256, 0, st>>>(c->win_of_cam.p, S.Cf, c->win_of_lm.p, S.Pf,
                                                                    c->win_state.p, c->x.p);
  G2OC_LAUNCH_CHECK();
  G2OC_TRY(oplus(c));
  G2OC_TRY(window_chi2(c, 1));
  G2OC_K(K_LM_CONTROL) win_scale<256><<<c->nw, 256, 0, st>>>(c->x.p, c->b.p, S.Cf, W, c->win_state.p);
  G2OC_K(K_LM_CONTROL) win_decide<<<cdiv(c->nw, 128), 128, 0, st>>>(c->win_state.p, c->nw,
                                                                    c->prm.max_trials_after_failure, c->win_iterations,
                                                                    c->win_active.p);
  G2OC_K(K_LM_CONTROL) win_pop<<<cdiv((long long)S.C * 8 + (long long)S.P * 4, 256), 256, 0, st>>>(
      c->win_of_pose.p, S.C, c->win_of_point.p, S.P, c->win_state.p, c->pose_bak.p, c->pose.p, c->point_bak.p,
      c->point.p);
  G2OC_LAUNCH_CHECK();
  return G2OC_OK;
}

int g2oc_optimize_windows(g2oc_ctx* c, int32_t iterations, g2oc_window_stats* stats) {
  G2OC_TRY(check_ctx(c, true));
  if (!c->batch) {
    set_error("no windows uploaded (g2oc_upload_windows)");
    return G2OC_ERR_STATE;
  }
  if (iterations < 0) {
    set_error("iterations < 0");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  if (c->prm.algorithm != G2OC_ALGO_LEVENBERG) {
    set_error("batched windows run Levenberg-Marquardt");
    return G2OC_ERR_NOT_SUPPORTED;
  }
  cudaStream_t st = c->stream;
  // window states: windows without edges are finished from the start
  std::vector<WinState> ws0(c->nw);
  memset(ws0.data(), 0, ws0.size() * sizeof(WinState));
  std::vector<int> we(c->nw + 1);
  G2OC_CUDA_TRY(cudaMemcpy(we.data(), c->win_edge.p, we.size() * sizeof(int), cudaMemcpyDeviceToHost));
  for (int i = 0; i < c->nw; ++i) {
    ws0[i].solve_ok = 1;
    ws0[i].result = G2OC_RESULT_OK;
    if (we[i + 1] == we[i] || iterations == 0) ws0[i].done = 1;
  }
  G2OC_CUDA_TRY(cudaMemcpyAsync(c->win_state.p, ws0.data(), ws0.size() * sizeof(WinState), cudaMemcpyHostToDevice,
                                st));
  G2OC_CUDA_TRY(cudaStreamSynchronize(st));
  const bool timing = c->timing;
  if (iterations != c->win_iterations && c->win_graph) {
    cudaGraphExecDestroy(c->win_graph);
    c->win_graph = nullptr;
  }
  c->win_iterations = iterations;
  const int max_rounds = iterations * std::max(c->prm.max_trials_after_failure, 1);
  int rounds = 0, active = 1;
  // first round eagerly (it also tunes the dense solve), then a captured round
  if (max_rounds > 0) {
    G2OC_TRY(window_round(c, true));
    ++rounds;
    G2OC_CUDA_TRY(cudaMemcpyAsync(&active, c->win_active.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    G2OC_CUDA_TRY(cudaStreamSynchronize(st));
  }
  if (active > 0 && rounds < max_rounds && !c->win_graph) {
    c->timing = false;  // no per-launch events inside the graph
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    int rs = e == cudaSuccess ? window_round(c, false) : G2OC_ERR_CUDA;
    cudaError_t e2 = cudaStreamEndCapture(st, &graph);
    c->timing = timing;
    if (e != cudaSuccess || rs != G2OC_OK || e2 != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      set_error("capturing the window round failed");
      return G2OC_ERR_CUDA;
    }
    e = cudaGraphInstantiate(&c->win_graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      c->win_graph = nullptr;
      set_error("instantiating the window round failed: %s", cudaGetErrorString(e));
      return G2OC_ERR_CUDA;
    }
  }
  // replay the round, checking the count of unfinished windows every few rounds
  while (active > 0 && rounds < max_rounds) {
    const int k = std::min(4, max_rounds - rounds);
    for (int i = 0; i < k; ++i) G2OC_CUDA_TRY(cudaGraphLaunch(c->win_graph, st));
    rounds += k;
    G2OC_CUDA_TRY(cudaMemcpyAsync(&active, c->win_active.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    G2OC_CUDA_TRY(cudaStreamSynchronize(st));
  }
  c->system_built = false;
  c->chi2_carry = false;
  c->win_rounds = rounds;
  if (stats) {
    std::vector<WinState> ws(c->nw);
    G2OC_CUDA_TRY(cudaMemcpy(ws.data(), c->win_state.p, ws.size() * sizeof(WinState), cudaMemcpyDeviceToHost));
    for (int i = 0; i < c->nw; ++i) {
      g2oc_window_stats& o = stats[i];
      o.iterations = ws[i].iteration;
      o.trials = ws[i].trials;
      o.result = ws[i].result;
      o.solve_ok = ws[i].solve_ok;
      o.cholesky_threads = c->win_threads.empty() ? 0 : c->win_threads[i];
      o.rounds = rounds;
      o.chi2_initial = ws[i].chi2_init;
      o.chi2 = ws[i].chi2_cur;
      o.lambda = ws[i].lambda;
    }
  }
  return G2OC_OK;
}

int g2oc_download_window(g2oc_ctx* c, int32_t window, double* pose, double* point) {
  G2OC_TRY(check_ctx(c, true));
  if (!c->batch || window < 0 || window >= c->nw) {
    set_error("no such window");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  const Structure& S = c->S;
  std::vector<double> ps((size_t)S.C * 7), pt((size_t)std::max(S.P, 1) * 3);
  G2OC_TRY(g2oc_download(c, ps.data(), pt.data()));
  const int p0 = c->win_pose_h[window], p1 = c->win_pose_h[window + 1];
  const int q0 = c->win_point_h[window], q1 = c->win_point_h[window + 1];
  if (pose) memcpy(pose, ps.data() + (size_t)p0 * 7, (size_t)(p1 - p0) * 7 * sizeof(double));
  if (point && q1 > q0) memcpy(point, pt.data() + (size_t)q0 * 3, (size_t)(q1 - q0) * 3 * sizeof(double));
  return G2OC_OK;
}

// a caller's block matrix (upper blocks listed column-major, row-major
// values) as a device system in the internal row order
struct CallerSystem {
  Structure tmp;
  std::vector<int32_t> rcv;
  int bs = 0;
  DBuf<int> rp, rcl, brw, dg, cp, cb, pm;
  DBuf<double> val;
  SysDev<double> A;
};

static int caller_system(cudaStream_t st, int32_t nb, const int32_t* offs, int32_t nnzb, const int32_t* rc,
                         const double* values, CallerSystem& cs) {
  if (nb <= 0 || !offs || nnzb <= 0 || !rc || !values) {
    set_error("invalid block system arguments");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  const int bs = offs[1] - offs[0];
  for (int i = 0; i < nb; ++i)
    if (offs[i + 1] - offs[i] != bs) {
      set_error("only uniform block sizes are supported");
      return G2OC_ERR_NOT_SUPPORTED;
    }
  if (bs != 3 && bs != 6) {
    set_error("block size %d not supported (3 or 6)", bs);
    return G2OC_ERR_NOT_SUPPORTED;
  }
  cs.bs = bs;
  cs.rcv.assign(rc, rc + 2 * (size_t)nnzb);
  for (int k = 0; k < nnzb; ++k) {
    const int r = rc[2 * k], cc = rc[2 * k + 1];
    if (r < 0 || cc < 0 || r >= nb || cc >= nb || r > cc ||
        (k > 0 && (rc[2 * k - 1] > cc || (rc[2 * k - 1] == cc && rc[2 * k - 2] >= r)))) {
      set_error("blocks must be upper-triangular and listed column-major");
      return G2OC_ERR_INVALID_ARGUMENT;
    }
  }
  Structure& tmp = cs.tmp;
  build_sym_lists(nb, cs.rcv, tmp);
  for (int i = 0; i < nb; ++i)
    if (tmp.sys_diag[i] < 0) {
      set_error("diagonal block %d missing", i);
      return G2OC_ERR_INVALID_ARGUMENT;
    }
  const size_t per = (size_t)bs * bs;
  std::vector<double> vint((size_t)nnzb * per);
  for (int k = 0; k < nnzb; ++k) {
    const int r = tmp.sys_brow[k], rb = tmp.sys_rptr[r], nblk = tmp.sys_rptr[r + 1] - rb;
    for (size_t e = 0; e < per; ++e)
      vint[(size_t)rb * per + e * nblk + (k - rb)] = values[(size_t)tmp.sys_perm[k] * per + e];
  }
  G2OC_TRY(cs.rp.upload(tmp.sys_rptr, st));
  G2OC_TRY(cs.rcl.upload(tmp.sys_rcol, st));
  G2OC_TRY(cs.brw.upload(tmp.sys_brow, st));
  G2OC_TRY(cs.dg.upload(tmp.sys_diag, st));
  G2OC_TRY(cs.cp.upload(tmp.sys_cptr, st));
  G2OC_TRY(cs.cb.upload(tmp.sys_cblk.empty() ? std::vector<int>{0} : tmp.sys_cblk, st));
  G2OC_TRY(cs.val.upload(vint, st));
  G2OC_TRY(cs.pm.upload(tmp.sys_perm, st));
  cs.A = SysDev<double>{nb, nnzb, cs.rp.p, cs.rcl.p, cs.brw.p, cs.dg.p, cs.cp.p, cs.cb.p, cs.pm.p, cs.val.p};
  return G2OC_OK;
}

int g2oc_solve_block_system(g2oc_ctx* c, int32_t linear_solver, int32_t nb, const int32_t* offs, int32_t nnzb,
                            const int32_t* rc, const double* values, const double* b, double* x, int32_t* iters) {
  G2OC_TRY(check_ctx(c, false));
  if (!b || !x) {
    set_error("invalid block system arguments");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  cudaStream_t st = c->stream;
  CallerSystem cs;
  G2OC_TRY(caller_system(st, nb, offs, nnzb, rc, values, cs));
  const int bs = cs.bs;
  const SysDev<double>& A = cs.A;
  DBuf<double> rhs, xo, mi, r, s, d0, d1, q, qrow, tb;
  const int n = nb * bs;
  G2OC_TRY(rhs.upload(std::vector<double>(b, b + n), st));
  G2OC_TRY(xo.alloc(n));
  int it = 0, ok = 1;
  if (linear_solver == G2OC_LINEAR_CHOLESKY) {
    CholPlan P;
    G2OC_TRY(chol_plan_build(P, nb, bs, cs.rcv, true, st));
    G2OC_TRY(chol_solve<double>(P, st, A, rhs.p, xo.p, &ok, &c->kcount[K_CHOLESKY]));
  } else {
    G2OC_TRY(mi.alloc((size_t)nb * bs * bs));
    G2OC_TRY(r.alloc(n));
    G2OC_TRY(s.alloc(n));
    G2OC_TRY(d0.alloc(n));
    G2OC_TRY(d1.alloc(n));
    G2OC_TRY(q.alloc(n));
    G2OC_TRY(qrow.alloc(n));
    G2OC_TRY(tb.alloc((size_t)nnzb * bs + 1));
    G2OC_TRY(reset_pcg(c));
    if (bs == 3) {
      G2OC_K(K_PCG_DIAG_INV) pcg_diag_inv<double, 3><<<cdiv(nb, 128), 128, 0, st>>>(A, mi.p, c->flag.p);
      G2OC_TRY((run_pcg<double, 3>(c, A, mi.p, rhs.p, xo.p, r.p, s.p, d0.p, d1.p, q.p, qrow.p, tb.p, false, &it)));
    } else {
      G2OC_K(K_PCG_DIAG_INV) pcg_diag_inv<double, 6><<<cdiv(nb, 128), 128, 0, st>>>(A, mi.p, c->flag.p);
      G2OC_TRY((run_pcg<double, 6>(c, A, mi.p, rhs.p, xo.p, r.p, s.p, d0.p, d1.p, q.p, qrow.p, tb.p, false, &it)));
    }
  }
  G2OC_CUDA_TRY(cudaStreamSynchronize(st));
  G2OC_CUDA_TRY(cudaMemcpy(x, xo.p, n * sizeof(double), cudaMemcpyDeviceToHost));
  if (iters) *iters = it;
  return ok ? G2OC_OK : G2OC_ERR_NOT_PD;
}

// blocks of the inverse of a caller system (LinearSolver::solvePattern)
static int solve_pattern(g2oc_ctx* c, CallerSystem& cs, int32_t nb, int32_t nreq, const int32_t* req, double* out) {
  if (nreq < 0 || (nreq > 0 && (!req || !out))) {
    set_error("invalid block index arguments");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  std::vector<int32_t> extra(req, req + 2 * (size_t)nreq);
  std::vector<int2> pairs(nreq > 0 ? nreq : 1, make_int2(0, 0));
  for (int q = 0; q < nreq; ++q) {
    const int r = req[2 * q], cc = req[2 * q + 1];
    if (r < 0 || cc < 0 || r >= nb || cc >= nb) {
      set_error("block index pair (%d, %d) out of range [0, %d)", r, cc, nb);
      return G2OC_ERR_INVALID_ARGUMENT;
    }
    pairs[q] = make_int2(r, cc);
  }
  cudaStream_t st = c->stream;
  CholPlan P;
  G2OC_TRY(chol_plan_build(P, nb, cs.bs, cs.rcv, true, st, &extra));
  DBuf<int2> d_req;
  DBuf<double> d_out;
  G2OC_TRY(d_req.upload(pairs, st));
  G2OC_TRY(d_out.alloc((size_t)(nreq > 0 ? nreq : 1) * cs.bs * cs.bs));
  int ok = 1;
  G2OC_TRY(chol_selected_inverse<double>(P, st, cs.A, d_req.p, nreq, d_out.p, &ok, &c->kcount[K_CHOLESKY]));
  if (!ok) {
    set_error("the matrix is not positive definite");
    return G2OC_ERR_NOT_PD;
  }
  if (nreq > 0)
    G2OC_CUDA_TRY(cudaMemcpy(out, d_out.p, (size_t)nreq * cs.bs * cs.bs * sizeof(double), cudaMemcpyDeviceToHost));
  return G2OC_OK;
}

int g2oc_solve_pattern_block_system(g2oc_ctx* c, int32_t nb, const int32_t* offs, int32_t nnzb, const int32_t* rc,
                                    const double* values, int32_t num_blocks, const int32_t* block_indices,
                                    double* out) {
  G2OC_TRY(check_ctx(c, false));
  CallerSystem cs;
  G2OC_TRY(caller_system(c->stream, nb, offs, nnzb, rc, values, cs));
  return solve_pattern(c, cs, nb, num_blocks, block_indices, out);
}

int g2oc_compute_marginals(g2oc_ctx* c, int32_t num_blocks, const int32_t* block_indices, double* out) {
  G2OC_TRY(check_ctx(c, true));
  if (c->shard_world > 1 || c->batch) {
    set_error("marginals of a sharded bundle adjustment or of batched windows are not supported");
    return G2OC_ERR_NOT_SUPPORTED;
  }
  const Structure& S = c->S;
  const int nb = S.Cf;
  if (nb <= 0) {
    set_error("the graph has no free pose");
    return G2OC_ERR_BAD_GRAPH;
  }
  // H at the current estimates, then its pose part Hpp
  G2OC_TRY(g2oc_build_system(c));
  const int pd = S.pd;
  const size_t nnzb = S.hpp_rc.size() / 2;
  std::vector<double> hpp(nnzb * pd * pd);
  G2OC_TRY(c->eng->get_hessian(hpp.data(), nullptr, nullptr));
  std::vector<int32_t> offs(nb + 1);
  for (int i = 0; i <= nb; ++i) offs[i] = i * pd;
  CallerSystem cs;
  G2OC_TRY(caller_system(c->stream, nb, offs.data(), (int32_t)nnzb, S.hpp_rc.data(), hpp.data(), cs));
  return solve_pattern(c, cs, nb, num_blocks, block_indices, out);
}

int g2oc_get_stream(g2oc_ctx* c, void** stream) {
  G2OC_TRY(check_ctx(c, false));
  if (!stream) {
    set_error("stream is NULL");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  *stream = (void*)c->stream;
  return G2OC_OK;
}

int g2oc_restore_initial_estimates(g2oc_ctx* c) {
  G2OC_TRY(check_ctx(c, true));
  c->chi2_carry = false;
  G2OC_CUDA_TRY(cudaMemcpyAsync(c->pose.p, c->pose_init.p, c->pose.bytes(), cudaMemcpyDeviceToDevice, c->stream));
  if (c->point.n)
    G2OC_CUDA_TRY(cudaMemcpyAsync(c->point.p, c->point_init.p, c->point.bytes(), cudaMemcpyDeviceToDevice, c->stream));
  G2OC_CUDA_TRY(cudaMemsetAsync(c->oplus_count.p, 0, c->oplus_count.bytes(), c->stream));
  G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->system_built = false;
  return G2OC_OK;
}

int g2oc_set_kernel_timing(g2oc_ctx* c, int enable) {
  G2OC_TRY(check_ctx(c, false));
  G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->flush_timing();
  for (int k = 0; k < K_COUNT; ++k) {
    c->kcount[k] = 0;
    c->ktime_ms[k] = 0.0;
  }
  c->timing = enable != 0;
  return G2OC_OK;
}

int g2oc_get_kernel_stats(g2oc_ctx* c, g2oc_kernel_stat* out, int capacity, int* count, int64_t* total) {
  G2OC_TRY(check_ctx(c, false));
  G2OC_CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->flush_timing();
  int n = 0;
  long long t = 0;
  for (int k = 0; k < K_COUNT; ++k) {
    t += c->kcount[k];
    if (c->kcount[k] == 0) continue;
    if (out && n < capacity) {
      memset(out[n].name, 0, sizeof(out[n].name));
      strncpy(out[n].name, kKernelNames[k], sizeof(out[n].name) - 1);
      out[n].launches = c->kcount[k];
      out[n].total_ms = c->ktime_ms[k];
    }
    ++n;
  }
  if (count) *count = n;
  if (total) *total = t;
  return G2OC_OK;
}

}  // extern "C"

